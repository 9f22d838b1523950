// CPU oracle for the sparkalog binary recursive operator pipeline.
//
// TEST INFRASTRUCTURE ONLY. This library is what the CUDA path is compared
// against (tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline arm). Nothing in the product package links, loads or calls it.
//
// Every function restates the reference's CPU semantics and cites the file and
// line it follows; paths are relative to the rdaum/sparkalog source tree.
//   - operators:       crates/sparkalog-execution/src/lib.rs
//   - range index:     crates/sparkalog-storage/src/lib.rs
//   - semi-naive loop: crates/sparkalog-recursion/src/generic.rs
// The reference is Rust and cannot be compiled in this environment (no cargo or
// rustc); parity is pinned by the reference's own known-answer tests, which
// tests/golden/ restates, and by the serial-versus-parallel equality the
// reference asserts for every operator.

#include <algorithm>
#include <atomic>
#include <chrono>
#include <set>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <vector>
#include <unordered_map>

namespace {

using u32 = std::uint32_t;
using u64 = std::uint64_t;

// ---------------------------------------------------------------------------
// Thread helpers (stand-in for the persistent Rayon pool used by *_cpu_parallel)
// ---------------------------------------------------------------------------

int clamp_threads(int threads) {
    if (threads <= 0) {
        unsigned hw = std::thread::hardware_concurrency();
        threads = hw == 0 ? 1 : static_cast<int>(hw);
    }
    return threads;
}

template <class F>
void parallel_for(size_t tasks, int threads, F&& body) {
    if (tasks == 0) return;
    threads = std::min<size_t>(clamp_threads(threads), tasks);
    if (threads <= 1) {
        for (size_t t = 0; t < tasks; ++t) body(t);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> pool;
    pool.reserve(threads);
    for (int w = 0; w < threads; ++w) {
        pool.emplace_back([&]() {
            for (;;) {
                size_t t = next.fetch_add(1);
                if (t >= tasks) break;
                body(t);
            }
        });
    }
    for (auto& th : pool) th.join();
}

inline u64 pack_tuple(u32 first, u32 second) {  // execution/src/lib.rs:344-346
    return (static_cast<u64>(first) << 32) | static_cast<u64>(second);
}

// execution/src/lib.rs:348-357
size_t deduplicate_sorted(u64* packed, size_t len) {
    size_t unique = 0;
    for (size_t read = 0; read < len; ++read) {
        if (unique == 0 || packed[read] != packed[unique - 1]) {
            packed[unique] = packed[read];
            ++unique;
        }
    }
    return unique;
}

// Merge-path split, execution/src/lib.rs:981-997.
size_t merge_partition(const u64* left, size_t left_len, const u64* right, size_t right_len,
                       size_t output_position) {
    size_t low = output_position > right_len ? output_position - right_len : 0;
    size_t high = std::min(output_position, left_len);
    while (low < high) {
        size_t left_position = low + (high - low) / 2;
        size_t right_position = output_position - left_position;
        if (left_position < left_len && right_position > 0 &&
            right[right_position - 1] > left[left_position]) {
            low = left_position + 1;
        } else {
            high = left_position;
        }
    }
    return low;
}

// execution/src/lib.rs:999-1012 (ties take the left element first).
void merge_packed_range(const u64* left, size_t left_len, const u64* right, size_t right_len,
                        size_t output_start, u64* output, size_t output_len) {
    size_t left_row = merge_partition(left, left_len, right, right_len, output_start);
    size_t right_row = output_start - left_row;
    for (size_t i = 0; i < output_len; ++i) {
        if (right_row == right_len || (left_row < left_len && left[left_row] <= right[right_row])) {
            output[i] = left[left_row++];
        } else {
            output[i] = right[right_row++];
        }
    }
}

void parallel_merge(const u64* a, size_t na, const u64* b, size_t nb, u64* out, int threads) {
    size_t total = na + nb;
    if (total == 0) return;
    int workers = static_cast<int>(std::min<size_t>(clamp_threads(threads), total));
    size_t chunk = (total + workers - 1) / workers;
    size_t chunks = (total + chunk - 1) / chunk;
    parallel_for(chunks, threads, [&](size_t c) {
        size_t start = c * chunk;
        size_t len = std::min(chunk, total - start);
        merge_packed_range(a, na, b, nb, start, out + start, len);
    });
}

// Stand-in for rayon's par_sort_unstable over u64 keys (lib.rs:431): chunked
// std::sort followed by rounds of parallel merge-path merges. Sorting u64 keys
// is deterministic, so the result equals the serial sort (lib.rs:409).
void parallel_sort(std::vector<u64>& keys, int threads) {
    threads = clamp_threads(threads);
    size_t n = keys.size();
    if (threads <= 1 || n < 65536) {
        std::sort(keys.begin(), keys.end());
        return;
    }
    size_t runs = static_cast<size_t>(threads);
    size_t chunk = (n + runs - 1) / runs;
    std::vector<size_t> bounds;
    for (size_t s = 0; s < n; s += chunk) bounds.push_back(s);
    bounds.push_back(n);
    parallel_for(bounds.size() - 1, threads, [&](size_t r) {
        std::sort(keys.begin() + bounds[r], keys.begin() + bounds[r + 1]);
    });
    std::vector<u64> scratch(n);
    u64* src = keys.data();
    u64* dst = scratch.data();
    while (bounds.size() > 2) {
        std::vector<size_t> next_bounds;
        size_t pairs = (bounds.size() - 1) / 2;
        int per_pair = std::max(1, threads / static_cast<int>(std::max<size_t>(pairs, 1)));
        for (size_t r = 0; r + 1 < bounds.size(); r += 2) {
            next_bounds.push_back(bounds[r]);
            if (r + 2 < bounds.size()) {
                size_t a0 = bounds[r], a1 = bounds[r + 1], b1 = bounds[r + 2];
                parallel_merge(src + a0, a1 - a0, src + a1, b1 - a1, dst + a0, per_pair);
            } else {
                std::memcpy(dst + bounds[r], src + bounds[r], (bounds[r + 1] - bounds[r]) * 8);
            }
        }
        next_bounds.push_back(n);
        bounds.swap(next_bounds);
        std::swap(src, dst);
    }
    if (src != keys.data()) std::memcpy(keys.data(), src, n * 8);
}

// ---------------------------------------------------------------------------
// U32RangeIndex::build_slice, storage/src/lib.rs:357-393
// ---------------------------------------------------------------------------

struct RangeIndex {
    std::vector<u32> keys;
    std::vector<u32> starts;
    std::vector<u32> rows;
    size_t source_rows = 0;

    // IndexView::lookup, execution/src/lib.rs:1221-1227
    void lookup(u32 key, size_t* begin, size_t* end) const {
        auto it = std::lower_bound(keys.begin(), keys.end(), key);
        if (it == keys.end() || *it != key) {
            *begin = *end = 0;
            return;
        }
        size_t index = static_cast<size_t>(it - keys.begin());
        *begin = starts[index];
        *end = starts[index + 1];
    }
};

RangeIndex build_range_index(const u32* values, size_t n) {
    RangeIndex index;
    index.source_rows = n;
    index.rows.resize(n);
    for (size_t i = 0; i < n; ++i) index.rows[i] = static_cast<u32>(i);
    std::sort(index.rows.begin(), index.rows.end(), [&](u32 a, u32 b) {
        return values[a] != values[b] ? values[a] < values[b] : a < b;
    });
    for (size_t p = 0; p < n; ++p) {
        u32 key = values[index.rows[p]];
        if (p == 0 || index.keys.back() != key) {
            index.keys.push_back(key);
            index.starts.push_back(static_cast<u32>(p));
        }
    }
    index.starts.push_back(static_cast<u32>(n));
    return index;
}

// ---------------------------------------------------------------------------
// Relations: two u32 columns (the binary subset's canonical SoA layout)
// ---------------------------------------------------------------------------

struct Rel {
    std::vector<u32> c[2];
    size_t len() const { return c[0].size(); }
    void clear() { c[0].clear(); c[1].clear(); }
};

struct JoinPlan {          // relational/src/lib.rs:46-50
    u32 left_key;
    u32 right_key;
    u32 proj_side[2];      // 0 = left, 1 = right (JoinInput)
    u32 proj_col[2];
};

// join_cpu_serial / join_cpu_parallel, execution/src/lib.rs:1309-1423.
// Output is left-row-major; the matches of one left row follow index order.
void join_op(const Rel& left, const Rel& right, const RangeIndex& index, const JoinPlan& plan,
             int threads, Rel* out) {
    const std::vector<u32>& left_key = left.c[plan.left_key];
    size_t n = left.len();
    std::vector<u64> counts(n), offsets(n);
    parallel_for((n + 65535) / 65536, threads, [&](size_t chunk) {
        size_t s = chunk * 65536, e = std::min(n, s + 65536);
        for (size_t r = s; r < e; ++r) {
            size_t b, en;
            index.lookup(left_key[r], &b, &en);
            counts[r] = en - b;
        }
    });
    u64 total = 0;
    for (size_t r = 0; r < n; ++r) {
        offsets[r] = total;
        total += counts[r];
    }
    out->c[0].assign(total, 0);
    out->c[1].assign(total, 0);
    parallel_for((n + 65535) / 65536, threads, [&](size_t chunk) {
        size_t s = chunk * 65536, e = std::min(n, s + 65536);
        for (size_t r = s; r < e; ++r) {
            size_t b, en;
            index.lookup(left_key[r], &b, &en);
            u64 o = offsets[r];
            for (size_t m = b; m < en; ++m, ++o) {
                u32 right_row = index.rows[m];
                for (int j = 0; j < 2; ++j) {
                    out->c[j][o] = plan.proj_side[j] == 0 ? left.c[plan.proj_col[j]][r]
                                                          : right.c[plan.proj_col[j]][right_row];
                }
            }
        }
    });
}

// distinct_cpu_serial / distinct_cpu_parallel, execution/src/lib.rs:398-434.
void distinct_op(const Rel& input, const u32 columns[2], int threads, Rel* out) {
    size_t n = input.len();
    std::vector<u64> packed(n);
    const std::vector<u32>& a = input.c[columns[0]];
    const std::vector<u32>& b = input.c[columns[1]];
    for (size_t i = 0; i < n; ++i) packed[i] = pack_tuple(a[i], b[i]);
    parallel_sort(packed, threads);
    size_t unique = deduplicate_sorted(packed.data(), n);
    out->c[0].resize(unique);
    out->c[1].resize(unique);
    for (size_t i = 0; i < unique; ++i) {
        out->c[0][i] = static_cast<u32>(packed[i] >> 32);
        out->c[1][i] = static_cast<u32>(packed[i]);
    }
}

// compare_pair / lower_bound_pair, execution/src/lib.rs:570-600.
inline bool pair_less(u32 a0, u32 a1, u32 b0, u32 b1) {
    return a0 != b0 ? a0 < b0 : a1 < b1;
}

size_t lower_bound_pair(const u32* f, const u32* s, size_t n, u32 first, u32 second) {
    size_t low = 0, high = n;
    while (low < high) {
        size_t middle = low + (high - low) / 2;
        if (pair_less(f[middle], s[middle], first, second)) low = middle + 1;
        else high = middle;
    }
    return low;
}

// anti_join_chunk_count/emit + anti_join_cpu_serial/parallel,
// execution/src/lib.rs:602-783. Stable: the output keeps the left order.
void anti_join_op(const Rel& left, const u32 lcols[2], const Rel& right, const u32 rcols[2],
                  int threads, Rel* out) {
    const u32* lf = left.c[lcols[0]].data();
    const u32* ls = left.c[lcols[1]].data();
    const u32* rf = right.c[rcols[0]].data();
    const u32* rs = right.c[rcols[1]].data();
    size_t ln = left.len(), rn = right.len();
    int workers = static_cast<int>(std::min<size_t>(clamp_threads(threads), std::max<size_t>(ln, 1)));
    size_t chunk = ln == 0 ? 1 : (ln + workers - 1) / workers;
    size_t chunks = ln == 0 ? 0 : (ln + chunk - 1) / chunk;
    std::vector<u64> selected(chunks, 0);
    auto scan = [&](size_t c, bool emit, u64 out_at) {
        size_t row_start = c * chunk, row_end = std::min(ln, row_start + chunk);
        if (row_start == row_end) return;
        size_t right_row = lower_bound_pair(rf, rs, rn, lf[row_start], ls[row_start]);
        u64 count = 0;
        for (size_t l = row_start; l < row_end; ++l) {
            while (right_row < rn && pair_less(rf[right_row], rs[right_row], lf[l], ls[l])) ++right_row;
            bool matched = right_row < rn && rf[right_row] == lf[l] && rs[right_row] == ls[l];
            if (!matched) {
                if (emit) {
                    out->c[0][out_at + count] = lf[l];
                    out->c[1][out_at + count] = ls[l];
                }
                ++count;
            }
        }
        if (!emit) selected[c] = count;
    };
    parallel_for(chunks, threads, [&](size_t c) { scan(c, false, 0); });
    u64 total = 0;
    std::vector<u64> offsets(chunks);
    for (size_t c = 0; c < chunks; ++c) {
        offsets[c] = total;
        total += selected[c];
    }
    out->c[0].assign(total, 0);
    out->c[1].assign(total, 0);
    parallel_for(chunks, threads, [&](size_t c) { scan(c, true, offsets[c]); });
}

// union_cpu_serial / union_cpu_parallel, execution/src/lib.rs:934-1066.
void union_op(const Rel& left, const u32 lcols[2], const Rel& right, const u32 rcols[2],
              int threads, Rel* out) {
    size_t ln = left.len(), rn = right.len();
    std::vector<u64> pl(ln), pr(rn), merged(ln + rn);
    for (size_t i = 0; i < ln; ++i) pl[i] = pack_tuple(left.c[lcols[0]][i], left.c[lcols[1]][i]);
    for (size_t i = 0; i < rn; ++i) pr[i] = pack_tuple(right.c[rcols[0]][i], right.c[rcols[1]][i]);
    parallel_merge(pl.data(), ln, pr.data(), rn, merged.data(), threads);
    size_t unique = deduplicate_sorted(merged.data(), ln + rn);
    out->c[0].resize(unique);
    out->c[1].resize(unique);
    for (size_t i = 0; i < unique; ++i) {
        out->c[0][i] = static_cast<u32>(merged[i] >> 32);
        out->c[1][i] = static_cast<u32>(merged[i]);
    }
}

// ---------------------------------------------------------------------------
// RelationStore / RecursiveExecutor, recursion/src/generic.rs:16-525
// ---------------------------------------------------------------------------

struct RelState {
    Rel full;
    Rel delta;
    Rel newt;
    bool recursive = false;
    u64 version = 0;
};

struct Store {
    std::map<u32, RelState> relations;
    std::string error;
};

}  // namespace

extern "C" {

// One RecursiveRulePlan (relational/src/lib.rs:74-82) as a flat record.
struct oracle_rule_plan {
    u32 target;
    u32 delta_input;
    u32 right_input;
    u32 left_key;
    u32 right_key;
    u32 proj_side[2];
    u32 proj_col[2];
    u32 distinct_cols[2];
    u32 anti_left[2];
    u32 anti_right[2];
    u32 union_left[2];
    u32 union_right[2];
};

// ---------------- generators ----------------

// splitmix64 output for counter i (state = seed + (i + 1) * golden gamma).
u64 oracle_splitmix64(u64 seed, u64 i) {
    u64 z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Seeded directed Erdos-Renyi edge set: candidate j is
// (hi32(z(2j)) * n >> 32, hi32(z(2j+1)) * n >> 32); self-loops are rejected and
// the first `edges` distinct candidates (in j order) are kept. The result is
// written sorted by (src, dst), i.e. the BTreeSet order execute_binary gives
// the EDB (datalog/src/subset.rs:381-398). Returns the number of edges written
// (smaller than `edges` only if n*(n-1) < edges).
u64 oracle_er_edges(u32 n, u64 edges, u64 seed, u32* src, u32* dst) {
    if (n < 2) return 0;
    u64 possible = static_cast<u64>(n) * (n - 1);
    if (edges > possible) edges = possible;
    std::vector<u64> accepted;
    accepted.reserve(edges);
    std::vector<u64> seen;  // sorted set of accepted keys
    // A hash set keeps this O(E); unordered_set of u64 is fine for test code.
    std::vector<u64> table(1, 0);
    size_t mask = 0;
    size_t count = 0;
    auto rebuild = [&](size_t cap) {
        std::vector<u64> fresh(cap, ~0ull);
        size_t m = cap - 1;
        for (u64 k : accepted) {
            size_t h = static_cast<size_t>((k * 0x9E3779B97F4A7C15ull) >> 17) & m;
            while (fresh[h] != ~0ull) h = (h + 1) & m;
            fresh[h] = k;
        }
        table.swap(fresh);
        mask = m;
    };
    rebuild(1024);
    for (u64 j = 0; count < edges; ++j) {
        u64 zu = oracle_splitmix64(seed, 2 * j);
        u64 zv = oracle_splitmix64(seed, 2 * j + 1);
        u32 u = static_cast<u32>(((zu >> 32) * static_cast<u64>(n)) >> 32);
        u32 v = static_cast<u32>(((zv >> 32) * static_cast<u64>(n)) >> 32);
        if (u == v) continue;
        u64 key = pack_tuple(u, v);
        size_t h = static_cast<size_t>((key * 0x9E3779B97F4A7C15ull) >> 17) & mask;
        bool found = false;
        while (table[h] != ~0ull) {
            if (table[h] == key) { found = true; break; }
            h = (h + 1) & mask;
        }
        if (found) continue;
        table[h] = key;
        accepted.push_back(key);
        ++count;
        if (count * 2 > mask + 1) rebuild((mask + 1) * 2);
    }
    std::sort(accepted.begin(), accepted.end());
    for (size_t i = 0; i < accepted.size(); ++i) {
        src[i] = static_cast<u32>(accepted[i] >> 32);
        dst[i] = static_cast<u32>(accepted[i]);
    }
    (void)seen;
    return accepted.size();
}

// ---------------- range index ----------------

// Returns the number of unique keys. keys needs n slots, starts n + 1, rows n.
u64 oracle_range_index_build(const u32* values, u64 n, u32* keys, u32* starts, u32* rows) {
    RangeIndex index = build_range_index(values, n);
    std::copy(index.keys.begin(), index.keys.end(), keys);
    std::copy(index.starts.begin(), index.starts.end(), starts);
    std::copy(index.rows.begin(), index.rows.end(), rows);
    return index.keys.size();
}

// ---------------- operators ----------------

namespace {
Rel make_rel(const u32* c0, const u32* c1, u64 n) {
    Rel r;
    r.c[0].assign(c0, c0 + n);
    r.c[1].assign(c1, c1 + n);
    return r;
}
void copy_out(const Rel& r, u32* o0, u32* o1) {
    if (r.len() == 0) return;
    std::memcpy(o0, r.c[0].data(), r.len() * 4);
    std::memcpy(o1, r.c[1].data(), r.len() * 4);
}
}  // namespace

// Join output size (count pass of join_cpu_serial, lib.rs:1283-1307).
u64 oracle_join_count(const u32* lc0, const u32* lc1, u64 ln, const u32* rc0, const u32* rc1, u64 rn,
                      u32 left_key, u32 right_key) {
    const u32* lk = left_key == 0 ? lc0 : lc1;
    const u32* rk = right_key == 0 ? rc0 : rc1;
    RangeIndex index = build_range_index(rk, rn);
    u64 total = 0;
    for (u64 r = 0; r < ln; ++r) {
        size_t b, e;
        index.lookup(lk[r], &b, &e);
        total += e - b;
    }
    return total;
}

u64 oracle_join(const u32* lc0, const u32* lc1, u64 ln, const u32* rc0, const u32* rc1, u64 rn,
                u32 left_key, u32 right_key, u32 side0, u32 col0, u32 side1, u32 col1, int threads,
                u32* out0, u32* out1) {
    Rel left = make_rel(lc0, lc1, ln), right = make_rel(rc0, rc1, rn), out;
    RangeIndex index = build_range_index(right.c[right_key].data(), rn);
    JoinPlan plan{left_key, right_key, {side0, side1}, {col0, col1}};
    join_op(left, right, index, plan, threads, &out);
    copy_out(out, out0, out1);
    return out.len();
}

u64 oracle_distinct(const u32* c0, const u32* c1, u64 n, u32 col0, u32 col1, int threads, u32* out0,
                    u32* out1) {
    Rel in = make_rel(c0, c1, n), out;
    u32 cols[2] = {col0, col1};
    distinct_op(in, cols, threads, &out);
    copy_out(out, out0, out1);
    return out.len();
}

u64 oracle_anti_join(const u32* lc0, const u32* lc1, u64 ln, const u32* rc0, const u32* rc1, u64 rn,
                     int threads, u32* out0, u32* out1) {
    Rel left = make_rel(lc0, lc1, ln), right = make_rel(rc0, rc1, rn), out;
    u32 cols[2] = {0, 1};
    anti_join_op(left, cols, right, cols, threads, &out);
    copy_out(out, out0, out1);
    return out.len();
}

u64 oracle_union(const u32* lc0, const u32* lc1, u64 ln, const u32* rc0, const u32* rc1, u64 rn,
                 int threads, u32* out0, u32* out1) {
    Rel left = make_rel(lc0, lc1, ln), right = make_rel(rc0, rc1, rn), out;
    u32 cols[2] = {0, 1};
    union_op(left, cols, right, cols, threads, &out);
    copy_out(out, out0, out1);
    return out.len();
}

// ---------------- store and executor ----------------

void* oracle_store_new() { return new Store(); }
void oracle_store_free(void* s) { delete static_cast<Store*>(s); }

// RelationStore::insert_static, generic.rs:36-51. Returns 0, or -2 on a duplicate id.
int oracle_store_insert_static(void* s, u32 id, const u32* c0, const u32* c1, u64 n) {
    Store* store = static_cast<Store*>(s);
    if (store->relations.count(id)) return -2;
    RelState st;
    st.full = make_rel(c0, c1, n);
    store->relations[id] = std::move(st);
    return 0;
}

// RelationStore::insert_recursive, generic.rs:53-79.
int oracle_store_insert_recursive(void* s, u32 id, const u32* f0, const u32* f1, u64 fn,
                                  const u32* d0, const u32* d1, u64 dn) {
    Store* store = static_cast<Store*>(s);
    if (store->relations.count(id)) return -2;
    RelState st;
    st.full = make_rel(f0, f1, fn);
    st.delta = make_rel(d0, d1, dn);
    st.recursive = true;
    store->relations[id] = std::move(st);
    return 0;
}

// version: 0 = FULL, 1 = DELTA. Returns ~0 for a missing relation.
u64 oracle_store_len(void* s, u32 id, int version) {
    Store* store = static_cast<Store*>(s);
    auto it = store->relations.find(id);
    if (it == store->relations.end()) return ~0ull;
    return version == 0 ? it->second.full.len() : it->second.delta.len();
}

int oracle_store_copy(void* s, u32 id, int version, u32* c0, u32* c1) {
    Store* store = static_cast<Store*>(s);
    auto it = store->relations.find(id);
    if (it == store->relations.end()) return -1;
    copy_out(version == 0 ? it->second.full : it->second.delta, c0, c1);
    return 0;
}

// RecursiveExecutor::compile + run, generic.rs:407-525 (with RuleRuntime::evaluate
// :197-259, TargetRuntime::combine :299-358 and ::apply :360-397).
// Return codes: 0 ok; -1 missing relation; -3 not recursive; -4 empty SCC;
// -5 duplicate SCC relation; -6 delta outside SCC; -7 target outside SCC;
// -8 incompatible target plans; -9 missing rule target; -10 iteration limit.
int oracle_run_scc(void* s, const u32* relations, u64 n_relations, const oracle_rule_plan* rules,
                   u64 n_rules, u64 max_iterations, int threads, u64* iterations_out,
                   u64* total_new_out) {
    Store* store = static_cast<Store*>(s);
    auto& rels = store->relations;
    if (n_relations == 0) return -4;
    for (u64 i = 0; i < n_relations; ++i) {
        for (u64 j = 0; j < i; ++j)
            if (relations[j] == relations[i]) return -5;
        auto it = rels.find(relations[i]);
        if (it == rels.end()) return -1;
        if (!it->second.recursive) return -3;
    }
    auto in_scc = [&](u32 id) {
        for (u64 i = 0; i < n_relations; ++i)
            if (relations[i] == id) return true;
        return false;
    };
    for (u64 r = 0; r < n_rules; ++r) {
        if (!rels.count(rules[r].delta_input) || !rels.count(rules[r].right_input)) return -1;
        if (!in_scc(rules[r].delta_input)) return -6;
        if (!in_scc(rules[r].target)) return -7;
    }
    // Group rules by target in SCC relation order (generic.rs:434-462).
    std::vector<std::vector<u64>> target_rules(n_relations);
    for (u64 t = 0; t < n_relations; ++t) {
        for (u64 r = 0; r < n_rules; ++r)
            if (rules[r].target == relations[t]) target_rules[t].push_back(r);
        if (target_rules[t].empty()) return -9;
        const oracle_rule_plan& first = rules[target_rules[t][0]];
        for (u64 r : target_rules[t]) {
            const oracle_rule_plan& p = rules[r];
            if (std::memcmp(p.anti_left, first.anti_left, 8) || std::memcmp(p.anti_right, first.anti_right, 8) ||
                std::memcmp(p.union_left, first.union_left, 8) || std::memcmp(p.union_right, first.union_right, 8))
                return -8;
        }
    }
    struct CachedIndex {
        bool valid = false;
        u32 relation = 0;
        u64 version = 0;
        u32 column = 0;
        RangeIndex index;
    };
    std::vector<CachedIndex> cache(n_rules);
    std::vector<Rel> rule_out(n_rules);
    u64 iterations = 0, total_new = 0;
    auto has_delta = [&]() {
        for (u64 i = 0; i < n_relations; ++i)
            if (rels[relations[i]].delta.len() != 0) return true;
        return false;
    };
    while (has_delta()) {
        if (iterations >= max_iterations) {
            *iterations_out = iterations;
            *total_new_out = total_new;
            return -10;
        }
        // RuleRuntime::evaluate for every rule (generic.rs:197-259).
        for (u64 r = 0; r < n_rules; ++r) {
            const oracle_rule_plan& p = rules[r];
            RelState& delta_state = rels[p.delta_input];
            RelState& right_state = rels[p.right_input];
            CachedIndex& ci = cache[r];
            if (!ci.valid || ci.relation != p.right_input || ci.version != right_state.version ||
                ci.column != p.right_key) {
                ci.valid = true;
                ci.relation = p.right_input;
                ci.version = right_state.version;
                ci.column = p.right_key;
                ci.index = build_range_index(right_state.full.c[p.right_key].data(), right_state.full.len());
            }
            Rel joined;
            JoinPlan jp{p.left_key, p.right_key, {p.proj_side[0], p.proj_side[1]}, {p.proj_col[0], p.proj_col[1]}};
            join_op(delta_state.delta, right_state.full, ci.index, jp, threads, &joined);
            distinct_op(joined, p.distinct_cols, threads, &rule_out[r]);
        }
        // TargetRuntime::combine for every target (generic.rs:299-358).
        for (u64 t = 0; t < n_relations; ++t) {
            Rel contributions;
            for (size_t k = 0; k < target_rules[t].size(); ++k) {
                u64 r = target_rules[t][k];
                if (k == 0) {
                    contributions = rule_out[r];
                    continue;
                }
                Rel merged;
                union_op(contributions, rules[r].union_left, rule_out[r], rules[r].union_right, threads, &merged);
                contributions = std::move(merged);
            }
            const oracle_rule_plan& first = rules[target_rules[t][0]];
            RelState& target = rels[relations[t]];
            anti_join_op(contributions, first.anti_left, target.full, first.anti_right, threads, &target.newt);
        }
        // TargetRuntime::apply for every target (generic.rs:360-397).
        for (u64 t = 0; t < n_relations; ++t) {
            const oracle_rule_plan& first = rules[target_rules[t][0]];
            RelState& target = rels[relations[t]];
            Rel merged;
            union_op(target.full, first.union_left, target.newt, first.union_right, threads, &merged);
            target.full = std::move(merged);
            target.delta = std::move(target.newt);
            target.newt.clear();
            target.version += 1;
            total_new += target.delta.len();
        }
        iterations += 1;
    }
    *iterations_out = iterations;
    *total_new_out = total_new;
    return 0;
}

// load_binary_u32 (crates/sparkalog-storage/src/io.rs:72-138) on one thread,
// the way the reference reads a graph: count_rows (a Git LFS pointer header
// anywhere is an error), then populate_columns line by line. Returns 0, or
// 1 (Git LFS pointer), 2 (field count), 3 (invalid u32) with *line (1-based)
// and *column. The columns must hold `capacity` rows.
int oracle_load_binary_u32(const char* text, u64 bytes, uint32_t* first, uint32_t* second, u64 capacity, u64* rows,
                           u64* line_out, int* column_out) {
    auto space = [](char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; };
    static const char kLfs[] = "version https://git-lfs.github.com/spec/v1";
    auto for_lines = [&](auto&& visit) -> int {
        u64 b = 0, index = 0;
        while (b < bytes) {
            u64 e = b;
            while (e < bytes && text[e] != '\n') ++e;
            int rc = visit(b, e, index);
            if (rc) return rc;
            ++index;
            b = e + 1;
        }
        return 0;
    };
    auto trim = [&](u64& b, u64& e) {
        while (b < e && space(text[b])) ++b;
        while (e > b && space(text[e - 1])) --e;
    };
    int rc = for_lines([&](u64 b, u64 e, u64) {
        trim(b, e);
        if (b == e || text[b] == '#' || text[b] == '%') return 0;
        if (e - b == sizeof(kLfs) - 1 && std::memcmp(text + b, kLfs, e - b) == 0) return 1;
        return 0;
    });
    if (rc) {
        *line_out = 0;
        return rc;
    }
    u64 n = 0;
    return for_lines([&](u64 b, u64 e, u64 index) {
        trim(b, e);
        if (b == e || text[b] == '#' || text[b] == '%') return 0;
        u64 fb[2] = {0, 0}, fe[2] = {0, 0};
        int fields = 0;
        for (u64 p = b; p < e;) {
            while (p < e && space(text[p])) ++p;
            if (p == e) break;
            const u64 q = p;
            while (p < e && !space(text[p])) ++p;
            if (fields < 2) {
                fb[fields] = q;
                fe[fields] = p;
            }
            if (++fields > 2) break;
        }
        *line_out = index + 1;
        if (fields != 2) return 2;
        uint32_t v[2];
        for (int c = 0; c < 2; ++c) {
            u64 i = fb[c];
            if (i < fe[c] && text[i] == '+') ++i;
            bool ok = i < fe[c];
            u64 x = 0;
            for (; ok && i < fe[c]; ++i) {
                ok = text[i] >= '0' && text[i] <= '9';
                x = x * 10 + static_cast<u64>(text[i] - '0');
                ok = ok && x <= 0xffffffffull;
            }
            if (!ok) {
                *column_out = c + 1;
                return 3;
            }
            v[c] = static_cast<uint32_t>(x);
        }
        if (n < capacity) {
            first[n] = v[0];
            second[n] = v[1];
        }
        *rows = ++n;
        return 0;
    });
}

// ValueCatalog::intern (crates/sparkalog-datalog/src/catalog.rs:108-117) for
// each value in order, with a hash map as the reference's HashMap.
void oracle_intern_u32(const uint32_t* values, u64 n, uint32_t* ids) {
    std::unordered_map<uint32_t, uint32_t> by_value;
    by_value.reserve(n);
    for (u64 i = 0; i < n; ++i) {
        auto it = by_value.find(values[i]);
        if (it == by_value.end()) it = by_value.emplace(values[i], static_cast<uint32_t>(by_value.size())).first;
        ids[i] = it->second;
    }
}

// GeneralCpu on the transitive-closure program (execute_scc and
// evaluate_clause, crates/sparkalog-datalog/src/general.rs:393-447 and
// :478-536): FULL is an ordered set seeded with the edges, DELTA = FULL; a
// round binds path(x, y) from every DELTA tuple (|DELTA| tests), then tests
// every edge tuple against y (|DELTA| x |edge| tests: the nested loop),
// collects (x, z), and keeps the tuples absent from FULL as the next DELTA.
// Single-threaded, as GeneralCpu is. Stops after max_rounds rounds, or once
// time_cap_s has passed (checked every 64 DELTA tuples, so a sample can end
// inside a round). Reports completed rounds, new tuples of those rounds, the
// tuple tests made and the seconds spent; *converged = 1 if DELTA emptied.
// A test here is a plain compare, where the reference clones a binding per
// tested pair, so times measured here bound GeneralCpu's from below.
int oracle_general_tc(const uint32_t* src, const uint32_t* dst, u64 n, u64 max_rounds, double time_cap_s,
                      u64* rounds_out, u64* new_out, u64* tests_out, double* seconds_out, int* converged_out) {
    const auto start = std::chrono::steady_clock::now();
    auto elapsed = [&] { return std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count(); };
    std::vector<u64> edges(n);
    for (u64 i = 0; i < n; ++i) edges[i] = (static_cast<u64>(src[i]) << 32) | dst[i];
    std::sort(edges.begin(), edges.end());
    edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
    std::vector<uint32_t> edge_first(edges.size()), edge_second(edges.size());
    for (size_t i = 0; i < edges.size(); ++i) {
        edge_first[i] = static_cast<uint32_t>(edges[i] >> 32);
        edge_second[i] = static_cast<uint32_t>(edges[i]);
    }
    std::set<u64> full(edges.begin(), edges.end());
    std::vector<u64> delta(edges.begin(), edges.end());
    u64 rounds = 0, total_new = 0, tests = 0;
    bool capped = false;
    const size_t m = edges.size();
    while (!delta.empty() && rounds < max_rounds && !capped) {
        std::vector<u64> joined;
        for (size_t d = 0; d < delta.size(); ++d) {
            if ((d & 63) == 0 && elapsed() > time_cap_s) {
                capped = true;
                break;
            }
            const u64 x = delta[d] >> 32;
            const uint32_t y = static_cast<uint32_t>(delta[d]);
            tests += 1 + m;
            for (size_t i = 0; i < m; ++i)
                if (edge_first[i] == y) joined.push_back((x << 32) | edge_second[i]);
        }
        if (capped) break;
        std::sort(joined.begin(), joined.end());
        joined.erase(std::unique(joined.begin(), joined.end()), joined.end());
        std::vector<u64> next;
        for (u64 t : joined)
            if (!full.count(t)) next.push_back(t);
        full.insert(next.begin(), next.end());
        total_new += next.size();
        delta.swap(next);
        ++rounds;
    }
    *rounds_out = rounds;
    *new_out = total_new;
    *tests_out = tests;
    *seconds_out = elapsed();
    *converged_out = delta.empty() ? 1 : 0;
    return 0;
}

}  // extern "C"
