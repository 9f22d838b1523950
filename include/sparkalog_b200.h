/*
 * sparkalog_b200 — B200-native (sm_100a) binary recursive operator pipeline.
 *
 * C ABI of libsparkalog_b200.so. Plain pointers and sizes only.
 *
 * Tier A: the reference's own FFI for the pipeline's operators, with the same
 * names, signatures, argument meaning, null-pointer checks and empty-input
 * behaviour as the launchers in crates/sparkalog-execution/native/column_ops.cu
 * (bound from Rust at crates/sparkalog-execution/src/lib.rs:28-169). A build of
 * the reference links this library in place of its libsparkalog_cuda.a.
 * Return values are cudaError_t codes (0 = success); counts are written to
 * device (or managed) memory asynchronously on `stream`.
 *
 * Tier B: a device-resident RelationStore / RecursiveExecutor
 * (crates/sparkalog-recursion/src/generic.rs:16-525) that keeps FULL, DELTA
 * and NEWT on the device as packed 64-bit rows and runs the whole semi-naive
 * loop without copying relations back to the host. Return values are 0 on
 * success, a positive cudaError_t, or a negative SPARKALOG_E_* code;
 * sparkalog_last_error() describes the last failure of the calling thread.
 */
#ifndef SPARKALOG_B200_H
#define SPARKALOG_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define SPARKALOG_API __attribute__((visibility("default")))
#else
#define SPARKALOG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Tier A: reference-compatible operator entry points                        */
/* ------------------------------------------------------------------------ */

/* column_ops.cu:248-250; lib.rs:32. */
SPARKALOG_API int sparkalog_stream_synchronize(void* stream);

/* Scratch size for the join's count stage. column_ops.cu:339-355; lib.rs:59-65. */
SPARKALOG_API int sparkalog_join_u32_temporary_bytes(const uint64_t* counts, uint64_t* offsets, size_t left_rows,
                                                     size_t* temporary_bytes, void* stream);

/* Per left row match counts, their exclusive scan and the total.
 * column_ops.cu:357-401; lib.rs:66-78. */
SPARKALOG_API int sparkalog_join_u32_count(const uint32_t* left_keys, size_t left_rows, const uint32_t* index_keys,
                                           const uint32_t* index_starts, size_t unique_keys, uint64_t* counts,
                                           uint64_t* offsets, uint64_t* total, void* temporary,
                                           size_t temporary_bytes, void* stream);

/* Projected join output, left-row-major, matches in index order.
 * A side value of 0 selects the left row, 1 the right row.
 * column_ops.cu:403-444; lib.rs:79-94. */
SPARKALOG_API int sparkalog_join_u32_emit(const uint32_t* left_keys, size_t left_rows, const uint32_t* index_keys,
                                          const uint32_t* index_starts, const uint32_t* index_rows,
                                          size_t unique_keys, const uint32_t* projection0,
                                          uint32_t projection0_side, const uint32_t* projection1,
                                          uint32_t projection1_side, const uint64_t* offsets, uint32_t* output0,
                                          uint32_t* output1, void* stream);

/* column_ops.cu:446-487; lib.rs:95-102. */
SPARKALOG_API int sparkalog_distinct_u32_temporary_bytes(uint64_t* packed, uint64_t* scratch, uint64_t* unique_rows,
                                                         size_t rows, size_t* temporary_bytes, void* stream);

/* Sort and deduplicate (first, second) pairs; sorted unique output and its
 * u64 count. `packed`/`scratch` (rows u64 each) are the sort's buffers.
 * column_ops.cu:489-549; lib.rs:103-115. */
SPARKALOG_API int sparkalog_distinct_u32(const uint32_t* first, const uint32_t* second, size_t rows,
                                         uint64_t* packed, uint64_t* scratch, uint64_t* unique_rows,
                                         uint32_t* output_first, uint32_t* output_second, void* temporary,
                                         size_t temporary_bytes, void* stream);

/* column_ops.cu:551-574; lib.rs:116-123. */
SPARKALOG_API int sparkalog_anti_join_u32_temporary_bytes(const uint32_t* flags, uint32_t* selected,
                                                          uint32_t* selected_rows, size_t left_rows,
                                                          size_t* temporary_bytes, void* stream);

/* Stable left - right over lexicographically sorted pairs. flags[row] = 1 for
 * kept rows, selected[] = kept row ids, *selected_rows = u32 count.
 * column_ops.cu:576-641; lib.rs:124-139. */
SPARKALOG_API int sparkalog_anti_join_u32(const uint32_t* left_first, const uint32_t* left_second, size_t left_rows,
                                          const uint32_t* right_first, const uint32_t* right_second,
                                          size_t right_rows, uint32_t* flags, uint32_t* selected,
                                          uint32_t* selected_rows, uint32_t* output_first, uint32_t* output_second,
                                          void* temporary, size_t temporary_bytes, void* stream);

/* Filter: output[] = ascending row ids i with compare(input[i], operation,
 * operand), flags[i] = 1 / 0, *count = u32 number of ids. Operation codes:
 * 0 ==, 1 !=, 2 <, 3 <=, 4 >, 5 >=, anything else matches no row.
 * column_ops.cu:252-318; lib.rs:33-52. */
SPARKALOG_API int sparkalog_filter_u32_temporary_bytes(const uint32_t* flags, uint32_t* output, uint32_t* count,
                                                       size_t len, size_t* temporary_bytes, void* stream);
SPARKALOG_API int sparkalog_filter_u32(const uint32_t* input, size_t len, uint32_t operation, uint32_t operand,
                                       uint32_t* flags, uint32_t* output, uint32_t* count, void* temporary,
                                       size_t temporary_bytes, void* stream);

/* output[i] = i % modulus. column_ops.cu:320-336; lib.rs:53-58. */
SPARKALOG_API int sparkalog_fill_mod_u32(uint32_t* output, size_t len, uint32_t modulus, void* stream);

/* data[i] += 1 (the reference's workspace smoke test). column_ops.cu:231-246;
 * lib.rs:31. */
SPARKALOG_API int sparkalog_add_one_i32(int32_t* data, size_t len, void* stream);

/* column_ops.cu:643-690; lib.rs:140-150. */
SPARKALOG_API int sparkalog_union_u32_temporary_bytes(const uint64_t* left, size_t left_rows, const uint64_t* right,
                                                      size_t right_rows, uint64_t* merged, uint64_t* unique,
                                                      uint64_t* unique_rows, size_t* temporary_bytes, void* stream);

/* Merge two sorted pair lists and deduplicate; sorted output and u64 count.
 * column_ops.cu:692-775; lib.rs:151-168. */
SPARKALOG_API int sparkalog_union_u32(const uint32_t* left_first, const uint32_t* left_second, size_t left_rows,
                                      const uint32_t* right_first, const uint32_t* right_second, size_t right_rows,
                                      uint64_t* left, uint64_t* right, uint64_t* merged, uint64_t* unique,
                                      uint64_t* unique_rows, uint32_t* output_first, uint32_t* output_second,
                                      void* temporary, size_t temporary_bytes, void* stream);

/* sparkalog_anti_join_u32 without the `temporary` buffer, for callers that
 * cannot allocate device memory (a runtime whose HBM budget is fully handed to
 * relation buffers, a binding with no device allocator, a pipeline that must
 * not take cudaMalloc's implicit synchronisation). No counterpart in the
 * reference. The kernel's scratch is a fixed static array in the library
 * (about 513 KiB per device, kept until exit), shared by every call on a
 * device: calls that overlap on the GPU race, so order them on one stream.
 * left_rows above SPARKALOG_ANTI_JOIN_NO_ALLOC_MAX_LEFT_ROWS is rejected with
 * cudaErrorInvalidValue. The first call on a device looks up the array's
 * address; make it before any stream capture. Allocates nothing. */
#define SPARKALOG_ANTI_JOIN_NO_ALLOC_MAX_LEFT_ROWS (1ull << 27)
SPARKALOG_API int sparkalog_anti_join_u32_no_alloc(const uint32_t* left_first, const uint32_t* left_second,
                                                   size_t left_rows, const uint32_t* right_first,
                                                   const uint32_t* right_second, size_t right_rows, uint32_t* flags,
                                                   uint32_t* selected, uint32_t* selected_rows,
                                                   uint32_t* output_first, uint32_t* output_second, void* stream);

/* Error bits of sparkalog_anti_join_u32_no_alloc on the current device (a
 * look-back wait that hit its spin cap), accumulated over every call since
 * the last reset; reset != 0 clears them. The bits live in a static device
 * word that the entry point's per-call clearing never touches, and this
 * getter reads it with a synchronous symbol copy, so it allocates nothing.
 * Call it after the stream of the calls it covers has finished. No
 * counterpart in the reference. */
SPARKALOG_API int sparkalog_anti_join_u32_no_alloc_error(uint32_t* bits, int reset);

/* Asynchronous error bits of this device's allocating Tier A kernels (a
 * decoupled look-back that hit its spin cap); the no-alloc anti-join reports
 * through sparkalog_anti_join_u32_no_alloc_error instead. No counterpart in
 * the reference, whose CUB kernels have no such wait. reset != 0 clears the
 * bits. */
SPARKALOG_API int sparkalog_b200_device_error(uint32_t* bits, int reset);

/* ------------------------------------------------------------------------ */
/* Tier B: device-resident store and executor                                */
/* ------------------------------------------------------------------------ */

enum {
    SPARKALOG_E_MISSING = -1,              /* RelationStoreError::Missing */
    SPARKALOG_E_DUPLICATE = -2,            /* RelationStoreError::Duplicate */
    SPARKALOG_E_NOT_RECURSIVE = -3,        /* RelationStoreError::NotRecursive */
    SPARKALOG_E_EMPTY_SCC = -4,            /* GenericExecutionError::EmptyScc */
    SPARKALOG_E_DUPLICATE_SCC_RELATION = -5,
    SPARKALOG_E_DELTA_OUTSIDE_SCC = -6,
    SPARKALOG_E_TARGET_OUTSIDE_SCC = -7,
    SPARKALOG_E_INCOMPATIBLE_TARGET_PLANS = -8,
    SPARKALOG_E_MISSING_RULE_TARGET = -9,
    SPARKALOG_E_ITERATION_LIMIT = -10,
    SPARKALOG_E_TOO_MANY_ROWS = -11,       /* execution::Error::TooManyRows */
    SPARKALOG_E_MISSING_COLUMN = -12,      /* MissingPlanColumn / MissingColumn */
    SPARKALOG_E_DEVICE_FAULT = -20,        /* a kernel reported an error bit */
    SPARKALOG_E_INVALID_ARGUMENT = -21,
    SPARKALOG_E_UNSORTED_FULL = -22,       /* FULL must be sorted for anti-join/union */
    SPARKALOG_E_LOAD = -23,                /* storage::LoadError; details in sparkalog_load_error */
};

/* JoinInput: 0 = Left (the DELTA side), 1 = Right. */
typedef struct sparkalog_rule_plan {
    uint32_t target;          /* RecursiveRulePlan::target, relational/src/lib.rs:74-82 */
    uint32_t delta_input;
    uint32_t right_input;
    uint32_t left_key;        /* BinaryEqualityJoin, relational/src/lib.rs:46-50 */
    uint32_t right_key;
    uint32_t proj_side[2];
    uint32_t proj_col[2];
    uint32_t distinct_cols[2];   /* BinaryDistinct */
    uint32_t anti_left[2];       /* SortedBinaryAntiJoin */
    uint32_t anti_right[2];
    uint32_t union_left[2];      /* SortedBinaryUnion */
    uint32_t union_right[2];
} sparkalog_rule_plan;

/* SccSummary, recursion/src/generic.rs:536-542 (placements omitted: every
 * operator runs on the GPU). relation_rows has one entry per SCC relation, in
 * plan order; the caller provides room for relation_count entries. */
typedef struct sparkalog_scc_summary {
    uint64_t iterations;
    uint64_t total_new_rows;
    uint64_t relation_count;
    uint32_t* relation_ids;
    uint64_t* relation_rows;
} sparkalog_scc_summary;

typedef struct sparkalog_store sparkalog_store;
typedef struct sparkalog_executor sparkalog_executor;

/* Location of caller buffers: host memory (pageable or pinned) or device. */
enum { SPARKALOG_HOST = 0, SPARKALOG_DEVICE = 1 };
/* Relation versions, RelationVersion (relational/src/lib.rs:10-14). */
enum { SPARKALOG_FULL = 0, SPARKALOG_DELTA = 1 };

/* RelationStore::new, generic.rs:29-34. Work runs on `stream` (0 = legacy). */
SPARKALOG_API int sparkalog_store_create(void* stream, sparkalog_store** out);
SPARKALOG_API void sparkalog_store_destroy(sparkalog_store* store);

/* RelationStore::insert_static, generic.rs:36-51. */
SPARKALOG_API int sparkalog_store_insert_static(sparkalog_store* store, uint32_t id, const uint32_t* first,
                                                const uint32_t* second, size_t rows, int location);

/* RelationStore::insert_recursive, generic.rs:53-79. */
SPARKALOG_API int sparkalog_store_insert_recursive(sparkalog_store* store, uint32_t id, const uint32_t* full_first,
                                                   const uint32_t* full_second, size_t full_rows,
                                                   const uint32_t* delta_first, const uint32_t* delta_second,
                                                   size_t delta_rows, int location);

/* Row count of FULL or DELTA (RelationStore::full/delta, generic.rs:81-92). */
SPARKALOG_API int sparkalog_store_rows(sparkalog_store* store, uint32_t id, int version, size_t* rows);

/* Copies FULL or DELTA out as two u32 columns (sorted for FULL of recursive
 * relations after a run, as the reference's RelationBuffer is). */
SPARKALOG_API int sparkalog_store_read(sparkalog_store* store, uint32_t id, int version, uint32_t* first,
                                       uint32_t* second, int location);

/* Stratified negation over completed relations: stores
 *   out(x, y) :- left(x, y), !right(x, y).
 * as a new static relation `out_id` holding the sorted, deduplicated rows of
 * FULL(left) that are absent from FULL(right). This is the GeneralCpu
 * evaluation of such a clause (general.rs:478-551: positive atom scan, then a
 * negated atom checked against the completed FULL of an earlier stratum),
 * which outputs a BTreeSet (sorted, unique); the reference's binary lowering
 * rejects the clause (subset.rs:56-63), so this extends the device path. */
SPARKALOG_API int sparkalog_store_anti_join(sparkalog_store* store, uint32_t left_id, uint32_t right_id,
                                            uint32_t out_id);

/* ---- Non-recursive clauses on the device ----
 * GeneralCpu evaluates every non-recursive clause of a stratified program
 * with nested loops (crates/sparkalog-datalog/src/general.rs:478-551:
 * positive atoms matched term by term, constants compared, negated atoms
 * checked against a completed relation), and the binary lowering rejects
 * such clauses (subset.rs:56-63). These two operations, with
 * sparkalog_store_anti_join, evaluate the binary ones on the GPU; each
 * stores its result as a new static relation (sorted, deduplicated: the
 * BTreeSet GeneralCpu builds) and fails with SPARKALOG_E_DUPLICATE when
 * out_id exists. */

/* Merges the levels of relation id's FULL into one sorted run on the device
 * (the single sorted FULL that TargetRuntime::apply keeps after every round,
 * crates/sparkalog-recursion/src/generic.rs:360-397; here FULL is kept as
 * disjoint sorted levels and merged on demand). Reads merge implicitly; this
 * call does it ahead of them. Synchronises the store's stream. */
SPARKALOG_API int sparkalog_store_compact(sparkalog_store* store, uint32_t id);

/* Removes relation id from the store and frees its device memory (stream-
 * ordered). */
SPARKALOG_API int sparkalog_store_drop(sparkalog_store* store, uint32_t id);

/* out(c0, c1) :- in(x, y), where(x, y): where_mask bit 0 keeps rows with
 * x == where_value[0], bit 1 rows with y == where_value[1], bit 2 rows with
 * x == y (an atom with constants or a repeated variable, the equality
 * predicate of the reference's filter, column_ops.cu:20-43); out column k
 * is x (out_source[k] = 0), y (1) or the constant out_value[k] (2). */
typedef struct sparkalog_select {
    uint32_t where_mask;
    uint32_t where_value[2];
    uint32_t out_source[2];
    uint32_t out_value[2];
} sparkalog_select;
SPARKALOG_API int sparkalog_store_select(sparkalog_store* store, uint32_t in_id, const sparkalog_select* spec,
                                         uint32_t out_id, size_t* rows);

/* out(p0, p1) :- left(..), right(..) joined on left's column left_key equal
 * to right's column right_key; output column k is column proj_col[k] of the
 * left (proj_side[k] = 0) or right (1) row (BinaryEqualityJoin,
 * relational/src/lib.rs:46-50), deduplicated. */
SPARKALOG_API int sparkalog_store_join(sparkalog_store* store, uint32_t left_id, uint32_t right_id,
                                       uint32_t left_key, uint32_t right_key, const uint32_t* proj_side,
                                       const uint32_t* proj_col, uint32_t out_id, size_t* rows);

/* RecursiveExecutor::compile, generic.rs:407-470. */
SPARKALOG_API int sparkalog_executor_compile(sparkalog_store* store, const uint32_t* relations,
                                             size_t relation_count, const sparkalog_rule_plan* rules,
                                             size_t rule_count, sparkalog_executor** out);
SPARKALOG_API void sparkalog_executor_destroy(sparkalog_executor* executor);

/* RecursiveExecutor::run, generic.rs:472-516. */
SPARKALOG_API int sparkalog_executor_run(sparkalog_executor* executor, sparkalog_store* store,
                                         size_t max_iterations, sparkalog_scc_summary* summary);

/* ---- Serving: relations stay resident while requests join and leave ----
 * No counterparts in the reference, whose Database re-runs every fixpoint
 * from scratch after an insert (database.rs:82-112). Requests are kept apart
 * by a tag in the high bits of both columns (a "segment": first >> shift). */

/* Runs at most `rounds` rounds of the loop (no error at the limit);
 * *converged = 1 when every DELTA of the SCC is empty afterwards. */
SPARKALOG_API int sparkalog_executor_step(sparkalog_executor* executor, sparkalog_store* store, size_t rounds,
                                          sparkalog_scc_summary* summary, int* converged);

/* FULL(id) u= rows, and for a recursive relation also DELTA(id) u= (rows not
 * already in FULL), so the next round derives from them: new facts join a
 * resident fixpoint. Rows may be unsorted and may repeat. */
SPARKALOG_API int sparkalog_store_append(sparkalog_store* store, uint32_t id, const uint32_t* first,
                                         const uint32_t* second, size_t rows, int location);

/* Copies the rows of FULL(id) whose first >> shift == segment, sorted, into
 * (first, second); with first == NULL only *rows is set. */
SPARKALOG_API int sparkalog_store_extract_segment(sparkalog_store* store, uint32_t id, uint32_t shift,
                                                  uint32_t segment, uint32_t* first, uint32_t* second,
                                                  int location, size_t* rows);

/* As sparkalog_store_extract_segment, with the segment tag (the bits at and
 * above `shift`) cleared on the device from the first column and, when
 * clear_second is non-zero, from the second column too: a tagged request's
 * rows come back in its own node ids without a host pass over them. */
SPARKALOG_API int sparkalog_store_extract_segment_untagged(sparkalog_store* store, uint32_t id, uint32_t shift,
                                                           uint32_t segment, int clear_second, uint32_t* first,
                                                           uint32_t* second, int location, size_t* rows);

/* Removes every row whose first >> shift is one of `segments` from FULL and
 * DELTA of relation id (a completed request's rows, freeing its tag). */
SPARKALOG_API int sparkalog_store_remove_segments(sparkalog_store* store, uint32_t id, uint32_t shift,
                                                  const uint32_t* segments, size_t count);

/* Per-kernel-class statistics of an executor, measured with CUDA events on
 * the executor's stream while profiling is enabled. No counterpart in the
 * reference (which has no tracing); used to report achieved HBM bandwidth.
 * bytes[] are algorithmic bytes: each input row read once, each output row
 * written once (8 bytes per packed pair). launches[] counts every kernel of
 * the class; total_launches counts every kernel the executor launched. */
enum {
    SPARKALOG_K_JOIN = 0,        /* fused count/scan/emit join */
    SPARKALOG_K_SORT_HIST = 1,   /* radix histogram + plan */
    SPARKALOG_K_SORT_PASS = 2,   /* radix scatter passes (active ones) */
    SPARKALOG_K_ANTI_JOIN = 3,   /* unique + anti-join against the FULL levels */
    SPARKALOG_K_MERGE = 4,       /* merge of NEWT / levels */
    SPARKALOG_K_INDEX = 5,       /* right-relation index build */
    SPARKALOG_K_FUSED = 6,       /* fused join + distinct (then the anti-join) */
    SPARKALOG_K_CLASSES = 8
};
typedef struct sparkalog_kernel_stats {
    uint64_t launches[SPARKALOG_K_CLASSES];
    double milliseconds[SPARKALOG_K_CLASSES];
    double bytes[SPARKALOG_K_CLASSES];
    uint64_t total_launches;
    uint64_t rounds;
} sparkalog_kernel_stats;

/* Per-segment activity for batched runs, where independent instances share
 * one SCC and a row's segment (instance) is its first column >> shift. After
 * each round the executor records, for every segment that gained NEWT rows,
 * round_index + 1 and the number of rows. An instance whose seed DELTA was
 * non-empty then ran last_active_round[s] + 1 rounds of its own fixpoint (the
 * count RecursiveExecutor::run would report for it alone). No counterpart in
 * the reference, which runs one instance at a time. */
SPARKALOG_API int sparkalog_executor_track_segments(sparkalog_executor* executor, uint32_t shift, uint32_t count);
SPARKALOG_API int sparkalog_executor_segment_stats(sparkalog_executor* executor, uint32_t* last_active_round,
                                                   uint64_t* new_rows);

SPARKALOG_API int sparkalog_executor_set_profiling(sparkalog_executor* executor, int enable);

/* Enables (default) or disables the fused join + distinct kernel for rules
 * whose join output starts with DELTA's first column. Disabled, every round
 * runs the general join, radix sort and anti-join; results are identical. No
 * counterpart in the reference. */
SPARKALOG_API int sparkalog_executor_set_fused(sparkalog_executor* executor, int enable);

/* Enables or disables (default) FULL's hash set for recursive relations. With
 * it, the anti-join of a round's candidates against FULL is one hash probe per
 * candidate instead of a search of each sorted level; the set is built from
 * the levels on first use (128 bytes of slots per row of FULL, only when the
 * device has that much free memory) and takes every round's NEWT. Results are
 * identical either way; on sorted candidates the level search keeps cache
 * locality that hashing gives up, so the set is opt-in. No counterpart in the
 * reference. */
SPARKALOG_API int sparkalog_executor_set_member_set(sparkalog_executor* executor, int enable);

/* Enables (default) or disables device-driven rounds: while a single
 * transitive-closure-shaped target's rounds stay within the group-searched
 * anti-join's candidate bound, the executor runs them as a CUDA graph whose
 * WHILE node repeats one round (fused join + order, anti-join, merge into
 * TAIL, and a round-end kernel that applies the round and tests convergence
 * on the device), with one host synchronisation per launch instead of one
 * per round. Results, iteration counts and the round trace are identical
 * either way. Profiling (sparkalog_executor_set_profiling) runs every round
 * from the host. The reference runs every round from the host
 * (generic.rs:472-516). */
SPARKALOG_API int sparkalog_executor_set_device_loop(sparkalog_executor* executor, int enable);
/* Graph launches of the device-driven loop and the rounds they applied, over
 * the executor's lifetime. */
SPARKALOG_API int sparkalog_executor_device_loop_stats(sparkalog_executor* executor, uint64_t* launches,
                                                       uint64_t* rounds);

/* Launch shapes and thresholds of the executor's kernels, chosen per device
 * by the autotuner (sparkalog_b200/autotune.py) on a short calibration
 * fixpoint. Every value gives identical results; only speed changes. The
 * reference fixes its analogue at compile time for one GPU
 * (crates/sparkalog-execution/src/placement.rs:34-38). */
typedef struct sparkalog_tuning {
    uint32_t dir_rows_log2;       /* 2^k rows per bucket of a FULL level's directory (0-10) */
    uint32_t group_lanes;         /* lanes that search one candidate together: 4, 8 or 16 */
    uint64_t group_candidates;    /* candidate bound up to which the group search runs */
    uint64_t sparse_candidates;   /* ... up to which the per-thread search runs; above: staged slices */
    uint32_t fused_rows_cap;      /* DELTA rows per fused join tile, at most (64-768) */
    uint32_t merge_items;         /* rows per thread of a merge tile: 7, 11 or 15 */
    uint32_t level_ratio;         /* a FULL level merges down past 1/ratio of the next (2-64) */
    uint32_t levels;              /* sorted runs that hold a recursive FULL (2-4) */
    uint32_t bloom_bits;          /* bits per FULL row of the anti-join's Bloom filter; 0: no filter (0, 4-32) */
    uint32_t merge_anti_ratio;    /* the merge-form anti-join runs while FULL rows <= ratio x the round's
                                     estimated candidates; 0: never (0-1024) */
    uint32_t sparse_items;        /* candidates per thread of the per-thread search: 2, 3 or 4 */
    uint32_t compact_index;       /* 1: the fused join probes 4-bit match counts and one word per key
                                     instead of CSR offsets; 0: offsets */
} sparkalog_tuning;

/* The built-in defaults (measured on a B200). */
SPARKALOG_API int sparkalog_tuning_defaults(sparkalog_tuning* out);
/* Replaces the executor's tuning; SPARKALOG_E_INVALID_ARGUMENT for a value
 * outside the ranges above. Takes effect at the next run or step. */
SPARKALOG_API int sparkalog_executor_set_tuning(sparkalog_executor* executor, const sparkalog_tuning* tuning);
SPARKALOG_API int sparkalog_executor_get_tuning(sparkalog_executor* executor, sparkalog_tuning* out);

/* Device value catalog: ValueCatalog (crates/sparkalog-datalog/src/
 * catalog.rs:98-127) for u32 values. intern gives every value of the batch
 * its dense id, new values numbered by first appearance after the catalog's
 * current size (as interning the values one by one in order would);
 * decode maps ids back to values (Database::query's decode, database.rs:
 * 179-213) and fails with SPARKALOG_E_INVALID_ARGUMENT on an id outside the
 * catalog. `location` applies to both the input and the output array. */
typedef struct sparkalog_catalog sparkalog_catalog;
SPARKALOG_API int sparkalog_catalog_create(void* stream, sparkalog_catalog** out);
SPARKALOG_API void sparkalog_catalog_destroy(sparkalog_catalog* catalog);
SPARKALOG_API int sparkalog_catalog_intern_u32(sparkalog_catalog* catalog, const uint32_t* values, size_t count,
                                               int location, uint32_t* ids, size_t* catalog_size);
SPARKALOG_API int sparkalog_catalog_decode_u32(sparkalog_catalog* catalog, const uint32_t* ids, size_t count,
                                               int location, uint32_t* values);
SPARKALOG_API int sparkalog_catalog_size(sparkalog_catalog* catalog, size_t* size);

/* storage::LoadError (crates/sparkalog-storage/src/io.rs:7-20). */
enum {
    SPARKALOG_LOAD_OK = 0,
    SPARKALOG_LOAD_GIT_LFS_POINTER = 1,
    SPARKALOG_LOAD_INVALID_FIELD_COUNT = 2,
    SPARKALOG_LOAD_INVALID_U32 = 3,
    /* DelimitedError (crates/sparkalog-datalog/src/ingest.rs:43-120), by message */
    SPARKALOG_LOAD_UNTERMINATED_QUOTE = 4,   /* "unterminated quoted field" */
    SPARKALOG_LOAD_EXPECTED_DELIMITER = 5,   /* "expected delimiter after quoted field" */
    SPARKALOG_LOAD_EMPTY_FIELD = 6,          /* "empty fields are not values" */
    SPARKALOG_LOAD_TRAILING_DELIMITER = 7,   /* "record ends with an empty field" */
    /* DatabaseError::Arity (crates/sparkalog-datalog/src/database.rs:98-104); column = values in the row */
    SPARKALOG_LOAD_ARITY = 8,
    /* a String or Symbol value where this entry point loads u32 relations */
    SPARKALOG_LOAD_NOT_U32 = 9
};
typedef struct sparkalog_load_error {
    int32_t kind;           /* SPARKALOG_LOAD_* */
    uint32_t column;        /* 1 or 2 for SPARKALOG_LOAD_INVALID_U32; the 1-based byte column for 4-7 and 9 */
    uint64_t line;          /* 1-based line number */
    uint64_t field_offset;  /* byte offset of the offending field in `text` */
    uint64_t field_length;  /* its length in bytes */
} sparkalog_load_error;

/* load_binary_u32 (crates/sparkalog-storage/src/io.rs:72-138) parsed on the
 * GPU and inserted as relation `id` (static, or recursive with FULL = DELTA
 * when `recursive` != 0). `text` holds `bytes` bytes of whitespace-separated
 * u32 pairs, one per line, in host or device memory (`location`); empty
 * lines and lines starting with '#' or '%' are skipped. On a malformed input
 * nothing is inserted, the call returns SPARKALOG_E_LOAD and *error (when not
 * null) names the first failing line as the reference would: a Git LFS
 * pointer anywhere first, then the lowest line with a wrong field count or a
 * field that is not a u32. Whitespace is ASCII whitespace. *rows receives the
 * number of rows read; they are inserted as read (in file order, duplicates
 * kept), as inserting load_binary_u32's relation would. */
SPARKALOG_API int sparkalog_store_load_binary_u32(sparkalog_store* store, uint32_t id, const char* text, size_t bytes,
                                                  int location, int recursive, size_t* rows,
                                                  sparkalog_load_error* error);

/* Database::load_delimited (crates/sparkalog-datalog/src/database.rs:165-177,
 * parse_delimited_parallel in crates/sparkalog-datalog/src/ingest.rs:20-120)
 * for a binary relation of u32 values, parsed on the GPU and inserted as
 * relation `id` like sparkalog_store_load_binary_u32. Lines are split at
 * '\n' (a '\r' before it dropped); with has_header the first line is
 * skipped; lines that trim to nothing are skipped; every other line is a
 * record split at `delimiter`: a field starting with '"' is a quoted string,
 * any other is trimmed (Unicode whitespace) and must parse as a u32. A
 * whitespace delimiter other than tab is SPARKALOG_E_INVALID_ARGUMENT. On a
 * syntax error anywhere (kinds 4-7, the first failing line) nothing is
 * inserted and the call returns SPARKALOG_E_LOAD; otherwise the first line
 * whose record is not two u32 values reports SPARKALOG_LOAD_ARITY or
 * SPARKALOG_LOAD_NOT_U32 (the reference would intern strings and symbols;
 * this entry point loads u32 relations only). Values are not interned here:
 * sparkalog_catalog_intern_u32 over the rows gives Database's value ids. */
SPARKALOG_API int sparkalog_store_load_delimited_u32(sparkalog_store* store, uint32_t id, const char* text,
                                                     size_t bytes, int location, unsigned char delimiter,
                                                     int has_header, int recursive, size_t* rows,
                                                     sparkalog_load_error* error);
/* Database::load_delimited (database.rs:165-177 over parse_delimited_parallel,
 * ingest.rs:20-120) for a binary relation of any values: U32, String (a
 * quoted field, '""' a quote) and Symbol (any other field that is not a
 * u32), parsed on the GPU, every value interned into `catalog` in row order
 * as Database::insert interns them (ValueCatalog::intern, catalog.rs:
 * 108-117: String, Symbol and U32 are distinct values), and the rows of
 * value ids inserted as relation `id`. Errors as for
 * sparkalog_store_load_delimited_u32, except that any two values make a
 * row (a row of another length reports SPARKALOG_LOAD_ARITY). Strings and
 * symbols are interned by a 62-bit key of their bytes and every value is
 * compared byte for byte with the value already holding its key, so a key
 * shared by two different values fails with SPARKALOG_E_DEVICE_FAULT (it
 * never merges them); a value may be at most 16 MiB - 1 bytes. The catalog's
 * U32 entry points still work on the same catalog; decode_u32 fails on the
 * id of a String or Symbol. */
SPARKALOG_API int sparkalog_store_load_delimited_values(sparkalog_store* store, sparkalog_catalog* catalog,
                                                        uint32_t id, const char* text, size_t bytes, int location,
                                                        unsigned char delimiter, int has_header, int recursive,
                                                        size_t* rows, sparkalog_load_error* error);

/* The catalog's values in id order, into host memory (Database::query's
 * decode, database.rs:179-213): kinds[i] 0 U32, 1 String, 2 Symbol;
 * numbers[i] a U32's value; a String's or Symbol's text is
 * bytes[offsets[i] .. offsets[i + 1]) (a String without its quotes and
 * with '""' undone). kinds, numbers and offsets (size + 1 entries) and
 * bytes may be null; *bytes_used is always set, so a first call with a null
 * `bytes` sizes the buffer. */
SPARKALOG_API int sparkalog_catalog_export(sparkalog_catalog* catalog, uint32_t* kinds, uint32_t* numbers,
                                           uint64_t* offsets, unsigned char* bytes, size_t bytes_capacity,
                                           size_t* bytes_used);

SPARKALOG_API int sparkalog_executor_stats(sparkalog_executor* executor, sparkalog_kernel_stats* out, int reset);

/* Per-round trace of an executor (the operator cardinalities of each round,
 * summed over the SCC's targets): the figures the reference's benchmark CSVs
 * report per operator. No counterpart in the reference's ABI. */
typedef struct sparkalog_round_trace {
    uint64_t round;        /* 1-based round number within the executor's lifetime */
    uint64_t delta_rows;   /* DELTA rows joined, over all rules */
    uint64_t join_rows;    /* BinaryEqualityJoin output rows */
    uint64_t unique_rows;  /* BinaryDistinct output rows (distinct join rows) */
    uint64_t new_rows;     /* SortedBinaryAntiJoin output rows (NEWT) */
    uint64_t full_rows;    /* FULL rows after the round (SortedBinaryUnion output) */
} sparkalog_round_trace;

/* Copies up to `capacity` recorded rounds (oldest first) to `out` (which may
 * be null when capacity is 0) and sets *count to the number recorded; with
 * reset != 0 the record is cleared afterwards. */
SPARKALOG_API int sparkalog_executor_trace(sparkalog_executor* executor, sparkalog_round_trace* out,
                                           size_t capacity, size_t* count, int reset);

/* Grows the current device's stream-ordered memory pool to at least `bytes`
 * and keeps it (relations are allocated from it), so a long-running process
 * does not pay for pool growth inside its first large requests. */
SPARKALOG_API int sparkalog_reserve_device_memory(size_t bytes, void* stream);

/* Thread-local description of the last failure. */
SPARKALOG_API const char* sparkalog_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* SPARKALOG_B200_H */
