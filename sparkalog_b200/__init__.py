"""sparkalog_b200: a B200-native (sm_100a) implementation of sparkalog's binary
recursive operator pipeline (the semi-naive fixpoint over u32 column pairs).

The work runs in ``lib/libsparkalog_b200.so`` (hand-written CUDA kernels plus
a C++ device-resident executor behind the C ABI of include/sparkalog_b200.h).
This package is the host-side mirror of the reference's Rust API for that
path:

* :mod:`sparkalog_b200.relational` — plan types (sparkalog-relational);
* :mod:`sparkalog_b200.execution` — operators through the reference's own
  operator ABI (sparkalog-execution's CUDA path);
* :mod:`sparkalog_b200.recursion` — RelationStore / RecursiveExecutor
  (sparkalog-recursion), device resident;
* :mod:`sparkalog_b200.datalog` — execute_binary (sparkalog-datalog's
  BinaryHybrid backend);
* :mod:`sparkalog_b200.generators` — seeded synthetic workloads.
"""

from . import _native

__all__ = ["load_library"]


def load_library():
    """Loads the CUDA library (raises if it has not been built)."""
    return _native.load()
