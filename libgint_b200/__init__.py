"""B200 (sm_100a) exchange-matrix engine behind the libGint C-ABI.

The engine is the native library libgint_b200/lib/libgint_b200.so (C-ABI in include/libgint.h).
`LibGint` mirrors the reference's Fortran/C interface method by method; `workload` generates
the synthetic systems and replays their quartet streams through the C-ABI.
"""
from .capi import LibGint, engine_path, load_engine  # noqa: F401
