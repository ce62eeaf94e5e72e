"""hacapk_b200: B200-native H-matrix matvec and BiCGSTAB engine (host side).

The product is the C ABI in include/hacapk_b200.h, implemented by
libhacapk_b200.so (sm_100a CUDA).  This package holds the ctypes bindings
used by the tests and the benchmark, and the host-side construction of the
leaf lists (libhacapk_build.so).
"""
from . import abi  # noqa: F401
