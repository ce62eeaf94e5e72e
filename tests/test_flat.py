"""CPU check of the flat drop-in solver's host loop (hbx_flat.cpp,
HACApK_SOLVER.c:254-417 restated): compiled here on its own and driven with
the oracle matvec, it must retrace the oracle BiCGSTAB."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

SRC = os.path.join(ROOT, "hacapk-magma_b200", "csrc", "hbx_flat.cpp")
LIB = os.path.join(ROOT, "tests", "emu", "_build", "libflat.so")
MV = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double))


@pytest.fixture(scope="module")
def flat(build_libs):
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-o", LIB, SRC], check=True)
    lib = C.CDLL(LIB)
    lib.hbx_test_flat_bicgstab.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double,
                                           C.c_int, MV, C.c_void_p]
    return lib


@pytest.mark.parametrize("level", [3, 4])
def test_flat_loop_retraces_oracle(flat, level):
    import oracle
    from hacapk_b200 import configs
    H, b = configs.c1(level)
    n = H.nd

    def mv(ctx, x, y):
        xa = np.ctypeslib.as_array(x, shape=(n,)).copy()
        np.ctypeslib.as_array(y, shape=(n,))[:] = oracle.matvec(H.st, xa)
        return 0

    cb = MV(mv)
    u = np.zeros(n)
    steps = flat.hbx_test_flat_bicgstab(n, u.ctypes.data_as(C.POINTER(C.c_double)),
                                        b.ctypes.data_as(C.POINTER(C.c_double)), 1e-8, 1000, cb, None)
    u_ref, n_ref, _, _ = oracle.bicgstab(H.st, b, tol=1e-8, max_iter=1000, kind="restated")
    assert steps == n_ref
    assert np.array_equal(u, u_ref)
