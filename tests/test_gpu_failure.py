"""Failure paths of the engine, exercised without faulting or hanging a GPU
(every device wait is bounded; the failures are made on purpose through the
host-side test hooks of include/hacapk_b200.h or through inputs):

  * a grid barrier that cannot complete: the launch's bounded waits expire
    after HBX_TIMEOUT_MS, hbx_sync reports HBX_ERR_TIMEOUT, and the engine
    gives a correct product on the next call;
  * NaN or Inf in b or x0: HBX_ERR_NONFINITE from the GPU solver (first
    step's stop test) and from the flat drop-in entry (host check), where
    the reference would iterate on NaN;
  * BiCGSTAB breakdown (r^.Ap = 0: a skew-symmetric operator and a unit
    right-hand side, all products exact): HBX_ERR_BREAKDOWN, u left at the
    last completed step; the reference divides by zero unchecked
    (HACApK_SOLVER.c:650, :694);
  * a device allocation that fails: hbx_create returns HBX_ERR_NOMEM,
    releases what it allocated, and the next create works; the reference
    exit(0)s (HACApK_BATCH_SORT.c:203-206)."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import sphere

pytestmark = pytest.mark.gpu


def test_expired_grid_barrier_reports_timeout_and_engine_recovers(gpu, build_libs, monkeypatch):
    import oracle
    from hacapk_b200.engine import Engine, HbxError
    monkeypatch.setenv("HBX_TIMEOUT_MS", "100")
    H = sphere(3)
    E = Engine(H.st, H.nd)
    x = np.random.default_rng(1).standard_normal(H.nd)
    assert E.lib.hbx_debug_stall_next_barrier(E._h) == 0
    with pytest.raises(HbxError) as ei:
        E.matvec_host(x)
    assert ei.value.status == 4
    assert "bounded device wait" in str(ei.value)
    y, _, _ = E.matvec_host(x)  # the next call works
    ref = oracle.matvec(H.st, x)
    assert np.abs(y - ref).max() / np.abs(ref).max() <= 1e-13
    E.close()


def test_nonfinite_inputs_are_rejected(gpu, build_libs):
    from hacapk_b200 import abi, configs
    from hacapk_b200.engine import Engine
    from test_gpu_bicgstab import _control
    H, b = configs.c1(3)
    E = Engine(H.st, H.nd)
    for bad in (np.nan, np.inf):
        bb = b.copy()
        bb[17] = bad
        u, info = E.bicgstab_host(bb, check=False)
        assert info["status"] == 7 and info["iterations"] == 0
        u0 = np.zeros(H.nd)
        u0[5] = bad
        u, info = E.bicgstab_host(b, u0=u0, check=False)
        assert info["status"] == 7 and info["iterations"] == 0
    u, info = E.bicgstab_host(b)  # still usable
    assert info["status"] == 0
    E.close()
    lib = abi.engine_lib()
    ctl, buf = _control()
    bb = b.copy()
    bb[3] = np.nan
    u = np.zeros(H.nd)
    nd, nstp, lrtrn = C.c_int(H.nd), C.c_int(-1), C.c_int(-1)
    lib.c_hacapk_bicgstab_cax_lfmtx_flat_(H.st, C.byref(ctl), abi.dptr(u), abi.dptr(bb), ctl.param, C.byref(nd),
                                          C.byref(nstp), C.byref(lrtrn))
    assert lrtrn.value == 7 and nstp.value == 0


def _skew(nd=64):
    """One dense leaf: A[2k, 2k+1] = 1, A[2k+1, 2k] = -1 (skew-symmetric, so
    x^T A x = 0 for every x; with b = e_0 every product and dot is exact)."""
    import test_plan as tp
    A = np.zeros((nd, nd))
    for k in range(0, nd, 2):
        A[k, k + 1], A[k + 1, k] = 1.0, -1.0
    P, keep = tp._custom([(2, 0, 1, nd, 1, nd, A.reshape(-1))], nd)
    return P, keep, A


def test_breakdown_is_reported(gpu, build_libs):
    from hacapk_b200 import abi
    from hacapk_b200.engine import Engine
    from test_gpu_bicgstab import _control
    P, keep, A = _skew()
    nd = A.shape[0]
    E = Engine(C.pointer(P), nd)
    b = np.zeros(nd)
    b[0] = 1.0
    u, info = E.bicgstab_host(b, check=False)
    assert info["status"] == 5
    assert np.all(np.isfinite(u))
    E.close()
    lib = abi.engine_lib()
    ctl, buf = _control()
    u = np.zeros(nd)
    n_, nstp, lrtrn = C.c_int(nd), C.c_int(-1), C.c_int(-1)
    lib.c_hacapk_bicgstab_cax_lfmtx_flat_(C.pointer(P), C.byref(ctl), abi.dptr(u), abi.dptr(b), ctl.param,
                                          C.byref(n_), C.byref(nstp), C.byref(lrtrn))
    assert lrtrn.value == 5 and np.all(np.isfinite(u))


def test_failed_device_allocation_reports_nomem(gpu, build_libs):
    from hacapk_b200 import abi
    from hacapk_b200.engine import Engine, HbxError
    lib = abi.engine_lib()
    H = sphere(2)
    for n in (0, 3):
        assert lib.hbx_debug_fail_alloc(n) == 0
        with pytest.raises(HbxError) as ei:
            Engine(H.st, H.nd)
        assert ei.value.status == 2
    assert lib.hbx_debug_fail_alloc(-1) == 0
    E = Engine(H.st, H.nd)
    y, _, _ = E.matvec_host(np.ones(H.nd))
    assert np.all(np.isfinite(y))
    E.close()
