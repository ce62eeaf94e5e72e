"""GPU GCR(m) through the C ABI against the CPU restatement of
HACApK_gcrm_lfmtx (m_HACApK_solve.f90:506-571) driving the reference's
compiled matvec.  Bar: the same iteration count within +-1 and a true residual
||b - H u||/||b|| below the tolerance."""
import numpy as np
import pytest

from conftest import reference_input_mesh, sphere

pytestmark = pytest.mark.gpu


def _oracle_kind():
    import oracle
    return "ref" if oracle.have_ref() else "restated"


@pytest.mark.parametrize("level,restart", [(3, 8), (4, 8), (5, 8), (4, 3), (5, 30)])
def test_iterations_and_residual_match_oracle(gpu, build_libs, level, restart):
    import oracle
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    H, b = configs.c1(level)
    E = Engine(H.st, H.nd)
    u, info = E.gcr_host(b, tol=1e-8, max_iter=1000, restart=restart)
    u_ref, n_ref, hist, _ = oracle.gcrm(H.st, b, tol=1e-8, max_iter=1000, restart=restart, kind=_oracle_kind())
    assert info["status"] == 0
    assert abs(info["iterations"] - n_ref) <= 1
    r = b - oracle.matvec(H.st, u)
    rel = np.linalg.norm(r) / np.linalg.norm(b)
    assert rel < 1e-8 * 1.05
    assert info["true_relres"] == pytest.approx(rel, rel=1e-3)
    assert info["relres"] < 1e-8
    assert np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref) < 1e-5


@pytest.mark.parametrize("level,restart", [(3, 8), (4, 3), (5, 8)])
def test_bitwise_equal_to_the_replay(gpu, build_libs, level, restart):
    """The device solve against its CPU replay (tests/conftest.py gcr_replay:
    the kernel-order product, the device's compensated dot order, the
    kernels' roundings): the same iterations and u bit for bit."""
    import torch
    from conftest import gcr_replay
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    H, b = configs.c1(level)
    E = Engine(H.st, H.nd)
    u, info = E.gcr_host(b, tol=1e-8, max_iter=1000, restart=restart)
    num_ctas = torch.cuda.get_device_properties(0).multi_processor_count
    ur, nr, relr = gcr_replay(H, b, tol=1e-8, max_iter=1000, restart=restart, num_ctas=num_ctas)
    assert info["iterations"] == nr and np.array_equal(u, ur) and info["relres"] == relr


def test_reference_input_file(gpu, build_libs):
    """The reference's own input_10ts.pbf mesh (committed fixture)."""
    import oracle
    from hacapk_b200 import abi, hmatrix
    from hacapk_b200.engine import Engine
    H = hmatrix.HostHMatrix(reference_input_mesh(), leaf_size=15, eta=2.0, aca_eps=1e-6,
                            kernel=abi.KERNEL_PPOHBEM)
    b = np.ones(H.nd)
    E = Engine(H.st, H.nd)
    u, info = E.gcr_host(b, tol=1e-8, max_iter=1000, restart=8)
    _, n_ref, _, _ = oracle.gcrm(H.st, b, tol=1e-8, max_iter=1000, restart=8, kind=_oracle_kind())
    assert info["status"] == 0 and abs(info["iterations"] - n_ref) <= 1
    assert info["true_relres"] < 1e-8 * 1.05


def test_repeated_solves_are_bitwise_identical(gpu, build_libs):
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    H, b = configs.c1(4)
    E = Engine(H.st, H.nd)
    u1, i1 = E.gcr_host(b)
    u2, i2 = E.gcr_host(b)
    assert i1["iterations"] == i2["iterations"] and np.array_equal(u1, u2)


def test_device_vectors_stream_and_restart_growth(gpu, build_libs):
    import torch
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    H, b = configs.c1(4)
    E = Engine(H.st, H.nd)
    bd = torch.from_numpy(b).to(gpu)
    ud = torch.zeros_like(bd)
    s = torch.cuda.current_stream().cuda_stream
    i4 = E.gcr_dev(bd.data_ptr(), ud.data_ptr(), restart=4, stream=s)
    assert i4["status"] == 0
    ud.zero_()
    i16 = E.gcr_dev(bd.data_ptr(), ud.data_ptr(), restart=16, stream=s)   # workspace grows
    assert i16["status"] == 0 and i16["iterations"] <= i4["iterations"]
    info2 = E.gcr_dev(bd.data_ptr(), ud.data_ptr(), restart=16, stream=s)  # start from the solution
    assert info2["iterations"] <= 1


def test_limits_zero_rhs_not_converged_and_bad_restart(gpu, build_libs):
    from hacapk_b200.engine import Engine
    H = sphere(3)
    E = Engine(H.st, H.nd)
    b = np.random.default_rng(3).standard_normal(H.nd)
    u, info = E.gcr_host(b, tol=1e-30, max_iter=3, check=False)
    assert info["status"] == 6 and info["iterations"] == 3
    u, info = E.gcr_host(np.zeros(H.nd), check=False)
    assert info["status"] == 0 and info["iterations"] == 0 and np.all(u == 0.0)
    with pytest.raises(RuntimeError):
        E.gcr_host(b, restart=65)


def test_nonfinite_rhs_is_reported(gpu, build_libs):
    from hacapk_b200.engine import Engine
    H = sphere(3)
    E = Engine(H.st, H.nd)
    b = np.ones(H.nd)
    b[5] = np.nan
    u, info = E.gcr_host(b, check=False)
    assert info["status"] == 7


@pytest.mark.parametrize("restart", [8, 30])
def test_entry_point_with_the_solvers_arguments(gpu, build_libs, restart):
    """c_hacapk_gcrm_lfmtx_gpu_ (the solvers' argument list; param(87) the
    restart length, param(83) the step limit, param(91) the tolerance) on the
    reference's own input_10ts mesh: the same solution as hbx_gcr_host, bit
    for bit, and the oracle's step count."""
    import ctypes as C
    import oracle
    from hacapk_b200 import abi, hmatrix
    from hacapk_b200.engine import Engine
    from test_gpu_bicgstab import _control
    lib = abi.engine_lib()
    H = hmatrix.HostHMatrix(reference_input_mesh(), leaf_size=15, eta=2.0, aca_eps=1e-6, kernel=abi.KERNEL_PPOHBEM)
    b = np.ones(H.nd)
    ctl, buf = _control(maxit=1000, tol=1e-8)
    buf[86] = restart
    u = np.zeros(H.nd)
    nd, nstp, lrtrn = C.c_int(H.nd), C.c_int(-1), C.c_int(-1)
    lib.c_hacapk_gcrm_lfmtx_gpu_(H.st, C.byref(ctl), abi.dptr(u), abi.dptr(b), ctl.param, C.byref(nd),
                                 C.byref(nstp), C.byref(lrtrn))
    assert lrtrn.value == 0
    E = Engine(H.st, H.nd)
    u2, info = E.gcr_host(b, tol=1e-8, max_iter=1000, restart=restart)
    assert nstp.value == info["iterations"] and np.array_equal(u, u2)
    _, n_ref, _, _ = oracle.gcrm(H.st, b, tol=1e-8, max_iter=1000, restart=restart, kind=_oracle_kind())
    assert abs(nstp.value - n_ref) <= 1
