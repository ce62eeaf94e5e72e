"""GPU pipelined BiCGSTAB (HACApK_SOLVER_PIPE.c:144-600; _pipe2_ at :640)
through the C ABI.

Two bars.  (1) Bit for bit: the device solve equals its CPU replay
(tests/conftest.py pipe_replay: the kernel-order product, the device's
compensated dot order, the kernels' roundings) in iterations and in every
entry of u.  (2) Against the oracle's restatement of the reference loop with
the reference's compiled product: the iteration count inside the oracle's own
rounding spread and a true residual below the tolerance.  The pipelined
recurrences amplify rounding: the oracle loop itself, given products
perturbed by 1e-15 * max|y|, stops after 14-15 steps at C1 L3, 19-21 at L4
and 29-34 at L5 (12 seeds each), against 14 / 21 / 34 unperturbed; the bands
below are that spread."""
import ctypes as C

import numpy as np
import pytest

from conftest import pipe_replay, reference_input_mesh, sphere

pytestmark = pytest.mark.gpu

BANDS = {3: (0, 1), 4: (2, 1), 5: (5, 1)}


def _oracle_kind():
    import oracle
    return "ref" if oracle.have_ref() else "restated"


@pytest.mark.parametrize("level", [3, 4, 5])
def test_bitwise_equal_to_the_replay_and_inside_the_oracle_spread(gpu, build_libs, level):
    import oracle
    import torch
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    H, b = configs.c1(level)
    E = Engine(H.st, H.nd)
    u, info = E.bicgstab_pipe_host(b, tol=1e-8, max_iter=1000)
    num_ctas = torch.cuda.get_device_properties(0).multi_processor_count
    ur, nr, relr, sr = pipe_replay(H, b, tol=1e-8, max_iter=1000, num_ctas=num_ctas)
    assert info["status"] == 0 and sr == 0
    assert info["iterations"] == nr and np.array_equal(u, ur)
    assert info["relres"] == relr
    _, n_ref, _, _ = oracle.bicgstab_pipe(H.st, b, tol=1e-8, max_iter=1000, kind=_oracle_kind())
    lo, hi = BANDS[level]
    assert n_ref - lo <= info["iterations"] <= n_ref + hi
    rel = np.linalg.norm(b - oracle.matvec(H.st, u)) / np.linalg.norm(b)
    assert rel < 1e-8 * 1.05
    assert info["true_relres"] == pytest.approx(rel, rel=1e-3)


def test_legacy_pipe_symbols_on_the_reference_input(gpu, build_libs):
    """The reference's own input_10ts mesh through c_hacapk_bicgstab_cax_lfmtx_pipe_
    and _pipe2_ (param(83) steps, param(91) tolerance): the same answer from
    both, inside the oracle's band, below the tolerance."""
    import oracle
    from hacapk_b200 import abi, hmatrix
    from test_gpu_bicgstab import _control
    lib = abi.engine_lib()
    H = hmatrix.HostHMatrix(reference_input_mesh(), leaf_size=15, eta=2.0, aca_eps=1e-6, kernel=abi.KERNEL_PPOHBEM)
    n = H.nd
    b = np.ones(n)
    ctl, _buf = _control(maxit=1000, tol=1e-8)
    _, n_ref, _, _ = oracle.bicgstab_pipe(H.st, b, tol=1e-8, max_iter=1000, kind=_oracle_kind())
    outs = []
    for fn in (lib.c_hacapk_bicgstab_cax_lfmtx_pipe_, lib.c_hacapk_bicgstab_cax_lfmtx_pipe2_):
        u = np.zeros(n)
        nd, nstp, lrtrn = C.c_int(n), C.c_int(0), C.c_int(-1)
        fn(H.st, C.byref(ctl), abi.dptr(u), abi.dptr(b), ctl.param, C.byref(nd), C.byref(nstp), C.byref(lrtrn))
        assert lrtrn.value == 0
        assert n_ref - 2 <= nstp.value <= n_ref + 1
        assert np.linalg.norm(b - oracle.matvec(H.st, u)) / np.linalg.norm(b) < 1e-8 * 1.05
        outs.append((nstp.value, u))
    assert outs[0][0] == outs[1][0] and np.array_equal(outs[0][1], outs[1][1])


def test_device_vectors_stream_and_warm_start(gpu, build_libs):
    import torch
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    H, b = configs.c1(4)
    E = Engine(H.st, H.nd)
    bd = torch.from_numpy(b).to(gpu)
    ud = torch.zeros_like(bd)
    s = torch.cuda.current_stream().cuda_stream
    i1 = E.bicgstab_pipe_dev(bd.data_ptr(), ud.data_ptr(), stream=s, batch=3)
    assert i1["status"] == 0
    u1 = ud.cpu().numpy().copy()
    ud.zero_()
    i2 = E.bicgstab_pipe_dev(bd.data_ptr(), ud.data_ptr(), stream=s, batch=8)  # another graph batch
    assert i2["iterations"] == i1["iterations"] and np.array_equal(ud.cpu().numpy(), u1)
    i3 = E.bicgstab_pipe_dev(bd.data_ptr(), ud.data_ptr(), stream=s)  # start from the solution
    assert i3["iterations"] <= 1


def test_limits_zero_rhs_nonfinite_and_not_converged(gpu, build_libs):
    from hacapk_b200.engine import Engine
    H = sphere(3)
    E = Engine(H.st, H.nd)
    b = np.random.default_rng(3).standard_normal(H.nd)
    u, info = E.bicgstab_pipe_host(b, tol=1e-30, max_iter=3, check=False)
    assert info["status"] == 6 and info["iterations"] == 3
    u, info = E.bicgstab_pipe_host(np.zeros(H.nd), check=False)
    assert info["status"] == 0 and info["iterations"] == 0 and np.all(u == 0.0)
    bn = b.copy()
    bn[7] = np.inf
    u, info = E.bicgstab_pipe_host(bn, check=False)
    assert info["status"] == 7
    u, info = E.bicgstab_pipe_host(b)  # the engine is still usable
    assert info["status"] == 0


def test_larger_iteration_limit_after_a_captured_solve(gpu, build_libs):
    """A second solve with a larger iteration limit replaces the residual
    history buffer that the first solve's captured steps write; the steps are
    captured again, and the solve is the same bit for bit."""
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    H, b = configs.c1(3)
    E = Engine(H.st, H.nd)
    u1, i1 = E.bicgstab_pipe_host(b, tol=1e-8, max_iter=40)
    u2, i2 = E.bicgstab_pipe_host(b, tol=1e-8, max_iter=4000)
    u3, i3 = E.bicgstab_pipe_host(b, tol=1e-8, max_iter=40)
    assert i1["status"] == i2["status"] == i3["status"] == 0
    assert i1["iterations"] == i2["iterations"] == i3["iterations"]
    assert np.array_equal(u1, u2) and np.array_equal(u1, u3)
