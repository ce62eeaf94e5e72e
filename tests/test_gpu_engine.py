"""GPU parity tests of the H-matvec through the C ABI (libhacapk_b200.so).

Bar: relative to max|y|, the engine matches the reference's CPU H-matvec to
1e-13 (FP64; the summation order differs), and is bit-reproducible."""
import ctypes as C
import importlib.util
import os

import numpy as np
import pytest

from conftest import ROOT, sphere

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(ROOT, "tests", "golden")
TOL = 1e-13


def _mg():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg


def relerr(y, ref):
    return np.abs(y - ref).max() / np.abs(ref).max()


@pytest.mark.parametrize("name", ["sphere_L2_dense", "sphere_L3_leaf32", "sphere_L3_leaf15_ppohbem",
                                  "sphere_L4_leaf32"])
def test_matvec_matches_golden_vectors(gpu, build_libs, name):
    from hacapk_b200.engine import Engine
    mg = _mg()
    case = [c for c in mg.CASES if c[0] == name][0]
    fx = np.load(os.path.join(GOLDEN, name + ".npz"))
    H, x = mg.build(case)
    E = Engine(H.st, H.nd)
    y, tk, tc = E.matvec_host(fx["x"])
    assert relerr(y, fx["y"]) <= TOL
    assert tk > 0.0


def test_matvec_c1_full_size_and_deterministic(gpu, build_libs):
    import oracle
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    H, b = configs.c1(5)
    E = Engine(H.st, H.nd)
    rng = np.random.default_rng(21)
    for _ in range(2):
        x = rng.standard_normal(H.nd)
        ref = oracle.matvec(H.st, x)
        y1, _, _ = E.matvec_host(x)
        y2, _, _ = E.matvec_host(x)
        assert relerr(y1, ref) <= TOL
        assert np.array_equal(y1, y2)
    # linearity at full size: H(a x + z) = a H x + H z
    x, z = rng.standard_normal(H.nd), rng.standard_normal(H.nd)
    hx, _, _ = E.matvec_host(x)
    hz, _, _ = E.matvec_host(z)
    hc, _, _ = E.matvec_host(2.5 * x + z)
    assert relerr(hc, 2.5 * hx + hz) <= 1e-13


def test_reference_self_check_with_unit_vector(gpu, build_libs):
    """The reference's own CPU-vs-GPU check (m_HACApK_solve.f90:705-735):
    x = 1, error(CPU-GPU) = ||y_cpu - y_gpu||_2 / ||y_cpu||_2, on the C1
    matrix through hbx_matvec_host."""
    import oracle
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    H, _ = configs.c1(5)
    E = Engine(H.st, H.nd)
    x = np.ones(H.nd)
    y_cpu = oracle.matvec(H.st, x)
    y_gpu, _, _ = E.matvec_host(x)
    err = np.linalg.norm(y_cpu - y_gpu) / np.linalg.norm(y_cpu)
    print(f"error(CPU-GPU) = {err:.3e}")
    assert err <= TOL


def test_device_api_alpha_beta_and_aliasing(gpu, build_libs):
    import torch
    import oracle
    from hacapk_b200.engine import Engine
    H = sphere(4)
    E = Engine(H.st, H.nd)
    x = torch.randn(H.nd, dtype=torch.float64, device=gpu)
    z = torch.randn(H.nd, dtype=torch.float64, device=gpu)
    y = torch.empty_like(x)
    s = torch.cuda.current_stream().cuda_stream
    hx = oracle.matvec(H.st, x.cpu().numpy())
    E.matvec_dev(x.data_ptr(), y.data_ptr(), alpha=-2.0, beta=0.5, yin_ptr=z.data_ptr(), stream=s)
    E.sync(s)
    assert relerr(y.cpu().numpy(), -2.0 * hx + 0.5 * z.cpu().numpy()) <= TOL
    w = z.clone()
    E.matvec_dev(x.data_ptr(), w.data_ptr(), alpha=1.0, beta=1.0, yin_ptr=w.data_ptr(), stream=s)  # in place
    E.sync(s)
    assert relerr(w.cpu().numpy(), hx + z.cpu().numpy()) <= TOL


@pytest.mark.parametrize("nc", [1, 7, 148])
def test_any_number_of_persistent_ctas(gpu, build_libs, nc):
    import oracle
    from hacapk_b200.engine import Engine
    H = sphere(4)
    E = Engine(H.st, H.nd, num_ctas=nc)
    x = np.random.default_rng(nc).standard_normal(H.nd)
    y, _, _ = E.matvec_host(x)
    assert relerr(y, oracle.matvec(H.st, x)) <= TOL


def _lib():
    from hacapk_b200 import abi
    return abi.engine_lib()


def test_legacy_batch_entry_points(gpu, build_libs):
    """c_hacapk_adot_body_lfcpy_batch_sorted_ / _lfmtx_batch_ / _lfdel_batch_
    (HACApK_BATCH_SORT.c:86, HACApK_BATCH.c:257, :812): zau += H zu."""
    import oracle
    from hacapk_b200 import abi
    lib = _lib()
    H = sphere(4)
    nd = C.c_int(H.nd)
    zu = np.random.default_rng(1).standard_normal(H.nd)
    zau = np.ones(H.nd)
    zbu = np.zeros(max(1, H.st.contents.ktmax))
    tb, ts, tc = C.c_double(0), C.c_double(0), C.c_double(0)
    lib.magma_init_()
    lib.c_hacapk_adot_body_lfcpy_batch_sorted_(C.byref(nd), H.st)
    lib.c_hacapk_adot_body_lfmtx_batch_(abi.dptr(zau), H.st, abi.dptr(zu), abi.dptr(zbu), C.byref(tb),
                                        C.byref(ts), C.byref(tc))
    assert relerr(zau, oracle.matvec(H.st, zu, np.ones(H.nd))) <= TOL
    assert tb.value > 0.0
    lib.c_hacapk_adot_body_lfdel_batch_(H.st)
    # per-leaf variants map onto the same engine
    zau2 = np.full(H.nd, -3.0)
    lib.c_hacapk_adot_body_lfcpy_gpu_(C.byref(nd), H.st)
    lib.c_hacapk_adot_body_lfmtx_gpu_(abi.dptr(zau2), H.st, abi.dptr(zu), abi.dptr(zbu))
    lib.c_hacapk_adot_body_lfdel_gpu_(H.st)
    assert relerr(zau2, oracle.matvec(H.st, zu, np.full(H.nd, -3.0))) <= TOL
    lib.magma_finalize_()


def test_fortran_leaf_stride_and_edge_leaves(gpu, build_libs):
    import oracle
    from hacapk_b200.engine import Engine
    import test_plan as tp
    H = sphere(3)
    P, keep = tp._fortran_like(H, 176)
    E = Engine(C.pointer(P), H.nd)
    x = np.random.default_rng(2).standard_normal(H.nd)
    y, _, _ = E.matvec_host(x)
    assert relerr(y, oracle.matvec(H.st, x)) <= TOL
    rng = np.random.default_rng(9)
    nd = 100
    leaves = [
        (2, 0, 1, 40, 1, 100, rng.standard_normal(40 * 100)),
        (1, 0, 41, 30, 1, 50, np.zeros(0)),
        (1, 3, 41, 30, 51, 50, rng.standard_normal(3 * (30 + 50))),
        (1, 70, 71, 30, 1, 100, rng.standard_normal(70 * 130)),
        (2, 0, 41, 30, 1, 50, rng.standard_normal(30 * 50)),
    ]
    P2, keep2 = tp._custom(leaves, nd)
    x = rng.standard_normal(nd)
    for nc in (1, 3, 148):
        E2 = Engine(C.pointer(P2), nd, num_ctas=nc)
        y, _, _ = E2.matvec_host(x)
        ref = tp._dense_of(leaves, nd) @ x
        assert relerr(y, ref) <= TOL
    P3, keep3 = tp._custom([], 33)
    E3 = Engine(C.pointer(P3), 33)
    y, _, _ = E3.matvec_host(np.ones(33))
    assert np.all(y == 0.0)


def test_invalid_inputs_report_status(gpu, build_libs):
    from hacapk_b200 import abi
    from hacapk_b200.engine import Engine, HbxError
    import test_plan as tp
    lib = _lib()
    h = C.c_void_p()
    assert lib.hbx_create(None, 10, None, C.byref(h)) == 1
    assert b"NULL" in lib.hbx_last_error()
    P, keep = tp._custom([(2, 0, 95, 10, 1, 10, np.ones(100))], 100)
    with pytest.raises(HbxError) as ei:
        Engine(C.pointer(P), 100)
    assert ei.value.status == 1
    H = sphere(2)
    E = Engine(H.st, H.nd)
    assert lib.hbx_matvec(E._h, 1.0, None, 0.0, None, None, None) == 1
    assert lib.hbx_matvec(E._h, 1.0, C.c_void_p(16), 1.0, None, C.c_void_p(16), None) == 1  # beta!=0, no yin
    y, _, _ = E.matvec_host(np.ones(H.nd))  # still usable
    assert np.isfinite(y).all()


@pytest.mark.parametrize("level", [3, 4, 5])
def test_matvec_equals_kernel_order_emulation_bitwise(gpu, build_libs, level):
    """k_matvec's arithmetic is fully specified: the CPU interpreter that sums
    in the kernel's order (per-warp fma accumulators over rotated panels,
    block sums in warp order; tests/emu) reproduces it bit for bit, on the
    engine's own CTA count."""
    import torch
    from conftest import kernel_order_matvec
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    H, _ = configs.c1(level)
    E = Engine(H.st, H.nd)
    x = np.random.default_rng(40 + level).standard_normal(H.nd)
    y, _, _ = E.matvec_host(x)
    y_emu = kernel_order_matvec(H, E.info["num_ctas"])(x)
    assert np.array_equal(y, y_emu)
    E.close()
