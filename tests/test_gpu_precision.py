"""The precision form on the GPU (no counterpart in the reference, which is
FP64 throughout): an engine created with precision = HBX_FP32 stores every
factor in float (half the bytes of the FP64 stream) and multiplies in
float; hbx_bicgstab_refined wraps BiCGSTAB on it in FP64 iterative
refinement.  Errors are stated against the FP64 oracle (the reference's own
CPU product, HACApK_MAGMA.c:5-57): the FP32 product within 1e-6 of it, the
refined solution's FP64 residual ||b - H u||/||b|| below the tolerance."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("level", [3, 5])
def test_fp32_matvec_error_against_fp64_oracle(gpu, build_libs, level):
    import oracle
    from hacapk_b200 import abi, configs
    from hacapk_b200.engine import Engine
    H, _ = configs.c1(level)
    E32 = Engine(H.st, H.nd, precision=abi.HBX_FP32)
    E64 = Engine(H.st, H.nd)
    assert E32.info["precision"] == abi.HBX_FP32
    assert E32.info["stream_bytes"] <= 0.52 * E64.info["stream_bytes"]
    x = np.random.default_rng(level).standard_normal(H.nd)
    y, _, _ = E32.matvec_host(x)
    ref = oracle.matvec(H.st, x)
    err = np.abs(y - ref).max() / np.abs(ref).max()
    assert err <= 1e-6
    y2, _, _ = E32.matvec_host(x)
    assert np.array_equal(y, y2)  # deterministic like the FP64 engine


@pytest.mark.parametrize("level", [3, 4, 5])
def test_refined_solve_reaches_fp64_tolerance(gpu, build_libs, level):
    import oracle
    from hacapk_b200 import abi, configs
    from hacapk_b200.engine import Engine
    H, b = configs.c1(level)
    E64 = Engine(H.st, H.nd)
    E32 = Engine(H.st, H.nd, precision=abi.HBX_FP32)
    u, info = E64.bicgstab_refined_host(E32, b, tol=1e-8, max_iter=1000)
    assert info["status"] == 0 and info["outer"] >= 1
    r = b - oracle.matvec(H.st, u)
    relres = np.linalg.norm(r) / np.linalg.norm(b)
    assert relres < 1.05e-8
    assert info["true_relres"] == pytest.approx(relres, rel=1e-3)
    u64, _ = E64.bicgstab_host(b, tol=1e-8, max_iter=1000)
    assert np.linalg.norm(u - u64) / np.linalg.norm(u64) < 1e-5


def test_fp32_plain_bicgstab_and_rejects_mismatch(gpu, build_libs):
    from hacapk_b200 import abi, configs
    from hacapk_b200.engine import Engine, HbxError
    H, b = configs.c1(3)
    E32 = Engine(H.st, H.nd, precision=abi.HBX_FP32)
    u, info = E32.bicgstab_host(b, tol=1e-5, max_iter=500)
    assert info["status"] == 0 and info["true_relres"] < 1e-4
    H2, b2 = configs.c1(2)
    E64_small = Engine(H2.st, H2.nd)
    with pytest.raises(HbxError):
        E64_small.bicgstab_refined_host(E32, b2)


# ---- BF16 storage ----


@pytest.mark.parametrize("level", [3, 5])
def test_bf16_matvec_error_against_fp64_oracle(gpu, build_libs, level):
    """bfloat16 factors (8 significant bits, unit roundoff 2^-9) times the
    float-rounded vector, float accumulation within a run: the product is
    within 2^-8 of the FP64 oracle in the relative 2-norm (measured value
    printed), streams a quarter of the FP64 bytes plus panel padding, and is
    bit-identical on repeat."""
    import oracle
    from hacapk_b200 import abi, configs
    from hacapk_b200.engine import Engine
    H, _ = configs.c1(level)
    E16 = Engine(H.st, H.nd, precision=abi.HBX_BF16)
    E64 = Engine(H.st, H.nd)
    assert E16.info["precision"] == abi.HBX_BF16
    assert E16.info["stream_bytes"] <= 0.27 * E64.info["stream_bytes"]
    x = np.random.default_rng(level + 16).standard_normal(H.nd)
    y, _, _ = E16.matvec_host(x)
    ref = oracle.matvec(H.st, x)
    rel = np.linalg.norm(y - ref) / np.linalg.norm(ref)
    print(f"L{level}: BF16 product relative error {rel:.2e}")
    assert rel <= 2.0**-8
    y2, _, _ = E16.matvec_host(x)
    assert np.array_equal(y, y2)


@pytest.mark.parametrize("level", [3, 4])
def test_bf16_refined_solve_reaches_fp64_tolerance(gpu, build_libs, level):
    """BiCGSTAB on the BF16 engine inside FP64 iterative refinement reaches
    1e-8 in the FP64 residual, recomputed by the oracle."""
    import oracle
    from hacapk_b200 import abi, configs
    from hacapk_b200.engine import Engine
    H, b = configs.c1(level)
    E64 = Engine(H.st, H.nd)
    E16 = Engine(H.st, H.nd, precision=abi.HBX_BF16)
    u, info = E64.bicgstab_refined_host(E16, b, tol=1e-8, max_iter=1000, inner_tol=1e-2)
    assert info["status"] == 0
    relres = np.linalg.norm(b - oracle.matvec(H.st, u)) / np.linalg.norm(b)
    print(f"L{level}: BF16 refined: {info['outer']} refinement steps, {info['iterations']} inner steps, "
          f"FP64 residual {relres:.2e}")
    assert relres < 1.05e-8
