"""The multi-RHS form on the GPU (no counterpart in the reference, whose
batched GEMV takes one vector): an engine created with nrhs = HBX_NRHS and
FP32 factors computes Y = alpha H X + beta Yin for 64 right-hand sides in one
launch, on the tensor cores (tcgen05, TF32 inputs, FP32 accumulation).
Errors are stated against the FP64 oracle (the reference's own CPU product,
HACApK_MAGMA.c:5-57) column by column: TF32 keeps 10 mantissa bits of every
factor and every X entry, so the bound is a relative error of 5e-3 in the
2-norm of each column (measured values are printed)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TF32_TOL = 5e-3


def _engine(H, nc=0):
    from hacapk_b200 import abi
    from hacapk_b200.engine import Engine
    return Engine(H.st, H.nd, precision=abi.HBX_FP32, nrhs=abi.HBX_NRHS, num_ctas=nc)


def _matmat(E, X, alpha=1.0, beta=0.0, Yin=None):
    import torch
    x = torch.from_numpy(np.ascontiguousarray(X, np.float32)).cuda()
    y = torch.zeros((X.shape[0], X.shape[1]), dtype=torch.float64, device="cuda")
    yin = torch.from_numpy(np.ascontiguousarray(Yin, np.float64)).cuda() if Yin is not None else None
    E.matmat_dev(x.data_ptr(), y.data_ptr(), alpha, beta, yin.data_ptr() if yin is not None else None)
    torch.cuda.synchronize()
    E.sync()
    return y.cpu().numpy()


def _col_errors(H, X, Y, cols):
    import oracle
    errs = []
    for j in cols:
        ref = oracle.matvec(H.st, X[:, j].astype(np.float64))
        errs.append(np.linalg.norm(Y[:, j] - ref) / np.linalg.norm(ref))
    return np.array(errs)


@pytest.mark.parametrize("level,nc", [(3, 148), (4, 148), (4, 7)])
def test_matmat_columns_match_oracle(gpu, build_libs, level, nc):
    from conftest import sphere
    H = sphere(level)
    E = _engine(H, nc)
    assert E.info["nrhs"] == 64
    X = np.random.default_rng(level * 10 + nc).standard_normal((H.nd, 64)).astype(np.float32)
    Y = _matmat(E, X)
    errs = _col_errors(H, X, Y, range(64))
    print(f"L{level} nc={nc}: TF32 column errors max {errs.max():.2e} median {np.median(errs):.2e}")
    assert errs.max() <= TF32_TOL
    # deterministic: the same product twice
    assert np.array_equal(Y, _matmat(E, X))


def test_matmat_alpha_beta(gpu, build_libs):
    from conftest import sphere
    H = sphere(3)
    E = _engine(H)
    rng = np.random.default_rng(5)
    X = rng.standard_normal((H.nd, 64)).astype(np.float32)
    Yin = rng.standard_normal((H.nd, 64))
    Y0 = _matmat(E, X)
    Y = _matmat(E, X, alpha=-0.5, beta=2.0, Yin=Yin)
    assert np.abs(Y - (-0.5 * Y0 + 2.0 * Yin)).max() <= 1e-12 * np.abs(Y).max()


def test_matmat_rhs_are_independent(gpu, build_libs):
    """Column j of Y depends on column j of X only (one RHS set to zero, one
    scaled: the rest unchanged)."""
    from conftest import sphere
    H = sphere(3)
    E = _engine(H)
    X = np.random.default_rng(7).standard_normal((H.nd, 64)).astype(np.float32)
    Y = _matmat(E, X)
    X2 = X.copy()
    X2[:, 5] = 0.0
    X2[:, 40] *= 2.0
    Y2 = _matmat(E, X2)
    keep = [j for j in range(64) if j not in (5, 40)]
    assert np.array_equal(Y[:, keep], Y2[:, keep])
    assert np.abs(Y2[:, 5]).max() == 0.0
    assert np.abs(Y2[:, 40] - 2.0 * Y[:, 40]).max() <= 1e-6 * np.abs(Y[:, 40]).max()


def test_single_vector_calls_are_refused(gpu, build_libs):
    from conftest import sphere
    from hacapk_b200.engine import HbxError
    H = sphere(3)
    E = _engine(H)
    with pytest.raises(HbxError):
        E.matvec_host(np.ones(H.nd))


def test_multi_rhs_needs_fp32(gpu, build_libs):
    from conftest import sphere
    from hacapk_b200 import abi
    from hacapk_b200.engine import Engine, HbxError
    H = sphere(3)
    with pytest.raises(HbxError):
        Engine(H.st, H.nd, precision=abi.HBX_FP64, nrhs=abi.HBX_NRHS)


@pytest.mark.parametrize("level", [3, 4])
def test_multi_rhs_solve_reaches_fp64_tolerance(gpu, build_libs, level):
    """hbx_bicgstab_multi: 64 right-hand sides (the unit-potential rhs of the
    BEM config plus 63 N(0,1) ones) solved to 1e-8 in the FP64 norm, each
    checked with the FP64 oracle product."""
    import oracle
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    H, b = configs.c1(level)
    E64 = Engine(H.st, H.nd)
    Em = _engine(H)
    rng = np.random.default_rng(2)
    B = rng.standard_normal((H.nd, 64))
    B[:, 0] = b
    U, infos = E64.bicgstab_multi_host(Em, B, tol=1e-8, max_iter=500)
    worst = 0.0
    for j in range(64):
        assert infos[j]["status"] == 0, (j, infos[j])
        ref = oracle.matvec(H.st, U[:, j])
        rel = np.linalg.norm(B[:, j] - ref) / np.linalg.norm(B[:, j])
        assert rel < 1e-8, (j, rel)
        assert abs(rel - infos[j]["true_relres"]) <= 1e-3 * rel + 1e-15
        worst = max(worst, rel)
    its = [i["iterations"] for i in infos]
    print(f"L{level}: 64 RHS, worst FP64 residual {worst:.2e}, inner steps {min(its)}..{max(its)}, "
          f"refinement steps {infos[0]['outer']}")


def test_multi_rhs_solve_masks_converged_columns(gpu, build_libs):
    """A right-hand side that is zero converges at once (x = 0) and leaves
    the others unchanged: the convergence mask holds it still."""
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    H, b = configs.c1(3)
    E64 = Engine(H.st, H.nd)
    Em = _engine(H)
    B = np.random.default_rng(3).standard_normal((H.nd, 64))
    B[:, 7] = 0.0
    U, infos = E64.bicgstab_multi_host(Em, B, tol=1e-8)
    assert np.all(U[:, 7] == 0.0) and infos[7]["iterations"] == 0
    assert all(i["status"] == 0 for i in infos)
