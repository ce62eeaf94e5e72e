"""The adjoint form on the GPU (no counterpart in the reference): an engine
created with hbx_options.transpose = 1 streams H^T through the same sm_100a
kernels.  Checked against the oracle's transposed product (oracle.c:
orc_adot_lfmtx_t, the loops of HACApK_MAGMA.c:5-57 with row/column roles and
U/V swapped), by the duality <H x, y> = <x, H^T y>, by the adjoint BiCGSTAB,
and by the gradient of J(g) = 0.5 ||sigma(g) - sigma_t||^2 (H sigma = g)
against central finite differences in random directions."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-13


@pytest.mark.parametrize("level", [3, 5])
def test_transposed_matvec_matches_oracle(gpu, build_libs, level):
    import oracle
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    H, _ = configs.c1(level)
    Et = Engine(H.st, H.nd, transpose=True)
    assert Et.info["transposed"] == 1
    x = np.random.default_rng(level).standard_normal(H.nd)
    y, _, _ = Et.matvec_host(x)
    ref = oracle.matvec_t(H.st, x)
    assert np.abs(y - ref).max() <= TOL * np.abs(ref).max()
    E = Engine(H.st, H.nd)
    assert Et.info["stream_bytes"] == E.info["stream_bytes"] or abs(Et.info["stream_bytes"] - E.info["stream_bytes"]) < 0.01 * E.info["stream_bytes"]
    z = np.random.default_rng(level + 1).standard_normal(H.nd)
    hx, _, _ = E.matvec_host(x)
    htz, _, _ = Et.matvec_host(z)
    assert abs(np.dot(hx, z) - np.dot(x, htz)) <= 1e-12 * np.linalg.norm(hx) * np.linalg.norm(z)


def test_adjoint_bicgstab(gpu, build_libs):
    import oracle
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    H, b = configs.c1(4)
    Et = Engine(H.st, H.nd, transpose=True)
    u, info = Et.bicgstab_host(b, tol=1e-8, max_iter=1000)
    assert info["status"] == 0
    r = b - oracle.matvec_t(H.st, u)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1.05e-8


def test_gradient_against_central_differences(gpu, build_libs):
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine
    H, _ = configs.c1(3)
    E, Et = Engine(H.st, H.nd), Engine(H.st, H.nd, transpose=True)
    rng = np.random.default_rng(3)
    g, sigma_t = rng.standard_normal(H.nd), rng.standard_normal(H.nd)
    tol = 1e-12
    J, grad, sigma, fi, ai = E.gradient_host(Et, g, sigma_t, tol=tol)
    assert fi["status"] == 0 and ai["status"] == 0
    assert J == pytest.approx(0.5 * np.sum((sigma - sigma_t) ** 2), rel=1e-12)

    def objective(gg):
        s, inf = E.bicgstab_host(gg, tol=tol, max_iter=1000)
        assert inf["status"] == 0
        return 0.5 * np.sum((s - sigma_t) ** 2)

    h = 1e-6
    for k in range(16):
        d = rng.standard_normal(H.nd)
        fd = (objective(g + h * d) - objective(g - h * d)) / (2 * h)
        assert fd == pytest.approx(np.dot(grad, d), rel=1e-4, abs=1e-6 * np.linalg.norm(grad) * np.linalg.norm(d))


def test_gradient_rejects_swapped_engines(gpu, build_libs):
    from hacapk_b200 import configs
    from hacapk_b200.engine import Engine, HbxError
    H, _ = configs.c1(2)
    E, Et = Engine(H.st, H.nd), Engine(H.st, H.nd, transpose=True)
    with pytest.raises(HbxError):
        Et.gradient_host(E, np.ones(H.nd), np.zeros(H.nd))
