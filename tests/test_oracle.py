"""CPU tests of the checker (oracle/) and of the host-side construction.

The oracle is pinned two ways: against the reference's own compiled CPU
H-matvec (oracle/_ref, HACApK_MAGMA.c:5-57) and against the golden fixtures
in tests/golden/ that were produced by it; the construction is pinned by the
known answers recorded in the reference's ivb/ log.
"""
import json
import os

import numpy as np
import pytest

from conftest import REFERENCE, ROOT, sphere

GOLDEN = os.path.join(ROOT, "tests", "golden")


def test_icosphere_counts(build_libs):
    from hacapk_b200 import hmatrix
    for L in range(4):
        m = hmatrix.icosphere(L)
        assert m.xyz.shape == (10 * 4 ** L + 2, 3)
        assert m.faces.shape == (20 * 4 ** L, 3)
        assert np.allclose(np.linalg.norm(m.xyz, axis=1), 1.0)
        assert m.faces.min() == 0 and m.faces.max() == m.xyz.shape[0] - 1


@pytest.mark.skipif(not os.path.exists(os.path.join(REFERENCE, "bem-bb_inputs", "input_10ts.pbs")),
                    reason="reference mesh input_10ts.pbs not available")
@pytest.mark.parametrize("aca_method", [1, 2])
def test_known_answers_input_10ts(build_libs, aca_method):
    """Construction counts of the recorded run (ivb/log0000.txt, ivb/job_cpu.sh.o78632)."""
    import ctypes as C
    from hacapk_b200 import abi, hmatrix
    ka = json.load(open(os.path.join(GOLDEN, "input_10ts_known_answers.json")))
    m = hmatrix.read_pbs(os.path.join(REFERENCE, "bem-bb_inputs", "input_10ts.pbs"))
    lib = abi.build_lib()
    p = hmatrix.default_params()
    p.leaf_size, p.eta, p.aca_eps, p.kernel, p.aca_method = 15, 2.0, 1e-6, abi.KERNEL_PPOHBEM, aca_method
    h = C.c_void_p()
    xyz, f = np.ascontiguousarray(m.xyz), np.ascontiguousarray(m.faces)
    assert lib.hbx_build(abi.dptr(xyz), xyz.shape[0], abi.iptr(f), f.shape[0], C.byref(p), C.byref(h)) == 0
    s = abi.BuildStats()
    lib.hbx_build_get_stats(h, C.byref(s))
    lib.hbx_build_free(h)
    assert s.nd == ka["nd"]
    assert s.nclst == ka["nclst"]
    assert (s.n_lowrank, s.n_dense, s.n_hnode) == (ka["n_lowrank"], ka["n_dense"], ka["n_hnode"])
    assert s.ncpc7 == ka["ncpc_kt7"]
    assert s.ktmax == ka["ktmax"]
    mb = s.memh_words * 8.0 / 1024.0 / 1024.0
    if aca_method == 1:  # the recorded revision used plain ACA
        assert mb == pytest.approx(ka["memory_mbyte"], rel=1e-12)
        assert 100.0 * mb / (s.nd * s.nd * 8.0 / 1024 / 1024) == pytest.approx(ka["memory_compression_pct"], rel=1e-10)


def test_read_pbs_small(build_libs):
    path = os.path.join(REFERENCE, "bem-bb_inputs", "input_1ts.pbs")
    if not os.path.exists(path):
        pytest.skip("reference mesh not available")
    from hacapk_b200 import hmatrix
    m = hmatrix.read_pbs(path)
    assert m.xyz.shape == (502, 3) and m.faces.shape == (1000, 3)
    assert m.dble.shape == (1000, 1) and np.all(m.dble == 1.0)


def test_restated_matvec_is_bitwise_the_reference(build_libs):
    import oracle
    if not oracle.have_ref():
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    H = sphere(3)
    x = np.random.default_rng(0).standard_normal(H.nd)
    z = np.random.default_rng(1).standard_normal(H.nd)
    assert np.array_equal(oracle.matvec(H.st, x), oracle.matvec_ref(H.st, x))
    assert np.array_equal(oracle.matvec(H.st, x, z), oracle.matvec_ref(H.st, x, z))


@pytest.mark.parametrize("name", ["sphere_L2_dense", "sphere_L3_leaf32", "sphere_L3_leaf15_ppohbem",
                                  "sphere_L4_leaf32"])
def test_oracle_against_golden_vectors(build_libs, name):
    import oracle
    sys_path_golden = os.path.join(GOLDEN)
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(sys_path_golden, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    case = [c for c in mg.CASES if c[0] == name][0]
    fx = np.load(os.path.join(GOLDEN, name + ".npz"))
    H, x = mg.build(case)
    assert np.array_equal(x, fx["x"])
    assert int(fx["nlf"]) == H.nlf
    y = oracle.matvec(H.st, x)
    scale = np.abs(fx["y"]).max()
    assert np.abs(y - fx["y"]).max() <= 1e-14 * scale
    if mg.leaf_digest(H) != str(fx["digest"]):
        pytest.skip("leaf bytes differ from the fixture's host (libm); values checked to 1e-14")


def test_blas_and_omp_matvec_agree(build_libs):
    import oracle
    H = sphere(3)
    x = np.random.default_rng(2).standard_normal(H.nd)
    y = oracle.matvec(H.st, x)
    for y2 in (oracle.matvec_blas(H.st, x), oracle.matvec_omp(H.st, x, nthreads=4)):
        assert np.abs(y2 - y).max() <= 1e-14 * np.abs(y).max()


def test_transposed_matvec(build_libs):
    import oracle
    H = sphere(2)
    Hm = np.stack([oracle.matvec(H.st, e) for e in np.eye(H.nd)], axis=1)
    x = np.random.default_rng(3).standard_normal(H.nd)
    yt = oracle.matvec_t(H.st, x)
    assert np.abs(Hm.T @ x - yt).max() <= 1e-13 * np.abs(yt).max()


def test_hmatrix_approximates_dense(build_libs):
    import oracle
    H = sphere(3, aca_eps=1e-5)
    A = H.dense()
    x = np.random.default_rng(4).standard_normal(H.nd)
    err = np.linalg.norm(A @ x - oracle.matvec(H.st, x)) / np.linalg.norm(A @ x)
    assert err < 1e-4


@pytest.mark.parametrize("aca_eps", [1e-5, 1e-7])
def test_accuracy_check_matches_the_assembled_matrix(build_libs, aca_eps):
    """The reference's H-matrix accuracy check (HACApK_accuracy_leafmtx,
    m_HACApK_base.f90:614-673) restated: its ||A - H||_F / ||A||_F equals
    the one of the H-matrix assembled densely from its leaves against the
    exact operator, and it follows the ACA+ tolerance."""
    H = sphere(3, aca_eps=aca_eps)
    zh, za = H.accuracy()
    A = H.dense()
    Hd = np.zeros_like(A)
    for ip in range(H.nlf):
        kind, r0, nr, c0, nc, kt, data = H.leaf_arrays(ip)
        Hd[r0 - 1:r0 - 1 + nr, c0 - 1:c0 - 1 + nc] = data[0] @ data[1].T if kind == 1 else data
    assert za == pytest.approx(np.linalg.norm(A), rel=1e-12)
    assert zh / za == pytest.approx(np.linalg.norm(A - Hd) / np.linalg.norm(A), rel=1e-6, abs=1e-15)
    assert zh / za < 10 * aca_eps
    print(f"ACA+ {aca_eps:.0e}: ||A - H||_F / ||A||_F = {zh / za:.2e}")


def test_oracle_bicgstab_converges(build_libs):
    import oracle
    from hacapk_b200 import configs
    H, b = configs.c1(3)
    u, n, hist, _ = oracle.bicgstab(H.st, b, tol=1e-8, max_iter=500, kind="restated")
    assert hist[-1] < 1e-8 and hist[0] == pytest.approx(1.0)
    r = b - oracle.matvec(H.st, u)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-8 * 1.01
    if oracle.have_ref():
        u2, n2, hist2, _ = oracle.bicgstab(H.st, b, tol=1e-8, max_iter=500, kind="ref")
        assert n2 == n and np.array_equal(u2, u)


def _gcrm_numpy(st, b, tol, mstep, m):
    """HACApK_gcrm_lfmtx (m_HACApK_solve.f90:506-571) line by line in numpy:
    products from the restated matvec, HACApK_dotp_d as a running sum
    (np.cumsum accumulates in index order), 1-based slots kept as written."""
    import oracle

    def dotp(x, y):
        return float(np.cumsum(x * y)[-1])

    nd = b.shape[0]
    u = np.zeros(nd)
    zp, zap, capap = np.zeros((m + 1, nd)), np.zeros((m + 1, nd)), np.zeros(m + 1)
    bnorm = np.sqrt(dotp(b, b))
    zr = b - oracle.matvec(st, u)
    zp[1] = zr
    zrnorm = np.sqrt(dotp(zr, zr))
    hist = [zrnorm / bnorm]
    if zrnorm / bnorm < tol:
        return u, 0, hist
    zap[1] = oracle.matvec(st, zp[1])
    for it in range(1, mstep + 1):
        ik = (it - 1) % m + 1
        znom = dotp(zap[ik], zr)
        capap[ik] = dotp(zap[ik], zap[ik])
        alpha = znom / capap[ik]
        u = u + alpha * zp[ik]
        zr = zr - alpha * zap[ik]
        zrnorm = np.sqrt(dotp(zr, zr))
        hist.append(zrnorm / bnorm)
        if zrnorm / bnorm < tol or it == mstep:
            break
        zar = oracle.matvec(st, zr)
        ikn = it % m + 1
        zp[ikn] = zr
        zap[ikn] = zar
        for il in range(1, ik + 1):
            beta = -dotp(zap[il], zar) / capap[il]
            zp[ikn] = zp[ikn] + beta * zp[il]
            zap[ikn] = zap[ikn] + beta * zap[il]
    return u, it, hist


@pytest.mark.parametrize("restart", [1, 3, 8])
def test_oracle_gcrm_is_the_fortran_loop(build_libs, restart):
    """The C restatement of GCR(m) against the Fortran loop restated in numpy:
    the same iterations, bit for bit (restart 1 and 3 exercise the slot-1
    aliasing at every restart)."""
    import oracle
    H = sphere(2)
    b = np.random.default_rng(11).standard_normal(H.nd)
    u, n, hist, _ = oracle.gcrm(H.st, b, tol=1e-8, max_iter=400, restart=restart, kind="restated")
    u2, n2, hist2 = _gcrm_numpy(H.st, b, 1e-8, 400, restart)
    assert n == n2 and np.array_equal(hist, np.array(hist2)) and np.array_equal(u, u2)


def test_oracle_gcrm_converges_monotonically(build_libs):
    """GCR minimises the residual over its search space, so the recorded
    residual never grows; the solution meets the tolerance in the true
    residual; the reference's compiled matvec gives the same iterations."""
    import oracle
    from hacapk_b200 import configs
    H, b = configs.c1(3)
    u, n, hist, _ = oracle.gcrm(H.st, b, tol=1e-8, max_iter=500, restart=8, kind="restated")
    assert hist[-1] < 1e-8 and np.all(np.diff(hist) <= 1e-15)
    assert np.linalg.norm(b - oracle.matvec(H.st, u)) / np.linalg.norm(b) < 1.05e-8
    if oracle.have_ref():
        u2, n2, _, _ = oracle.gcrm(H.st, b, tol=1e-8, max_iter=500, restart=8, kind="ref")
        assert n2 == n and np.array_equal(u2, u)
    _, n3, _, _ = oracle.gcrm(H.st, b, tol=1e-30, max_iter=4, restart=8, kind="restated")
    assert n3 == 4


def test_oracle_pipe_is_the_reference_loop(build_libs):
    """The C restatement of the pipelined BiCGSTAB (HACApK_SOLVER_PIPE.c:144-600)
    against the same loop in numpy (products from the restated matvec,
    running-sum dots, daxpy / dlascl roundings): bit for bit; it converges
    in the true residual."""
    import oracle

    def dotp(x, y):
        return float(np.cumsum(x * y)[-1])

    H = sphere(2)
    b = np.random.default_rng(12).standard_normal(H.nd)
    mv = lambda x: oracle.matvec(H.st, x)
    u = np.zeros(H.nd)
    bnorm = np.sqrt(dotp(b, b))
    r = b + (-1.0) * mv(u)
    r0 = r.copy()
    w = mv(r)
    t = mv(w)
    znorm = dotp(r, r)
    alpha = znorm / dotp(w, r)
    zr = np.sqrt(znorm)
    beta = zeta = 0.0
    hist = [zr / bnorm]
    for step in range(1, 401):
        if zr / bnorm < 1e-8:
            break
        if step > 1:
            p = (p + (-zeta) * s) * beta + r
            s, z = (s + (-zeta) * z) * beta + w, (z + (-zeta) * v) * beta + t
        else:
            p, s, z = r.copy(), w.copy(), t.copy()
        q = r + (-alpha) * s
        y = w + (-alpha) * z
        zeta = dotp(y, q) / dotp(y, y)
        v = mv(z)
        u = (u + alpha * p) + zeta * q
        r = q + (-zeta) * y
        w = (t + (-alpha) * v) * (-zeta) + y
        znormold, znorm = znorm, dotp(r, r0)
        zw, zs, zz, rr = dotp(w, r0), dotp(s, r0), dotp(z, r0), dotp(r, r)
        beta = (alpha / zeta) * (znorm / znormold)
        alpha = znorm / (zw + beta * zs - beta * zeta * zz)
        zr = np.sqrt(rr)
        hist.append(zr / bnorm)
        t = mv(w)
    u2, n2, hist2, _ = oracle.bicgstab_pipe(H.st, b, tol=1e-8, max_iter=400, kind="restated")
    assert n2 == len(hist) - 1 and np.array_equal(hist2, np.array(hist)) and np.array_equal(u2, u)
    assert np.linalg.norm(b - mv(u2)) / np.linalg.norm(b) < 1.05e-8
    if oracle.have_ref():
        u3, n3, _, _ = oracle.bicgstab_pipe(H.st, b, tol=1e-8, max_iter=400, kind="ref")
        assert n3 == n2 and np.array_equal(u3, u2)


def test_device_replays_against_the_oracle(build_libs):
    """The CPU replays of the device GCR(m) and pipelined solvers (kernel-order
    product, the device's compensated dot order) on C1 L3 / L4: GCR takes the
    oracle's iteration count; the pipelined solver lands inside the oracle's
    own spread under 1e-15 product noise; both meet the tolerance in the
    true residual.  The dot emulation is checked against exact sums."""
    import math
    import oracle
    from conftest import device_dots, gcr_replay, pipe_replay
    from hacapk_b200 import configs
    rng = np.random.default_rng(4)
    for n in (1, 255, 256, 257, 5000, 151552, 200003):
        x, y = rng.standard_normal(n), rng.standard_normal(n)
        d = device_dots([(x, y)])[0]
        # the exact dot, correctly rounded: each product split into p + e
        # (Veltkamp / Dekker), then one exactly rounded sum of all the parts
        p = x * y
        c = 134217729.0
        xh = x * c - (x * c - x)
        yh = y * c - (y * c - y)
        xl, yl = x - xh, y - yh
        e = ((xh * yh - p) + xh * yl + xl * yh) + xl * yl
        exact = math.fsum(np.concatenate([p, e]))
        assert abs(d - exact) <= 2 * math.ulp(exact)
    for level in (3, 4):
        H, b = configs.c1(level)
        tr = lambda u: np.linalg.norm(b - oracle.matvec(H.st, u)) / np.linalg.norm(b)
        u, n, _ = gcr_replay(H, b, restart=8)
        _, n_ref, _, _ = oracle.gcrm(H.st, b, restart=8, kind="restated")
        assert n == n_ref and tr(u) < 1.05e-8
        u, n, _, st = pipe_replay(H, b)
        _, n_ref, _, _ = oracle.bicgstab_pipe(H.st, b, kind="restated")
        assert st == 0 and n_ref - 2 <= n <= n_ref + 1 and tr(u) < 1.05e-8


def _pipe_with_noisy_products(H, b, seed, eps=1e-15, tol=1e-8, max_iter=1000):
    """The oracle's pipelined loop (orc_bicgstab_pipe) with every product
    H x (the restated reference product) perturbed by eps * max|Hx| * N(0,1),
    seeded: the loop's own sensitivity to rounding-sized changes of the
    product.  Returns the step count."""
    import ctypes as C
    import oracle
    nd = H.nd
    rng = np.random.default_rng(seed)
    DP = C.POINTER(C.c_double)

    def product(zau, _st, zu, _zbu):
        y = oracle.matvec(H.st, np.ctypeslib.as_array(zu, (nd,)))
        np.ctypeslib.as_array(zau, (nd,))[:] += y + eps * np.abs(y).max() * rng.standard_normal(nd)

    cb = C.CFUNCTYPE(None, DP, C.c_void_p, DP, DP)(product)
    u, hist, secs = np.zeros(nd), np.zeros(max_iter + 1), C.c_double(0.0)
    n = oracle.lib().orc_bicgstab_pipe(oracle._st(H.st), nd, oracle._d(u), oracle._d(np.ascontiguousarray(b)), tol,
                                       max_iter, oracle.MV_EXTERNAL, C.cast(cb, C.c_void_p), None, 0,
                                       oracle._d(hist), C.byref(secs))
    return int(n)


@pytest.mark.parametrize("level", [3, 4, 5])
def test_pipelined_bands_are_the_oracle_spread(build_libs, level):
    """The GPU test's step-count bands for the pipelined solver
    (tests/test_gpu_pipe.py BANDS) come from the oracle loop's own spread:
    over 12 seeds of 1e-15 * max|y| product noise it stops after 14-15 steps
    at C1 L3, 19-21 at L4 and 29-34 at L5 (unperturbed: 14 / 21 / 34).  Each
    band lies inside that spread (or +-1), and the device's step count (its
    kernel-order replay, which the GPU test holds equal to the device bit for
    bit) lies inside the spread too."""
    import oracle
    from conftest import pipe_replay
    from hacapk_b200 import configs
    from test_gpu_pipe import BANDS
    H, b = configs.c1(level)
    _, n_ref, _, _ = oracle.bicgstab_pipe(H.st, b, kind="restated")
    spread = [_pipe_with_noisy_products(H, b, seed) for seed in range(12)]
    lo, hi = BANDS[level]
    assert n_ref - lo >= min(spread) and n_ref + hi <= max(max(spread), n_ref + 1)
    _, n_dev, _, status = pipe_replay(H, b)
    assert status == 0 and min(spread) <= n_dev <= max(spread)


def test_two_body_precision_workload(build_libs):
    """C2 (the precision form's workload) at level 3: the sphere and the
    seeded ellipsoid are disjoint with the stated gap along x, the H-matrix
    over both bodies reproduces the dense operator to the ACA tolerance
    (1e-6), and the oracle's BiCGSTAB reaches 1e-8."""
    import oracle
    from hacapk_b200 import configs
    from hacapk_b200.hmatrix import ellipsoid, icosphere
    H, b = configs.c2(3)
    sphere3 = icosphere(3)
    assert H.nd == 2 * sphere3.nofc
    axes = np.random.default_rng(1).uniform(0.5, 2.0, 3)
    body2 = ellipsoid(3, axes, center=(1.0 + 3.0 + axes[0], 0.0, 0.0))
    assert body2.xyz[:, 0].min() - sphere3.xyz[:, 0].max() >= 3.0 - 1e-12
    A = H.dense()
    x = np.random.default_rng(6).standard_normal(H.nd)
    err = np.linalg.norm(A @ x - oracle.matvec(H.st, x)) / np.linalg.norm(A @ x)
    assert err < 1e-5
    u, n, hist, _ = oracle.bicgstab(H.st, b, tol=1e-8, max_iter=500, kind="restated")
    assert np.linalg.norm(b - oracle.matvec(H.st, u)) / np.linalg.norm(b) < 1.01e-8


def test_oracle_bicgstab_zero_rhs_and_limits(build_libs):
    import oracle
    H = sphere(2)
    b = np.random.default_rng(5).standard_normal(H.nd)
    u, n, hist, _ = oracle.bicgstab(H.st, b, tol=1e-30, max_iter=3, kind="restated")
    assert n == 3


def test_reference_input_end_to_end_to_vtk(build_libs, tmp_path):
    """The reference's own mesh input (bem-bb_inputs/input_1ts.pbs, ppohBEM
    kernel as in its runs) read, built, solved (CPU oracle BiCGSTAB to 1e-8)
    and written as the VTK result file of Print_result; the file reads back
    with the same points, triangles and values."""
    path = os.path.join(REFERENCE, "bem-bb_inputs", "input_1ts.pbs")
    if not os.path.exists(path):
        pytest.skip("reference mesh not available")
    import oracle
    from hacapk_b200 import abi, hmatrix
    m = hmatrix.read_pbs(path)
    H = hmatrix.HostHMatrix(m, leaf_size=15, eta=2.0, aca_eps=1e-6, kernel=abi.KERNEL_PPOHBEM)
    b = H.to_cluster(np.ones(H.nd))
    u, n, hist, _ = oracle.bicgstab(H.st, b, tol=1e-8, max_iter=500, kind="restated")
    assert hist[n] < 1e-8
    sol = H.from_cluster(u)
    out = str(tmp_path / "result.vtk")
    hmatrix.write_vtk(out, m, sol)
    xyz, tri, vals = hmatrix.read_vtk_cell_scalars(out)
    assert np.array_equal(tri, m.faces) and np.allclose(xyz, m.xyz, rtol=0, atol=1e-15)
    assert np.array_equal(vals, sol)
