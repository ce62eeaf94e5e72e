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
