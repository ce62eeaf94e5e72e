"""Shared test setup: import paths, markers, and cached problem builders."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "hacapk-magma_b200"))
sys.path.insert(0, ROOT)

# The reference tree (read only by the CPU tests that pin the oracle against
# it; absent where the GPU tests run): REFERENCE_DIR, else "reference" beside
# the repository.
REFERENCE = os.environ.get("REFERENCE_DIR", os.path.join(os.path.dirname(ROOT), "reference"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (sm_100)")


@pytest.fixture(scope="session")
def build_libs():
    """The two package libraries and the oracle are built once per session."""
    import subprocess
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "hacapk-magma_b200")], check=True)
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    return True


_cache = {}


def sphere(level, leaf_size=32, eta=2.0, aca_eps=1e-5, kernel=None):
    from hacapk_b200 import abi, hmatrix
    key = (level, leaf_size, eta, aca_eps, kernel)
    if key not in _cache:
        k = abi.KERNEL_LAPLACE if kernel is None else kernel
        _cache[key] = hmatrix.HostHMatrix(hmatrix.icosphere(level), leaf_size=leaf_size, eta=eta,
                                          aca_eps=aca_eps, kernel=k)
    return _cache[key]


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


_libs = {}


def emu_lib():
    """The test-only interpreter of the packed layout (tests/emu/plan_emu.cpp,
    linked with the product's planner), built once per session."""
    import ctypes as C
    import subprocess
    if "emu" not in _libs:
        src = os.path.join(ROOT, "tests", "emu", "plan_emu.cpp")
        lib = os.path.join(ROOT, "tests", "emu", "_build", "libplanemu.so")
        os.makedirs(os.path.dirname(lib), exist_ok=True)
        subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off", "-o", lib, src,
                        os.path.join(ROOT, "hacapk-magma_b200", "csrc", "hbx_plan.cpp")], check=True)
        L = C.CDLL(lib)
        DP = C.POINTER(C.c_double)
        L.emu_matvec_kernel_order.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, DP, C.c_double, DP, DP]
        L.emu_matvec_kernel_order_mk.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, DP, C.c_double,
                                                 DP, DP]
        L.emu_dots.argtypes = [C.c_int, C.POINTER(DP), C.POINTER(DP), C.c_size_t, DP]
        L.emu_dots.restype = None
        _libs["emu"] = L
    return _libs["emu"]


def device_dots(pairs):
    """[x . y for (x, y) in pairs], each summed as the device does
    (compensated, in the fixed block order of hbx_dots.cuh), bit for bit."""
    import ctypes as C
    import numpy as np
    L = emu_lib()
    DP = C.POINTER(C.c_double)
    k = len(pairs)
    xs = [np.ascontiguousarray(x, np.float64) for x, _ in pairs]
    ys = [np.ascontiguousarray(y, np.float64) for _, y in pairs]
    xa = (DP * k)(*[x.ctypes.data_as(DP) for x in xs])
    ya = (DP * k)(*[y.ctypes.data_as(DP) for y in ys])
    out = np.zeros(k)
    L.emu_dots(k, xa, ya, xs[0].shape[0], out.ctypes.data_as(DP))
    return [float(v) for v in out]


def kernel_order_residual(H, num_ctas=148, merge_keep=None):
    """r = b - H u in k_matvec's operation order (alpha = -1, beta = 1)."""
    import ctypes as C
    import numpy as np
    L = emu_lib()
    DP = C.POINTER(C.c_double)
    mk = engine_merge_keep() if merge_keep is None else merge_keep

    def res(b, u):
        u = np.ascontiguousarray(u, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        y = np.zeros_like(u)
        assert L.emu_matvec_kernel_order_mk(C.cast(H.st, C.c_void_p), H.nd, num_ctas, mk, -1.0,
                                            u.ctypes.data_as(DP), 1.0, b.ctypes.data_as(DP),
                                            y.ctypes.data_as(DP)) == 0
        return y
    return res


def gcr_replay(H, b, tol=1e-8, max_iter=1000, restart=8, num_ctas=148):
    """hbx_gcr's sequence on the CPU: the kernel-order product, the device's
    dot order, the vector updates as the kernels round them.  Returns (u,
    iterations, relres)."""
    import numpy as np
    mv, res = kernel_order_matvec(H, num_ctas), kernel_order_residual(H, num_ctas)
    m = restart
    u = np.zeros(H.nd)
    bnorm = np.sqrt(device_dots([(b, b)])[0])
    rel = lambda rn: rn / bnorm if bnorm > 0 else 0.0
    zr = res(b, u)
    P, AP, capap = [None] * m, [None] * m, [0.0] * m
    P[0] = zr.copy()
    zrnorm = np.sqrt(device_dots([(zr, zr)])[0])
    nstp = 0
    if not rel(zrnorm) < tol and max_iter > 0:
        AP[0] = mv(P[0])
        for it in range(1, max_iter + 1):
            ik = (it - 1) % m
            d = device_dots([(AP[ik], zr), (AP[ik], AP[ik])])
            capap[ik] = d[1]
            alpha = d[0] / d[1]
            u = u + alpha * P[ik]
            zr = zr - alpha * AP[ik]
            zrnorm = np.sqrt(device_dots([(zr, zr)])[0])
            nstp = it
            if rel(zrnorm) < tol or it == max_iter:
                break
            zar = mv(zr)
            ikn = it % m
            P[ikn], AP[ikn] = zr.copy(), zar.copy()
            d = device_dots([(AP[l], zar) for l in range(ik + 1)])
            beta = [-d[l] / capap[l] for l in range(ik + 1)]
            for l in range(ik + 1):
                P[ikn] = P[ikn] + beta[l] * P[l]
                AP[ikn] = AP[ikn] + beta[l] * AP[l]
    return u, nstp, rel(zrnorm)


def pipe_replay(H, b, tol=1e-8, max_iter=1000, num_ctas=148):
    """hbx_bicgstab_pipe's sequence on the CPU (k_pipe_init / _a / _b with the
    kernel-order product and the device's dot order).  Returns (u,
    iterations, relres, status)."""
    import numpy as np
    mv, res = kernel_order_matvec(H, num_ctas), kernel_order_residual(H, num_ctas)
    u = np.zeros(H.nd)
    r = res(b, u)
    r0 = r.copy()
    w = mv(r)
    t = mv(w)
    bb, rr, wr = device_dots([(b, b), (r, r), (w, r)])
    bnorm = np.sqrt(bb)
    znorm, alpha, beta, zeta = rr, rr / wr, 0.0, 0.0
    rel = np.sqrt(rr) / bnorm if bnorm > 0 else 0.0
    step, status = 0, 0
    if not np.isfinite(bb) or not np.isfinite(rr):
        return u, 0, rel, 7
    if rel < tol:
        return u, 0, rel, 0
    p = s = z = v = None
    while True:
        if step == 0:
            p, s, z = r.copy(), w.copy(), t.copy()
        else:
            p = beta * (p + (-zeta) * s) + r
            s, z = beta * (s + (-zeta) * z) + w, beta * (z + (-zeta) * v) + t
        q = r + (-alpha) * s
        y = w + (-alpha) * z
        yq, yy = device_dots([(y, q), (y, y)])
        zeta = yq / yy if yy != 0.0 else float("nan")
        if not np.isfinite(zeta):
            return u, step, rel, 5
        v = mv(z)
        u = (u + alpha * p) + zeta * q
        r = q + (-zeta) * y
        w = (-zeta) * (t + (-alpha) * v) + y
        d = device_dots([(r, r0), (w, r0), (s, r0), (z, r0), (r, r)])
        znormold, znorm = znorm, d[0]
        beta = (alpha / zeta) * (znorm / znormold)
        alpha = znorm / ((d[1] + beta * d[2]) - (beta * zeta) * d[3])
        rel = np.sqrt(d[4]) / bnorm if bnorm > 0 else 0.0
        step += 1
        if rel < tol:
            return u, step, rel, 0
        if not (np.isfinite(rel) and np.isfinite(alpha) and np.isfinite(beta)):
            return u, step, rel, 5
        if step >= max_iter:
            return u, step, rel, 6
        t = mv(w)


FLAT_MV = None


def flat_lib():
    """The flat solver's host loop (hbx_flat.cpp) compiled alone, callable
    with any product (hbx_test_flat_bicgstab)."""
    import ctypes as C
    import subprocess
    global FLAT_MV
    if "flat" not in _libs:
        src = os.path.join(ROOT, "hacapk-magma_b200", "csrc", "hbx_flat.cpp")
        lib = os.path.join(ROOT, "tests", "emu", "_build", "libflat.so")
        os.makedirs(os.path.dirname(lib), exist_ok=True)
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-o", lib, src],
                       check=True)
        L = C.CDLL(lib)
        DP = C.POINTER(C.c_double)
        FLAT_MV = C.CFUNCTYPE(C.c_int, C.c_void_p, DP, DP)
        L.hbx_test_flat_bicgstab.argtypes = [C.c_int, DP, DP, C.c_double, C.c_int, FLAT_MV, C.c_void_p]
        _libs["flat"] = L
    return _libs["flat"]


def kernel_order_matvec(H, num_ctas=148, merge_keep=None):
    """y = H x in the FP64 kernel's own operation order (bit for bit what
    k_matvec computes on num_ctas CTAs with the engine's block layout), on
    the CPU.  merge_keep: the planner's merged-D+U setting (None: the
    engine's default, HBX_MERGE_KEEP)."""
    import ctypes as C
    import numpy as np
    L = emu_lib()
    DP = C.POINTER(C.c_double)
    mk = engine_merge_keep() if merge_keep is None else merge_keep

    def mv(x):
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros_like(x)
        assert L.emu_matvec_kernel_order_mk(C.cast(H.st, C.c_void_p), H.nd, num_ctas, mk, 1.0,
                                            x.ctypes.data_as(DP), 0.0, None, y.ctypes.data_as(DP)) == 0
        return y
    return mv


def engine_merge_keep() -> int:
    """The merged-D+U setting the engine's planner uses (HBX_MERGE_KEEP)."""
    v = os.environ.get("HBX_MERGE_KEEP")
    return int(v) if v is not None else 4


def flat_solve(H, b, mv, tol=1e-8, max_iter=1000):
    """The flat solver's host loop driven by the product mv(x) -> H x;
    returns (u, steps)."""
    import ctypes as C
    import numpy as np
    L = flat_lib()
    n = H.nd
    DP = C.POINTER(C.c_double)

    def cb(ctx, x, y):
        xa = np.ctypeslib.as_array(x, shape=(n,)).copy()
        np.ctypeslib.as_array(y, shape=(n,))[:] = mv(xa)
        return 0

    fn = FLAT_MV(cb)
    u = np.zeros(n)
    b = np.ascontiguousarray(b, np.float64)
    steps = L.hbx_test_flat_bicgstab(n, u.ctypes.data_as(DP), b.ctypes.data_as(DP), tol, max_iter, fn, None)
    return u, steps


def reference_input_mesh():
    """The reference's own input bem-bb_inputs/input_10ts.pbs (10,400
    triangles) from its committed fixture (tests/golden/make_golden.py)."""
    import numpy as np
    from hacapk_b200 import hmatrix
    z = np.load(os.path.join(GOLDEN, "input_10ts_mesh.npz"))
    return hmatrix.Mesh(np.ascontiguousarray(z["xyz"]), np.ascontiguousarray(z["faces"]), None)
