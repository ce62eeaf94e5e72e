"""TEST INFRASTRUCTURE ONLY -- the CPU checker.

ctypes bindings to
  * oracle/_ref/libhacapk_ref.so: the reference's own CPU H-matvec
    c_hacapk_adot_body_lfmtx_ (HACApK_MAGMA.c:5-57), compiled from the
    reference sources by oracle/Makefile;
  * oracle/liboracle.so: the C restatement in oracle.c (matvec, per-leaf BLAS
    matvec, OpenMP "_hyp" matvec, transposed matvec, BiCGSTAB of
    HACApK_SOLVER.c:254-417, pipelined BiCGSTAB of HACApK_SOLVER_PIPE.c:144-600,
    GCR(m) of m_HACApK_solve.f90:506-571).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
The product library never links or calls anything here.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(_HERE, "liboracle.so")
REF_LIB = os.path.join(_HERE, "_ref", "libhacapk_ref.so")

_DP = C.POINTER(C.c_double)
_VP = C.c_void_p

MV_REF, MV_BLAS, MV_OMP, MV_EXTERNAL = 0, 1, 2, 3

_lib = None
_ref = None


def build():
    """Compiles the checker (and oracle/_ref when the reference tree exists)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_LIB):
            build()
        L = C.CDLL(ORACLE_LIB)
        L.orc_adot_lfmtx.argtypes = [_DP, _VP, _DP, _DP]
        L.orc_adot_lfmtx_blas.argtypes = [_DP, _VP, _DP, _DP, _VP]
        L.orc_adot_lfmtx_omp.argtypes = [_DP, _VP, _DP, C.c_int]
        L.orc_adot_lfmtx_t.argtypes = [_DP, _VP, _DP, _DP]
        L.orc_bicgstab.argtypes = [_VP, C.c_int, _DP, _DP, C.c_double, C.c_int, C.c_int, _VP,
                                   _VP, C.c_int, _DP, _DP]
        L.orc_bicgstab.restype = C.c_int
        L.orc_bicgstab_pipe.argtypes = L.orc_bicgstab.argtypes
        L.orc_bicgstab_pipe.restype = C.c_int
        L.orc_gcrm.argtypes = [_VP, C.c_int, _DP, _DP, C.c_double, C.c_int, C.c_int, C.c_int, _VP,
                               _VP, C.c_int, _DP, _DP]
        L.orc_gcrm.restype = C.c_int
        for f in ("orc_adot_lfmtx", "orc_adot_lfmtx_blas", "orc_adot_lfmtx_omp", "orc_adot_lfmtx_t"):
            getattr(L, f).restype = None
        _lib = L
    return _lib


def have_ref() -> bool:
    return os.path.exists(REF_LIB)


def ref_lib() -> C.CDLL:
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB):
            raise RuntimeError("oracle/_ref/libhacapk_ref.so is not built (needs the reference tree)")
        R = C.CDLL(REF_LIB)
        R.c_hacapk_adot_body_lfmtx_.argtypes = [_DP, _VP, _DP, _DP]
        R.c_hacapk_adot_body_lfmtx_.restype = None
        _ref = R
    return _ref


def _st(st):
    return C.cast(st, _VP)


class _CompactLeafMtxP(C.Structure):
    """The container as the reference compiles it WITHOUT HAVE_MAGMA
    (HACApK_MAGMA.h:28-32 then :104): the GPU/batch block is absent, so
    st_lf follows st_lf_stride directly.  The compiled reference matvec is
    built that way (MAGMA is not available here), so it is handed this view
    of the same leaves."""
    _fields_ = [("nd", C.c_int), ("nlf", C.c_int), ("nlfkt", C.c_int), ("ktmax", C.c_int),
                ("st_lf_stride", C.c_int), ("st_lf", C.c_void_p)]


def _compact(st):
    s = st.contents
    return _CompactLeafMtxP(s.nd, s.nlf, s.nlfkt, s.ktmax, s.st_lf_stride,
                            C.cast(s.st_lf, C.c_void_p))


def _d(a):
    return a.ctypes.data_as(_DP)


def _work(st):
    return np.zeros(max(1, int(st.contents.ktmax)), np.float64)


def matvec_ref(st, zu: np.ndarray, zau: np.ndarray | None = None) -> np.ndarray:
    """zau + H zu with the reference's own compiled c_hacapk_adot_body_lfmtx_."""
    zu = np.ascontiguousarray(zu, np.float64)
    out = np.zeros_like(zu) if zau is None else np.array(zau, np.float64, copy=True)
    cst = _compact(st)
    ref_lib().c_hacapk_adot_body_lfmtx_(_d(out), C.cast(C.byref(cst), _VP), _d(zu), _d(_work(st)))
    return out


def matvec(st, zu, zau=None) -> np.ndarray:
    zu = np.ascontiguousarray(zu, np.float64)
    out = np.zeros_like(zu) if zau is None else np.array(zau, np.float64, copy=True)
    lib().orc_adot_lfmtx(_d(out), _st(st), _d(zu), _d(_work(st)))
    return out


def matvec_t(st, zu, zau=None) -> np.ndarray:
    """zau + H^T zu."""
    zu = np.ascontiguousarray(zu, np.float64)
    out = np.zeros_like(zu) if zau is None else np.array(zau, np.float64, copy=True)
    lib().orc_adot_lfmtx_t(_d(out), _st(st), _d(zu), _d(_work(st)))
    return out


def matvec_omp(st, zu, zau=None, nthreads: int = 0) -> np.ndarray:
    zu = np.ascontiguousarray(zu, np.float64)
    out = np.zeros_like(zu) if zau is None else np.array(zau, np.float64, copy=True)
    lib().orc_adot_lfmtx_omp(_d(out), _st(st), _d(zu), nthreads)
    return out


def dgemv_pointer() -> int:
    """Address of OpenBLAS dgemv as bundled with scipy (stands in for MKL)."""
    from scipy.linalg import cython_blas
    cap = cython_blas.__pyx_capi__["dgemv"]
    get_name = C.pythonapi.PyCapsule_GetName
    get_name.restype = C.c_char_p
    get_name.argtypes = [C.py_object]
    get_ptr = C.pythonapi.PyCapsule_GetPointer
    get_ptr.restype = C.c_void_p
    get_ptr.argtypes = [C.py_object, C.c_char_p]
    return get_ptr(cap, get_name(cap))


def matvec_blas(st, zu, zau=None) -> np.ndarray:
    zu = np.ascontiguousarray(zu, np.float64)
    out = np.zeros_like(zu) if zau is None else np.array(zau, np.float64, copy=True)
    lib().orc_adot_lfmtx_blas(_d(out), _st(st), _d(zu), _d(_work(st)), C.c_void_p(dgemv_pointer()))
    return out


def gcrm(st, b: np.ndarray, u0: np.ndarray | None = None, tol: float = 1e-8, max_iter: int = 1000,
         restart: int = 8, kind: str = "ref", nthreads: int = 0):
    """GCR(m) of m_HACApK_solve.f90:506-571 on the CPU (restart m = param(87),
    8 by default).  kind: 'ref', 'restated', 'omp'.  Returns (u, nstp,
    hist[0..nstp], matvec_seconds)."""
    nd = int(b.shape[0])
    b = np.ascontiguousarray(b, np.float64)
    u = np.zeros(nd) if u0 is None else np.array(u0, np.float64, copy=True)
    hist = np.zeros(max_iter + 1)
    secs = C.c_double(0.0)
    fn = None
    cst = _compact(st)
    if kind == "ref":
        mk = MV_EXTERNAL
        fn = C.cast(ref_lib().c_hacapk_adot_body_lfmtx_, C.c_void_p)
    elif kind == "omp":
        mk = MV_OMP
    else:
        mk = MV_REF
    n = lib().orc_gcrm(_st(st), nd, _d(u), _d(b), tol, max_iter, restart, mk, fn, C.cast(C.byref(cst), _VP),
                       nthreads, _d(hist), C.byref(secs))
    return u, int(n), hist[: n + 1].copy(), secs.value


def bicgstab_pipe(st, b: np.ndarray, u0: np.ndarray | None = None, tol: float = 1e-8, max_iter: int = 1000,
                  kind: str = "ref", nthreads: int = 0):
    """Pipelined BiCGSTAB of HACApK_SOLVER_PIPE.c:144-600 on the CPU (the
    iterate accumulates in u).  kind: 'ref', 'restated', 'omp'.  Returns (u,
    nstp, hist[0..nstp], matvec_seconds)."""
    nd = int(b.shape[0])
    b = np.ascontiguousarray(b, np.float64)
    u = np.zeros(nd) if u0 is None else np.array(u0, np.float64, copy=True)
    hist = np.zeros(max_iter + 1)
    secs = C.c_double(0.0)
    fn = None
    cst = _compact(st)
    if kind == "ref":
        mk = MV_EXTERNAL
        fn = C.cast(ref_lib().c_hacapk_adot_body_lfmtx_, C.c_void_p)
    elif kind == "omp":
        mk = MV_OMP
    else:
        mk = MV_REF
    n = lib().orc_bicgstab_pipe(_st(st), nd, _d(u), _d(b), tol, max_iter, mk, fn, C.cast(C.byref(cst), _VP),
                                nthreads, _d(hist), C.byref(secs))
    return u, int(n), hist[: n + 1].copy(), secs.value


def bicgstab(st, b: np.ndarray, u0: np.ndarray | None = None, tol: float = 1e-8,
             max_iter: int = 1000, kind: str = "ref", nthreads: int = 0):
    """BiCGSTAB of HACApK_SOLVER.c:254-417 on the CPU.

    kind: 'ref' (compiled reference matvec), 'restated', 'blas', 'omp'.
    Returns (u, nstp, hist[0..nstp], matvec_seconds)."""
    nd = int(b.shape[0])
    b = np.ascontiguousarray(b, np.float64)
    u = np.zeros(nd) if u0 is None else np.array(u0, np.float64, copy=True)
    hist = np.zeros(max_iter + 1)
    secs = C.c_double(0.0)
    fn = None
    cst = _compact(st)
    if kind == "ref":
        mk = MV_EXTERNAL
        fn = C.cast(ref_lib().c_hacapk_adot_body_lfmtx_, C.c_void_p)
    elif kind == "blas":
        mk, fn = MV_BLAS, C.c_void_p(dgemv_pointer())
    elif kind == "omp":
        mk = MV_OMP
    else:
        mk = MV_REF
    n = lib().orc_bicgstab(_st(st), nd, _d(u), _d(b), tol, max_iter, mk, fn,
                           C.cast(C.byref(cst), _VP), nthreads, _d(hist), C.byref(secs))
    return u, int(n), hist[: n + 1].copy(), secs.value
