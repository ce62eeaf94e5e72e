"""Python handle on the sm_100a engine (libhacapk_b200.so) through its C ABI.

Every call goes through the hbx_* entry points of include/hacapk_b200.h; the
library fails loudly (RuntimeError) when it is missing or when the device
reports an error.  There is no host fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi


class HbxError(RuntimeError):
    def __init__(self, status: int, where: str):
        lib = abi.engine_lib()
        msg = lib.hbx_last_error().decode(errors="replace")
        super().__init__(f"{where}: {abi.STATUS.get(status, status)}: {msg}")
        self.status = status


def _check(status: int, where: str):
    if status != 0:
        raise HbxError(status, where)


class Engine:
    """Packed H-matrix resident on the current CUDA device."""

    @staticmethod
    def autotune(st, nd: int, precision: int = 0, nrhs: int = 0, transpose: bool = False, reps: int = 20):
        """Times a grid of CTA schedules and layouts on the current device
        (hbx_autotune); returns (keyword options for Engine(...) of the
        fastest, its us, the default's us)."""
        lib = abi.engine_lib()
        base = abi.Options()
        base.precision = precision
        base.nrhs = nrhs
        base.transpose = 1 if transpose else 0
        best = abi.Options()
        tb, td = C.c_double(0.0), C.c_double(0.0)
        _check(lib.hbx_autotune(st, nd, C.byref(base), reps, C.byref(best), C.byref(tb), C.byref(td)), "hbx_autotune")
        kw = {"num_ctas": best.num_ctas, "block_cost": best.block_cost, "run_cost": best.run_cost,
              "merge": best.merge, "l2_keep_mb": best.l2_keep_mb}
        return kw, tb.value, td.value

    def __init__(self, st, nd: int, num_ctas: int = 0, transpose: bool = False, precision: int = 0,
                 nrhs: int = 0, block_cost: int = 0, run_cost: int = 0, merge: int = 0, l2_keep_mb: int = 0):
        """transpose=True packs H^T: products and solves with the adjoint.
        precision=abi.HBX_FP32 stores the factors in float (half the bytes),
        abi.HBX_BF16 in bfloat16 (a quarter).
        nrhs=abi.HBX_NRHS (with HBX_FP32) makes a multi-RHS engine: matmat only."""
        self.lib = abi.engine_lib()
        opt = abi.Options()
        opt.precision = precision
        opt.num_ctas = num_ctas
        opt.transpose = 1 if transpose else 0
        opt.nrhs = nrhs
        opt.block_cost = block_cost
        opt.run_cost = run_cost
        opt.merge = merge  # merged D+U runs: k + 1 keeps each CTA's first k atoms split; -1 none; 0 default
        opt.l2_keep_mb = l2_keep_mb  # L2 budget of the stream in MB; -1 no cache hints; 0 default
        h = C.c_void_p()
        _check(self.lib.hbx_create(st, nd, C.byref(opt), C.byref(h)), "hbx_create")
        self._h = h
        self.nd = nd
        inf = abi.Info()
        _check(self.lib.hbx_get_info(h, C.byref(inf)), "hbx_get_info")
        self.info = {f: getattr(inf, f) for f, _ in abi.Info._fields_ if f != "reserved"}

    @classmethod
    def batch(cls, hmats, num_ctas: int = 0, precision: int = 0) -> "Engine":
        """One engine over independent H-matrices (objects with .st and .nd):
        block-diagonal, instance k at rows off[k]..off[k+1] (self.offsets)."""
        self = cls.__new__(cls)
        self.lib = abi.engine_lib()
        opt = abi.Options()
        opt.precision = precision
        opt.num_ctas = num_ctas
        k = len(hmats)
        sts = (C.POINTER(abi.LeafMtxP) * k)(*[C.cast(H.st, C.POINTER(abi.LeafMtxP)) for H in hmats])
        nds = (C.c_int * k)(*[int(H.nd) for H in hmats])
        h = C.c_void_p()
        _check(self.lib.hbx_create_batch(sts, nds, k, C.byref(opt), C.byref(h)), "hbx_create_batch")
        self._h = h
        self.offsets = np.concatenate([[0], np.cumsum([int(H.nd) for H in hmats])]).astype(np.int64)
        self.nd = int(self.offsets[-1])
        inf = abi.Info()
        _check(self.lib.hbx_get_info(h, C.byref(inf)), "hbx_get_info")
        self.info = {f: getattr(inf, f) for f, _ in abi.Info._fields_ if f != "reserved"}
        return self

    def bicgstab_batch_host(self, b: np.ndarray, u0: np.ndarray | None = None, tol: float = 1e-8,
                            max_iter: int = 1000, batch: int = 0):
        """Every instance of a batch engine solved at once; returns (u, [info per instance])."""
        b = np.ascontiguousarray(b, np.float64)
        u = np.zeros(self.nd) if u0 is None else np.array(u0, np.float64, copy=True)
        k = self.info["instances"]
        infos = (abi.SolveInfo * k)()
        o = self._opts(tol, max_iter, 0, batch)
        st = self.lib.hbx_bicgstab_batch_host(self._h, abi.dptr(b), abi.dptr(u), C.byref(o), infos)
        if st not in (0, 5, 6):
            _check(st, "hbx_bicgstab_batch_host")
        return u, [self._info(infos[j]) for j in range(k)]

    def bicgstab_batch_dev(self, b_ptr: int, u_ptr: int, tol: float = 1e-8, max_iter: int = 1000, batch: int = 0,
                           stream: int = 0, check: bool = True):
        k = self.info["instances"]
        infos = (abi.SolveInfo * k)()
        o = self._opts(tol, max_iter, 0, batch)
        st = self.lib.hbx_bicgstab_batch(self._h, C.c_void_p(b_ptr), C.c_void_p(u_ptr), C.byref(o), infos,
                                         C.c_void_p(stream) if stream else None)
        if check:
            _check(st, "hbx_bicgstab_batch")
        return [self._info(infos[j]) for j in range(k)]

    def bicgstab_batch_refined_host(self, low: "Engine", b: np.ndarray, u0: np.ndarray | None = None,
                                    tol: float = 1e-8, max_iter: int = 1000, inner_tol: float = 0.0, batch: int = 0):
        """Every instance solved at once to an FP64-verified tol, the
        corrections on `low` (an FP32 / BF16 batch engine of the same
        instances); returns (u, [info per instance])."""
        b = np.ascontiguousarray(b, np.float64)
        u = np.zeros(self.nd) if u0 is None else np.array(u0, np.float64, copy=True)
        k = self.info["instances"]
        infos = (abi.SolveInfo * k)()
        o = self._opts(tol, max_iter, 0, batch, inner_tol)
        st = self.lib.hbx_bicgstab_batch_refined_host(self._h, low._h, abi.dptr(b), abi.dptr(u), C.byref(o), infos)
        if st not in (0, 5, 6):
            _check(st, "hbx_bicgstab_batch_refined_host")
        return u, [self._info(infos[j]) for j in range(k)]

    def bicgstab_batch_refined_dev(self, low: "Engine", b_ptr: int, u_ptr: int, tol: float = 1e-8,
                                   max_iter: int = 1000, inner_tol: float = 0.0, batch: int = 0, stream: int = 0,
                                   check: bool = True):
        k = self.info["instances"]
        infos = (abi.SolveInfo * k)()
        o = self._opts(tol, max_iter, 0, batch, inner_tol)
        st = self.lib.hbx_bicgstab_batch_refined(self._h, low._h, C.c_void_p(b_ptr), C.c_void_p(u_ptr), C.byref(o),
                                                 infos, C.c_void_p(stream) if stream else None)
        if check:
            _check(st, "hbx_bicgstab_batch_refined")
        return [self._info(infos[j]) for j in range(k)]

    def close(self):
        if getattr(self, "_h", None):
            self.lib.hbx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- matvec -------------------------------------------------------------
    def matvec_host(self, zu: np.ndarray, zau: np.ndarray | None = None):
        """zau + H zu (zau=None: H zu) with host vectors; returns (y, kernel_s, copy_s)."""
        zu = np.ascontiguousarray(zu, np.float64)
        acc = zau is not None
        y = np.array(zau, np.float64, copy=True) if acc else np.zeros(self.nd)
        tk, tc = C.c_double(0.0), C.c_double(0.0)
        _check(self.lib.hbx_matvec_host(self._h, abi.dptr(zu), abi.dptr(y), 1 if acc else 0,
                                        C.byref(tk), C.byref(tc)), "hbx_matvec_host")
        return y, tk.value, tc.value

    def matvec_dev(self, x_ptr: int, y_ptr: int, alpha: float = 1.0, beta: float = 0.0,
                   yin_ptr: int | None = None, stream: int = 0):
        """y = alpha H x + beta yin on device pointers (async on `stream`)."""
        _check(self.lib.hbx_matvec(self._h, alpha, C.c_void_p(x_ptr), beta,
                                   C.c_void_p(yin_ptr) if yin_ptr else None, C.c_void_p(y_ptr),
                                   C.c_void_p(stream) if stream else None), "hbx_matvec")

    def matmat_dev(self, x_ptr: int, y_ptr: int, alpha: float = 1.0, beta: float = 0.0,
                   yin_ptr: int | None = None, stream: int = 0):
        """Y = alpha H X + beta Yin for HBX_NRHS right-hand sides: X nd x 64
        floats, Y (and Yin) nd x 64 doubles, row-major device arrays."""
        _check(self.lib.hbx_matmat(self._h, alpha, C.c_void_p(x_ptr), beta,
                                   C.c_void_p(yin_ptr) if yin_ptr else None, C.c_void_p(y_ptr),
                                   C.c_void_p(stream) if stream else None), "hbx_matmat")

    def bicgstab_multi_host(self, multi: "Engine", B: np.ndarray, U0: np.ndarray | None = None, tol: float = 1e-8,
                            max_iter: int = 1000, inner_tol: float = 0.0, batch: int = 0):
        """Solves H U = B for HBX_NRHS right-hand sides (B: nd x 64) with
        this FP64 engine for the refinement residuals and `multi` (a multi-RHS
        engine) for the inner products; returns (U, [info dict per RHS])."""
        B = np.ascontiguousarray(B, np.float64)
        U = np.zeros_like(B) if U0 is None else np.array(U0, np.float64, copy=True, order="C")
        infos = (abi.SolveInfo * abi.HBX_NRHS)()
        o = self._opts(tol, max_iter, 0, batch, inner_tol)
        st = self.lib.hbx_bicgstab_multi_host(self._h, multi._h, abi.dptr(B), abi.dptr(U), C.byref(o), infos)
        res = [self._info(infos[j]) for j in range(abi.HBX_NRHS)]
        if st not in (0, 5, 6):
            _check(st, "hbx_bicgstab_multi_host")
        return U, res

    def bicgstab_multi_dev(self, multi: "Engine", B_ptr: int, U_ptr: int, tol: float = 1e-8, max_iter: int = 1000,
                           inner_tol: float = 0.0, batch: int = 0, stream: int = 0, check: bool = True):
        """Device-array form of bicgstab_multi_host (nd x 64 row-major doubles)."""
        infos = (abi.SolveInfo * abi.HBX_NRHS)()
        o = self._opts(tol, max_iter, 0, batch, inner_tol)
        st = self.lib.hbx_bicgstab_multi(self._h, multi._h, C.c_void_p(B_ptr), C.c_void_p(U_ptr), C.byref(o), infos,
                                         C.c_void_p(stream) if stream else None)
        if check:
            _check(st, "hbx_bicgstab_multi")
        return [self._info(infos[j]) for j in range(abi.HBX_NRHS)]

    def sync(self, stream: int = 0):
        _check(self.lib.hbx_sync(self._h, C.c_void_p(stream) if stream else None), "hbx_sync")

    # -- BiCGSTAB -------------------------------------------------------------
    @staticmethod
    def _opts(tol, max_iter, verbose, batch, inner_tol=0.0):
        o = abi.SolveOpts()
        o.tol = tol
        o.max_iter = max_iter
        o.verbose = verbose
        o.batch = batch
        o.inner_tol = inner_tol
        return o

    @staticmethod
    def _info(si: abi.SolveInfo) -> dict:
        return {f: getattr(si, f) for f, _ in abi.SolveInfo._fields_ if f != "reserved"}

    def bicgstab_host(self, b: np.ndarray, u0: np.ndarray | None = None, tol: float = 1e-8,
                      max_iter: int = 1000, verbose: int = 0, batch: int = 8, check: bool = True,
                      inplace: bool = False):
        """Solve with host vectors; u0 is copied unless inplace=True (then u0,
        a contiguous float64 array, receives the solution)."""
        b = np.ascontiguousarray(b, np.float64)
        if inplace:
            u = u0
        else:
            u = np.zeros(self.nd) if u0 is None else np.array(u0, np.float64, copy=True)
        o = self._opts(tol, max_iter, verbose, batch)
        si = abi.SolveInfo()
        st = self.lib.hbx_bicgstab_host(self._h, abi.dptr(b), abi.dptr(u), C.byref(o), C.byref(si))
        if check:
            _check(st, "hbx_bicgstab_host")
        return u, self._info(si)

    def bicgstab_dev(self, b_ptr: int, u_ptr: int, tol: float = 1e-8, max_iter: int = 1000,
                     verbose: int = 0, batch: int = 8, stream: int = 0, check: bool = True) -> dict:
        o = self._opts(tol, max_iter, verbose, batch)
        si = abi.SolveInfo()
        st = self.lib.hbx_bicgstab(self._h, C.c_void_p(b_ptr), C.c_void_p(u_ptr), C.byref(o),
                                   C.byref(si), C.c_void_p(stream) if stream else None)
        if check:
            _check(st, "hbx_bicgstab")
        return self._info(si)

    # -- pipelined BiCGSTAB ----------------------------------------------------
    def bicgstab_pipe_host(self, b: np.ndarray, u0: np.ndarray | None = None, tol: float = 1e-8,
                           max_iter: int = 1000, verbose: int = 0, batch: int = 8, check: bool = True):
        """Pipelined BiCGSTAB (HACApK_SOLVER_PIPE.c:144-600) with host vectors;
        returns (u, info)."""
        b = np.ascontiguousarray(b, np.float64)
        u = np.zeros(self.nd) if u0 is None else np.array(u0, np.float64, copy=True)
        o = self._opts(tol, max_iter, verbose, batch)
        si = abi.SolveInfo()
        st = self.lib.hbx_bicgstab_pipe_host(self._h, abi.dptr(b), abi.dptr(u), C.byref(o), C.byref(si))
        if check:
            _check(st, "hbx_bicgstab_pipe_host")
        return u, self._info(si)

    def bicgstab_pipe_dev(self, b_ptr: int, u_ptr: int, tol: float = 1e-8, max_iter: int = 1000,
                          verbose: int = 0, batch: int = 8, stream: int = 0, check: bool = True) -> dict:
        o = self._opts(tol, max_iter, verbose, batch)
        si = abi.SolveInfo()
        st = self.lib.hbx_bicgstab_pipe(self._h, C.c_void_p(b_ptr), C.c_void_p(u_ptr), C.byref(o), C.byref(si),
                                        C.c_void_p(stream) if stream else None)
        if check:
            _check(st, "hbx_bicgstab_pipe")
        return self._info(si)

    # -- GCR(m) ----------------------------------------------------------------
    def gcr_host(self, b: np.ndarray, u0: np.ndarray | None = None, tol: float = 1e-8, max_iter: int = 1000,
                 restart: int = 8, check: bool = True):
        """GCR(restart) of HACApK_gcrm_lfmtx (m_HACApK_solve.f90:506-571) with
        host vectors; returns (u, info)."""
        b = np.ascontiguousarray(b, np.float64)
        u = np.zeros(self.nd) if u0 is None else np.array(u0, np.float64, copy=True)
        o = self._opts(tol, max_iter, 0, 0)
        o.restart = restart
        si = abi.SolveInfo()
        st = self.lib.hbx_gcr_host(self._h, abi.dptr(b), abi.dptr(u), C.byref(o), C.byref(si))
        if check:
            _check(st, "hbx_gcr_host")
        return u, self._info(si)

    def gcr_dev(self, b_ptr: int, u_ptr: int, tol: float = 1e-8, max_iter: int = 1000, restart: int = 8,
                stream: int = 0, check: bool = True) -> dict:
        o = self._opts(tol, max_iter, 0, 0)
        o.restart = restart
        si = abi.SolveInfo()
        st = self.lib.hbx_gcr(self._h, C.c_void_p(b_ptr), C.c_void_p(u_ptr), C.byref(o), C.byref(si),
                              C.c_void_p(stream) if stream else None)
        if check:
            _check(st, "hbx_gcr")
        return self._info(si)

    def gradient_host(self, adjoint: "Engine", g: np.ndarray, sigma_t: np.ndarray, tol: float = 1e-8,
                      max_iter: int = 1000):
        """dJ/dg for J = 0.5||sigma - sigma_t||^2 with H sigma = g (self holds H,
        `adjoint` holds H^T).  Returns (J, grad, sigma, forward info, adjoint info)."""
        g = np.ascontiguousarray(g, np.float64)
        sigma_t = np.ascontiguousarray(sigma_t, np.float64)
        sigma = np.zeros(self.nd)
        grad = np.zeros(self.nd)
        J = C.c_double(0.0)
        o = self._opts(tol, max_iter, 0, 8)
        fi, ai = abi.SolveInfo(), abi.SolveInfo()
        _check(self.lib.hbx_gradient_host(self._h, adjoint._h, abi.dptr(g), abi.dptr(sigma_t), abi.dptr(sigma),
                                          abi.dptr(grad), C.byref(J), C.byref(o), C.byref(fi), C.byref(ai)),
               "hbx_gradient_host")
        return J.value, grad, sigma, self._info(fi), self._info(ai)

    # -- mixed precision --------------------------------------------------------
    def bicgstab_refined_host(self, low: "Engine", b: np.ndarray, u0: np.ndarray | None = None, tol: float = 1e-8,
                              max_iter: int = 1000, inner_tol: float = 0.0, check: bool = True):
        """FP64 iterative refinement (self: FP64 engine) around BiCGSTAB on
        `low` (an FP32 or BF16 engine of the same matrix); host vectors."""
        b = np.ascontiguousarray(b, np.float64)
        u = np.zeros(self.nd) if u0 is None else np.array(u0, np.float64, copy=True)
        o = self._opts(tol, max_iter, 0, 8, inner_tol)
        si = abi.SolveInfo()
        st = self.lib.hbx_bicgstab_refined_host(self._h, low._h, abi.dptr(b), abi.dptr(u), C.byref(o), C.byref(si))
        if check:
            _check(st, "hbx_bicgstab_refined_host")
        return u, self._info(si)

    def bicgstab_refined_dev(self, low: "Engine", b_ptr: int, u_ptr: int, tol: float = 1e-8, max_iter: int = 1000,
                             inner_tol: float = 0.0, stream: int = 0, check: bool = True) -> dict:
        o = self._opts(tol, max_iter, 0, 8, inner_tol)
        si = abi.SolveInfo()
        st = self.lib.hbx_bicgstab_refined(self._h, low._h, C.c_void_p(b_ptr), C.c_void_p(u_ptr), C.byref(o),
                                           C.byref(si), C.c_void_p(stream) if stream else None)
        if check:
            _check(st, "hbx_bicgstab_refined")
        return self._info(si)
