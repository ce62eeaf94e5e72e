"""Row-partitioned H-matvec across ranks: the reference's MPI scheme.

* Row cuts at leaf row starts, balanced by stored words (HACApK_setcutrow,
  m_HACApK_base.f90:540-581): walking the leaves in row order, a cut is set
  at the first row of the leaf whose cumulative words pass the next multiple
  of total / nranks.  The reference balances before the fill with a nominal
  rank for every low-rank leaf; here the leaves are filled, so their own
  ranks are counted.
* Each rank keeps the leaves whose first row lies in its range
  (HACApK_generate_frame_leafmtx, m_HACApK_base.f90:511-521) and multiplies
  them on its own device.
* The combination of the ranks' products.  The reference all-gathers the
  owned row segments (MPI_Allgatherv, HACApK_SOLVER.c:106-251).  A leaf that
  starts in one range can reach rows below it, into the next ranges, so a
  rank's product also holds rows it does not own (its spill, usually a few
  leaves' worth).  Two collectives per product: the spills are all-gathered
  (padded to the longest), every rank adds the spills that reach its own
  rows to its own rows in rank order, and the owned segments are
  all-gathered (padded to the longest).  Per product a rank sends and
  receives about N + world * (longest spill) values, against world * N for
  gathering full-length partial products, and every rank holds the same
  vector, bit for bit, on every run.  The vectors of the solve are
  replicated, as in the reference's flat solver.

The local product is a callable built by a factory, so the same plumbing runs
an engine per GPU over NCCL or the CPU checker over gloo.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable

import numpy as np

from . import abi


def _leaf_ptr(st, ip: int) -> abi.LeafMtx:
    c = st.contents
    base = C.cast(c.st_lf, C.c_void_p).value
    return abi.LeafMtx.from_address(base + ip * c.st_lf_stride)


def leaf_words(L: abi.LeafMtx) -> int:
    """Stored words of a leaf: ndl*ndt dense, kt*(ndl+ndt) low-rank."""
    return int(L.ndl) * int(L.ndt) if L.ltmtx == 2 else int(L.kt) * (int(L.ndl) + int(L.ndt))


def row_cuts(st, nd: int, nranks: int) -> list[int]:
    """cuts[0] = 0 < ... < cuts[nranks] = nd; rank r owns rows [cuts[r], cuts[r+1])."""
    nlf = st.contents.nlf
    leaves = [_leaf_ptr(st, ip) for ip in range(nlf)]
    order = sorted(range(nlf), key=lambda ip: (leaves[ip].nstrtl, leaves[ip].nstrtt))
    total = sum(leaf_words(L) for L in leaves)
    per = total // max(1, nranks)
    cuts = [0] * (nranks + 1)
    cuts[nranks] = nd
    acc, ip_cut = 0, 1
    for ip in order:
        L = leaves[ip]
        acc += leaf_words(L)
        if ip_cut < nranks and acc > per * ip_cut and L.nstrtl - 1 > cuts[ip_cut - 1]:
            cuts[ip_cut] = L.nstrtl - 1
            ip_cut += 1
    for r in range(ip_cut, nranks):  # fewer leaf starts than ranks: empty ranges at the end
        cuts[r] = nd
    return cuts


class LeafSubset:
    """A leaf list holding the leaves of `st` whose first row (0-based) lies in
    [r0, r1), in the reference C layout; the factors are not copied."""

    def __init__(self, st, nd: int, r0: int, r1: int):
        c = st.contents
        keep = [ip for ip in range(c.nlf) if r0 <= _leaf_ptr(st, ip).nstrtl - 1 < r1]
        self._arr = (abi.LeafMtx * max(1, len(keep)))()
        for k, ip in enumerate(keep):
            C.memmove(C.addressof(self._arr[k]), C.addressof(_leaf_ptr(st, ip)), C.sizeof(abi.LeafMtx))
        self._cont = abi.LeafMtxP()
        self._cont.nd = nd
        self._cont.nlf = len(keep)
        self._cont.nlfkt = sum(1 for ip in keep if _leaf_ptr(st, ip).ltmtx == 1)
        self._cont.ktmax = max([_leaf_ptr(st, ip).kt for ip in keep] + [0])
        self._cont.st_lf_stride = C.sizeof(abi.LeafMtx)
        self._cont.st_lf = C.cast(self._arr, C.POINTER(abi.LeafMtx))
        self.st = C.pointer(self._cont)
        self.nd = nd
        self.nlf = len(keep)


class RowPartitionedMatvec:
    """y = H x with the leaves split over the ranks of a torch.distributed
    group.  `local_factory(st, nd)` returns the rank's product x -> y over its
    own leaves (full-length y, zero on rows none of them touch); x and y are
    torch tensors on the rank's device (CPU for gloo, CUDA for NCCL)."""

    def __init__(self, st, nd: int, local_factory: Callable, group=None):
        import torch.distributed as dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.cuts = row_cuts(st, nd, self.world)
        # reach[r]: one past the last row a leaf of rank r touches
        self.reach = list(self.cuts[1:])
        for ip in range(st.contents.nlf):
            L = _leaf_ptr(st, ip)
            r0 = L.nstrtl - 1
            r = next(k for k in range(self.world) if self.cuts[k] <= r0 < self.cuts[k + 1])
            self.reach[r] = max(self.reach[r], r0 + L.ndl)
        self.spill = [self.reach[r] - self.cuts[r + 1] for r in range(self.world)]
        self.max_spill = max(self.spill)
        self.max_own = max(self.cuts[r + 1] - self.cuts[r] for r in range(self.world))
        self.subset = LeafSubset(st, nd, self.cuts[self.rank], self.cuts[self.rank + 1])
        self.local = local_factory(self.subset.st, nd)
        self.nd = nd
        # values a rank sends per product (spill window, then owned segment)
        self.exchange_values = self.max_spill + self.max_own

    def __call__(self, x):
        import torch
        import torch.distributed as dist
        y = self.local(x)
        me, c = self.rank, self.cuts
        own = y[c[me]:c[me + 1]].clone()
        if self.max_spill > 0:
            mine = torch.zeros(self.max_spill, dtype=y.dtype, device=y.device)
            mine[:self.spill[me]] = y[c[me + 1]:self.reach[me]]
            spills = [torch.empty_like(mine) for _ in range(self.world)]
            dist.all_gather(spills, mine, group=self.group)
            for r in range(me):  # rank order: the same sum on every run
                lo, hi = max(c[r + 1], c[me]), min(self.reach[r], c[me + 1])
                if lo < hi:
                    own[lo - c[me]:hi - c[me]] += spills[r][lo - c[r + 1]:hi - c[r + 1]]
        seg = torch.zeros(self.max_own, dtype=y.dtype, device=y.device)
        seg[:own.numel()] = own
        segs = [torch.empty_like(seg) for _ in range(self.world)]
        dist.all_gather(segs, seg, group=self.group)
        return torch.cat([segs[r][:c[r + 1] - c[r]] for r in range(self.world)])


def engine_product(st, nd: int):
    """Local product of one rank on its GPU: an engine over the rank's leaves."""
    import torch
    from .engine import Engine
    E = Engine(st, nd)

    def prod(x):
        y = torch.empty_like(x)
        E.matvec_dev(x.data_ptr(), y.data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
        return y
    prod.engine = E
    return prod


def bicgstab(matvec: Callable, b, tol: float = 1e-8, max_iter: int = 1000):
    """BiCGSTAB of HACApK_SOLVER.c:254-417 on replicated vectors (torch
    tensors), the product given by `matvec`; returns (u, steps, relres).  A
    breakdown (a zero denominator) ends the loop with the last iterate, whose
    relres then stays at or above tol."""
    import torch
    u = torch.zeros_like(b)
    r = b - matvec(u)
    rh = r.clone()
    p = torch.zeros_like(b)
    ap = torch.zeros_like(b)
    bnorm = float(torch.linalg.norm(b))
    if bnorm == 0.0:  # u = 0 solves it (whatever tol)
        return u, 0, 0.0
    rho_old = alpha = zeta = 1.0
    steps = 0
    relres = float(torch.linalg.norm(r)) / bnorm if bnorm > 0 else 0.0
    while relres >= tol and steps < max_iter:
        if steps > 0 and (zeta == 0.0 or rho_old == 0.0):
            break
        rho = float(torch.dot(rh, r))
        if steps == 0:
            p = r.clone()
        else:
            beta = (alpha / zeta) * (rho / rho_old)
            p = r + beta * (p - zeta * ap)
        ap = matvec(p)
        den = float(torch.dot(rh, ap))
        if den == 0.0:
            break
        alpha = rho / den
        t = r - alpha * ap
        at = matvec(t)
        aa = float(torch.dot(at, at))
        zeta = float(torch.dot(at, t)) / aa if aa != 0.0 else 0.0
        u = u + alpha * p + zeta * t
        r = t - zeta * at
        rho_old = rho
        steps += 1
        relres = float(torch.linalg.norm(r)) / bnorm
    return u, steps, relres


def diagonal_scaling(st, nd: int) -> np.ndarray:
    """1/sqrt(|a_ii|) from the diagonal of the leaves that sit on the diagonal
    (nstrtl == nstrtt, dense), the right scaling of the pipelined solver of
    HACApK_SOLVER_PIPE.c:233-253 (1 where no dense diagonal leaf covers a row)."""
    d = np.zeros(nd)
    for ip in range(st.contents.nlf):
        L = _leaf_ptr(st, ip)
        if L.ltmtx == 2 and L.nstrtl == L.nstrtt and L.ndl > 0:
            a = np.ctypeslib.as_array(L.a1, shape=(L.ndl * L.ndt,))
            n = min(L.ndl, L.ndt)
            d[L.nstrtl - 1:L.nstrtl - 1 + n] = a[np.arange(n) * (L.ndt + 1)]
    out = np.ones(nd)
    nz = d != 0.0
    out[nz] = 1.0 / np.sqrt(np.abs(d[nz]))
    return out


def bicgstab_pipelined(matvec: Callable, b, tol: float = 1e-8, max_iter: int = 1000, scale=None):
    """Pipelined BiCGSTAB of HACApK_SOLVER_PIPE.c:144-600 ("version 1") on
    replicated vectors (torch tensors): the products of the auxiliary vectors
    s = A p and z = A s are carried by recurrences, so a step has two
    products (v = A z and t = A w) and two reduction points (zeta, then five
    dot products for beta and alpha) instead of four.  `scale` (a tensor,
    e.g. diagonal_scaling) applies the reference's right scaling: the solver
    iterates on A diag(scale) and returns u = diag(scale) x.  Returns
    (u, steps, relres) with relres the recursive residual.  A breakdown (a
    zero denominator) ends the loop with the last iterate."""
    import torch
    D = scale if scale is not None else None
    op = (lambda v: matvec(D * v)) if D is not None else matvec
    x = torch.zeros_like(b)
    if float(torch.linalg.norm(b)) == 0.0:  # u = 0 solves it (whatever tol)
        return x, 0, 0.0
    r = b - op(x)
    r0 = r.clone()
    w = op(r)
    t = op(w)
    bnorm = float(torch.linalg.norm(b))
    znorm = float(torch.dot(r, r))
    wr = float(torch.dot(w, r))
    alpha = znorm / wr if wr != 0.0 else 0.0
    beta = zeta = 0.0
    relres = (znorm ** 0.5) / bnorm if bnorm > 0 else 0.0
    p = s = z = None
    steps = 0
    while relres >= tol and steps < max_iter:
        if steps == 0:
            p, s, z = r.clone(), w.clone(), t.clone()
        else:
            p = r + beta * (p - zeta * s)
            s = w + beta * (s - zeta * z)
            z = t + beta * (z - zeta * v)
        q = r - alpha * s
        y = w - alpha * z
        yy = float(torch.dot(y, y))
        if yy == 0.0 or alpha == 0.0:
            break
        zeta = float(torch.dot(y, q)) / yy
        v = op(z)
        x = x + alpha * p + zeta * q
        r = q - zeta * y
        w = y - zeta * (t - alpha * v)
        znorm_old = znorm
        znorm = float(torch.dot(r, r0))
        zw, zs, zz = float(torch.dot(w, r0)), float(torch.dot(s, r0)), float(torch.dot(z, r0))
        rr = float(torch.dot(r, r))
        if zeta == 0.0 or znorm_old == 0.0:
            steps += 1
            relres = (rr ** 0.5) / bnorm
            break
        beta = (alpha / zeta) * (znorm / znorm_old)
        den = zw + beta * zs - beta * zeta * zz
        alpha = znorm / den if den != 0.0 else 0.0
        t = op(w)
        steps += 1
        relres = (rr ** 0.5) / bnorm
    u = D * x if D is not None else x
    return u, steps, relres
