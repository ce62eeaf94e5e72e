"""Meshes and host-side H-matrix construction (input side of the hot path).

`HostHMatrix` wraps libhacapk_build.so: the CPU restatement of HACApK's
cluster tree / block partition / ACA+ fill (m_HACApK_base.f90) over the
ppohBEM collocation kernel (m_ppohBEM_user_func.f90).  It exposes the leaf
list in the reference C layout (stc_HACApK_leafmtxp) which is what the
engine and the oracle both consume.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import abi


@dataclass
class Mesh:
    xyz: np.ndarray     # (nond, 3) float64
    faces: np.ndarray   # (nofc, 3) int32, 0-based vertex ids
    dble: np.ndarray | None = None  # per-face real parameters, if read from a file

    @property
    def nofc(self) -> int:
        return int(self.faces.shape[0])


def icosphere(level: int) -> Mesh:
    """Unit icosphere, 10*4^L+2 vertices and 20*4^L faces."""
    lib = abi.build_lib()
    nv, nf = 10 * 4 ** level + 2, 20 * 4 ** level
    xyz = np.zeros((nv, 3), np.float64)
    faces = np.zeros((nf, 3), np.int32)
    st = lib.hbx_mesh_icosphere(level, abi.dptr(xyz), abi.iptr(faces))
    if st != 0:
        raise RuntimeError(f"hbx_mesh_icosphere failed: {abi.STATUS.get(st, st)}")
    return Mesh(xyz, faces)


def ellipsoid(level: int, axes, center=(0.0, 0.0, 0.0)) -> Mesh:
    """Icosphere scaled by the semi-axes `axes` and moved to `center`."""
    m = icosphere(level)
    xyz = m.xyz * np.asarray(axes, np.float64)[None, :] + np.asarray(center, np.float64)[None, :]
    return Mesh(np.ascontiguousarray(xyz), m.faces)


def concat(*meshes: Mesh) -> Mesh:
    xyz, faces, off = [], [], 0
    for m in meshes:
        xyz.append(m.xyz)
        faces.append(m.faces + off)
        off += m.xyz.shape[0]
    return Mesh(np.ascontiguousarray(np.concatenate(xyz)),
                np.ascontiguousarray(np.concatenate(faces).astype(np.int32)))


def read_pbs(path: str) -> Mesh:
    """Reads a ppohBEM .pbf/.pbs mesh (list-directed, as Read_model_data in
    bem-bb-fw-HACApK-0.4.2.f90:411-640): nond, nond x (x y z), nofc,
    nond_on_face, nint_para_fc, ndble_para_fc, nofc x face2node (0-based),
    nofc x int params, nofc x real params."""
    with open(path) as f:
        tok = f.read().split()
    p = 0

    def take(n, conv):
        nonlocal p
        out = [conv(t.replace("D", "E").replace("d", "e")) for t in tok[p:p + n]]
        p += n
        return out

    nond = int(take(1, float)[0])
    xyz = np.array(take(3 * nond, float), np.float64).reshape(nond, 3)
    nofc = int(take(1, float)[0])
    non = int(take(1, float)[0])
    nint = int(take(1, float)[0])
    ndble = int(take(1, float)[0])
    if non != 3:
        raise ValueError(f"only triangles are supported (nond_on_face={non})")
    faces = np.array(take(non * nofc, lambda s: int(float(s))), np.int32).reshape(nofc, non)
    if nint > 0:
        take(nint * nofc, float)
    dble = np.array(take(ndble * nofc, float), np.float64).reshape(nofc, ndble) if ndble else None
    return Mesh(np.ascontiguousarray(xyz), np.ascontiguousarray(faces), dble)


def write_vtk(path: str, mesh: Mesh, values: np.ndarray, name: str = "solve") -> None:
    """Writes the mesh and one value per face (in the mesh's own face order,
    e.g. HostHMatrix.from_cluster(u)) as a legacy ASCII VTK unstructured grid
    of triangles -- the output of Print_result in bem-bb-fw-HACApK-0.4.2.f90
    (:755-855): POINTS, CELLS, CELL_TYPES (5 = triangle) and CELL_DATA with
    one scalar field."""
    values = np.asarray(values, np.float64)
    if values.shape != (mesh.nofc,):
        raise ValueError(f"need one value per face ({mesh.nofc}), got {values.shape}")
    nv, nf = mesh.xyz.shape[0], mesh.nofc
    lines = ["# vtk DataFile Version 2.0", "B200 H-matrix BiCGSTAB result", "ASCII",
             "DATASET UNSTRUCTURED_GRID", f"POINTS {nv} double"]
    lines += [f"{x:.16e} {y:.16e} {z:.16e}" for x, y, z in mesh.xyz]
    lines.append(f"CELLS {nf} {4 * nf}")
    lines += [f"3 {a} {b} {c}" for a, b, c in mesh.faces]
    lines.append(f"CELL_TYPES {nf}")
    lines += ["5"] * nf
    lines += [f"CELL_DATA {nf}", f"SCALARS {name} double 1", "LOOKUP_TABLE default"]
    lines += [f"{v:.17e}" for v in values]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def read_vtk_cell_scalars(path: str):
    """(points, triangles, values) of a file written by write_vtk."""
    tok = open(path).read().split("\n")
    i = tok.index(next(t for t in tok if t.startswith("POINTS")))
    nv = int(tok[i].split()[1])
    xyz = np.array([[float(v) for v in t.split()] for t in tok[i + 1:i + 1 + nv]])
    i = tok.index(next(t for t in tok if t.startswith("CELLS")))
    nf = int(tok[i].split()[1])
    tri = np.array([[int(v) for v in t.split()[1:]] for t in tok[i + 1:i + 1 + nf]], np.int32)
    i = tok.index("LOOKUP_TABLE default")
    vals = np.array([float(t) for t in tok[i + 1:i + 1 + nf]])
    return xyz, tri, vals


def default_params() -> abi.BuildParams:
    p = abi.BuildParams()
    abi.build_lib().hbx_build_default_params(C.byref(p))
    return p


class HostHMatrix:
    """H-matrix built on the host, leaves in the reference C layout.

    Vectors passed to the engine / oracle are in cluster order:
    `to_cluster(v) = v[lod-1]` (m_HACApK_use.f90:209, :285)."""

    def __init__(self, mesh: Mesh, leaf_size: int = 15, eta: float = 2.0,
                 aca_eps: float = 1e-6, kernel: int = abi.KERNEL_LAPLACE,
                 nthreads: int = 0, fill: bool | str = True):
        """fill: True fills the leaves on the host (C++ restatement of the
        reference's fill), "gpu" on the current CUDA device
        (hbx_fill_leaves), False leaves only the block partition."""
        lib = abi.build_lib()
        self._lib = lib
        self._fill = None
        self.mesh = mesh
        p = default_params()
        p.leaf_size = leaf_size
        p.eta = eta
        p.aca_eps = aca_eps
        p.kernel = kernel
        p.nthreads = nthreads
        p.fill = 1 if fill is True else 0
        self.params = p
        h = C.c_void_p()
        xyz = np.ascontiguousarray(mesh.xyz, np.float64)
        faces = np.ascontiguousarray(mesh.faces, np.int32)
        st = lib.hbx_build(abi.dptr(xyz), xyz.shape[0], abi.iptr(faces), faces.shape[0],
                           C.byref(p), C.byref(h))
        if st != 0:
            raise RuntimeError(f"hbx_build failed: {abi.STATUS.get(st, st)}")
        self._h = h
        self.st = lib.hbx_build_leafmtxp(h)
        self.nd = int(faces.shape[0])
        lod = lib.hbx_build_lod(h)
        self.lod = np.ctypeslib.as_array(lod, shape=(self.nd,)).copy()
        s = abi.BuildStats()
        lib.hbx_build_get_stats(h, C.byref(s))
        self.stats = {f: getattr(s, f) for f, _ in abi.BuildStats._fields_ if f != "reserved"}
        if fill == "gpu":
            self.fill_stats = self._fill_gpu(xyz, faces)

    def _fill_gpu(self, xyz, faces) -> dict:
        """The ACA+ / dense fill on the GPU (hbx_fill_leaves) into this
        partition's leaves; keeps the stats of the host fill in step."""
        fp = abi.FillParams()
        p = self.params
        if p.aca_method != 2:
            raise ValueError("the GPU fill runs ACA+ (aca_method 2) only")
        fp.kernel, fp.aca_eps, fp.aca_abs_factor, fp.kmax, fp.kmin = p.kernel, p.aca_eps, p.aca_abs_factor, p.kmax, p.kmin
        f = C.c_void_p()
        fs = abi.FillStats()
        lod = np.ascontiguousarray(self.lod, np.int32)
        st = abi.engine_lib().hbx_fill_leaves(abi.dptr(xyz), xyz.shape[0], abi.iptr(faces), faces.shape[0],
                                              abi.iptr(lod), C.byref(fp), self.st, C.byref(f), C.byref(fs))
        if st != 0:
            raise RuntimeError(f"hbx_fill_leaves failed: {abi.STATUS.get(st, st)}")
        self._fill = f
        d, lr = self.storage_words()
        self.stats["ktmax"] = fs.ktmax
        self.stats["mem_words"] = d + lr
        self.stats["memh_words"] = d + lr + self.nlf
        return {k: getattr(fs, k) for k, _ in abi.FillStats._fields_ if k != "reserved"}

    def close(self):
        if getattr(self, "_fill", None):
            abi.engine_lib().hbx_fill_free(self._fill)
            self._fill = None
        if getattr(self, "_h", None):
            self._lib.hbx_build_free(self._h)
            self._h = None
            self.st = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- vector ordering ---------------------------------------------------
    def to_cluster(self, v: np.ndarray) -> np.ndarray:
        return np.ascontiguousarray(v[self.lod - 1])

    def from_cluster(self, u: np.ndarray) -> np.ndarray:
        out = np.empty_like(u)
        out[self.lod - 1] = u
        return out

    # -- inspection --------------------------------------------------------
    @property
    def nlf(self) -> int:
        return int(self.st.contents.nlf)

    def leaf(self, ip: int) -> abi.LeafMtx:
        return self.st.contents.st_lf[ip]

    def leaf_arrays(self, ip: int):
        """(kind, nstrtl, ndl, nstrtt, ndt, kt, A_or_(U, V)) with numpy views."""
        L = self.leaf(ip)
        if L.ltmtx == 1:
            V = np.ctypeslib.as_array(L.a1, shape=(L.kt * L.ndt,)).reshape(L.kt, L.ndt).T if L.kt else np.zeros((L.ndt, 0))
            U = np.ctypeslib.as_array(L.a2, shape=(L.kt * L.ndl,)).reshape(L.kt, L.ndl).T if L.kt else np.zeros((L.ndl, 0))
            return 1, L.nstrtl, L.ndl, L.nstrtt, L.ndt, L.kt, (U, V)
        A = np.ctypeslib.as_array(L.a1, shape=(L.ndl * L.ndt,)).reshape(L.ndl, L.ndt)
        return 2, L.nstrtl, L.ndl, L.nstrtt, L.ndt, 0, A

    def dense(self, r0: int = 0, nr: int | None = None, c0: int = 0, nc: int | None = None) -> np.ndarray:
        """Exact matrix block in cluster order (for small problems)."""
        nr = self.nd - r0 if nr is None else nr
        nc = self.nd - c0 if nc is None else nc
        out = np.zeros((nc, nr), np.float64)  # column-major (r + c*nr)
        st = self._lib.hbx_build_dense_block(self._h, r0, nr, c0, nc, abi.dptr(out))
        if st != 0:
            raise RuntimeError("hbx_build_dense_block failed")
        return out.T

    def entry(self, i: int, j: int) -> float:
        return float(self._lib.hbx_build_entry(self._h, i, j))

    def storage_words(self) -> tuple[int, int]:
        """(dense words, low-rank words)."""
        d = lr = 0
        arr = self.st.contents.st_lf
        for ip in range(self.nlf):
            L = arr[ip]
            if L.ltmtx == 1:
                lr += L.kt * (L.ndl + L.ndt)
            else:
                d += L.ndl * L.ndt
        return d, lr

    def accuracy(self) -> tuple[float, float]:
        """(||A - H||_F, ||A||_F) over the leaves, as HACApK_accuracy_leafmtx
        (m_HACApK_base.f90:614-673) reports them: a low-rank leaf adds its
        exact entries to ||A|| and their difference from U V^T to ||A - H||;
        a dense leaf, which holds the exact entries, adds them to ||A|| only."""
        zh = za = 0.0
        for ip in range(self.nlf):
            kind, nstrtl, ndl, nstrtt, ndt, kt, data = self.leaf_arrays(ip)
            if kind == 1:
                U, V = data
                A = self.dense(nstrtl - 1, ndl, nstrtt - 1, ndt)
                za += float(np.sum(A * A))
                E = A - U @ V.T
                zh += float(np.sum(E * E))
            else:
                za += float(np.sum(data * data))
        return float(np.sqrt(zh)), float(np.sqrt(za))
