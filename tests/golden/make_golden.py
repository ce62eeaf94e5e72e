"""Generates tests/golden/*.npz from the reference's own compiled CPU
H-matvec (oracle/_ref/libhacapk_ref.so, built from HACApK_MAGMA.c).

Each fixture stores the inputs of one case (mesh recipe + construction
parameters + a seeded x), a digest of the leaf list the construction produced,
and y = H x as computed by the reference code.

It also stores the reference's own mesh input bem-bb_inputs/input_10ts.pbs
(10,400 flat triangles) as input_10ts_mesh.npz -- the vertices and faces as
read by hmatrix.read_pbs, and the SHA-256 of the source file -- so that the
GPU tests, which run where the reference tree is absent, can take the
reference's inputs through the drop-in entry points.  Run from the repository
root (REFERENCE_DIR: the reference tree, default ../reference beside the
repository):
    python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "hacapk-magma_b200"))
sys.path.insert(0, ROOT)

from hacapk_b200 import abi, hmatrix  # noqa: E402
import oracle  # noqa: E402

CASES = [
    # name, level, leaf, eta, aca_eps, kernel, seed
    ("sphere_L2_dense", 2, 32, 2.0, 1e-5, abi.KERNEL_LAPLACE, 11),
    ("sphere_L3_leaf32", 3, 32, 2.0, 1e-5, abi.KERNEL_LAPLACE, 12),
    ("sphere_L3_leaf15_ppohbem", 3, 15, 2.0, 1e-6, abi.KERNEL_PPOHBEM, 13),
    ("sphere_L4_leaf32", 4, 32, 2.0, 1e-5, abi.KERNEL_LAPLACE, 14),
]


def leaf_digest(H) -> str:
    """SHA-256 over every leaf's metadata and factor bytes, in leaf order."""
    h = hashlib.sha256()
    arr = H.st.contents.st_lf
    for ip in range(H.nlf):
        L = arr[ip]
        h.update(np.array([L.ltmtx, L.kt, L.nstrtl, L.ndl, L.nstrtt, L.ndt], np.int64).tobytes())
        n = L.kt * (L.ndl + L.ndt) if L.ltmtx == 1 else L.ndl * L.ndt
        if n:
            h.update(np.ctypeslib.as_array(L.a1, shape=(n,)).tobytes())
    return h.hexdigest()


def build(case):
    name, level, leaf, eta, eps, kernel, seed = case
    H = hmatrix.HostHMatrix(hmatrix.icosphere(level), leaf_size=leaf, eta=eta, aca_eps=eps, kernel=kernel,
                            nthreads=1)
    x = np.random.default_rng(seed).standard_normal(H.nd)
    return H, x


def reference_dir() -> str:
    return os.environ.get("REFERENCE_DIR", os.path.join(os.path.dirname(ROOT), "reference"))


def save_reference_mesh(out: str):
    src = os.path.join(reference_dir(), "bem-bb_inputs", "input_10ts.pbs")
    if not os.path.exists(src):
        print("reference mesh not found:", src)
        return
    m = hmatrix.read_pbs(src)
    digest = hashlib.sha256(open(src, "rb").read()).hexdigest()
    np.savez_compressed(os.path.join(out, "input_10ts_mesh.npz"), xyz=m.xyz, faces=m.faces, source_sha256=digest)
    print("input_10ts_mesh", m.xyz.shape, m.faces.shape, digest)


def main():
    out = os.path.dirname(os.path.abspath(__file__))
    save_reference_mesh(out)
    for case in CASES:
        H, x = build(case)
        y = oracle.matvec_ref(H.st, x)
        np.savez_compressed(os.path.join(out, case[0] + ".npz"), x=x, y=y, digest=leaf_digest(H),
                            nlf=H.nlf, stats=np.array([H.stats["nclst"], H.stats["n_lowrank"],
                                                       H.stats["n_dense"], H.stats["ktmax"],
                                                       H.stats["memh_words"]]))
        print(case[0], H.nd, H.nlf, np.linalg.norm(y))


if __name__ == "__main__":
    main()
