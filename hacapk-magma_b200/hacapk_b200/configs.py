"""Synthetic workloads of the benchmark configurations.

Seeded stand-ins for the reference's inputs (the .pbf meshes it timed are not
available): unit icospheres and ellipsoids, piecewise-constant collocation of
the Laplace single layer 1/(4 pi r) with the analytic flat-triangle integral
(including the self term), HACApK's cluster tree / admissibility / ACA+.

  C1  plain FP64: icosphere L5 (20,480 faces), leaf 32, eta 2, ACA+ 1e-5,
      rhs = 1 + N(0, (1e-3)^2) per element (seed 0), BiCGSTAB to 1e-8.
  C2  precision: icosphere L7 (327,680 faces) and, as a second body, an
      ellipsoid of the same subdivision level with semi-axes U(0.5, 2)
      (seed 1), centred on the x axis so that the gap between the two
      surfaces along x is 3; leaf 32, eta 2, ACA+ 1e-6; rhs as C1.
  C3  multi-RHS: icosphere L6 (81,920 faces) as C1, 64 right-hand sides
      N(0,1) per element (seed 2).
  C4  differentiation: icosphere L6 as C1; g and sigma_t N(0,1) (seeds 3, 4).
  C5  uneven batch: `count` ellipsoids (256 in the config), semi-axes
      U(0.3, 3), subdivision levels drawn uniformly from {2, 3, 4, 5} (so the
      sizes 320 .. 20,480 are log-uniform), seed 5; leaf 32, eta 2, ACA+ 1e-5;
      rhs of instance k = 1 + N(0, (1e-3)^2) per element with seed 5 + k.
"""
from __future__ import annotations

import numpy as np

from . import abi
from .hmatrix import HostHMatrix, concat, ellipsoid, icosphere


def rhs_unit_plus_noise(n: int, seed: int = 0, sigma: float = 1e-3) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return 1.0 + sigma * rng.standard_normal(n)


def laplace_sphere(level: int, leaf_size: int = 32, eta: float = 2.0, aca_eps: float = 1e-5,
                   nthreads: int = 0, fill=True) -> HostHMatrix:
    return HostHMatrix(icosphere(level), leaf_size=leaf_size, eta=eta, aca_eps=aca_eps,
                       kernel=abi.KERNEL_LAPLACE, nthreads=nthreads, fill=fill)


# fill: True builds the leaves on the host (the C++ restatement of the
# reference's fill), "gpu" on the current CUDA device (hbx_fill_leaves).


def c1(level: int = 5, nthreads: int = 0, fill=True):
    """(H-matrix, rhs in cluster order) of configuration C1 (level 5 by default)."""
    H = laplace_sphere(level, 32, 2.0, 1e-5, nthreads, fill)
    b = H.to_cluster(rhs_unit_plus_noise(H.nd, seed=0))
    return H, b


def c2(level: int = 7, seed: int = 1, gap: float = 3.0, aca_eps: float = 1e-6, nthreads: int = 0, fill=True):
    """(H-matrix, rhs in cluster order) of configuration C2: the unit
    icosphere and a seeded ellipsoid of the same level, one H-matrix over
    both bodies."""
    axes = np.random.default_rng(seed).uniform(0.5, 2.0, 3)
    body2 = ellipsoid(level, axes, center=(1.0 + gap + axes[0], 0.0, 0.0))
    H = HostHMatrix(concat(icosphere(level), body2), leaf_size=32, eta=2.0, aca_eps=aca_eps,
                    kernel=abi.KERNEL_LAPLACE, nthreads=nthreads, fill=fill)
    b = H.to_cluster(rhs_unit_plus_noise(H.nd, seed=0))
    return H, b


def c5(count: int = 256, seed: int = 5, max_level: int = 5, nthreads: int = 0, fill=True):
    """[(H-matrix, rhs in cluster order)] of configuration C5: `count` independent
    ellipsoids of uneven sizes (the batch form's workload)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        level = int(rng.integers(2, max_level + 1))
        axes = rng.uniform(0.3, 3.0, 3)
        H = HostHMatrix(ellipsoid(level, axes), leaf_size=32, eta=2.0, aca_eps=1e-5,
                        kernel=abi.KERNEL_LAPLACE, nthreads=nthreads, fill=fill)
        out.append((H, H.to_cluster(rhs_unit_plus_noise(H.nd, seed=seed + k))))
    return out


def c3(level: int = 6, nrhs: int = 64, seed: int = 2, fill=True):
    """(H-matrix, nd x nrhs right-hand sides in cluster order) of configuration C3."""
    H = laplace_sphere(level, 32, 2.0, 1e-5, 0, fill)
    B = np.random.default_rng(seed).standard_normal((H.nd, nrhs))
    return H, np.ascontiguousarray(B[H.lod - 1])


def c4(level: int = 6, fill=True):
    """(H-matrix, g, sigma_t) of configuration C4, vectors in cluster order."""
    H = laplace_sphere(level, 32, 2.0, 1e-5, 0, fill)
    g = np.random.default_rng(3).standard_normal(H.nd)
    st = np.random.default_rng(4).standard_normal(H.nd)
    return H, H.to_cluster(g), H.to_cluster(st)
