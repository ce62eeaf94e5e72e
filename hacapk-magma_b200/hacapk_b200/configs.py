"""Synthetic workloads of the benchmark configurations.

Seeded stand-ins for the reference's inputs (the .pbf meshes it timed are not
available): unit icospheres and ellipsoids, piecewise-constant collocation of
the Laplace single layer 1/(4 pi r) with the analytic flat-triangle integral
(including the self term), HACApK's cluster tree / admissibility / ACA+.

  C1  plain FP64: icosphere L5 (20,480 faces), leaf 32, eta 2, ACA+ 1e-5,
      rhs = 1 + N(0, (1e-3)^2) per element (seed 0), BiCGSTAB to 1e-8.
"""
from __future__ import annotations

import numpy as np

from . import abi
from .hmatrix import HostHMatrix, icosphere


def rhs_unit_plus_noise(n: int, seed: int = 0, sigma: float = 1e-3) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return 1.0 + sigma * rng.standard_normal(n)


def laplace_sphere(level: int, leaf_size: int = 32, eta: float = 2.0, aca_eps: float = 1e-5,
                   nthreads: int = 0) -> HostHMatrix:
    return HostHMatrix(icosphere(level), leaf_size=leaf_size, eta=eta, aca_eps=aca_eps,
                       kernel=abi.KERNEL_LAPLACE, nthreads=nthreads)


def c1(level: int = 5, nthreads: int = 0):
    """(H-matrix, rhs in cluster order) of configuration C1 (level 5 by default)."""
    H = laplace_sphere(level, 32, 2.0, 1e-5, nthreads)
    b = H.to_cluster(rhs_unit_plus_noise(H.nd, seed=0))
    return H, b
