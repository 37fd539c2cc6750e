"""Named synthetic workloads with their Wave3d options.

Each workload fixes a geometry, N, wavenumber box K, accuracy ACCU
(P = 4/6/8 equivalent points per edge, src/wave3d.cpp:145-158), kernel,
NPQ=4 wedges per quadrant and ptsmax=100, as the reference driver's
-wave3d_* options would (src/wave3d_setup.cpp:30-61).
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

from . import geometry, precompute

OPERATOR_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_operators")


@dataclass(frozen=True)
class Workload:
    name: str
    geometry: str          # "sphere" | "ellipsoid"
    K: float               # root-box width in wavelengths
    N: int
    accu: int = 1
    kernel: int = 0        # 0: exp(ir)/r, 1: exp(ir)
    ptsmax: int = 100
    npq: int = 4
    seed: int = 0

    @property
    def P(self) -> int:
        return precompute.accu_to_p(self.accu)

    @property
    def nc(self) -> int:
        return geometry.cells_for(self.K)

    @property
    def maxlevel(self) -> int:
        return geometry.maxlevel_for(self.K)

    @property
    def wmax(self) -> int:
        """Widest high-frequency box: the cell-level width K/NC."""
        return max(1, int(round(self.K / self.nc)))

    def points(self) -> np.ndarray:
        if self.geometry == "sphere":
            return geometry.sphere_points(self.N, self.K, self.seed)
        if self.geometry == "ellipsoid":
            return geometry.ellipsoid_points(self.N, self.K, self.seed)
        if self.geometry == "cluster":
            return geometry.cluster_points(self.N, self.K, self.seed)
        raise ValueError("unknown geometry %r" % self.geometry)

    def densities(self, dtype=np.complex128) -> np.ndarray:
        return geometry.densities(self.N, self.seed, dtype)

    def check_ids(self, count: int = 200) -> np.ndarray:
        return geometry.check_ids(self.N, count, self.seed)

    def operators(self, workers=None):
        return precompute.ensure_operators(OPERATOR_DIR, self.kernel, self.accu, self.wmax, workers)

    def options(self) -> dict:
        return {
            "-wave3d_ACCU": str(self.accu),
            "-wave3d_NPQ": str(self.npq),
            "-wave3d_K": repr(float(self.K)),
            "-wave3d_ctr": "0 0 0",
            "-wave3d_ptsmax": str(self.ptsmax),
            "-wave3d_maxlevel": str(self.maxlevel),
        }


def sphere(K, N=None, accu=1, kernel=0, seed=0, ptsmax=100):
    N = N if N is not None else geometry.sphere_n_for(K)
    return Workload("sphere_K%g_N%d_P%d_k%d" % (K, N, precompute.accu_to_p(accu), kernel),
                    "sphere", float(K), int(N), accu, kernel, ptsmax, 4, seed)


def ellipsoid(K, N, accu=1, kernel=0, seed=0, ptsmax=100):
    return Workload("ellipsoid_K%g_N%d_P%d_k%d" % (K, N, precompute.accu_to_p(accu), kernel),
                    "ellipsoid", float(K), int(N), accu, kernel, ptsmax, 4, seed)


def cluster(K, N, accu=1, kernel=0, seed=0, ptsmax=8):
    return Workload("cluster_K%g_N%d_P%d_k%d_m%d" % (K, N, precompute.accu_to_p(accu), kernel, ptsmax),
                    "cluster", float(K), int(N), accu, kernel, ptsmax, 4, seed)


def instance_mix(Ks, seed0, accu=2):
    """Spheres and ellipsoids (alternating) of the given K, N = 25 pi K^2
    points, P=6 by default, seeded from seed0 on: the instances of the
    batched (64 uneven instances) and served (16 sessions) configurations."""
    out = []
    for j, K in enumerate(Ks):
        n = geometry.sphere_n_for(K)
        seed = seed0 + j
        out.append(sphere(K, n, accu=accu, seed=seed) if j % 2 == 0 else ellipsoid(K, n, accu=accu, seed=seed))
    return out


# the small plain-method case the reference binary runs in seconds
SMALL = sphere(8, 5000, accu=1)
# the large single instance (about 25 points per square wavelength)
LARGE = sphere(64, None, accu=2)
# a quarter-size instance of the same family (profiling captures)
MEDIUM = sphere(32, None, accu=2)
