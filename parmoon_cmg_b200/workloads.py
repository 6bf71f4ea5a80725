"""Synthetic workloads of the batched and serving configurations (seeded, no datasets).

``batched_cd2d``: independent CD2D problems on the unit square, mesh N x N with N
log-uniform in [16, 256], Q1 or Q2 with equal probability, eps log-uniform in [1e-6, 1e-1],
convection angle uniform in [0, 2 pi) with |b| = 1, f = 1, Dirichlet 0.  The multigrid
hierarchy of an N x N mesh has L = floor(log2(N / 2)) + 1 levels on a coarsest mesh of
n0 = round(N / 2^(L-1)) in {2, 3, 4} cells per side (a small exact coarse solve), so N is
rounded to n0 * 2^(L-1) (within 20 %); the rounded N is recorded with every instance.

``serving_stream``: Poisson arrivals of CD2D/CD3D requests (70 % 2D, 30 % 3D, Q1/Q2 50/50),
DOF counts log-uniform in [1e3, 2e6] mapped to the nearest admissible N, eps log-uniform in
[1e-6, 1e-1], a random unit convection direction, f = 1, Dirichlet 0.
"""
import math

import numpy as np

from . import mesh


def hierarchy_shape(n):
    """(levels, coarsest cells per side, rounded n) of the multigrid hierarchy of an n^d mesh."""
    L = max(1, int(math.floor(math.log2(n / 2.0))) + 1)
    n0 = max(1, int(round(n / 2 ** (L - 1))))
    return L, n0, n0 * 2 ** (L - 1)


def batched_cd2d(n_instances=4096, seed=20261203):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_instances):
        n = int(round(math.exp(rng.uniform(math.log(16), math.log(256)))))
        order = 1 if rng.random() < 0.5 else 2
        eps = 10.0 ** rng.uniform(-6, -1)
        ang = rng.uniform(0, 2 * math.pi)
        L, n0, nr = hierarchy_shape(n)
        out.append(dict(dim=2, n=n, n_used=nr, levels=L, n0=n0, order=order, eps=eps,
                        b=(math.cos(ang), math.sin(ang)), angle=ang))
    return out


def dofs(dim, order, n):
    return (order * n + 1) ** dim


def n_for_dofs(dim, order, target):
    """Cells per side whose DOF count is nearest to target, rounded to its hierarchy."""
    best = None
    for n in range(4, 2049):
        L, n0, nr = hierarchy_shape(n)
        if nr != n:
            continue
        d = abs(math.log(dofs(dim, order, n) / target))
        if best is None or d < best[0]:
            best = (d, n)
    return best[1]


def serving_stream(n_requests, rate_per_s, seed=20261204):
    """Requests with arrival times (s) of a Poisson process of the given rate."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for _ in range(n_requests):
        t += rng.exponential(1.0 / rate_per_s)
        dim = 2 if rng.random() < 0.7 else 3
        order = 1 if rng.random() < 0.5 else 2
        target = 10.0 ** rng.uniform(3, math.log10(2e6))
        n = n_for_dofs(dim, order, target)
        eps = 10.0 ** rng.uniform(-6, -1)
        v = rng.normal(size=dim)
        v /= np.linalg.norm(v)
        L, n0, _ = hierarchy_shape(n)
        out.append(dict(t=t, dim=dim, order=order, n=n, levels=L, n0=n0, eps=eps, b=tuple(v),
                        n_dof=dofs(dim, order, n)))
    return out


class StructureCache:
    """One uploaded multigrid hierarchy per (dim, order, n) for a Batch."""

    def __init__(self, batch):
        self.batch = batch
        self.ids = {}

    def get(self, dim, order, n):
        key = (dim, order, n)
        if key not in self.ids:
            L, n0, nr = hierarchy_shape(n)
            assert nr == n, "n must be admissible (rounded by hierarchy_shape)"
            spaces, parents = mesh.structured_hierarchy(dim, order, n0, L)
            self.ids[key] = (self.batch.add_structure(spaces, parents), int(spaces[-1]["n_dof"]))
        return self.ids[key]
