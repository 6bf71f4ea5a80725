"""The seeded synthetic workloads of the batched and serving configurations."""
import math

import numpy as np

from parmoon_cmg_b200 import workloads as W


def test_hierarchy_shape_rounds_within_20_percent():
    for n in range(16, 257):
        L, n0, nr = W.hierarchy_shape(n)
        assert n0 in (2, 3, 4) and nr == n0 * 2 ** (L - 1)
        assert abs(nr - n) <= 0.2 * n
        # an admissible size is its own rounding
        assert W.hierarchy_shape(nr)[2] == nr


def test_batched_cd2d_is_seeded_and_in_range():
    a, b = W.batched_cd2d(512), W.batched_cd2d(512)
    assert a == b  # same seed, same instances
    n = np.array([r["n"] for r in a])
    assert n.min() >= 16 and n.max() <= 256
    orders = np.array([r["order"] for r in a])
    assert set(orders) == {1, 2} and 0.4 < (orders == 1).mean() < 0.6
    eps = np.array([r["eps"] for r in a])
    assert eps.min() >= 1e-6 and eps.max() <= 1e-1
    assert all(abs(math.hypot(*r["b"]) - 1) < 1e-12 for r in a)
    assert all(r["n_used"] == W.hierarchy_shape(r["n"])[2] for r in a)
    # log-uniform N: about half the instances below the geometric mean 64
    assert 0.4 < (n < 64).mean() < 0.6


def test_serving_stream_mix_and_arrivals():
    reqs = W.serving_stream(400, 40.0)
    assert reqs == W.serving_stream(400, 40.0)
    t = np.array([r["t"] for r in reqs])
    assert np.all(np.diff(t) > 0)
    # Poisson arrivals at 40/s: mean gap 25 ms
    assert 0.02 < np.diff(t).mean() < 0.03
    dims = np.array([r["dim"] for r in reqs])
    assert 0.6 < (dims == 2).mean() < 0.8
    nd = np.array([r["n_dof"] for r in reqs])
    assert nd.min() >= 0.5e3 and nd.max() <= 4e6
    for r in reqs:
        assert W.hierarchy_shape(r["n"])[2] == r["n"]
        assert r["n_dof"] == W.dofs(r["dim"], r["order"], r["n"])
        assert abs(np.linalg.norm(r["b"]) - 1) < 1e-12
