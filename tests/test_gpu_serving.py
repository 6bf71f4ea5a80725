"""Serving loop: continuous batching of solve requests under a device-memory budget.

Requests arrive over time and are admitted into one running batch as memory frees up; each
result must equal the result of the same request solved alone (bit-identical: an instance's
arithmetic does not depend on the other instances of the batch), and the admission budget
must be respected.
"""
import math

import numpy as np
import pytest

from parmoon_cmg_b200 import workloads as W
from parmoon_cmg_b200.serving import Server
from parmoon_cmg_b200.system import Context

pytestmark = pytest.mark.gpu


def small_requests():
    rng = np.random.default_rng(5)
    reqs = []
    t = 0.0
    for k in range(10):
        dim = 2 if k % 3 else 3
        order = 1 + (k % 2)
        n = int(rng.choice([8, 12, 16])) if dim == 2 else int(rng.choice([4, 6]))
        L, n0, nr = W.hierarchy_shape(n)
        ang = rng.uniform(0, 2 * math.pi)
        b = (math.cos(ang), math.sin(ang)) if dim == 2 else tuple(np.array([1.0, -0.5, 0.25]) / np.linalg.norm([1.0, -0.5, 0.25]))
        reqs.append(dict(t=t, dim=dim, order=order, n=nr, eps=10.0 ** rng.uniform(-4, -1), b=b))
        t += 0.002
    return reqs


@pytest.fixture(scope="module")
def ctx():
    from parmoon_cmg_b200 import _build
    _build.build()
    c = Context(0)
    yield c
    c.close()


def test_serving_results_equal_alone(ctx):
    reqs = small_requests()
    srv = Server(ctx, budget_bytes=10 ** 10, iterations_per_round=2)
    done = srv.run([dict(r) for r in reqs], keep_solutions=True)
    assert len(done) == len(reqs)
    assert all(r["status"] == 0 for r in done)
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["p99_latency_s"] >= st["p50_latency_s"] > 0
    for r in done:
        alone = Server(ctx, budget_bytes=10 ** 10, iterations_per_round=2)
        one = dict(r)
        one["t"] = 0.0
        res = alone.run([one], keep_solutions=True)[0]
        assert res["iterations"] == r["iterations"]
        assert np.array_equal(res["solution"], r["solution"])


def test_serving_respects_the_budget(ctx):
    reqs = small_requests()
    probe = Server(ctx, budget_bytes=0)
    need = [probe.batch.instance_bytes(probe.cache.get(r["dim"], r["order"], r["n"])[0]) for r in reqs]
    budget = 2 * max(need)  # at most two of the largest at once
    srv = Server(ctx, budget_bytes=budget, iterations_per_round=1)
    peak = [0]
    orig = srv.batch.advance

    def advance(k):
        peak[0] = max(peak[0], srv.batch.memory())
        return orig(k)

    srv.batch.advance = advance
    done = srv.run([dict(r, t=0.0) for r in reqs])
    assert len(done) == len(reqs) and all(r["status"] == 0 for r in done)
    assert peak[0] <= budget
