"""Request loop for convection-diffusion solves with continuous batching on one GPU.

Requests arrive over time (each: dimension, order, mesh size, coefficients).  The loop keeps
every admitted solve's matrices, hierarchy vectors and Krylov iterates on the device
(a ``Batch``), admits waiting requests whenever the device memory they need fits under the
budget, and advances all running solves together a few FGMRES iterations at a time; a
solve that finishes frees its memory at once, so the next waiting request is admitted at
the next round while the others keep iterating.  Latency = completion time - arrival time.
"""
import time

import numpy as np

from .system import SUPG, Batch, coeffs, solver_params
from .workloads import StructureCache


def default_params():
    """FGMRES(30) to ||r|| <= 1e-10 ||r0||, V(2,2) multicolour SSOR, exact coarse solve."""
    return solver_params(smoother=3, omega=1.0, pre=2, post=2, stop_rule=1, red_factor=1e-10, restart=30,
                         maxit=2000)


class Server:
    def __init__(self, ctx, budget_bytes, params=None, iterations_per_round=4, batch=None):
        # batch: an existing Batch (or an object with its methods) instead of a new one
        self.batch = batch if batch is not None else Batch(params or default_params(), ctx)
        self.cache = StructureCache(self.batch)
        self.budget = budget_bytes
        self.k = iterations_per_round
        self.waiting = []   # requests not yet admitted, arrival order
        self.running = {}   # slot -> request
        self.done = []      # finished requests with latency and status

    def prepare(self, requests):
        """Upload the mesh structures the requests need (the meshes are known in advance)."""
        for r in requests:
            self.cache.get(r["dim"], r["order"], r["n"])

    def _admit(self, now):
        held = self.batch.memory()
        while self.waiting:
            r = self.waiting[0]
            sid, n_dof = self.cache.get(r["dim"], r["order"], r["n"])
            need = self.batch.instance_bytes(sid)
            if held + need > self.budget and self.running:
                break
            self.waiting.pop(0)
            co = coeffs(0, eps=r["eps"], b=r["b"], f=1.0, poly_degree=r["order"])
            slot = self.batch.submit(sid, co, SUPG)
            r["admitted"] = now
            r["n_dof_used"] = n_dof
            self.running[slot] = r
            held += need

    def run(self, requests, keep_solutions=False):
        """Replay the requests at their arrival times (seconds from the start); returns the
        finished requests with 'latency', 'iterations', 'status'.  keep_solutions: True, or a
        predicate of the request, selects the requests whose solution is fetched into
        r['solution']."""
        pending = sorted(requests, key=lambda r: r["t"])
        t0 = time.perf_counter()
        i = 0
        while i < len(pending) or self.waiting or self.running:
            now = time.perf_counter() - t0
            while i < len(pending) and pending[i]["t"] <= now:
                self.waiting.append(pending[i])
                i += 1
            if not self.running and not self.waiting:
                # idle until the next arrival
                time.sleep(max(0.0, min(pending[i]["t"] - now, 0.01)))
                continue
            self._admit(now)
            self.batch.advance(self.k)
            finished = self.batch.poll()
            tnow = time.perf_counter() - t0
            for slot in finished:
                r = self.running.pop(slot)
                keep = keep_solutions(r) if callable(keep_solutions) else keep_solutions
                x, info = self.batch.fetch(slot, r["n_dof_used"] if keep else 0)
                r["latency"] = tnow - r["t"]
                r["iterations"] = info.iterations
                r["status"] = info.status
                if keep:
                    r["solution"] = x
                self.batch.release(slot)
                self.done.append(r)
        self.elapsed = time.perf_counter() - t0
        return self.done

    def stats(self):
        lat = np.array([r["latency"] for r in self.done])
        ok = sum(1 for r in self.done if r["status"] == 0)
        return dict(completed=len(self.done), converged=ok, solves_per_s=len(self.done) / self.elapsed,
                    p50_latency_s=float(np.percentile(lat, 50)) if len(lat) else None,
                    p99_latency_s=float(np.percentile(lat, 99)) if len(lat) else None,
                    elapsed_s=self.elapsed)
