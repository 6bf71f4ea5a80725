"""The request loop's host logic (admission under the memory budget, continuous batching,
arrival order, latency bookkeeping) on the CPU, with a stand-in for the device batch."""
import types

from parmoon_cmg_b200.serving import Server


class FakeBatch:
    """The Batch methods the loop uses; an instance finishes after a fixed number of rounds
    that depends on its mesh size."""

    def __init__(self):
        self.structures = []
        self.slots = {}
        self.next_slot = 0
        self.held = 0
        self.events = []  # (kind, slot, running slots after the event, held bytes)

    def add_structure(self, spaces, parents):
        self.structures.append(int(spaces[-1]["n_dof"]))
        return len(self.structures) - 1

    def memory(self):
        return self.held

    def instance_bytes(self, sid):
        return 1000 * self.structures[sid]

    def submit(self, sid, co, disc):
        slot = self.next_slot
        self.next_slot += 1
        need = self.instance_bytes(sid)
        self.slots[slot] = dict(left=2 + self.structures[sid] // 100, bytes=need, polled=False)
        self.held += need
        self.events.append(("submit", slot, sorted(self.slots), self.held))
        return slot

    def advance(self, k):
        for v in self.slots.values():
            v["left"] -= 1

    def poll(self):
        out = [s for s, v in self.slots.items() if v["left"] <= 0 and not v["polled"]]
        for s in out:
            self.slots[s]["polled"] = True
        return out

    def fetch(self, slot, n_dof):
        return None, types.SimpleNamespace(iterations=7, status=0)

    def release(self, slot):
        self.held -= self.slots.pop(slot)["bytes"]
        self.events.append(("release", slot, sorted(self.slots), self.held))


def requests(sizes):
    return [dict(t=0.0, dim=2, order=1, n=n, eps=1e-2, b=(1.0, 0.0), id=i) for i, n in enumerate(sizes)]


def test_admission_under_budget_and_continuous_batching():
    fb = FakeBatch()
    sizes = [16, 8, 16, 8, 8, 16]
    reqs = requests(sizes)
    # 16^2 Q1: 289 DOFs -> 289,000 bytes; 8^2: 81 DOFs -> 81,000 bytes
    budget = 289_000 + 81_000 + 1
    srv = Server(None, budget, batch=fb, iterations_per_round=1)
    srv.prepare(reqs)
    done = srv.run(reqs)
    assert len(done) == len(reqs) and all(r["status"] == 0 and r["latency"] >= 0 for r in done)
    submits = [e for e in fb.events if e[0] == "submit"]
    # arrival order is admission order
    assert [e[1] for e in submits] == list(range(len(reqs)))
    # the budget holds whenever another solve is running
    assert all(held <= budget or len(running) == 1 for _, _, running, held in submits)
    # continuous batching: solves are admitted while others are still running
    assert any(len(running) > 1 for _, _, running, _ in submits)
    assert fb.held == 0 and not fb.slots
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["converged"] == len(reqs)


def test_request_larger_than_budget_runs_alone():
    fb = FakeBatch()
    reqs = requests([16, 8])
    srv = Server(None, 10, batch=fb, iterations_per_round=1)  # smaller than any instance
    srv.prepare(reqs)
    done = srv.run(reqs)
    assert len(done) == 2
    submits = [e for e in fb.events if e[0] == "submit"]
    assert all(len(running) == 1 for _, _, running, _ in submits)
