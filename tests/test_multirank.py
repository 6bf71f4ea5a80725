"""The N > 1 path of bench.py on the CPU: two gloo ranks.

The workload shards as independent replicas (one solve per rank, no data-path collective);
the only collectives are the barrier around the timed region and the maximum of the ranks'
times.  These tests run bench.py's own helpers in two processes over gloo on 127.0.0.1, and
check that the reference arm does its work on rank 0 only.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import bench
    import torch.distributed as dist
    r, w, local = bench.dist_init(None)
    try:
        bench.barrier(w)
        # every rank reports its own time; the job's time is the slowest rank's
        m = bench.max_over_ranks(1.0 + r, w)
        out[r] = (r, w, local, m, dist.get_backend())
        bench.barrier(w)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_max_over_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        for p in procs:
            if p.is_alive():
                p.kill()
        assert all(p.exitcode == 0 for p in procs)
        res = dict(out)
    assert sorted(res) == [0, 1]
    for r, (rank, world, local, m, backend) in res.items():
        assert (rank, world, local) == (r, 2, r)
        assert m == 2.0  # the maximum over both ranks
        assert backend == "gloo"


def test_reference_arm_runs_on_rank_zero_only(capsys):
    """Under torchrun every rank calls the reference arm; ranks other than 0 return at once
    without work or output (the driver reads rank 0's line)."""
    import bench
    assert bench.run_reference_arm(None, 1, 2) is None
    assert capsys.readouterr().out == ""
