"""Multi-GPU plumbing of bench.py on CPU: two gloo ranks.

Runs are independent, so N GPUs run N replicas with no data-path collective; the
only cross-rank operations are the barrier around the timed region, the maximum of
the ranks' device times and the sum of their run-steps.  These tests run that
plumbing as two processes over gloo (127.0.0.1) and check the aggregation the
bench reports: value = sum(run-steps) / max(time).
"""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist(world, backend="gloo")
    d.barrier()
    ms = [120.0, 150.0][rank]        # each rank's device time of its timed region
    steps = [16 * 2000, 16 * 2000][rank]
    ms_max = d.max(ms)
    total = d.sum(steps)
    d.barrier()
    d.close()
    # the reference arm prints from rank 0 only; other ranks exit 0 without work
    rc = bench.run_reference(bench.parse(["--gpus", str(world)])) if rank == 1 else 0
    q.put((rank, ms_max, total, rc))


def test_two_gloo_ranks_aggregate_like_the_bench():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms_max, total, rc in out:
        assert ms_max == 150.0          # the slowest rank sets the time
        assert total == 2 * 16 * 2000   # run-steps of all ranks
        assert rc == 0
    value = out[0][2] / (out[0][1] / 1000.0)
    assert value == pytest.approx(2 * 16 * 2000 / 0.150)


def test_single_process_dist_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        os.environ.pop(k, None)
    d = bench.Dist(1)
    assert d.world == 1 and d.pg is None
    assert d.max(3.5) == 3.5 and d.sum(7.0) == 7.0
    d.barrier()
    d.close()
