"""The bench's N > 1 path on the CPU (gloo, world size 2): every rank takes
the same collective steps, the reported time is the slowest rank's, the rate
counts every rank's work, and each replica runs its own event."""
import multiprocessing as mp
import os
import sys

import pytest

import vahlib as V

sys.path.insert(0, V.ROOT)


def _rank(rank, world, port, q):
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        elapsed = bench.max_over_ranks(dist, 1.0 + rank, device="cpu")  # rank 1 is the slow one
        dist.barrier()
        q.put((rank, elapsed, bench.whole_job_rate(world, 100, elapsed), bench.rank_seed(rank, 1),
               bench.batch_events(2, bench.rank_seed(rank, 1000))))
    finally:
        dist.destroy_process_group()


def test_two_ranks_report_the_slowest_time_and_whole_job_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, t0, v0, s0, ev0), (r1, t1, v1, s1, ev1) = res
    assert t0 == t1 == 2.0          # max over ranks
    assert v0 == v1 == 2 * 100 / 2.0  # all ranks' units over the slowest time
    assert s0 != s1 and ev0 != ev1    # replicas run different events


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    import bench

    calls = []
    monkeypatch.setattr(bench, "cpu_step_rate", lambda *a, **k: calls.append(a) or (1.0, "reference", [1.0]))

    class Args:
        steps, warmup, gpus = 1, 0, 2
    bench.run_reference(Args, 1, 2)
    assert calls == []


def test_reference_arm_blocks_cover_the_event_once():
    """The reference arm's per-step sample is the whole 121x121x81 event, cut
    into blocks of whole x rows: every cell in exactly one block, each block
    at least 3 eta planes deep (3+1D arithmetic), at most one block per
    worker."""
    import numpy as np

    import bench

    for workers in (1, 2, 7, 16, 27, 40, 64, 200):
        blocks = bench.ref_blocks(workers)
        assert 1 <= len(blocks) <= workers
        hits = np.zeros((bench.NZ, bench.NY), int)
        for j0, j1, k0, k1 in blocks:
            assert k1 - k0 >= 3 and j1 > j0
            hits[k0:k1, j0:j1] += 1
        assert np.all(hits == 1), workers
