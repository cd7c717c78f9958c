"""Replicas through the library path: two ranks (processes joined by a gloo
process group, as bench.py's N > 1 path joins its ranks) each run their own
event of the benchmark workload through vah.Event on the one GPU this test
has, with no collective between their kernels: only the host-side barrier
and the max over ranks of the device-timed interval. Each rank's final state
must equal a single-process run of the same seed, bit for bit, and the
reported time must be the slower rank's."""
import multiprocessing as mp
import os
import sys
import tempfile

import numpy as np
import pytest

import vahlib as V

sys.path.insert(0, V.ROOT)

pytestmark = pytest.mark.gpu

NX, NY, NZ, STEPS = 41, 43, 9, 6


def _run_event(vah, bench, table, seed, stream=None):
    e0 = bench.initial_energy_density(vah, table, seed, NX, NY, NZ)
    ev = vah.Event(NX, NY, NZ, bench.DX, bench.DX, bench.DZ, bench.ETA_S, physics=vah.VAH_PIMUNU_PI,
                   eos=vah.VAH_EOS_TABLE, zeta=vah.VAH_ZETA_CROSSOVER, table=table, t0=bench.T0, stream=stream)
    ev.init_from_e(bench.T0, e0, vah.VAH_PL_REFERENCE)
    return ev


def _rank(rank, world, port, outdir):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, os.path.join(V.ROOT, "gpu-vah_b200"))
    import bench
    import vah

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        stream = torch.cuda.Stream()
        table = vah.eos_table()
        ev = _run_event(vah, bench, table, bench.rank_seed(rank, 1), stream.cuda_stream)
        dist.barrier()
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        ev.run(bench.T0, bench.DT, STEPS)
        end.record(stream)
        torch.cuda.synchronize()
        elapsed = start.elapsed_time(end) / 1000.0
        slowest = bench.max_over_ranks(dist, elapsed, device="cpu")
        dist.barrier()
        np.save(os.path.join(outdir, f"e{rank}.npy"), ev.get_field(V.E))
        np.save(os.path.join(outdir, f"t{rank}.npy"), np.array([elapsed, slowest]))
        ev.close()
    finally:
        dist.destroy_process_group()


def test_two_replica_ranks_match_single_process_runs():
    ctx = mp.get_context("spawn")
    port = 29700 + os.getpid() % 1000
    with tempfile.TemporaryDirectory() as outdir:
        procs = [ctx.Process(target=_rank, args=(r, 2, port, outdir)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
            assert p.exitcode == 0
        e = [np.load(os.path.join(outdir, f"e{r}.npy")) for r in range(2)]
        t = [np.load(os.path.join(outdir, f"t{r}.npy")) for r in range(2)]

    import bench
    vah = V.product
    table = vah.eos_table()
    assert t[0][1] == t[1][1] == max(t[0][0], t[1][0])  # both ranks report the slower rank's time
    for rank in range(2):
        ev = _run_event(vah, bench, table, bench.rank_seed(rank, 1))
        ev.run(bench.T0, bench.DT, STEPS)
        alone = ev.get_field(V.E)
        ev.close()
        assert np.array_equal(e[rank], alone), rank
    assert not np.array_equal(e[0], e[1])  # the replicas ran different events
