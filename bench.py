"""Benchmark of the VAH time step on B200.

Workload: one 3+1D MC-Glauber Au+Au event (b = 7 fm) on a 121x121x81 grid,
dx = dy = 0.1 fm, d(eta) = 0.1, tabulated crossover EoS, eta/s = 0.16,
crossover zeta/s, shear + bulk (N_q = 16), FP64, tau0 = 0.25 fm/c,
d(tau) = 0.005 fm/c. A step is one Heun RK2 step of the whole grid; the
metric is interior cell-updates per second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun each rank advances its own event (seed 1 + rank): events are
independent, so multi-GPU is replicas with weak scaling and no data-path
collective. Rank 0 prints one JSON line.

--impl reference times the reference's own CPU step (oracle/_ref, compiled
from the reference's sources) on the same event: one worker process per host
core (bounded by memory), each advancing its own copy of the full grid, with
the inputs built by the oracle library -- no product code is loaded.
"""
import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gpu-vah_b200"))

NX, NY, NZ = 121, 121, 81
DX, DZ = 0.1, 0.1
T0, DT, ETA_S = 0.25, 0.005, 0.16
B_IMPACT = 7.0
NQ = 16
BYTES_PER_CELL_UPDATE = (5 * NQ + 32) * 8  # algorithmic HBM bytes, FP64 storage
WORKLOAD = ("vah 3+1D MC-Glauber Au+Au b=7fm 121x121x81 dx=0.1 deta=0.1 table-EoS shear+bulk FP64, "
            "reference initialisation (P_L = 0.0154483 e, u = 0, pi = Pi = 0)")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="vah", choices=["vah", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="event", choices=["event", "batch", "serve", "precision"],
                    help="event: one 121x121x81 3+1D event; batch: 256 2+1D events of uneven size; "
                         "serve: Poisson request stream served to freeze-out")
    ap.add_argument("--serve-seconds", type=float, default=10.0, help="serve: arrival window (s)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"],
                    help="fp32: state stored and updated in FP32, inversion in FP64")
    ap.add_argument("--events", type=int, default=256)
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the untuned launch configuration (the autotuner runs during warm-up otherwise)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the FP32-form, batch and serving measurements that the default N=1 run adds")
    ap.add_argument("--extras-serve-seconds", type=float, default=2.0,
                    help="arrival window of the serving measurement in the extras (s)")
    ap.add_argument("--flux", default="per_cell", choices=["per_cell", "shared", "fused"],
                    help="per_cell: reference face semantics, face+cell launches; fused: the same in one "
                         "launch per stage; shared: each face evaluated once")
    return ap.parse_args()


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def initial_energy_density(vah, table, seed, nx=NX, ny=NY, nz=NZ):
    """MC-Glauber transverse profile x plateau+Gaussian longitudinal profile,
    peak temperature 0.6 GeV under the tabulated EoS, plus 1e-3 fm^-4 after the
    product as InitialConditions.cpp:247 adds it (interior, x fastest)."""
    e_peak = vah.table_energy_density(table, 0.6 / vah.HBARC)
    exy, _ = vah.mc_glauber(nx, ny, DX, DX, B_IMPACT, seed, e_peak=e_peak, e_floor=0.0)
    f = vah.longitudinal(NZ, DZ)
    k0 = (NZ - nz) // 2
    return np.ascontiguousarray((f[k0:k0 + nz, None] * exy[None, :]).ravel() + 1e-3)


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.dev)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"),
                                 parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------- ranks ----
# N > 1: one process per GPU, each running its own replica (the events are
# independent: no data-path collective). Only the timing crosses ranks.
def max_over_ranks(dist, seconds, device="cuda"):
    """The slowest rank's time (the whole job ends when it does)."""
    if dist is None:
        return seconds
    import torch

    t = torch.tensor([seconds], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, units_per_rank, seconds):
    """Units all ranks processed per second of the slowest rank (weak scaling)."""
    return world * units_per_rank / seconds


def rank_seed(rank, base):
    """Each replica runs its own seeded event(s)."""
    return base + rank


# ------------------------------------------------------------ CPU baseline --
def event_config(cells=NX * NY * NZ):
    """The workload both arms time (identical dicts in both JSON lines)."""
    return {"workload": WORKLOAD, "cells": cells, "tau0_fm": T0, "dt_fm": DT, "eta_over_s": ETA_S,
            "b_fm": B_IMPACT, "seed": 1, "l2": "inputs larger than L2 (state 0.55 GB per event)"}


def _ref_worker(args):
    """One worker process: the reference's own CPU step (oracle/_ref, built from
    the reference's sources; the C restatement where it was not built)
    advancing its block (rows j0..j1, planes k0..k1, all of x) of the
    121x121x81 event, with the reference's own ghost fill around the block.
    The EoS table and the initial condition come from the oracle library's
    copy of the workload's generators (bit-identical to the library's), so
    this process maps no product code."""
    conn, steps, warm, seed, (j0, j1, k0, k1) = args
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import vahlib as V
    table = V.oracle_eos_table()
    ny, nz = j1 - j0, k1 - k0
    g = V.Grid(NX, ny, nz, DX, DX, DZ, ETA_S, physics="pimunu_pi", eos="table", zeta="crossover", table=table)
    use_ref = V.ref_available(g.physics, g.eos)
    impl = V.Reference(g) if use_ref else V.Oracle(g)
    e_peak = V.table_energy_density(table, 0.6 / 0.197326938)
    exy, _ = V.oracle_mc_glauber(NX, NY, DX, DX, B_IMPACT, seed, e_peak=e_peak, e_floor=0.0)
    f = V.oracle_longitudinal(NZ, DZ)
    e = ((f[:, None] * exy[None, :]) + 1e-3).reshape(NZ, NY, NX)[k0:k1, j0:j1, :]
    full = np.zeros(g.shape)
    full[2:-2, 2:-2, 2:-2] = e
    n = int(table[0])
    p = np.interp(np.log(np.maximum(full, 1e-300)), table[1] + table[3] * np.arange(n), table[8:8 + n])
    V.load_state(impl, {V.E: full.ravel(), V.PP: p.ravel(), V.UT: np.ones(g.ncell), V.PL: p.ravel()})
    if use_ref:
        impl.set_conserved(T0)  # the reference's own initialisation
    else:
        impl.set_conserved(T0, 0)
    impl.set_ghost_cells()
    conn.send(("ready", "reference" if use_ref else "port"))
    t = T0
    for n in range(warm + steps):
        conn.recv()
        a = time.perf_counter()
        impl.step(t, DT)
        conn.send(time.perf_counter() - a)
        t += DT
    conn.close()


def ref_blocks(workers):
    """The 121x121x81 event cut into at most `workers` blocks of whole x rows:
    eta slabs of at least 3 planes (3+1D arithmetic in every block), then y
    bands; the blocks cover every cell once."""
    def cuts(n, parts):
        return [round(n * q / parts) for q in range(parts + 1)]
    pz = max(1, min(workers, NZ // 3))
    py = max(1, min(workers // pz, NY // 8))
    kz, jy = cuts(NZ, pz), cuts(NY, py)
    return [(jy[a], jy[a + 1], kz[b], kz[b + 1]) for b in range(pz) for a in range(py)]


def cpu_step_rate(workers, steps, warmup, seed=1):
    """One RK2 step of the event per step, its blocks (ref_blocks) stepped in
    lockstep by spawned workers, one per block and host core; returns
    (cell-updates/s of the event, kind, per-step wall s)."""
    ctx = mp.get_context("spawn")
    pipes, procs = [], []
    blocks = ref_blocks(workers)
    for box in blocks:
        a, b = ctx.Pipe()
        p = ctx.Process(target=_ref_worker, args=((b, steps, warmup, seed, box),))
        p.start()
        pipes.append(a)
        procs.append(p)
    kinds = {pipe.recv()[1] for pipe in pipes}
    walls = []
    for n in range(warmup + steps):
        a = time.perf_counter()
        for pipe in pipes:
            pipe.send("go")
        for pipe in pipes:
            pipe.recv()
        if n >= warmup:
            walls.append(time.perf_counter() - a)
    for p in procs:
        p.join(timeout=60)
    rate = NX * NY * NZ * len(walls) / sum(walls)
    return rate, kinds.pop(), walls


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


REF_EVENT_BYTES = 1.3e9  # resident size of one reference process on the full event (measured: 1.02 GB)


def available_memory_bytes():
    """MemAvailable, bounded by the cgroup limit when one is set."""
    avail = None
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    avail = int(line.split()[1]) * 1024
    except Exception:
        pass
    for path in ("/sys/fs/cgroup/memory.max", "/sys/fs/cgroup/memory/memory.limit_in_bytes"):
        try:
            with open(path) as f:
                v = f.read().strip()
            if v != "max":
                lim = int(v)
                if lim < (1 << 60):
                    avail = lim if avail is None else min(avail, lim)
        except Exception:
            pass
    return avail


# -------------------------------------------------------------- main arms --
def run_reference(args, rank, world):
    if rank != 0:
        return
    cores = host_cores()
    workers = max(1, min(cores, 64))
    mem = available_memory_bytes()
    if mem is not None:  # a block's process: the interpreter plus its share of the event's arrays
        while workers > 1 and len(ref_blocks(workers)) * (0.2e9 + REF_EVENT_BYTES / len(ref_blocks(workers))) > 0.6 * mem:
            workers -= 1
    blocks = ref_blocks(workers)
    rate, kind, walls = cpu_step_rate(workers, args.steps, args.warmup)
    ms = 1000 * statistics.mean(walls)
    pz = len({b[2:] for b in blocks})
    sample = (f"one RK2 step of the {NX}x{NY}x{NZ} event (seed 1) per step, cut into {len(blocks)} blocks "
              f"({pz} eta slabs x {len(blocks) // pz} y bands, the reference's ghost fill around each) stepped in "
              f"lockstep by as many worker processes; {cores} host cores")
    workers = len(blocks)
    line = {"impl": "reference", "metric": "cell-updates/s", "value": rate, "unit": "cell-updates/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": event_config(),
            "cpu_baseline": {"value": rate, "unit": "cell-updates/s", "cores": workers, "kind": kind,
                             "sample": sample},
            "e2e": {"value": rate, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# Nominal FP64 vector peak: 64 DFMA per cycle per SM (the profiler's
# peak_sustained for sm__sass_thread_inst_executed_op_dfma_pred_on) x 2 FLOP
# x 148 SMs x 1965 MHz; the bench measures the device's own (vah_fp64_peak).
FP64_PEAK_TFLOPS = 64 * 2 * 148 * 1.965e9 / 1e12


def fp64_roofline(cells, flux, precision, stage_s, peak=None):
    """FP64 FLOP/s of one RK stage against the FP64 peak (measured when given,
    else nominal), from the FLOP count per cell and stage in the committed ncu
    summary (the FP32 form: the tile kernel's)."""
    tile = precision == "fp32"
    path = os.path.join(ROOT, "profiles", "tile_stage_dram.json" if tile else "split_stage_dram.json")
    if (flux != "per_cell" and not tile) or not os.path.exists(path) or not stage_s:
        return None
    with open(path) as f:
        d = json.load(f)
    per = d.get("fp64_flop_per_cell_per_stage") if tile else d.get("fp64_flop_per_cell_per_stage", {}).get(precision)
    if not per:
        return None
    achieved = per * cells / stage_s / 1e12
    if peak:
        return {"achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "flop_per_cell_update": 2 * per,
                "peak_kind": "measured FP64 FMA throughput (vah_fp64_peak: independent DFMA chains, this run)",
                "nominal_peak": FP64_PEAK_TFLOPS}
    return {"achieved": achieved, "peak": FP64_PEAK_TFLOPS, "unit": "TFLOP/s", "frac": achieved / FP64_PEAK_TFLOPS,
            "flop_per_cell_update": 2 * per, "peak_kind": "nominal FP64 vector peak (64 DFMA/cycle/SM at 1965 MHz)"}


def traffic_per_launch(cells, flux, precision):
    """DRAM bytes of one RK stage (its launches) from the committed ncu
    summaries (bytes per interior cell, scaled to this event), or None. The
    FP32 form runs the tile kernel whatever the face option."""
    if precision == "fp32":
        path = os.path.join(ROOT, "profiles", "tile_stage_dram.json")
        if not os.path.exists(path):
            return None
        with open(path) as f:
            per = json.load(f).get("dram_bytes_per_cell_per_stage", {}).get("mean")
        return per * cells if per else None
    if flux == "fused":
        name, key = "stage_kernel_dram.json", None
    elif flux == "per_cell":
        name, key = "split_stage_dram.json", precision
    else:
        return None
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    if key is None:
        per = d.get("dram_bytes_per_cell_per_launch") if precision == "fp64" else None
    else:
        per = d.get("dram_bytes_per_cell_per_stage", {}).get(key)
    return per * cells if per else None


BATCH_SIDES = (81, 121, 161, 201)
BATCH_DT = 0.01


def batch_events(n, seed):
    """The 2+1D batch: sides drawn from {81,121,161,201}, b uniform in [0,12] fm."""
    rng = np.random.default_rng(seed)
    return [(int(rng.choice(BATCH_SIDES)), float(rng.uniform(0, 12)), int(rng.integers(1, 2 ** 31))) for _ in range(n)]


def run_batch(args, rank, world, dist):
    import torch
    import vah

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    table = vah.eos_table()
    prec = vah.VAH_FP32 if args.precision == "fp32" else vah.VAH_FP64
    flux = {"per_cell": vah.VAH_FLUX_PER_CELL, "shared": vah.VAH_FLUX_SHARED}[args.flux]
    batch = vah.Batch(table=table, precision=prec, flux=flux, device=local, stream=stream.cuda_stream,
                      capacity_bytes=150 << 30)
    e_peak = vah.table_energy_density(table, 0.6 / vah.HBARC)
    cells = 0
    for side, b, seed in batch_events(args.events, rank_seed(rank, 1000)):
        exy, _ = vah.mc_glauber(side, side, DX, DX, b, seed, e_peak=e_peak)
        slot = batch.add(side, side, 1, DX, DX, DZ, T0, BATCH_DT, ETA_S, exy)
        assert slot is not None, "batch capacity"
        cells += side * side
    batch.step(args.warmup)
    batch.sync()
    tune = [] if args.no_autotune else batch.autotune(3)  # before the timed region; the state is unchanged
    batch.step(1)  # re-capture the step graph with the chosen variants (untimed)
    batch.sync()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        start.record(stream)
        batch.step(args.steps)
        end.record(stream)
        torch.cuda.synchronize()
    elapsed = max_over_ranks(dist, start.elapsed_time(end) / 1000.0)
    batch.close()
    if rank != 0:
        return
    w = 4 if prec == vah.VAH_FP32 else 8
    bpc = (5 * NQ + 32) * w
    value = whole_job_rate(world, cells * args.steps, elapsed)
    peak, peak_kind = measured_peaks()
    achieved = bpc * cells * args.steps / elapsed / 1e9
    line = {"metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * elapsed / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64-inversion" if prec == vah.VAH_FP32 else "f64", "data": "synthetic",
            "config": {"workload": f"vah batch: {args.events} 2+1D MC-Glauber events, sides {BATCH_SIDES}, dx=0.1, "
                                   f"b~U[0,12], table EoS, shear+bulk, dtau={BATCH_DT}",
                       "events": args.events, "cells_per_step": cells, "faces": args.flux,
                       "l2": "inputs larger than L2", "launch": "persistent tile work-list, CUDA graph per step",
                       "autotune": {k: c for k, c in zip(("face_x", "face_y", "face_z", "cell_2d", "cell_3d"), tune)}},
            "events_step_per_s": world * args.events * args.steps / elapsed,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_kind": f"{peak_kind} copy bandwidth",
                         "algorithmic_bytes_per_cell_update": bpc, "kernel": "whole step (graph)"}}
    s = clk.summary()
    if s:
        line["clocks"] = s
    print(json.dumps(line), flush=True)


def run_serve(args, rank, world, dist):
    import vah

    if rank != 0:
        return
    prec = vah.VAH_FP32 if args.precision == "fp32" else vah.VAH_FP64
    flux = {"per_cell": vah.VAH_FLUX_PER_CELL, "shared": vah.VAH_FLUX_SHARED}[args.flux]
    res, lat = vah.serve(rate=50.0, duration_s=args.serve_seconds, seed=1, precision=prec, flux=flux,
                         T0_GeV=0.4, e_floor=1e-2, t_max=100.0, ic_threads=max(2, min(host_cores(), 32)),
                         ic_on_device=1)
    line = {"metric": "events/s", "value": res["events_per_s"], "unit": "events/s", "n_gpus": 1,
            "steps": None, "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64-inversion" if prec == vah.VAH_FP32 else "f64",
            "data": "synthetic",
            "config": {"workload": "vah serving: Poisson 50 events/s, 70% 2+1D side U[61,261], 30% 3+1D "
                                   "81^2x41..161^2x81, b~U[0,14], dx=0.2, deta=0.2, dtau=0.02, MC-Glauber peak "
                                   "T0=0.4 GeV + 0.01 fm^-4 floor, table EoS, eta/s=0.16, retired at max T<150 MeV "
                                   "over converged cells (timeout tau=100 fm/c); ICs generated on the GPU at "
                                   "admission",
                       "arrival_window_s": args.serve_seconds, "faces": args.flux},
            "latency_p50_s": res["p50_s"], "latency_p99_s": res["p99_s"], "serve": res}
    print(json.dumps(line), flush=True)


def run_precision(args, rank, world, dist):
    """FP32 form against the FP64 form on the same events: per-event total
    energy, momentum anisotropy eps_p and <u_T> along the evolution (FP64
    device reductions over converged cells), and the freeze-out surface volume.
    (1) 2+1D events of the serving workload (side U[61, 261], b U[0, 14] fm,
        dx = 0.2, dtau = 0.02, peak T0 = 0.4 GeV, 0.01 fm^-4 floor), run to
        freeze-out;
    (2) 32 events of the batch workload (sides {81, 121, 161, 201}, b U[0, 12]
        fm, dx = 0.1, dtau = 0.01, peak T0 = 0.6 GeV), run to freeze-out;
    (3) the 201x201x101 3+1D event (dx = 0.1, deta = 0.08) to tau = 1.2 fm/c,
        where the reference algorithm is still stable on it.
    Errors are stated over two windows per event: while neither run has had an
    inversion fallback (cell or face), and up to the FP64 run's freeze-out. A
    fallback (e = 0.999 e_prev, u = (1, 0, 0, 0) for the cell or face state)
    is a discontinuous event whose place and step depend on the last bits of
    an ill-conditioned inversion at the dilute edge, so from the first one on
    the two runs' edges evolve differently; once the reference's fallback
    spreads through the dilute front (tens of percent of the inversions there,
    in the reference's own CPU code too), edge cells evolve chaotically in
    both forms. The FP32 form evaluates
    each face once (shared faces); the same comparison for the FP64 form with
    shared faces separates that part of the difference from FP32 rounding."""
    import vah

    if rank != 0:
        return
    table = vah.eos_table()

    def compare(events, dx, dt, t_end, sample, e_peak_GeV, floor, nz=1, deta=DZ):
        runs = []
        forms = ((vah.VAH_FP64, vah.VAH_FLUX_PER_CELL), (vah.VAH_FP32, vah.VAH_FLUX_PER_CELL),
                 (vah.VAH_FP64, vah.VAH_FLUX_SHARED))
        for prec, flux in forms:
            b = vah.Batch(table=table, precision=prec, flux=flux, capacity_bytes=150 << 30)
            e_peak = vah.table_energy_density(table, e_peak_GeV / vah.HBARC)
            ef = vah.table_energy_density(table, 0.150 / vah.HBARC)
            slots = []
            for side, bimp, seed in events:
                exy, _ = vah.mc_glauber(side, side, dx, dx, bimp, seed, e_peak=e_peak, e_floor=0.0)
                f = vah.longitudinal(nz, deta) if nz > 1 else np.ones(1)
                slots.append(b.add(side, side, nz, dx, dx, deta, T0, dt, ETA_S,
                                   (f[:, None] * exy[None, :]).ravel() + floor))
            n = max(slots) + 1
            t, obs, vol, frozen, fb = T0, [], [], [], []
            done = np.zeros(len(slots), bool)
            while t < t_end - 1e-9 and not done.all():
                b.step(sample)
                t += sample * dt
                obs.append(b.observables(n)[slots].copy())
                vol.append(b.freezeout_volume(n)[slots].copy())
                done |= b.max_energy_density(n)[slots] < ef
                frozen.append(done.copy())
                fb.append([(b.info(s).cell_fallbacks, b.info(s).face_fallbacks) for s in slots])
            b.close()
            runs.append((np.array(obs), np.array(vol), np.array(frozen), np.array(fb)))
        o64, v64, f64, fb64 = runs[0]

        def errs(a, b_):
            big = np.abs(b_[:, 1]) >= 0.01
            return {"E_tot": float(np.max(np.abs(a[:, 0] - b_[:, 0]) / np.abs(b_[:, 0]))),
                    "eps_p_abs": float(np.max(np.abs(a[:, 1] - b_[:, 1]))),
                    "eps_p_rel": float(np.max(np.abs(a[big, 1] - b_[big, 1]) / np.abs(b_[big, 1]))) if big.any()
                    else 0.0,
                    "uT_mean": float(np.max(np.abs(a[:, 2] - b_[:, 2]) / np.abs(b_[:, 2])))}

        def against_fp64(run):
            o32, v32, _, fb32 = run
            m = min(len(o64), len(o32))
            any64, any32 = fb64[:m].sum(axis=2), fb32[:m].sum(axis=2)  # cell + face fallbacks so far
            keys = ("E_tot", "eps_p_abs", "eps_p_rel", "uT_mean")
            clean, full = dict.fromkeys(keys, 0.0), dict.fromkeys(keys, 0.0)
            full["freezeout_volume"] = 0.0
            tau_clean, tau_f, frozen_events = [], [], 0
            for k in range(len(events)):
                hits = np.nonzero(f64[:m, k])[0]
                last = int(hits[0]) if len(hits) else m - 1
                dirty = np.nonzero((any64[:, k] > 0) | (any32[:, k] > 0))[0]
                ck = (int(dirty[0]) - 1) if len(dirty) else last
                if ck >= 0:
                    for key, v in errs(o32[:ck + 1, k], o64[:ck + 1, k]).items():
                        clean[key] = max(clean[key], v)
                    tau_clean.append(T0 + (ck + 1) * sample * dt)
                if len(hits) or nz > 1:
                    for key, v in errs(o32[:last + 1, k], o64[:last + 1, k]).items():
                        full[key] = max(full[key], v)
                if len(hits):
                    frozen_events += 1
                    tau_f.append(T0 + (last + 1) * sample * dt)
                    full["freezeout_volume"] = max(full["freezeout_volume"],
                                                   float(abs(v32[last, k] - v64[last, k]) / abs(v64[last, k])))
            if not frozen_events:
                del full["freezeout_volume"]
            return {"before_any_fallback": dict(clean, tau_end_median=float(np.median(tau_clean)) if tau_clean else None),
                    "to_freezeout": dict(full, tau_freeze_median=float(np.median(tau_f)) if tau_f else None),
                    "frozen_events": frozen_events, "cell_fallbacks": int(fb32[m - 1, :, 0].sum()),
                    "face_fallbacks": int(fb32[m - 1, :, 1].sum())}

        return {"events": len(events), "fp64_cell_fallbacks": int(fb64[-1, :, 0].sum()),
                "fp64_face_fallbacks": int(fb64[-1, :, 1].sum()),
                "fp32_form": against_fp64(runs[1]), "fp64_shared_faces": against_fp64(runs[2])}

    rng = np.random.default_rng(7)
    events2d = [(int(rng.integers(61, 262)), float(rng.uniform(0, 14)), int(rng.integers(1, 2 ** 31)))
                for _ in range(32)]
    t0 = time.perf_counter()
    out = {"2+1D_32_events": compare(events2d, 0.2, 0.02, 40.0, 10, 0.4, 1e-2),
           "2+1D_batch_32_events": compare(batch_events(32, 1000), DX, BATCH_DT, 40.0, 10, 0.6, 1e-3),
           "3+1D_201x201x101_to_tau_1.2": compare([(201, 7.0, 1)], DX, DT, 1.2, 10, 0.6, 1e-3, nz=101, deta=0.08)}
    worst = max(max(v["fp32_form"]["before_any_fallback"][k] for k in ("E_tot", "eps_p_rel", "uT_mean"))
                for v in out.values())
    line = {"metric": "FP32-form max relative observable error vs FP64", "value": worst, "unit": "relative",
            "higher_is_better": False, "n_gpus": 1, "data": "synthetic", "dtype": "f32+f64-inversion vs f64",
            "config": {"workload": "precision: E_tot(tau), eps_p(tau) (relative where |eps_p| >= 0.01, and absolute), "
                                   "<u_T>(tau), freeze-out volume; FP32 form (shared faces) and FP64 form with shared "
                                   "faces vs the FP64 form (reference faces) on the same events; value = worst "
                                   "relative error of the FP32 form while neither run has had an inversion fallback",
                       "wall_s": round(time.perf_counter() - t0, 1)},
            "errors": out}
    print(json.dumps(line), flush=True)


# ------------------------------------------------ the rest of the metric --
# The workload's metric covers cell-updates/s and events/s in the FP64 form
# and the FP32 form, and p50/p99 latency for serving. The default N=1 run
# measures each of them after the headline (FP64 event) number, with its own
# clock record, and adds them to the same JSON line.

def event_form_rate(vah, table, e0, precision, steps, warmup, local, stream, e2e_steps=0):
    """One event of the workload in the given form: cell-updates/s over `steps`
    device-timed steps after `warmup`, with the average stage time; then, when
    e2e_steps > 0, the same through the host-buffer entry point (pinned FP64
    host state in and out every step, wall-clocked)."""
    import torch

    ev = vah.Event(NX, NY, NZ, DX, DX, DZ, ETA_S, physics=vah.VAH_PIMUNU_PI, eos=vah.VAH_EOS_TABLE,
                   zeta=vah.VAH_ZETA_CROSSOVER, table=table, t0=T0, device=local, stream=stream.cuda_stream,
                   precision=precision)
    ev.init_from_e(T0, e0, vah.VAH_PL_REFERENCE)
    t = T0
    ev.run(t, DT, warmup)
    t += warmup * DT
    ev.sync()
    torch.cuda.synchronize()
    ev.set_timing(True)
    ev.kernel_time()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        start.record(stream)
        ev.run(t, DT, steps)
        end.record(stream)
        torch.cuda.synchronize()
    elapsed = start.elapsed_time(end) / 1000.0
    kms, launches = ev.kernel_time()
    ev.set_timing(False)
    ev.sync()
    stats = ev.stats()
    t += steps * DT
    cells = NX * NY * NZ
    out = {"value": cells * steps / elapsed, "ms_per_step": 1000 * elapsed / steps,
           "avg_stage_ms": kms / max(launches, 1), "stage_launches": launches, "clocks": clk.summary(),
           "fallbacks": {"face": stats.face_fallbacks, "cell": stats.cell_fallbacks, "nan": stats.nan_cells}}
    if e2e_steps > 0:
        host = {fid: torch.from_numpy(ev.get_field(fid)).pin_memory() for fid in range(26)}
        ptrs = [host[fid].data_ptr() if fid in host else 0 for fid in range(vah.NUM_FIELDS)]
        ev.step_host(t, DT, ptrs)  # warm
        t += DT
        a = time.perf_counter()
        for n in range(e2e_steps):
            ev.step_host(t, DT, ptrs)
            t += DT
        state_bytes = sum(h.numel() * 8 for h in host.values())
        out["e2e"] = {"value": cells * e2e_steps / (time.perf_counter() - a), "unit": "cell-updates/s",
                      "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes, "steps": e2e_steps}
    ev.close()
    return out


def late_regime_rates(vah, table, e0, precision, local, stream, steps=20):
    """The same event later in its evolution: device-timed `steps` steps from
    tau = 1.0 fm/c (flow developed, no inversion fallback yet) and from
    tau = 1.4 fm/c (the reference's inversion fallback spreading through the
    dilute edge; the event reaches NaN soon after 1.5), with the fallbacks per
    step in each window; a window that meets a NaN says so instead."""
    import torch

    ev = vah.Event(NX, NY, NZ, DX, DX, DZ, ETA_S, physics=vah.VAH_PIMUNU_PI, eos=vah.VAH_EOS_TABLE,
                   zeta=vah.VAH_ZETA_CROSSOVER, table=table, t0=T0, device=local, stream=stream.cuda_stream,
                   precision=precision)
    ev.init_from_e(T0, e0, vah.VAH_PL_REFERENCE)
    t, out = T0, {}
    for start in (1.0, 1.4):
        n = int(round((start - t) / DT))
        ev.run(t, DT, n)
        t += n * DT
        s0 = ev.stats()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ev.run(t, DT, steps)
        b.record(stream)
        torch.cuda.synchronize()
        t += steps * DT
        s1 = ev.stats()
        key = f"tau_{start:.1f}"
        if s1.nan_cells:
            out[key] = {"nan_cells": s1.nan_cells}
            break
        ms = a.elapsed_time(b) / steps
        out[key] = {"ms_per_step": ms, "value": NX * NY * NZ / (ms / 1000.0),
                    "face_fallbacks_per_step": (s1.face_fallbacks - s0.face_fallbacks) / steps,
                    "cell_fallbacks_per_step": (s1.cell_fallbacks - s0.cell_fallbacks) / steps}
    ev.close()
    return out


def batch_form_rate(vah, table, precision, nevents, steps, warmup, local, stream):
    """The 2+1D batch workload (nevents MC-Glauber events, sides from
    {81, 121, 161, 201}, b uniform in [0, 12] fm, dx = 0.1 fm, initial
    conditions generated on the device): cell-updates/s and event-steps/s."""
    import torch

    b = vah.Batch(table=table, precision=precision, device=local, stream=stream.cuda_stream,
                  capacity_bytes=150 << 30)
    e_peak = vah.table_energy_density(table, 0.6 / vah.HBARC)
    cells = 0
    for side, bimp, seed in batch_events(nevents, 1000):
        slot = b.add_glauber(side, side, 1, DX, DX, DZ, T0, BATCH_DT, ETA_S, bimp, seed, e_peak, e_floor=1e-3)
        assert slot is not None, "batch capacity"
        cells += side * side
    b.step(warmup)
    b.sync()
    if precision == vah.VAH_FP64:
        b.autotune(3)
        b.step(1)  # re-capture with the chosen variants (untimed)
        b.sync()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        start.record(stream)
        b.step(steps)
        end.record(stream)
        torch.cuda.synchronize()
    elapsed = start.elapsed_time(end) / 1000.0
    b.close()
    return {"cell_updates_per_s": cells * steps / elapsed, "event_steps_per_s": nevents * steps / elapsed,
            "ms_per_step": 1000 * elapsed / steps, "events": nevents, "cells_per_step": cells,
            "clocks": clk.summary()}


def serve_form_stats(vah, precision, seconds, local):
    """A short window of the serving workload: Poisson arrivals at 50/s, 70%
    2+1D (side U[61, 261]) and 30% 3+1D (81^2 x 41 .. 161^2 x 81), served to
    freeze-out; events/s and p50/p99 latency."""
    with ClockSampler(local) as clk:
        res, lat = vah.serve(rate=50.0, duration_s=seconds, seed=1, precision=precision, T0_GeV=0.4, e_floor=1e-2,
                             t_max=100.0, ic_threads=max(2, min(host_cores(), 32)), ic_on_device=1, device=local)
    keys = ("offered", "completed", "failed", "timeouts", "events_per_s", "p50_s", "p99_s", "cell_updates_per_s",
            "max_resident", "wall_s")
    out = {k: res[k] for k in keys}
    out["window_s"] = seconds
    out["clocks"] = clk.summary()
    return out


def run_vah(args, rank, world, dist):
    import torch
    import vah

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()  # a real stream handle: the library queues its kernels on it
    table = vah.eos_table()
    e0 = initial_energy_density(vah, table, seed=rank_seed(rank, 1))
    prec = vah.VAH_FP32 if args.precision == "fp32" else vah.VAH_FP64
    ev = vah.Event(NX, NY, NZ, DX, DX, DZ, ETA_S, physics=vah.VAH_PIMUNU_PI, eos=vah.VAH_EOS_TABLE,
                   zeta=vah.VAH_ZETA_CROSSOVER, table=table, t0=T0, device=local, stream=stream.cuda_stream,
                   precision=prec,
                   flux={"per_cell": vah.VAH_FLUX_PER_CELL, "shared": vah.VAH_FLUX_SHARED,
                         "fused": vah.VAH_FLUX_PER_CELL_FUSED}[args.flux])
    ev.init_from_e(T0, e0, vah.VAH_PL_REFERENCE)  # as the reference initialises (the reference arm does the same)
    t = T0
    ev.run(t, DT, args.warmup)
    t += args.warmup * DT
    ev.sync()
    tune = [] if args.no_autotune else ev.autotune(3)  # before the timed region; the state is unchanged
    ev.sync()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    barrier()
    ev.set_timing(True)
    ev.kernel_time()  # reset
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        start.record(stream)
        ev.run(t, DT, args.steps)
        end.record(stream)
        torch.cuda.synchronize()
    t += args.steps * DT
    elapsed = start.elapsed_time(end) / 1000.0
    kms, launches = ev.kernel_time()
    ev.set_timing(False)
    ev.sync()
    elapsed = max_over_ranks(dist, elapsed)
    cells = NX * NY * NZ
    value = whole_job_rate(world, cells * args.steps, elapsed)

    # end to end through the host-buffer entry point (pinned host state, H2D + step + D2H per step)
    ids = list(range(16)) + list(range(16, 26))
    host = {fid: torch.from_numpy(ev.get_field(fid)).pin_memory() for fid in ids}
    ptrs = [host[fid].data_ptr() if fid in host else 0 for fid in range(vah.NUM_FIELDS)]
    ev.step_host(t, DT, ptrs)  # warm
    t += DT
    barrier()
    a = time.perf_counter()
    for n in range(args.e2e_steps):
        ev.step_host(t, DT, ptrs)
        t += DT
    e2e_s = max_over_ranks(dist, time.perf_counter() - a)
    e2e_value = whole_job_rate(world, cells * args.e2e_steps, e2e_s)
    state_bytes = sum(h.numel() * 8 for h in host.values())
    stats = ev.stats()
    ev.close()

    if rank != 0:
        return
    peak, peak_kind = measured_peaks()
    fp64_peak = vah.fp64_peak(local)[0]  # measured FP64 FMA throughput of this device (TFLOP/s)
    avg_launch_s = kms / 1000.0 / max(launches, 1)
    bpc = BYTES_PER_CELL_UPDATE if prec == vah.VAH_FP64 else BYTES_PER_CELL_UPDATE // 2
    bytes_per_launch = bpc / 2 * cells
    achieved = bytes_per_launch / avg_launch_s / 1e9
    line = {"metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * elapsed / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64-inversion" if prec == vah.VAH_FP32 else "f64", "data": "synthetic",
            "config": event_config(cells) if prec == vah.VAH_FP64 else
            dict(event_config(cells), workload=WORKLOAD.replace("FP64", "FP32 state")),
            "launch": {"faces": args.flux, "global_batch": world, "parallelism": "replicas",
                       "autotune": {k: c for k, c in zip(("face_x", "face_y", "face_z", "cell"), tune)}},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic_per_launch(cells, args.flux, args.precision),
                         "peak_kind": f"{peak_kind} copy bandwidth",
                         "algorithmic_bytes_per_cell_update": bpc,
                         "kernel": ("tile_kernel (one TMA-tiled launch per RK stage)" if prec == vah.VAH_FP32
                                    else "stage_kernel (one fused RK stage)" if args.flux == "fused"
                                    else "one RK stage: face_kernel x3 + cell_kernel") + ", average over the two stages",
                         "avg_stage_ms": 1000 * avg_launch_s,
                         "fp64": fp64_roofline(cells, args.flux, args.precision, avg_launch_s, fp64_peak)},
            "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": state_bytes,
                    "d2h_bytes_per_step": state_bytes, "steps": args.e2e_steps,
                    "path": "vah_rk2_step_host (pinned host state in, one step, state out)"},
            "gpu_launches": launches * (1 if args.flux == "fused" or prec == vah.VAH_FP32 else 4),
            "stats": {"face_fallbacks": stats.face_fallbacks, "cell_fallbacks": stats.cell_fallbacks,
                      "nan_cells": stats.nan_cells}}
    clk_summary = clk.summary()
    if clk_summary:
        line["clocks"] = clk_summary
    if world == 1 and not args.no_extras and args.flux == "per_cell":
        other = vah.VAH_FP32 if prec == vah.VAH_FP64 else vah.VAH_FP64
        form = event_form_rate(vah, table, e0, other, args.steps, args.warmup, local, stream, args.e2e_steps)
        bpc_o = BYTES_PER_CELL_UPDATE // 2 if other == vah.VAH_FP32 else BYTES_PER_CELL_UPDATE
        ach = bpc_o / 2 * cells / (form["avg_stage_ms"] / 1000.0) / 1e9
        form.update({"unit": "cell-updates/s", "dtype": "f32+f64-inversion" if other == vah.VAH_FP32 else "f64",
                     "ratio_to_headline": form["value"] / value,
                     "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                                  "traffic": traffic_per_launch(cells, args.flux,
                                                                "fp32" if other == vah.VAH_FP32 else "fp64"),
                                  "algorithmic_bytes_per_cell_update": bpc_o,
                                  "fp64": fp64_roofline(cells, args.flux,
                                                        "fp32" if other == vah.VAH_FP32 else "fp64",
                                                        form["avg_stage_ms"] / 1000.0, fp64_peak),
                                  "kernel": "tile_kernel (one TMA-tiled launch per stage)" if other == vah.VAH_FP32
                                  else "one RK stage: face_kernel x3 + cell_kernel"}})
        line["fp32_form" if other == vah.VAH_FP32 else "fp64_form"] = form
        line["late"] = {name: late_regime_rates(vah, table, e0, p, local, stream)
                        for name, p in (("fp64", vah.VAH_FP64), ("fp32", vah.VAH_FP32))}
        line["batch"] = {name: batch_form_rate(vah, table, p, 256, args.steps, args.warmup, local, stream)
                         for name, p in (("fp64", vah.VAH_FP64), ("fp32", vah.VAH_FP32))}
        line["batch"]["workload"] = ("256 2+1D MC-Glauber events, sides {81,121,161,201}, dx=0.1, b~U[0,12] fm, "
                                     f"table EoS, shear+bulk, dtau={BATCH_DT}, ICs on the device")
        line["serve"] = {name: serve_form_stats(vah, p, args.extras_serve_seconds, local)
                         for name, p in (("fp64", vah.VAH_FP64), ("fp32", vah.VAH_FP32))}
        line["serve"]["workload"] = ("Poisson 50 events/s, 70% 2+1D side U[61,261], 30% 3+1D 81^2x41..161^2x81, "
                                     "b~U[0,14], dx=deta=0.2, dtau=0.02, peak T0=0.4 GeV, served to max T<150 MeV")
    if world == 1 and not args.no_cpu_baseline:
        rate, kind, walls = cpu_step_rate(1, 1, 0)
        line["cpu_baseline"] = {"value": rate, "unit": "cell-updates/s", "cores": 1, "kind": kind,
                                "sample": f"one RK2 step of the full {NX}x{NY}x{NZ} event on one core "
                                          f"({walls[0]:.1f} s)"}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod
        if args.impl == "reference":
            if rank != 0:
                return
        else:
            dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
            dist = dist_mod
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        elif args.workload == "batch":
            run_batch(args, rank, world, dist)
        elif args.workload == "serve":
            run_serve(args, rank, world, dist)
        elif args.workload == "precision":
            run_precision(args, rank, world, dist)
        else:
            run_vah(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
