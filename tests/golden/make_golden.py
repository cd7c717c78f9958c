"""Regenerate the golden fixtures of tests/golden from the reference's own CPU
step (oracle/_ref, built from the reference sources by oracle/Makefile).

Each fixture is a short run of a small grid (every field of the physics
variant, interior + ghost layers): the seeded primitives (prim_*), the state
after the reference's setConservedVariables (cons_*, P_L = 0.0154483 e) and
setGhostCells (init_*), and the state after n reference steps (final_*). Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import vahlib as V  # noqa: E402

CASES = [
    # name, physics, eos, nx, ny, nz, dx, dz, dt, t0, steps, pi_amp
    ("ideal_conf_2d", "ideal", "conformal", 9, 8, 1, 0.2, 0.2, 0.02, 0.5, 10, 0.0),
    ("pimunu_conf_2d", "pimunu", "conformal", 9, 8, 1, 0.2, 0.2, 0.02, 0.5, 10, 0.1),
    ("pimunu_conf_3d", "pimunu", "conformal", 7, 6, 5, 0.2, 0.2, 0.02, 0.5, 5, 0.1),
    ("pimunu_pi_table_3d", "pimunu_pi", "table", 7, 6, 5, 0.2, 0.2, 0.02, 0.5, 5, 0.1),
]


def run_case(name, physics, eos, nx, ny, nz, dx, dz, dt, t0, steps, pi_amp):
    table = V.eos_table() if eos == "table" else None
    g = V.Grid(nx, ny, nz, dx, dx, dz, 0.2, physics=physics, eos=eos,
               zeta="crossover" if eos == "table" else "reference", table=table)
    r = V.Reference(g)
    f = V.smooth_initial_state(g, t0, pi_amp=pi_amp)
    V.load_state(r, f)
    prim = {fid: r.field(fid).copy() for fid in V.state_ids(g.physics)}
    r.set_conserved(t0)          # the reference's own initialisation (P_L = 0.0154483 e)
    init = {fid: r.field(fid).copy() for fid in V.state_ids(g.physics)}
    r.set_ghost_cells()
    init_g = {fid: r.field(fid).copy() for fid in V.state_ids(g.physics)}
    for n in range(steps):
        r.step(t0 + n * dt, dt)
    final = {fid: r.field(fid).copy() for fid in V.state_ids(g.physics)}
    out = {"meta": np.array([g.physics, g.eos, nx, ny, nz, dx, dz, dt, t0, steps], dtype=np.float64)}
    for fid in init:
        out[f"prim_{fid}"] = prim[fid]
        out[f"cons_{fid}"] = init[fid]
        out[f"init_{fid}"] = init_g[fid]
        out[f"final_{fid}"] = final[fid]
    if table is not None:
        out["table"] = table
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


if __name__ == "__main__":
    for case in CASES:
        run_case(*case)
        print("wrote", case[0])
