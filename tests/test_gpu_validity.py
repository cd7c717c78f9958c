"""Validity diagnostics on the GPU (vah_event_set_validity): the Knudsen and
inverse Reynolds numbers, shear combinations and regulator maps the
reference computes at the end of every step, against the CPU oracle (itself
pinned bit for bit to the reference's VALIDITY_DOMAIN arrays); and turning
them on leaves the evolution bit-identical."""
import numpy as np
import pytest

import vahlib as V
from test_gpu_parity import conformal_workload, start_both
from test_hostcheck import validity_errors

pytestmark = pytest.mark.gpu


def table_slab():
    tab = V.eos_table()
    nx, ny, nz = 25, 23, 9
    g = V.Grid(nx, ny, nz, 0.1 * 121 / nx, 0.1 * 121 / ny, 0.1, 0.16, physics="pimunu_pi", eos="table",
               zeta="crossover", table=tab)
    e_peak = V.product.table_energy_density(tab, 0.6 / 0.197326938)
    exy, _ = V.product.mc_glauber(nx, ny, g.dx, g.dy, 7.0, seed=5, e_peak=e_peak)
    return g, (V.product.longitudinal(nz, g.dz)[:, None] * exy[None, :]).ravel(), 0.25, 0.005


@pytest.mark.parametrize("case", ["conformal_2d", "table_3d_bulk"])
@pytest.mark.parametrize("flux", [0, 2], ids=["split", "fused"])
def test_gpu_validity_matches_oracle(case, flux):
    if case == "conformal_2d":
        g, e, t0, dt = (*conformal_workload(31, 29), 0.5, 0.02)
    else:
        g, e, t0, dt = table_slab()
    o, ev = start_both(g, e, t0, flux=flux)
    o.set_validity(1)
    ev.set_validity(1)
    o.run(t0, dt, 12)
    ev.run(t0, dt, 12)
    ev.sync()
    errs = validity_errors(g, o.validity, ev.get_validity)
    assert max(errs) < 1e-8, [(k, e) for k, e in enumerate(errs) if e >= 1e-8]
    nonzero = sum(bool(np.any(g.interior(ev.get_validity(k)) != 0)) for k in range(V.NUM_VALIDITY))
    assert nonzero >= (27 if g.physics == 2 else 24)
    ev.close()


def test_gpu_validity_leaves_the_evolution_unchanged():
    g, e, t0, dt = table_slab()
    states = []
    for on in (False, True):
        ev = V.Event(g, t0=t0)
        ev.init_from_e(t0, e, 1)
        ev.set_validity(on)
        ev.run(t0, dt, 6)
        ev.sync()
        states.append({fid: ev.get_field(fid) for fid in V.state_ids(g.physics)})
        ev.close()
    for fid in states[0]:
        np.testing.assert_array_equal(states[1][fid], states[0][fid], err_msg=f"field {fid}")
