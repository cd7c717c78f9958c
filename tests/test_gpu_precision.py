"""The FP32 form (state stored and updated in FP32, Newton inversion and
reductions in FP64) against the FP64 form on the same event: per-event total
energy, momentum anisotropy and mean transverse flow within 1e-4 relative."""
import os
import sys

import numpy as np
import pytest

import vahlib as V

sys.path.insert(0, os.path.join(V.ROOT, "gpu-vah_b200"))
import observables as OBS  # noqa: E402

pytestmark = pytest.mark.gpu


def run(precision, flux, steps, nx=61, ny=61, nz=21):
    tab = V.eos_table()
    g = V.Grid(nx, ny, nz, 0.2, 0.2, 0.1, 0.16, physics="pimunu_pi", eos="table", zeta="crossover", table=tab)
    e_peak = V.product.table_energy_density(tab, 0.6 / 0.197326938)
    exy, _ = V.product.mc_glauber(nx, ny, 0.2, 0.2, 5.0, seed=9, e_peak=e_peak)
    e3 = (V.product.longitudinal(nz, g.dz)[:, None] * exy[None, :]).ravel()
    ev = V.Event(g, t0=0.25, precision=precision, flux=flux)
    ev.init_from_e(0.25, e3, 1)
    ev.run(0.25, 0.005, steps)
    ev.sync()
    tau = 0.25 + 0.005 * steps
    obs = OBS.observables(lambda f: ev.get_field(f, with_ghosts=False), tau, g.dx, g.dy, g.dz, g.physics)
    fields = {f: ev.get_field(f, with_ghosts=False) for f in (V.E, V.PL, V.UX, V.UY)}
    ev.close()
    return obs, fields


@pytest.mark.parametrize("flux", [0, 1], ids=["reference_faces", "shared_faces"])
def test_fp32_form_observables_within_1e4(flux):
    o64, f64 = run(0, flux, 100)
    o32, f32 = run(1, flux, 100)
    for k in o64:
        rel = abs(o32[k] - o64[k]) / abs(o64[k])
        assert rel < 1e-4, (k, o64[k], o32[k], rel)
    # fields stay close too (FP32 storage: ~1e-6 of the field scale)
    for fid in f64:
        assert np.max(np.abs(f32[fid] - f64[fid])) / np.max(np.abs(f64[fid])) < 1e-3, fid
