"""The launch autotuner (vah_event_autotune, vah_batch_autotune): it picks a
configuration from the documented search space, leaves the event state as it
was, and the steps after it give bit-identical results (launch shape and
register cap change scheduling, not arithmetic)."""
import numpy as np
import pytest

import vahlib as V

pytestmark = pytest.mark.gpu
vah = V.product

FACE_MINB, CELL_MINB, SHAPES = {3, 4, 5}, {2, 3, 4}, {(32, 4), (64, 2)}
FIELDS = list(range(16)) + [16, 17, 18, 19, 20, 21]


def event_e(tab, nx, ny, nz, dx, dz, b, seed):
    exy, _ = vah.mc_glauber(nx, ny, dx, dx, b, seed, e_peak=vah.table_energy_density(tab, 0.5 / vah.HBARC),
                            e_floor=0.0)
    return (vah.longitudinal(nz, dz)[:, None] * exy[None, :]).ravel() + 1e-3


@pytest.mark.parametrize("precision,flux", [(0, 0), (0, 1)], ids=["fp64", "fp64-shared"])
def test_event_autotune_keeps_results_bit_identical(precision, flux):
    tab = V.eos_table()
    nx, ny, nz = 45, 39, 11
    e = event_e(tab, nx, ny, nz, 0.2, 0.2, 5.0, 3)
    runs = []
    for tuned in (False, True):
        ev = vah.Event(nx, ny, nz, 0.2, 0.2, 0.2, 0.16, table=tab, t0=0.4, precision=precision, flux=flux)
        ev.init_from_e(0.4, e)
        ev.run(0.4, 0.01, 3)
        ev.sync()
        if tuned:
            before = {f: ev.get_field(f) for f in FIELDS}
            choice = ev.autotune(2)
            assert len(choice) == 4
            for k, c in enumerate(choice):
                assert tuple(c["block"]) in SHAPES
                assert c["minb"] in (CELL_MINB if k == 3 else FACE_MINB)
                assert c["ms_best"] > 0 and c["ms_best"] <= c["ms_default"] + 1e-12
            for f in FIELDS:  # the state is as it was
                np.testing.assert_array_equal(ev.get_field(f), before[f])
            s = ev.stats()
        ev.run(0.43, 0.01, 4)
        ev.sync()
        runs.append({f: ev.get_field(f) for f in FIELDS})
        if tuned:
            assert ev.stats().cell_fallbacks >= s.cell_fallbacks  # counters restored, then counting on
        ev.close()
    for f in FIELDS:
        np.testing.assert_array_equal(runs[1][f], runs[0][f], err_msg=f"field {f}")


def test_event_autotune_fp32_tile_form_has_nothing_to_tune():
    """The FP32 form runs one persistent tile launch per stage: no kinds to tune."""
    tab = V.eos_table()
    ev = vah.Event(21, 19, 9, 0.2, 0.2, 0.2, 0.16, table=tab, t0=0.4, precision=vah.VAH_FP32)
    ev.init_from_e(0.4, event_e(tab, 21, 19, 9, 0.2, 0.2, 2.0, 4))
    assert ev.autotune(1) == []
    ev.close()


def test_event_autotune_fused_mode_has_nothing_to_tune():
    tab = V.eos_table()
    ev = vah.Event(21, 21, 1, 0.2, 0.2, 0.2, 0.16, table=tab, t0=0.4, flux=vah.VAH_FLUX_PER_CELL_FUSED)
    ev.init_from_e(0.4, event_e(tab, 21, 21, 1, 0.2, 0.2, 2.0, 4))
    assert ev.autotune(1) == []
    ev.close()


def test_batch_autotune_keeps_results_bit_identical():
    tab = V.eos_table()
    events = [(41, 37, 1, 4.0, 11), (29, 33, 7, 6.0, 12), (64, 20, 1, 2.0, 13)]
    out = []
    for tuned in (False, True):
        b = vah.Batch(table=tab, capacity_bytes=4 << 30)
        slots = [b.add(nx, ny, nz, 0.25, 0.25, 0.2, 0.4, 0.01, 0.16, event_e(tab, nx, ny, nz, 0.25, 0.2, bb, s))
                 for (nx, ny, nz, bb, s) in events]
        b.step(3)
        if tuned:
            choice = b.autotune(2)
            assert len(choice) == 5
            for k, c in enumerate(choice):
                assert tuple(c["block"]) == (32, 4)
                assert c["minb"] in (CELL_MINB if k >= 3 else FACE_MINB)
        b.step(4)
        b.sync()
        out.append([{f: b.get_field(s, f, False) for f in FIELDS} for s in slots])
        for s in slots:
            assert b.info(s).steps == 7
        b.close()
    for k in range(len(events)):
        for f in FIELDS:
            np.testing.assert_array_equal(out[1][k][f], out[0][k][f], err_msg=f"event {k} field {f}")
