"""2+1D lattices: no stencil reads the eta ghost layers, so the steps of the
event and batch paths leave them and fill them (the eta pass of the
reference's ghost fill, DynamicalVariables.cpp:449-489) when a caller reads
fields with ghosts: vah_event_get_field, vah_batch_get_field, the host-buffer
step. Whoever reads them sees each eta ghost plane equal to the one interior
plane, as after the reference's setGhostCells; the interior is unchanged by
the fill."""
import numpy as np
import pytest

import vahlib as V

pytestmark = pytest.mark.gpu
vah = V.product

FIELDS = (V.TTT, V.TTX, V.PL, V.PIXY, V.PI, V.E, V.PP, V.UT, V.UX, V.UY)


def check_eta_planes(g, a):
    a = a.reshape(g.shape)
    mid = a[2]
    for k in (0, 1, 3, 4):
        np.testing.assert_array_equal(a[k][2:, 2:], mid[2:, 2:])  # the reference's ranges: from the first interior row


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_event_reads_fill_the_eta_ghost_layers(precision):
    tab = V.eos_table()
    g = V.Grid(37, 29, 1, 0.2, 0.2, 0.2, 0.16, physics="pimunu_pi", eos="table", zeta="crossover", table=tab)
    e_peak = vah.table_energy_density(tab, 0.5 / vah.HBARC)
    exy, _ = vah.mc_glauber(37, 29, 0.2, 0.2, 5.0, 3, e_peak=e_peak)
    ev = V.Event(g, t0=0.4, precision=precision)
    ev.init_from_e(0.4, exy, 1)
    ev.run(0.4, 0.01, 3)
    ev.sync()
    inner = {fid: ev.get_field(fid, with_ghosts=False) for fid in FIELDS}
    for fid in FIELDS:
        full = ev.get_field(fid)
        check_eta_planes(g, full)
        np.testing.assert_array_equal(g.interior(full).ravel(), inner[fid])
    # the host-buffer step returns them filled too
    host = {fid: ev.get_field(fid) for fid in V.state_ids(g.physics)}
    ev.step_host(0.43, 0.01, [host[f].ctypes.data if f in host else 0 for f in range(V.NUM_FIELDS)])
    for fid in FIELDS:
        check_eta_planes(g, host[fid])
    ev.close()


def test_batch_reads_fill_the_eta_ghost_layers():
    tab = V.eos_table()
    e_peak = vah.table_energy_density(tab, 0.5 / vah.HBARC)
    for precision in (0, 1):
        b = vah.Batch(table=tab, precision=precision, capacity_bytes=1 << 30)
        slot = b.add_glauber(41, 33, 1, 0.2, 0.2, 0.2, 0.4, 0.01, 0.16, b=4.0, seed=9, e_peak=e_peak)
        b.step(3)
        g = V.Grid(41, 33, 1, 0.2, 0.2, 0.2, 0.16, physics="pimunu_pi", eos="table", zeta="crossover", table=tab)
        for fid in FIELDS:
            check_eta_planes(g, b.get_field(slot, fid, True))
        b.close()
