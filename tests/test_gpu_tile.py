"""The FP32 form on the TMA-tiled stage kernel (vah_tile.cuh), through the C
ABI. The kernel runs the arithmetic of vah_tile_cell.cuh (state, flux and
sources in FP32; Newton inversions and closure fits in FP64; each face once
with the left cell's guess). Its references:
  * the host build of the same arithmetic (tests/hostcheck/vah_tilecheck.cpp):
    equal to FP32 rounding (the device contracts products into FMAs);
  * the FP64 shared-face form on the same state (the same scheme in FP64):
    equal to FP32 rounding -- an indexing, halo, shuffle or tile-boundary
    error would show as O(1);
  * a run of steps within 1e-4 of the FP64 shared-face form.
Grids are not multiples of the tiles (8x8x4 in 3+1D, 16x16 in 2+1D), so
partial tiles sit on every upper edge."""
import numpy as np
import pytest

import vahlib as V

pytestmark = pytest.mark.gpu
STATE = [V.E, V.PP, V.UT, V.UX, V.UY, V.UN, V.PL]


def rel(a, b, floor=1e-12):
    d = np.max(np.abs(a - b))
    return 0.0 if d == 0 else float(d / max(np.max(np.abs(b)), floor))


def start(g, f, t0):
    """The same initial state in an FP32 tile event, an FP64 shared-face event
    and the host build of the FP32 form (state from the oracle's set-up)."""
    o = V.Oracle(g)
    V.load_state(o, f)
    o.set_conserved(t0, 1)
    o.set_ghost_cells()
    state = {fid: o.field(fid).copy() for fid in V.state_ids(g.physics)}
    evs = []
    for prec, flux in ((1, 0), (0, 1)):
        ev = V.Event(g, t0=t0, precision=prec, flux=flux)
        for fid, arr in state.items():
            ev.set_field(fid, arr, with_ghosts=True)
        evs.append(ev)
    host = V.TileCheck(g)
    host.load(state)
    return evs[0], evs[1], host


CASES = [("pimunu_pi", "table", (21, 19, 11)), ("pimunu", "conformal", (21, 19, 11)),
         ("ideal", "table", (13, 9, 6)), ("pimunu_pi", "table", (37, 35, 1)), ("pimunu", "conformal", (17, 33, 1))]


@pytest.mark.parametrize("physics,eos,shape", CASES, ids=[f"{p}-{e}-{'x'.join(map(str, s))}" for p, e, s in CASES])
def test_tile_fp32_step_matches_its_host_build_and_the_fp64_shared_form(physics, eos, shape):
    tab = V.eos_table() if eos == "table" else None
    g = V.Grid(*shape, 0.2, 0.2, 0.2, 0.16, physics=physics, eos=eos,
               zeta="crossover" if eos == "table" else "reference", table=tab)
    f = V.smooth_initial_state(g, 0.5, amp=60.0, floor=0.5, flow=0.3, pi_amp=0.3)
    ev32, ev64, host = start(g, f, 0.5)
    worst_h, worst_64 = {}, {}
    for n in range(2):
        ev32.step(0.5 + 0.01 * n, 0.01)
        ev64.step(0.5 + 0.01 * n, 0.01)
        host.step(0.5 + 0.01 * n, 0.01)
        ev32.sync()
        ev64.sync()
        scale_e = np.max(np.abs(g.interior(ev64.get_field(V.E))))
        # velocity scale: u^eta is a small difference in 2+1D (set by the seeded shear noise)
        scale_u = max(np.max(np.abs(g.interior(ev64.get_field(V.UX)))), np.max(np.abs(g.interior(ev64.get_field(V.UY)))))
        for fid in STATE + list(range(V.NQ[g.physics])):
            a = g.interior(ev32.get_field(fid))
            h = g.interior(host.field(fid).astype(np.float64))
            b = g.interior(ev64.get_field(fid))
            floor = scale_u if V.UT <= fid <= V.UN else 1e-6 * scale_e
            worst_h[fid] = max(worst_h.get(fid, 0.0), rel(a, h, floor))
            worst_64[fid] = max(worst_64.get(fid, 0.0), rel(a, b, floor))
    print(physics, eos, shape, "vs host build", {k: f"{v:.1e}" for k, v in worst_h.items()})
    print(physics, eos, shape, "vs FP64 shared", {k: f"{v:.1e}" for k, v in worst_64.items()})
    for fid in worst_h:
        tol = 1e-4 if 5 <= fid < 16 else 2e-5
        assert worst_h[fid] < tol, ("host", fid, worst_h[fid])
        assert worst_64[fid] < tol, ("fp64", fid, worst_64[fid])
    s32 = ev32.stats()
    assert s32.nan_cells == 0 and s32.steps == 2
    ev32.close()
    ev64.close()


def test_tile_fp32_face_ghosts_copy_the_boundary_cells():
    """After a step every face ghost layer holds its boundary cell's values
    (zero-gradient ghosts, DynamicalVariables.cpp:349-489), in the padded device
    layout read back through vah_event_get_field."""
    tab = V.eos_table()
    g = V.Grid(21, 19, 11, 0.2, 0.2, 0.2, 0.16, physics="pimunu_pi", eos="table", zeta="crossover", table=tab)
    f = V.smooth_initial_state(g, 0.5, pi_amp=0.3)
    ev, ev64, _ = start(g, f, 0.5)
    ev64.close()
    ev.step(0.5, 0.01)
    ev.sync()
    for fid in (V.E, V.UX, V.PL, V.PIXY):
        a = ev.get_field(fid).reshape(g.shape)
        c = a[2:-2, 2:-2, 2:-2]
        np.testing.assert_array_equal(a[2:-2, 2:-2, 0], c[:, :, 0])
        np.testing.assert_array_equal(a[2:-2, 2:-2, 1], c[:, :, 0])
        np.testing.assert_array_equal(a[2:-2, 2:-2, -1], c[:, :, -1])
        np.testing.assert_array_equal(a[2:-2, 0, 2:-2], c[:, 0, :])
        np.testing.assert_array_equal(a[2:-2, -2, 2:-2], c[:, -1, :])
        np.testing.assert_array_equal(a[0, 2:-2, 2:-2], c[0])
        np.testing.assert_array_equal(a[-1, 2:-2, 2:-2], c[-1])
    ev.close()


def test_tile_fp32_mc_glauber_run_tracks_fp64_shared_faces():
    """40 steps of a 3+1D MC-Glauber event (47x45x21, shear + bulk, table EoS):
    e, P_L and u^mu within 1e-4 of the FP64 shared-face form."""
    tab = V.eos_table()
    nx, ny, nz = 47, 45, 21
    g = V.Grid(nx, ny, nz, 0.2, 0.2, 0.1, 0.16, physics="pimunu_pi", eos="table", zeta="crossover", table=tab)
    e_peak = V.product.table_energy_density(tab, 0.6 / 0.197326938)
    exy, _ = V.product.mc_glauber(nx, ny, 0.2, 0.2, 6.0, seed=4, e_peak=e_peak)
    e3 = (V.product.longitudinal(nz, g.dz)[:, None] * exy[None, :]).ravel()
    evs = []
    for prec, flux in ((1, 0), (0, 1)):
        ev = V.Event(g, t0=0.25, precision=prec, flux=flux)
        ev.init_from_e(0.25, e3, 1)
        ev.run(0.25, 0.005, 40)
        ev.sync()
        evs.append(ev)
    errs = {fid: rel(g.interior(evs[0].get_field(fid)), g.interior(evs[1].get_field(fid)))
            for fid in (V.E, V.PL, V.UT, V.UX, V.UY, V.UN)}
    print("FP32 tile vs FP64 shared, 40 steps:", {k: f"{v:.1e}" for k, v in errs.items()})
    assert max(errs.values()) < 1e-4, errs
    for ev in evs:
        ev.close()


@pytest.mark.parametrize("shape,dx,dz", [((105, 97, 45), 0.1, 0.1), ((401, 389, 1), 0.1, 0.1)], ids=["3+1D", "2+1D"])
def test_tile_fp32_many_tiles_per_block_match_the_host_build(shape, dx, dz):
    """An event with several tiles per block of the persistent grid (3+1D:
    2184 tiles of 8x8x4; 2+1D: 650 tiles of 16x16, on 296 blocks), so that
    each block's next tile is loaded while it finishes the current one: the
    benchmark's resolution and initialisation (MC-Glauber, P_L = 0.0154483 e,
    u = 0), 4 steps against the host build of the same arithmetic -- e, P_L and
    u^mu within 2e-5, the same cell-inversion fallbacks (none), and face
    fallbacks within a few: in the wide dilute floor of the 2+1D grid a face
    state can sit on the edge of the fallback test, where the device's fused
    multiply-adds move the reconstruction's last bit (measured: host 11, GPU 0
    of 2.4 million face inversions)."""
    tab = V.eos_table()
    nx, ny, nz = shape
    g = V.Grid(nx, ny, nz, dx, dx, dz, 0.16, physics="pimunu_pi", eos="table", zeta="crossover", table=tab)
    e_peak = V.product.table_energy_density(tab, 0.6 / 0.197326938)
    exy, _ = V.product.mc_glauber(nx, ny, dx, dx, 7.0, seed=1, e_peak=e_peak, e_floor=0.0)
    f = V.product.longitudinal(nz, dz) if nz > 1 else np.ones(1)
    e3 = (f[:, None] * exy[None, :]).ravel() + 1e-3
    t0, dt = 0.25, 0.005
    ev = V.Event(g, t0=t0, precision=1, flux=0)
    ev.init_from_e(t0, e3, 0)  # the reference's initialisation
    host = V.TileCheck(g)
    host.load({fid: ev.get_field(fid) for fid in V.state_ids(g.physics)})
    t = t0
    for n in range(4):
        ev.step(t, dt)
        host.step(t, dt)
        t += dt
    ev.sync()
    scale_u = max(np.max(np.abs(g.interior(host.field(V.UX)))), np.max(np.abs(g.interior(host.field(V.UY)))))
    errs = {}
    for fid in (V.E, V.PL, V.UT, V.UX, V.UY, V.UN):
        floor = scale_u if V.UT <= fid <= V.UN else 1e-12
        errs[fid] = rel(g.interior(ev.get_field(fid)), g.interior(host.field(fid).astype(np.float64)), floor)
    s = ev.stats()
    print(shape, "vs host build, 4 steps:", {k: f"{v:.1e}" for k, v in errs.items()}, "GPU fallbacks",
          s.face_fallbacks, s.cell_fallbacks, "host", host.counters())
    assert max(errs.values()) < 2e-5, errs
    hc = host.counters()
    assert [s.cell_fallbacks, s.nan_cells] == hc[1:]
    assert abs(s.face_fallbacks - hc[0]) <= 32, (s.face_fallbacks, hc[0])
    ev.close()
