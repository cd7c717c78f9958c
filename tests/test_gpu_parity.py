"""GPU parity: the library's CUDA step (through the C ABI) against the CPU
oracle and the reference fixtures. Tolerances are normwise relative L-inf,
max|gpu - cpu| / max|cpu| per field, on e, P_L and u^mu (the quantities the
drop-in must reproduce to 1e-9 after 200 steps); pi components use a floor of
their natural scale because several are analytically ~0."""
import glob
import os

import numpy as np
import pytest

import vahlib as V

pytestmark = pytest.mark.gpu
GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
KEY_FIELDS = [V.E, V.PL, V.UT, V.UX, V.UY, V.UN]


def rel_err(a, b, floor=0.0):
    d = np.max(np.abs(a - b))
    if d == 0:
        return 0.0
    return float(d / max(np.max(np.abs(a)), floor))


def upload(ev, g, fields):
    for fid, arr in fields.items():
        if fid < 16 and fid >= V.NQ[g.physics] and not (fid == V.PI and g.physics == 2):
            continue
        ev.set_field(fid, arr, with_ghosts=True)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_gpu_matches_reference_fixture(path):
    z = np.load(path)
    phys, eos, nx, ny, nz, dx, dz, dt, t0, steps = z["meta"]
    table = z["table"] if "table" in z.files else None
    g = V.Grid(int(nx), int(ny), int(nz), dx, dx, dz, 0.2, physics=int(phys), eos=int(eos),
               zeta=1 if int(eos) == 1 else 0, table=table)
    ev = V.Event(g, t0=t0)
    # setConservedVariables on the device from the reference's primitives
    upload(ev, g, {int(k[5:]): z[k] for k in z.files if k.startswith("prim_")})
    ev.set_conserved(t0, 0)
    for fid in V.state_ids(g.physics):
        assert rel_err(g.interior(z[f"cons_{fid}"]), g.interior(ev.get_field(fid))) < 1e-14, fid
    # ghost fill on the device: exact copies, edges included
    upload(ev, g, {fid: z[f"cons_{fid}"] for fid in V.state_ids(g.physics)})
    ev.set_ghost_cells()
    for fid in V.state_ids(g.physics):
        assert rel_err(z[f"init_{fid}"], ev.get_field(fid)) < 1e-14, fid
    # steps
    upload(ev, g, {fid: z[f"init_{fid}"] for fid in V.state_ids(g.physics)})
    ev.run(t0, dt, int(steps))
    ev.sync()
    for fid in KEY_FIELDS:
        assert rel_err(g.interior(z[f"final_{fid}"]), g.interior(ev.get_field(fid)), 1e-12) < 1e-11, fid
    ev.close()


def conformal_workload(nx=61, ny=61):
    """The 2+1D conformal case: optical Glauber Au+Au b = 7 fm, peak T0 = 0.6 GeV,
    P_L = P_T = p, u = (1,0,0,0), pi = 0, eta/s = 0.2, dx = 0.2, dt = 0.02, tau0 = 0.5."""
    g = V.Grid(nx, ny, 1, 0.2, 0.2, 0.2, 0.2, physics="pimunu", eos="conformal")
    e_peak = 13.8997 * (0.6 / 0.197326938) ** 4
    e2 = V.product.optical_glauber(nx, ny, 0.2, 0.2, b=7.0, e_peak=e_peak)
    return g, e2


def start_both(g, e_int, t0, pl_mode=1, flux=0):
    o = V.Oracle(g)
    full = np.zeros(g.shape)
    full[2:-2, 2:-2, 2:-2] = e_int.reshape(g.nz, g.ny, g.nx)
    p = full / 3 if g.eos == 0 else np.vectorize(lambda x: V.eos_point_oracle(g, x)[0])(full)
    V.load_state(o, {V.E: full.ravel(), V.PP: p.ravel(), V.UT: np.ones(g.ncell), V.PL: p.ravel()})
    o.set_conserved(t0, pl_mode)
    o.set_ghost_cells()
    ev = V.Event(g, t0=t0, flux=flux)
    ev.init_from_e(t0, e_int, pl_mode)
    return o, ev


# reference face semantics: split face/cell launches (0) and the fused stage (2)
FLUX = pytest.mark.parametrize("flux", [0, 2], ids=["split", "fused"])


@FLUX
def test_gpu_conformal_2d_200_steps_within_1e9(flux):
    g, e2 = conformal_workload()
    o, ev = start_both(g, e2, 0.5, flux=flux)
    for fid in V.state_ids(g.physics):
        assert rel_err(g.interior(o.field(fid)), g.interior(ev.get_field(fid)), 1e-12) < 1e-13, fid
    dt = 0.02
    o.run(0.5, dt, 200)
    ev.run(0.5, dt, 200)
    ev.sync()
    errs = {fid: rel_err(g.interior(o.field(fid)), g.interior(ev.get_field(fid)), 1e-12) for fid in KEY_FIELDS}
    assert max(errs.values()) < 1e-9, errs
    s = ev.stats()
    assert s.nan_cells == 0 and s.steps == 200
    ev.close()


@FLUX
def test_gpu_table_3d_bulk_within_1e9(flux):
    """3+1D MC-Glauber slab with the tabulated EoS, shear + bulk, eta/s = 0.16."""
    tab = V.eos_table()
    nx, ny, nz = 25, 23, 9
    g = V.Grid(nx, ny, nz, 0.1 * 121 / nx, 0.1 * 121 / ny, 0.1, 0.16, physics="pimunu_pi", eos="table",
               zeta="crossover", table=tab)
    e_peak = V.product.table_energy_density(tab, 0.6 / 0.197326938)
    exy, _ = V.product.mc_glauber(nx, ny, g.dx, g.dy, 7.0, seed=5, e_peak=e_peak)
    f = V.product.longitudinal(nz, g.dz)
    e3 = (f[:, None] * exy[None, :]).ravel()
    o, ev = start_both(g, e3, 0.25, flux=flux)
    dt = 0.005
    o.run(0.25, dt, 40)
    ev.run(0.25, dt, 40)
    ev.sync()
    errs = {fid: rel_err(g.interior(o.field(fid)), g.interior(ev.get_field(fid)), 1e-12) for fid in KEY_FIELDS}
    assert max(errs.values()) < 1e-9, errs
    ev.close()


def test_gpu_shared_faces_match_oracle_where_inversions_converge():
    """VAH_FLUX_SHARED evaluates each face once; on a state without inversion
    fallbacks it equals the reference to the Newton tolerance squared."""
    tab = V.eos_table()
    g = V.Grid(24, 20, 10, 0.2, 0.2, 0.2, 0.16, physics="pimunu_pi", eos="table", zeta="crossover", table=tab)
    f = V.smooth_initial_state(g, 0.5, amp=200.0, floor=1.0, flow=0.3)
    o = V.Oracle(g)
    V.load_state(o, f)
    o.set_conserved(0.5, 1)
    o.set_ghost_cells()
    ev = V.Event(g, t0=0.5, flux=1)
    upload(ev, g, {fid: o.field(fid).copy() for fid in V.state_ids(g.physics)})
    for n in range(30):
        o.step(0.5 + 0.01 * n, 0.01)
        assert o.stats()[0] == 0
    ev.run(0.5, 0.01, 30)
    ev.sync()
    assert ev.stats().face_fallbacks == 0
    for fid in KEY_FIELDS:
        assert rel_err(g.interior(o.field(fid)), g.interior(ev.get_field(fid)), 1e-12) < 1e-10, fid
    ev.close()


def test_gpu_ideal_3d_matches_oracle():
    g = V.Grid(12, 10, 8, 0.2, 0.2, 0.2, 0.2, physics="ideal", eos="conformal")
    f = V.smooth_initial_state(g, 0.5, flow=0.4)
    o = V.Oracle(g)
    V.load_state(o, f)
    o.set_conserved(0.5, 1)
    o.set_ghost_cells()
    ev = V.Event(g, t0=0.5)
    upload(ev, g, {fid: o.field(fid).copy() for fid in V.state_ids(g.physics)})
    o.run(0.5, 0.02, 20)
    ev.run(0.5, 0.02, 20)
    ev.sync()
    for fid in KEY_FIELDS:
        assert rel_err(g.interior(o.field(fid)), g.interior(ev.get_field(fid)), 1e-12) < 1e-11, fid
    ev.close()


@pytest.mark.parametrize("flux", [0, 2], ids=["split", "fused"])
def test_gpu_tall_lattice_beyond_the_grid_y_limit(flux):
    """1 x 512 x 512 cells: 262,144 rows of (j, k), more row blocks than a
    grid's y dimension holds (65,535 blocks of 4 rows); the launches continue
    along z. Two steps against the oracle."""
    g = V.Grid(1, 512, 512, 0.2, 0.2, 0.2, 0.2, physics="ideal", eos="conformal")
    f = V.smooth_initial_state(g, 0.5, flow=0.4)
    o = V.Oracle(g)
    V.load_state(o, f)
    o.set_conserved(0.5, 1)
    o.set_ghost_cells()
    ev = V.Event(g, t0=0.5, flux=flux)
    upload(ev, g, {fid: o.field(fid).copy() for fid in V.state_ids(g.physics)})
    o.run(0.5, 0.02, 2)
    ev.run(0.5, 0.02, 2)
    ev.sync()
    for fid in KEY_FIELDS:
        assert rel_err(g.interior(o.field(fid)), g.interior(ev.get_field(fid)), 1e-12) < 1e-11, fid
    ev.close()


def test_gpu_host_buffer_step_matches_device_step():
    g, e2 = conformal_workload(21, 19)
    ev = V.Event(g, t0=0.5)
    ev.init_from_e(0.5, e2, 1)
    ev.run(0.5, 0.02, 3)
    ids = [fid for fid in range(V.NUM_FIELDS) if fid < 15 or fid >= 16]
    state0 = {fid: ev.get_field(fid) for fid in ids}
    state = {fid: a.copy() for fid, a in state0.items()}
    ptrs = [state[fid].ctypes.data if fid in state else 0 for fid in range(V.NUM_FIELDS)]
    ev.step_host(0.56, 0.02, ptrs)  # host arrays in, one step, host arrays out
    dev = V.Event(g, t0=0.5)
    upload(dev, g, state0)
    dev.step(0.56, 0.02)            # the same step on a device-resident copy
    for fid in KEY_FIELDS:
        np.testing.assert_array_equal(state[fid], dev.get_field(fid))
    dev.close()
    ev.close()


@pytest.mark.parametrize("nz", [9, 22, 23])
@pytest.mark.parametrize("flux", [0, 1], ids=["reference_faces", "shared_faces"])
def test_gpu_host_buffer_step_overlapped_slabs_match_device_step(nz, flux):
    """3+1D host-buffer steps take the overlapped path (copies and stages of
    eta slabs on three streams; nz = 9: slabs of 3, 2, 2, 2 planes, nz = 22:
    4, 3 x 6, nz = 23: 4, 4, 3 x 5). Two steps in a row equal set_field + step
    + get_field bit for bit on every field, ghosts included."""
    tab = V.eos_table()
    nx, ny = 25, 23
    g = V.Grid(nx, ny, nz, 0.1 * 121 / nx, 0.1 * 121 / ny, 0.1, 0.16, physics="pimunu_pi", eos="table",
               zeta="crossover", table=tab)
    e_peak = V.product.table_energy_density(tab, 0.6 / 0.197326938)
    exy, _ = V.product.mc_glauber(nx, ny, g.dx, g.dy, 7.0, seed=5, e_peak=e_peak)
    e3 = (V.product.longitudinal(nz, g.dz)[:, None] * exy[None, :]).ravel()
    ev = V.Event(g, t0=0.25, flux=flux)
    ev.init_from_e(0.25, e3, 1)
    ev.run(0.25, 0.005, 4)
    ids = list(range(V.NUM_FIELDS))
    state0 = {fid: ev.get_field(fid) for fid in ids}
    state = {fid: a.copy() for fid, a in state0.items()}
    ptrs = [state[fid].ctypes.data for fid in range(V.NUM_FIELDS)]
    ev.step_host(0.27, 0.005, ptrs)
    ev.step_host(0.275, 0.005, ptrs)
    dev = V.Event(g, t0=0.25, flux=flux)
    upload(dev, g, state0)
    dev.step(0.27, 0.005)
    dev.step(0.275, 0.005)
    for fid in ids:
        np.testing.assert_array_equal(state[fid], dev.get_field(fid), err_msg=f"field {fid}")
    dev.close()
    ev.close()


def test_gpu_host_buffer_step_fp32_storage_matches_device_step():
    """FP32 storage: the host-buffer step narrows and widens on the device;
    the result equals set_field + step + get_field bit for bit."""
    g, e2 = conformal_workload(21, 19)
    ev = V.Event(g, t0=0.5, precision=1)
    ev.init_from_e(0.5, e2, 1)
    ev.run(0.5, 0.02, 3)
    ids = [fid for fid in range(V.NUM_FIELDS) if fid < 15 or fid >= 16]
    state0 = {fid: ev.get_field(fid) for fid in ids}
    state = {fid: a.copy() for fid, a in state0.items()}
    ptrs = [state[fid].ctypes.data if fid in state else 0 for fid in range(V.NUM_FIELDS)]
    ev.step_host(0.56, 0.02, ptrs)
    ev.step_host(0.58, 0.02, ptrs)
    dev = V.Event(g, t0=0.5, precision=1)
    upload(dev, g, state0)
    dev.step(0.56, 0.02)
    dev.step(0.58, 0.02)
    for fid in ids:
        np.testing.assert_array_equal(state[fid], dev.get_field(fid), err_msg=f"field {fid}")
    dev.close()
    ev.close()


@pytest.mark.parametrize("nz", [5, 9, 23, 41])
def test_gpu_host_buffer_step_fp32_overlapped_slabs_match_device_step(nz):
    """FP32 form, 3+1D: host-buffer steps take the overlapped path, in slabs
    of whole 4-plane tile layers (nz = 9: 4, 4, 1 planes; nz = 23: 4 x 5, 3;
    nz = 41: 12, 8, 8, 8, 5), each slab's stage one tile launch over its run
    of the work-list, its planes narrowed after their copy-in and widened
    before their copy-out; nz = 5 (two tile layers, fewer than three slabs)
    takes the plain path. Two steps in a row equal set_field + step +
    get_field bit for bit on every field, ghosts included."""
    tab = V.eos_table()
    nx, ny = 25, 23
    g = V.Grid(nx, ny, nz, 0.1 * 121 / nx, 0.1 * 121 / ny, 0.1, 0.16, physics="pimunu_pi", eos="table",
               zeta="crossover", table=tab)
    e_peak = V.product.table_energy_density(tab, 0.6 / 0.197326938)
    exy, _ = V.product.mc_glauber(nx, ny, g.dx, g.dy, 7.0, seed=5, e_peak=e_peak)
    e3 = (V.product.longitudinal(nz, g.dz)[:, None] * exy[None, :]).ravel()
    ev = V.Event(g, t0=0.25, precision=1)
    ev.init_from_e(0.25, e3, 1)
    ev.run(0.25, 0.005, 4)
    ids = list(range(V.NUM_FIELDS))
    state0 = {fid: ev.get_field(fid) for fid in ids}
    state = {fid: a.copy() for fid, a in state0.items()}
    ptrs = [state[fid].ctypes.data for fid in range(V.NUM_FIELDS)]
    ev.step_host(0.27, 0.005, ptrs)
    ev.step_host(0.275, 0.005, ptrs)
    dev = V.Event(g, t0=0.25, precision=1)
    upload(dev, g, state0)
    dev.step(0.27, 0.005)
    dev.step(0.275, 0.005)
    for fid in ids:
        np.testing.assert_array_equal(state[fid], dev.get_field(fid), err_msg=f"field {fid}")
    dev.close()
    ev.close()


def test_gpu_nan_is_reported_not_fatal():
    g, e2 = conformal_workload(9, 9)
    ev = V.Event(g, t0=0.5)
    ev.init_from_e(0.5, e2, 1)
    ttt = ev.get_field(V.TTT)
    ttt[g.ncell // 2] = np.nan
    ev.set_field(V.TTT, ttt)
    ev.step(0.5, 0.02)
    with pytest.raises(V.product.VahError) as info:
        ev.sync()
    assert info.value.rc == -4
    assert ev.stats().nan_cells > 0
    ev.close()


def test_gpu_rejects_bad_arguments():
    L = V.library()
    lat = V.product.Lattice(0, 5, 1, 0.1, 0.1, 0.1)
    hyd = V.product.Hydro(0.5, 0.2, 0.155)
    opt = V.product.Options(1, 0, 0, 0, 0, 0, None)
    h = V.C.c_void_p()
    assert L.vah_event_create(V.C.byref(lat), V.C.byref(hyd), V.C.byref(opt), None, V.C.byref(h)) == -1
    lat = V.product.Lattice(5, 5, 1, 0.1, 0.1, 0.1)
    opt = V.product.Options(1, 1, 0, 0, 0, 0, None)  # table EoS without a table
    assert L.vah_event_create(V.C.byref(lat), V.C.byref(hyd), V.C.byref(opt), None, V.C.byref(h)) == -1
