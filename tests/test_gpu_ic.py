"""Initial energy densities generated on the GPU (vah_event_init_glauber,
vah_event_init_optical_glauber, and vah_batch_add_glauber through the same
device code) against the host generators (vah_ic_mc_glauber,
vah_ic_optical_glauber, vah_ic_longitudinal) that build the workloads' events.

The device MC-Glauber sampler walks the host sampler's random streams, so the
participants are the same nucleons; positions and e differ only by the last
bits of the GPU's exp, sin and cos. The optical profile integrates the same
thickness table in the same order."""
import numpy as np
import pytest

import vahlib as V

pytestmark = pytest.mark.gpu
vah = V.product


def rel(a, b):
    d = np.max(np.abs(a - b))
    return 0.0 if d == 0 else d / np.max(np.abs(b))


def host_event(g, e3d, t0, precision=0):
    ev = V.Event(g, t0=t0, flux=1, precision=precision)
    ev.init_from_e(t0, e3d)
    return ev


@pytest.mark.parametrize("nz,dz,precision", [(1, 0.2, 0), (9, 0.3, 0), (7, 0.4, 1)], ids=["2+1D", "3+1D", "3+1D-fp32"])
@pytest.mark.parametrize("b,seed", [(0.0, 5), (6.5, 17), (11.0, 40)])
def test_device_mc_glauber_event_equals_the_host_generator(nz, dz, precision, b, seed):
    tab = V.eos_table()
    nx, ny, dx = 47, 41, 0.3
    g = V.Grid(nx, ny, nz, dx, dx, dz, 0.16, physics="pimunu_pi", eos="table", zeta="crossover", table=tab)
    e_peak = vah.table_energy_density(tab, 0.5 / vah.HBARC)
    t0 = 0.4
    exy, npart = vah.mc_glauber(nx, ny, dx, dx, b, seed, e_peak=e_peak, e_floor=0.0)
    f = vah.longitudinal(nz, dz) if nz > 1 else np.ones(1)
    host_e = (f[:, None] * exy[None, :]).ravel() + 2e-3
    assert npart > 2
    ev = V.Event(g, t0=t0, flux=1, precision=precision)
    ev.init_glauber(t0, b, seed, e_peak, e_floor=2e-3)
    ref = host_event(g, host_e, t0, precision)
    tol = 1e-13 if precision == 0 else 2e-7
    assert rel(ev.get_field(V.E, False), host_e) <= tol
    # the whole initial state (conserved variables, ghosts) follows
    for fid in (0, 3, 4, V.E, V.PP):
        assert rel(ev.get_field(fid), ref.get_field(fid)) <= tol, fid
    ev.close()
    ref.close()


def test_device_mc_glauber_without_collision_is_the_flat_floor():
    g = V.Grid(21, 19, 1, 0.3, 0.3, 0.2, 0.16, physics="pimunu_pi", eos="conformal")
    exy, npart = vah.mc_glauber(21, 19, 0.3, 0.3, 40.0, 3, e_peak=5.0, e_floor=0.01)
    assert npart == 0 and np.all(exy == 0.01)
    ev = V.Event(g, t0=0.5, flux=1)
    ev.init_glauber(0.5, 40.0, 3, 5.0, e_floor=0.01)
    assert np.all(ev.get_field(V.E, False) == 0.01)
    ev.close()


@pytest.mark.parametrize("nz,dz", [(1, 0.2), (11, 0.25)], ids=["2+1D", "3+1D"])
@pytest.mark.parametrize("b,A,x_coll", [(0.0, 197, 0.15), (7.0, 197, 0.15), (9.5, 208, 0.3)])
def test_device_optical_glauber_event_equals_the_host_generator(nz, dz, b, A, x_coll):
    nx, ny, dx = 61, 55, 0.25
    g = V.Grid(nx, ny, nz, dx, dx, dz, 0.16, physics="pimunu", eos="conformal")
    R, a = (6.38, 0.535) if A == 197 else (6.62, 0.546)
    exy = vah.optical_glauber(nx, ny, dx, dx, b=b, A=A, R=R, a=a, x_coll=x_coll, e_peak=40.0, e_floor=0.0)
    f = vah.longitudinal(nz, dz) if nz > 1 else np.ones(1)
    host_e = (f[:, None] * exy[None, :]).ravel() + 1e-3
    ev = V.Event(g, t0=0.6, flux=1)
    ev.init_optical_glauber(0.6, b, 40.0, e_floor=1e-3, A=A, R=R, a=a, x_coll=x_coll)
    assert rel(ev.get_field(V.E, False), host_e) <= 1e-12
    ev.close()


def test_device_initial_conditions_reject_bad_arguments():
    import ctypes as C
    g = V.Grid(9, 9, 5, 0.3, 0.3, 0.2, 0.16, physics="pimunu", eos="conformal")
    ev = V.Event(g, t0=0.5, flux=1)
    L = vah.library()
    gl = vah.Glauber(6.0, 4.2, 300, 6.38, 0.535, 0.5, 1, 5.0, 0.01, 1.5, 1.3)  # A beyond the sampling block
    L.vah_event_init_glauber.argtypes = [C.c_void_p, C.c_double, C.POINTER(vah.Glauber), C.c_int]
    assert L.vah_event_init_glauber(ev.ev, 0.5, C.byref(gl), 1) == -1
    gl.A, gl.sigma_eta = 197, 0.0  # no longitudinal width on a 3+1D lattice
    assert L.vah_event_init_glauber(ev.ev, 0.5, C.byref(gl), 1) == -1
    gl.sigma_eta, gl.width = 1.3, 0.0
    assert L.vah_event_init_glauber(ev.ev, 0.5, C.byref(gl), 1) == -1
    gl.width, gl.ws_a = 0.5, 0.0  # no Woods-Saxon surface thickness
    assert L.vah_event_init_glauber(ev.ev, 0.5, C.byref(gl), 1) == -1
    gl.ws_a, gl.ws_R = 0.535, float("inf")
    assert L.vah_event_init_glauber(ev.ev, 0.5, C.byref(gl), 1) == -1
    op = vah.Optical(6.0, 0.0, 197, 6.38, 0.535, 0.15, 5.0, 0.01, 1.5, 1.3)  # sigma_NN = 0
    L.vah_event_init_optical_glauber.argtypes = [C.c_void_p, C.c_double, C.POINTER(vah.Optical), C.c_int]
    assert L.vah_event_init_optical_glauber(ev.ev, 0.5, C.byref(op), 1) == -1
    assert L.vah_event_init_optical_glauber(ev.ev, 0.5, None, 1) == -1
    ev.close()
