"""The CPU oracle (oracle/vah_oracle.c) pinned against the reference itself:
bit-for-bit against the committed golden fixtures (generated by running the
reference's own CPU sources, tests/golden/make_golden.py), live against
oracle/_ref when it is built, and against the conformal Bjorken ODE of
python/conformal_bjorken_test.py:46-68."""
import glob
import os

import numpy as np
import pytest

import vahlib as V

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def golden_grid(z):
    phys, eos, nx, ny, nz, dx, dz, dt, t0, steps = z["meta"]
    table = z["table"] if "table" in z.files else None
    g = V.Grid(int(nx), int(ny), int(nz), dx, dx, dz, 0.2, physics=int(phys), eos=int(eos),
               zeta=1 if int(eos) == 1 else 0, table=table)
    return g, dt, t0, int(steps)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_reproduces_reference_fixture_bitwise(path):
    z = np.load(path)
    g, dt, t0, steps = golden_grid(z)
    o = V.Oracle(g)
    # setConservedVariables, DynamicalVariables.cpp:197-287
    V.load_state(o, {int(k[5:]): z[k] for k in z.files if k.startswith("prim_")})
    o.set_conserved(t0, 0)
    for fid in V.state_ids(g.physics):
        np.testing.assert_array_equal(o.field(fid), z[f"cons_{fid}"], err_msg=f"set_conserved field {fid}")
    o.set_ghost_cells()
    for fid in V.state_ids(g.physics):
        np.testing.assert_array_equal(o.field(fid), z[f"init_{fid}"], err_msg=f"ghosts field {fid}")
    for n in range(steps):
        o.step(t0 + n * dt, dt)
    for fid in V.state_ids(g.physics):
        np.testing.assert_array_equal(o.field(fid), z[f"final_{fid}"], err_msg=f"step field {fid}")


LIVE = [("ideal", "conformal", (8, 7, 6), 0.0), ("pimunu", "conformal", (11, 9, 1), 0.1),
        ("pimunu", "table", (7, 6, 5), 0.1), ("pimunu_pi", "table", (9, 8, 1), 0.1)]


@pytest.mark.parametrize("physics,eos,shape,pi_amp", LIVE)
def test_oracle_matches_reference_build_live(physics, eos, shape, pi_amp):
    g = V.Grid(*shape, 0.2, 0.2, 0.2, 0.2, physics=physics, eos=eos,
               zeta="crossover" if eos == "table" else "reference",
               table=V.eos_table() if eos == "table" else None)
    if not V.ref_available(g.physics, g.eos):
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    r, o = V.Reference(g), V.Oracle(g)
    f = V.smooth_initial_state(g, 0.5, pi_amp=pi_amp, seed=7)
    V.load_state(r, f)
    V.load_state(o, f)
    r.set_conserved(0.5)
    o.set_conserved(0.5, 0)
    r.set_ghost_cells()
    o.set_ghost_cells()
    for n in range(4):
        r.step(0.5 + 0.02 * n, 0.02)
        o.step(0.5 + 0.02 * n, 0.02)
        for fid in V.state_ids(g.physics):
            np.testing.assert_array_equal(o.field(fid), r.field(fid), err_msg=f"step {n} field {fid}")


def bjorken_ode(e0, pl0, t0, t1, etabar):
    """python/conformal_bjorken_test.py:46-68 (equationsAH): de/dt = -(e+P_L)/t,
    dP_L/dt = -(P_L - e/3)/tau_pi - (3 P_L - Rtilde(P_L/e) e)/t, tau_pi = 5 etabar/T,
    T = (e/13.8997)^(1/4)."""
    from scipy.integrate import solve_ivp
    num = [-6.674731906076046e-6, 0.004617789933500251, 0.7207562721999754, 9.097427250602184,
           -4.475814747302824, -36.37501529319408, 46.868405146729316, -15.833867583743228]
    den = [0.06856675185266, 2.9181587012768597, 11.951184087839218, -29.708257843442173,
           -2.618233802059826, 34.646239784689065, -19.62596366454439, 2.374808442453899]

    def rtilde(a):
        return np.polyval(num[::-1], a) / np.polyval(den[::-1], a)

    def rhs(t, y):
        e, pl = y
        T = (e / 13.8997) ** 0.25
        return [-(e + pl) / t, -(pl - e / 3) * T / (5 * etabar) - (3 * pl - rtilde(pl / e) * e) / t]

    sol = solve_ivp(rhs, (t0, t1), [e0, pl0], method="LSODA", rtol=1e-12, atol=1e-12)
    return sol.y[0, -1], sol.y[1, -1]


def run_bjorken(dt, t0=0.5, t1=10.0):
    g = V.Grid(1, 1, 1, 0.1, 0.1, 0.1, 0.2, physics="pimunu")
    o = V.Oracle(g)
    e0 = 13.8997 * (0.6 / 0.197326938) ** 4 + 1e-3
    n = g.ncell
    V.load_state(o, {V.E: np.full(n, e0), V.PP: np.full(n, e0 / 3), V.UT: np.ones(n)})
    o.set_conserved(t0, 0)  # P_L = 0.0154483 e, DynamicalVariables.cpp:246-248
    o.set_ghost_cells()
    steps = int(round((t1 - t0) / dt))
    o.run(t0, dt, steps)
    s = 2 + 5 * (2 + 5 * 2)
    return e0, o.field(V.E)[s], o.field(V.PL)[s]


def test_oracle_reproduces_conformal_bjorken_known_answer():
    e0, e1, pl1 = run_bjorken(0.02)
    e_ode, pl_ode = bjorken_ode(e0, 0.0154483 * e0, 0.5, 10.0, 0.2)
    # RK2 at dt = 0.02: 8.7e-5 relative (dt^2-limited)
    assert abs(e1 / e_ode - 1) < 2e-4
    assert abs(pl1 / pl_ode - 1) < 2e-4
    # second-order convergence in dt
    _, e2, pl2 = run_bjorken(0.01)
    assert abs(e2 / e_ode - 1) < 0.35 * abs(e1 / e_ode - 1)
    assert abs(pl2 / pl_ode - 1) < 0.35 * abs(pl1 / pl_ode - 1)


def test_limiter_matches_minmod_definition():
    L = V.oracle_lib()
    rng = np.random.default_rng(3)
    for _ in range(200):
        a, b, c = rng.standard_normal(3)
        l, cc, r = 1.1 * (b - a), (c - a) / 2, 1.1 * (c - b)

        def mm(x, y):
            sx = -1.0 if x < 0 else 1.0
            sy = -1.0 if y < 0 else 1.0
            return (sx + sy) * min(abs(x), abs(y)) / 2

        assert L.vo_approx_derivative(a, b, c) == mm(l, mm(cc, r))
    assert L.vo_approx_derivative(1.0, 1.0, 1.0) == 0.0


@pytest.mark.parametrize("physics,eos,shape", [("pimunu", "conformal", (9, 8, 5)), ("pimunu_pi", "table", (9, 8, 5)),
                                               ("pimunu", "table", (11, 9, 1))])
def test_validity_diagnostics_match_the_reference_bit_for_bit(physics, eos, shape):
    """The oracle's restatement of the validity diagnostics and regulator maps
    against the reference's own VALIDITY_DOMAIN arrays after three steps."""
    if not V.ref_available(V.PHYSICS[physics], {"conformal": 0, "table": 1}[eos]):
        pytest.skip("reference build not present")
    tab = V.eos_table() if eos == "table" else None
    g = V.Grid(*shape, 0.2, 0.2, 0.2, 0.2, physics=physics, eos=eos,
               zeta="crossover" if eos == "table" else "reference", table=tab)
    o, r = V.Oracle(g), V.Reference(g)
    o.set_validity(1)
    f = V.smooth_initial_state(g, 0.5, pi_amp=0.3)
    V.load_state(o, f)
    V.load_state(r, f)
    o.set_conserved(0.5, 0)
    r.set_conserved(0.5)
    o.set_ghost_cells()
    r.set_ghost_cells()
    for n in range(3):
        o.step(0.5 + 0.02 * n, 0.02)
        r.step(0.5 + 0.02 * n, 0.02)
    nonzero = 0
    for vid in range(V.NUM_VALIDITY):
        a, b = g.interior(o.validity(vid)), g.interior(r.validity(vid))
        np.testing.assert_array_equal(a, b, err_msg=f"validity field {vid}")
        nonzero += bool(np.any(b != 0))
    assert nonzero >= (27 if physics == "pimunu_pi" else 24)


def test_oracle_workload_inputs_equal_the_library_generators_bit_for_bit():
    """The oracle's copy of the workloads' inputs (the benchmark's reference
    arm builds its event from it, loading no product code) equals the
    library's host generators exactly: EoS table, MC-Glauber profile and
    longitudinal profile."""
    tab_o, tab_p = V.oracle_eos_table(), V.eos_table()
    assert np.array_equal(tab_o, tab_p)
    for b, seed in ((7.0, 1), (11.5, 12345)):
        eo, no = V.oracle_mc_glauber(121, 117, 0.1, 0.1, b, seed, e_peak=1234.5, e_floor=1e-3)
        ep, np_ = V.product.mc_glauber(121, 117, 0.1, 0.1, b, seed, e_peak=1234.5, e_floor=1e-3)
        assert no == np_ and np.array_equal(eo, ep)
    assert np.array_equal(V.oracle_longitudinal(81, 0.1), V.product.longitudinal(81, 0.1))
    T = 0.6 / 0.197326938
    assert V.table_energy_density(tab_o, T) == V.product.table_energy_density(tab_p, T)
