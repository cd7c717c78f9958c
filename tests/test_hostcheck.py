"""The library's per-cell stage code (gpu-vah_b200/csrc/vah_stage.cuh,
vah_physics.cuh) compiled for the host and checked against the CPU oracle:
the device formulas differ from the reference only by rounding."""
import numpy as np
import pytest

import vahlib as V

CASES = [("ideal", "conformal", (9, 8, 1), 0.0, 5), ("pimunu", "conformal", (9, 8, 1), 0.1, 5),
         ("pimunu", "conformal", (7, 6, 5), 0.1, 3), ("pimunu", "table", (7, 6, 5), 0.1, 3),
         ("pimunu_pi", "table", (9, 8, 1), 0.1, 5), ("pimunu_pi", "table", (7, 6, 5), 0.1, 3)]


def field_scale(g, fid, arr):
    """Normwise scale of a field; pi components that are analytically ~0 get
    the energy-density scale (times t^-2 per eta index) as a floor."""
    m = np.max(np.abs(arr))
    if V.PITT <= fid <= V.PI:
        eta_idx = {V.PITN: 1, V.PIXN: 1, V.PIYN: 1, V.PINN: 2}.get(fid, 0)
        m = max(m, 1e-3 * 50.0 * 0.5 ** (-2 * eta_idx))
    return m


@pytest.mark.parametrize("split", [0, 1, 2], ids=["fused", "split_reference_faces", "split_shared_faces"])
@pytest.mark.parametrize("physics,eos,shape,pi_amp,steps", CASES)
def test_host_build_of_device_code_matches_oracle(physics, eos, shape, pi_amp, steps, split):
    table = V.eos_table() if eos == "table" else None
    g = V.Grid(*shape, 0.2, 0.2, 0.2, 0.2, physics=physics, eos=eos,
               zeta="crossover" if eos == "table" else "reference", table=table)
    o, h = V.Oracle(g), V.HostCheck(g, split=split)
    f = V.smooth_initial_state(g, 0.5, pi_amp=pi_amp)
    V.load_state(o, f)
    V.load_state(h, f)
    o.set_conserved(0.5, 1)
    h.set_conserved(0.5, 1)
    for fid in V.state_ids(g.physics):
        np.testing.assert_allclose(h.field(fid), o.field(fid), rtol=1e-14, atol=0)
    o.set_ghost_cells()
    for fid in V.state_ids(g.physics):
        h.field(fid)[:] = o.field(fid)
    for n in range(steps):
        o.step(0.5 + 0.02 * n, 0.02)
        h.step(0.5 + 0.02 * n, 0.02)
    for fid in V.state_ids(g.physics):
        a, b = g.interior(o.field(fid)), g.interior(h.field(fid))
        diff = np.max(np.abs(a - b))
        err = 0.0 if diff == 0 else diff / field_scale(g, fid, a)
        assert err < 1e-11, (fid, err)


def validity_errors(g, a_get, b_get):
    """Normwise relative differences of the 27 validity fields; the stored
    shear combinations (ids 12-15: the trace of sigma and projections that
    nearly cancel) are measured against the expansion rate's scale."""
    th = np.max(np.abs(g.interior(a_get(11))))
    errs = []
    for vid in range(V.NUM_VALIDITY):
        a, b = g.interior(a_get(vid)), g.interior(b_get(vid))
        d = np.max(np.abs(a - b))
        m = np.max(np.abs(a))
        if 12 <= vid <= 15:
            m = max(m, th)
        errs.append(0.0 if d == 0 else float(d / m))
    return errs


@pytest.mark.parametrize("split", [0, 1], ids=["fused", "split_reference_faces"])
@pytest.mark.parametrize("physics,eos,shape", [("pimunu", "conformal", (9, 8, 5)), ("pimunu_pi", "table", (9, 8, 5)),
                                               ("pimunu", "table", (11, 9, 1)), ("ideal", "conformal", (9, 8, 1))])
def test_host_build_of_validity_code_matches_oracle(physics, eos, shape, split):
    table = V.eos_table() if eos == "table" else None
    g = V.Grid(*shape, 0.2, 0.2, 0.2, 0.2, physics=physics, eos=eos,
               zeta="crossover" if eos == "table" else "reference", table=table)
    o, h = V.Oracle(g), V.HostCheck(g, split=split)
    o.set_validity(1)
    h.set_validity(1)
    f = V.smooth_initial_state(g, 0.5, pi_amp=0.3)
    V.load_state(o, f)
    V.load_state(h, f)
    o.set_conserved(0.5, 1)
    h.set_conserved(0.5, 1)
    o.set_ghost_cells()
    for fid in V.state_ids(g.physics):
        h.field(fid)[:] = o.field(fid)
    for n in range(3):
        o.step(0.5 + 0.02 * n, 0.02)
        h.step(0.5 + 0.02 * n, 0.02)
    errs = validity_errors(g, o.validity, h.validity)
    assert max(errs) < 1e-10, [(k, e) for k, e in enumerate(errs) if e >= 1e-10]


def _minmod_reference(x, y):
    """FluxLimiter.cpp:15-22: (sign x + sign y) min(|x|, |y|) / 2, sign(0) = +1."""
    sx = np.where(x < 0, -1.0, 1.0)
    sy = np.where(y < 0, -1.0, 1.0)
    return (sx + sy) * np.minimum(np.abs(x), np.abs(y)) / 2


def test_limiter_equals_the_nested_minmod():
    """The device limiter (one sign test and a three-way min) against the
    reference's minmod(1.1 (y - x), minmod((z - x)/2, 1.1 (z - y)))
    (FluxLimiter.cpp:28-33) on edge values and a million random triples,
    ties and tiny and huge scales included: equal values everywhere."""
    edge = np.array([0.0, -0.0, 1.0, -1.0, 2.0, 3.0, 1e-300, -1e-300, 5e-324, -5e-324, 1e300, -1e300])
    x, y, z = (a.ravel() for a in np.meshgrid(edge, edge, edge, indexing="ij"))
    rng = np.random.default_rng(7)
    n = 1_000_000
    r = rng.uniform(-1, 1, (3, n))
    kind = rng.integers(0, 6, n)
    r[1] = np.where(kind == 1, r[0], r[1])          # y == x
    r[2] = np.where(kind == 2, r[1], r[2])          # z == y
    r[2] = np.where(kind == 3, r[0], r[2])          # z == x
    r *= np.where(kind == 4, 1e-300, np.where(kind == 5, 1e300, 1.0))
    x, y, z = (np.ascontiguousarray(np.concatenate([a, b])) for a, b in zip((x, y, z), r))
    ref = _minmod_reference(1.1 * (y - x), _minmod_reference((z - x) * 0.5, 1.1 * (z - y)))
    out = np.empty_like(x)
    p = [a.ctypes.data_as(V.P) for a in (x, y, z, out)]
    V.hostcheck_lib().hc_approx_derivative(*p, len(x))
    assert np.array_equal(out, ref)


def test_regulator_largest_ratio_path_equals_the_nine_divisions():
    """The regulator's largest shear ratio taken as one division of the largest
    numerator (the path without validity maps) gives the same regulated state,
    bit for bit, as the nine divisions of the path that reports them: random
    cells with shear from small to far above the regulation threshold, a
    light-like pi.pi = 0 and an all-zero pi included."""
    L = V.hostcheck_lib()
    rng = np.random.default_rng(11)
    cases = []
    for k in range(20000):
        e = 10 ** rng.uniform(-3, 3)
        p = e / 3
        q = np.zeros(16)
        q[4] = p * rng.uniform(0.05, 1.5)
        scale = e * 10 ** rng.uniform(-4, 1)
        q[5:15] = scale * rng.standard_normal(10)
        q[15] = scale * 0.1 * rng.standard_normal()
        ux, uy, un = rng.normal(0, 1.0, 3) * [1, 1, 0.5]
        t = rng.uniform(0.2, 5)
        ut = np.sqrt(1 + ux * ux + uy * uy + t * t * un * un)
        cases.append((t, e, p, q, np.array([ut, ux, uy, un])))
    q0 = np.zeros(16)
    q0[4] = 1.0
    cases.append((1.0, 3.0, 1.0, q0, np.array([1.0, 0.0, 0.0, 0.0])))
    ql = np.zeros(16)
    ql[4], ql[5], ql[6], ql[7] = 1.0, 2.0, 1.0, 1.0  # pi.pi = 2^2 - 2 (1^2) - 2 (1^2) = 0 exactly
    cases.append((1.0, 3.0, 1.0, ql, np.array([1.0, 0.0, 0.0, 0.0])))
    for t, e, p, q, u in cases:
        a, b = q.copy(), q.copy()
        L.hc_regulate(t, e, p, a.ctypes.data_as(V.P), u.ctypes.data_as(V.P), 0)
        L.hc_regulate(t, e, p, b.ctypes.data_as(V.P), u.ctypes.data_as(V.P), 1)
        assert np.array_equal(a.view(np.int64), b.view(np.int64))


@pytest.mark.parametrize("physics,eos,shape", [("pimunu_pi", "table", (21, 19, 11)), ("pimunu", "conformal", (37, 35, 1)),
                                               ("ideal", "table", (13, 9, 6))])
def test_fp32_form_host_build_tracks_the_fp64_shared_face_form(physics, eos, shape):
    """The FP32 form (vah_tile_cell.cuh: state and arithmetic in FP32, Newton
    inversions and the closure fits in FP64, each face once with the left
    cell's guess) compiled for the host, against the FP64 shared-face form
    (vah_stage.cuh) on the same state: two steps within 2e-5 on e, P_L, u^mu and
    T^{tau mu}, 1e-4 on the (randomly seeded) pi and Pi fields -- FP32 rounding;
    any difference in the scheme would be O(1)."""
    tab = V.eos_table() if eos == "table" else None
    g = V.Grid(*shape, 0.2, 0.2, 0.2, 0.16, physics=physics, eos=eos,
               zeta="crossover" if eos == "table" else "reference", table=tab)
    f = V.smooth_initial_state(g, 0.5, amp=60.0, floor=0.5, flow=0.3, pi_amp=0.3)
    o = V.Oracle(g)
    V.load_state(o, f)
    o.set_conserved(0.5, 1)
    o.set_ghost_cells()
    state = {fid: o.field(fid).copy() for fid in V.state_ids(g.physics)}
    h64 = V.HostCheck(g, split=2)
    V.load_state(h64, state)
    t32 = V.TileCheck(g)
    t32.load(state)
    for n in range(2):
        h64.step(0.5 + 0.01 * n, 0.01)
        t32.step(0.5 + 0.01 * n, 0.01)
    for fid in [V.E, V.PL, V.UT, V.UX, V.UY, V.UN] + list(range(V.NQ[g.physics])):
        a, b = g.interior(t32.field(fid).astype(np.float64)), g.interior(h64.field(fid))
        scale = max(np.max(np.abs(b)), 1e-6 * np.max(np.abs(g.interior(h64.field(V.E)))))
        assert np.max(np.abs(a - b)) / scale < (1e-4 if 5 <= fid < 16 else 2e-5), fid
