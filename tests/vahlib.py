"""ctypes bindings used by the tests: the library (libvah.so), the CPU oracle
(oracle/_build/libvah_oracle.so), the reference's own CPU step
(oracle/_ref/libvahref_<variant>.so) and the host build of the library's cell
code (tests/hostcheck). Only tests, the smoke check and the benchmark's
CPU-baseline leg use the oracle pieces.
"""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
D, I, P = C.c_double, C.c_int, C.POINTER(C.c_double)

# field ids (include/vah.h)
TTT, TTX, TTY, TTN, PL = 0, 1, 2, 3, 4
PITT, PITX, PITY, PITN, PIXX, PIXY, PIXN, PIYY, PIYN, PINN, PI = range(5, 16)
E, PP, UT, UX, UY, UN, UPT, UPX, UPY, UPN = range(16, 26)
NUM_FIELDS = 26
PHYSICS = {"ideal": 0, "pimunu": 1, "pimunu_pi": 2}
NQ = {0: 5, 1: 15, 2: 16}


def conserved_ids(physics):
    nq = NQ[physics]
    return list(range(nq)) if nq < 16 else list(range(16))


def state_ids(physics):
    return conserved_ids(physics) + [E, PP, UT, UX, UY, UN, UPT, UPX, UPY, UPN]


def make(target_dir, *targets):
    subprocess.run(["make", "-s", "-C", target_dir, *targets], check=True)


# --------------------------------------------------------------- the oracle --
class VOConfig(C.Structure):
    _fields_ = [("nx", I), ("ny", I), ("nz", I), ("dx", D), ("dy", D), ("dz", D), ("etabar", D),
                ("physics", I), ("eos", I), ("zeta", I), ("eos_table", P)]


_oracle = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        path = os.path.join(ROOT, "oracle", "_build", "libvah_oracle.so")
        if not os.path.exists(path):
            make(os.path.join(ROOT, "oracle"), "restate")
        L = C.CDLL(path)
        L.vo_create.restype = C.c_void_p
        L.vo_create.argtypes = [C.POINTER(VOConfig)]
        L.vo_destroy.argtypes = [C.c_void_p]
        L.vo_field.restype = P
        L.vo_field.argtypes = [C.c_void_p, I]
        L.vo_num_cells.argtypes = [C.c_void_p]
        L.vo_set_conserved.argtypes = [C.c_void_p, D, I]
        L.vo_set_ghost_cells.argtypes = [C.c_void_p]
        L.vo_step.argtypes = [C.c_void_p, D, D]
        L.vo_run.argtypes = [C.c_void_p, D, D, I]
        L.vo_run.restype = D
        L.vo_last_step_stats.argtypes = [C.c_void_p, C.POINTER(C.c_longlong)]
        L.vo_infer.argtypes = [C.POINTER(VOConfig), D, P, D, D, P]
        L.vo_infer.restype = I
        L.vo_approx_derivative.argtypes = [D, D, D]
        L.vo_approx_derivative.restype = D
        L.vo_eos_eval.argtypes = [C.POINTER(VOConfig), D, P]
        L.vo_set_validity.argtypes = [C.c_void_p, I]
        L.vo_validity_field.restype = P
        L.vo_validity_field.argtypes = [C.c_void_p, I]
        L.vo_last_step_face_fallbacks.argtypes = [C.c_void_p, C.POINTER(C.c_longlong)]
        L.vo_fallback_mask.restype = C.POINTER(C.c_ubyte)
        L.vo_fallback_mask.argtypes = [C.c_void_p, I]
        L.vo_eos_table_build.argtypes = [I, P, C.c_size_t]
        L.vo_ic_mc_glauber.argtypes = [I, I, D, D, D, D, I, D, D, D, C.c_ulonglong, D, D, P, C.POINTER(I)]
        L.vo_ic_longitudinal.argtypes = [I, D, D, D, P]
        _oracle = L
    return _oracle


# The workloads' inputs built by the oracle library (no product code): the
# reference arm of the benchmark uses these.
def oracle_eos_table(n=4096):
    out = np.zeros(8 + 3 * n)
    assert oracle_lib().vo_eos_table_build(n, out.ctypes.data_as(P), out.size) == 0
    return out


def oracle_mc_glauber(nx, ny, dx, dy, b, seed, sigma_nn_fm2=4.2, A=197, R=6.38, a=0.535, width=0.5, e_peak=1.0,
                      e_floor=1e-3):
    out = np.zeros(nx * ny)
    npart = C.c_int()
    assert oracle_lib().vo_ic_mc_glauber(nx, ny, dx, dy, b, sigma_nn_fm2, A, R, a, width, seed, e_peak, e_floor,
                                         out.ctypes.data_as(P), C.byref(npart)) == 0
    return out, npart.value


def oracle_longitudinal(nz, dz, eta_flat=1.5, sigma_eta=1.3):
    out = np.zeros(nz)
    assert oracle_lib().vo_ic_longitudinal(nz, dz, eta_flat, sigma_eta, out.ctypes.data_as(P)) == 0
    return out


def table_energy_density(tab, T_fm):
    """e(T) by inverting a table's T(e) (interpolation in ln e)."""
    n = int(tab[0])
    Ts = tab[8 + n:8 + 2 * n]
    lne = tab[1] + tab[3] * np.arange(n)
    return float(np.exp(np.interp(np.log(T_fm), np.log(Ts), lne)))


class Grid:
    """Grid + physics description shared by every implementation."""

    def __init__(self, nx, ny, nz, dx, dy, dz, etabar, physics="pimunu", eos="conformal", zeta="reference",
                 table=None):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.dx, self.dy, self.dz = dx, dy, dz
        self.etabar = etabar
        self.physics = PHYSICS[physics] if isinstance(physics, str) else physics
        self.eos = {"conformal": 0, "table": 1}[eos] if isinstance(eos, str) else eos
        self.zeta = {"reference": 0, "crossover": 1}[zeta] if isinstance(zeta, str) else zeta
        self.table = None if table is None else np.ascontiguousarray(table, dtype=np.float64)
        self.shape = (nz + 4, ny + 4, nx + 4)
        self.ncell = int(np.prod(self.shape))

    def interior(self, a):
        return a.reshape(self.shape)[2:-2, 2:-2, 2:-2]

    def coords(self):
        k, j, i = np.meshgrid(np.arange(self.shape[0]), np.arange(self.shape[1]), np.arange(self.shape[2]),
                              indexing="ij")
        x = (i - 2 - (self.nx - 1) / 2) * self.dx
        y = (j - 2 - (self.ny - 1) / 2) * self.dy
        z = (k - 2 - (self.nz - 1) / 2) * self.dz
        return x, y, z


class Oracle:
    def __init__(self, g: Grid):
        self.g = g
        self.L = oracle_lib()
        tab = g.table.ctypes.data_as(P) if g.table is not None else None
        self.cfg = VOConfig(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, g.etabar, g.physics, g.eos, g.zeta, tab)
        self.st = self.L.vo_create(C.byref(self.cfg))
        assert self.st, "oracle create failed"

    def __del__(self):
        try:
            self.L.vo_destroy(self.st)
        except Exception:
            pass

    def field(self, fid):
        return np.ctypeslib.as_array(self.L.vo_field(self.st, fid), (self.g.ncell,))

    def set_conserved(self, t, pl_from_field):
        self.L.vo_set_conserved(self.st, t, int(pl_from_field))

    def set_ghost_cells(self):
        self.L.vo_set_ghost_cells(self.st)

    def step(self, t, dt):
        self.L.vo_step(self.st, t, dt)

    def run(self, t0, dt, n):
        return self.L.vo_run(self.st, t0, dt, n)

    def stats(self):
        out = (C.c_longlong * 3)()
        self.L.vo_last_step_stats(self.st, out)
        return list(out)

    def face_fallbacks_by_axis(self):
        out = (C.c_longlong * 3)()
        self.L.vo_last_step_face_fallbacks(self.st, out)
        return list(out)

    def fallback_mask(self, stage):
        """Per ghosted cell, 1 where the last step's stage-`stage` inversion fell back."""
        return np.ctypeslib.as_array(self.L.vo_fallback_mask(self.st, stage), (self.g.ncell,)).copy()

    def set_validity(self, on):
        self.L.vo_set_validity(self.st, int(on))

    def validity(self, vid):
        return np.ctypeslib.as_array(self.L.vo_validity_field(self.st, vid), (self.g.ncell,))


# ---------------------------------------------------- the reference itself --
# Validity ids (include/vah.h VAH_V_*) -> member index in the reference's
# VALIDITY_DOMAIN (DynamicalVariables.h:86-117): knTaupiT, knTaupiL, knTaupi,
# knTauPi, Rpi, RPi, Rpi2, RPi2, taupi, dxux, dyuy, theta, stt, sxx, syy, snn,
# regulations, regMag, regTr, regU0-3, regZ0-3.
REF_VALIDITY_MEMBER = [0, 1, 2, 3, 4, 5, 7, 8, 26, 27, 28, 29, 22, 23, 24, 25, 11, 12, 13, 14, 15, 16, 17, 18, 19,
                       20, 21]
NUM_VALIDITY = 27
V_RPI2, V_RPI2_BULK, V_REGULATIONS = 6, 7, 16  # VAH_V_RPI2, VAH_V_RPI2_BULK, VAH_V_REGULATIONS


def ref_path(physics, eos):
    name = {0: "ideal", 1: "pimunu", 2: "pimunu_pi"}[physics]
    return os.path.join(ROOT, "oracle", "_ref", f"libvahref_{name}_{'conf' if eos == 0 else 'table'}.so")


def ref_available(physics=1, eos=0):
    return os.path.exists(ref_path(physics, eos))


class Reference:
    """The reference's own CPU step (process globals; one grid per library)."""

    _libs = {}

    def __init__(self, g: Grid):
        self.g = g
        path = ref_path(g.physics, g.eos)
        L = Reference._libs.get(path)
        if L is None:
            L = C.CDLL(path, mode=C.RTLD_LOCAL)
            L.vref_init.argtypes = [I, I, I, D, D, D, D, D, D]
            L.vref_field.restype = P
            L.vref_field.argtypes = [I]
            L.vref_step.argtypes = [D, D]
            L.vref_run.argtypes = [D, D, I]
            L.vref_run.restype = D
            L.vref_set_conserved.argtypes = [D]
            L.vref_set_eos_table.argtypes = [P]
            Reference._libs[path] = L
        self.L = L
        n = L.vref_init(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, 0.0, g.etabar, 0.0)
        assert n == g.ncell
        if g.table is not None:
            L.vref_set_eos_table(g.table.ctypes.data_as(P))

    def field(self, fid):
        p = self.L.vref_field(fid)
        return np.ctypeslib.as_array(p, (self.g.ncell,)) if p else None

    def validity(self, vid):
        """The reference's own VALIDITY_DOMAIN array for a VAH_V_* id."""
        self.L.vref_validity.restype = P
        self.L.vref_validity.argtypes = [I]
        p = self.L.vref_validity(REF_VALIDITY_MEMBER[vid])
        return np.ctypeslib.as_array(p, (self.g.ncell,)) if p else None

    def set_conserved(self, t):
        self.L.vref_set_conserved(t)

    def set_ghost_cells(self):
        self.L.vref_set_ghost_cells()

    def step(self, t, dt):
        self.L.vref_step(t, dt)

    def run(self, t0, dt, n):
        return self.L.vref_run(t0, dt, n)


# ------------------------------------------------- host build of the cells --
_hc = None


def hostcheck_lib():
    global _hc
    if _hc is None:
        make(os.path.join(ROOT, "tests", "hostcheck"))
        L = C.CDLL(os.path.join(ROOT, "tests", "hostcheck", "_build", "libvah_hostcheck.so"))
        L.hc_create.restype = C.c_void_p
        L.hc_create.argtypes = [I, I, I, D, D, D, D, I, I, I, P, C.c_void_p, I]
        L.hc_destroy.argtypes = [C.c_void_p]
        L.hc_field.restype = P
        L.hc_field.argtypes = [C.c_void_p, I]
        L.hc_set_conserved.argtypes = [C.c_void_p, D, I]
        L.hc_step.argtypes = [C.c_void_p, D, D]
        L.hc_counters.argtypes = [C.c_void_p, C.POINTER(C.c_ulonglong)]
        L.hc_set_split.argtypes = [C.c_void_p, I]
        L.hc_approx_derivative.argtypes = [P, P, P, P, C.c_longlong]
        L.hc_regulate.argtypes = [D, D, D, P, P, I]
        _hc = L
    return _hc


class TileCheck:
    """Host build of the FP32 form (the tile kernel's face and cell arithmetic,
    gpu-vah_b200/csrc/vah_tile_cell.cuh): float state in the reference layout."""

    def __init__(self, g: Grid):
        self.g = g
        self.L = hostcheck_lib()
        L = self.L
        if not getattr(L, "_tc_ready", False):
            L.tc_create.restype = C.c_void_p
            L.tc_create.argtypes = [I, I, I, D, D, D, D, I, I, I, P]
            L.tc_destroy.argtypes = [C.c_void_p]
            L.tc_field.restype = C.POINTER(C.c_float)
            L.tc_field.argtypes = [C.c_void_p, I]
            L.tc_step.argtypes = [C.c_void_p, D, D]
            L.tc_counters.argtypes = [C.c_void_p, C.POINTER(C.c_ulonglong)]
            L._tc_ready = True
        tab = g.table.ctypes.data_as(P) if g.table is not None else None
        self.h = L.tc_create(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, g.etabar, g.physics, g.eos, g.zeta, tab)

    def __del__(self):
        try:
            self.L.tc_destroy(self.h)
        except Exception:
            pass

    def field(self, fid):
        p = self.L.tc_field(self.h, fid)
        return np.ctypeslib.as_array(p, (self.g.ncell,)) if p else None

    def load(self, fields):
        for fid, arr in fields.items():
            dst = self.field(fid)
            if dst is not None:
                dst[:] = np.asarray(arr, dtype=np.float32)

    def step(self, t, dt):
        self.L.tc_step(self.h, t, dt)

    def counters(self):
        out = (C.c_ulonglong * 3)()
        self.L.tc_counters(self.h, out)
        return list(out)


class HostCheck:
    def __init__(self, g: Grid, libm_exceptions=True, split=0):
        """libm_exceptions: reproduce the host libm's powf rounding in the
        conformal temperature (as the library does) or not. split: 0 = fused
        per-cell stage, 1 = face/cell split with reference faces, 2 = split
        with shared faces."""
        self.g = g
        self.L = hostcheck_lib()
        tab = g.table.ctypes.data_as(P) if g.table is not None else None
        excp = None
        nexc = -1 if libm_exceptions else 0
        self.h = self.L.hc_create(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, g.etabar, g.physics, g.eos, g.zeta, tab, excp,
                                  nexc)
        self.L.hc_set_split(self.h, int(split))

    def __del__(self):
        try:
            self.L.hc_destroy(self.h)
        except Exception:
            pass

    def field(self, fid):
        p = self.L.hc_field(self.h, fid)
        return np.ctypeslib.as_array(p, (self.g.ncell,)) if p else None

    def set_conserved(self, t, pl_from_field):
        self.L.hc_set_conserved(self.h, t, int(pl_from_field))

    def step(self, t, dt):
        self.L.hc_step(self.h, t, dt)

    def set_validity(self, on):
        self.L.hc_set_validity(self.h, int(on))

    def validity(self, vid):
        self.L.hc_validity_field.restype = P
        self.L.hc_validity_field.argtypes = [C.c_void_p, I]
        return np.ctypeslib.as_array(self.L.hc_validity_field(self.h, vid), (self.g.ncell,))


# ------------------------------------------------------------- the library --
import sys as _sys

_sys.path.insert(0, os.path.join(ROOT, "gpu-vah_b200"))
import vah as product  # noqa: E402  (gpu-vah_b200/vah.py)

EXPORTS = product.EXPORTS
library = product.library
lib_path = product.lib_path


def eos_table(n=4096):
    return product.eos_table(n)


class Event(product.Event):
    """A device event built from a Grid."""

    def __init__(self, g: "Grid", t0=0.5, precision=0, flux=0, device=0, stream=None):
        self.g = g
        super().__init__(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, g.etabar, physics=g.physics, eos=g.eos, zeta=g.zeta,
                         table=g.table, t0=t0, precision=precision, flux=flux, device=device, stream=stream)


# ------------------------------------------------------- shared test inputs --
def smooth_initial_state(g: Grid, t0, amp=50.0, floor=0.5, flow=0.3, pi_amp=0.0, seed=1):
    """A smooth anisotropic Gaussian blob with radial transverse flow and
    optionally random shear/bulk (to exercise the regulator): dict field -> array."""
    rng = np.random.default_rng(seed)
    x, y, z = g.coords()
    e = amp * np.exp(-(x ** 2 / 8 + y ** 2 / 5 + z ** 2 / 4)) + floor
    w = np.exp(-(x ** 2 + y ** 2) / 10)
    ux = flow * x / 4 * w
    uy = flow * y / 5 * w
    ut = np.sqrt(1 + ux ** 2 + uy ** 2)
    if g.eos == 1:
        p = np.array([eos_point_oracle(g, ev)[0] for ev in e.ravel()]).reshape(e.shape)
    else:
        p = e / 3
    fields = {E: e, PP: p, UT: ut, UX: ux, UY: uy, UN: 0 * e, PL: p}
    if g.physics >= 1:
        for f in range(PITT, PINN + 1):
            fields[f] = pi_amp * 0.01 * e * rng.standard_normal(e.shape)
    if g.physics == 2:
        fields[PI] = pi_amp * 0.01 * e * rng.standard_normal(e.shape)
    return {k: np.ascontiguousarray(v.ravel()) for k, v in fields.items()}


def eos_point_oracle(g: Grid, e):
    L = oracle_lib()
    tab = g.table.ctypes.data_as(P) if g.table is not None else None
    cfg = VOConfig(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz, g.etabar, g.physics, g.eos, g.zeta, tab)
    out = (D * 3)()
    L.vo_eos_eval(C.byref(cfg), e, out)
    return list(out)


def load_state(impl, fields):
    for fid, arr in fields.items():
        dst = impl.field(fid)
        if dst is not None:
            dst[:] = arr


def rel_linf(a, b):
    """Normwise relative L-infinity: max|a-b| / max|a|."""
    scale = np.max(np.abs(a))
    return float(np.max(np.abs(a - b)) / scale) if scale > 0 else float(np.max(np.abs(a - b)))
