"""Python binding of libvah.so (include/vah.h) through ctypes.

The library is the product; this module only loads it and wraps the C ABI
for Python callers (tests, bench, notebooks). There is no Python or CPU
implementation of the step behind it: if libvah.so is missing or no CUDA
device is present, creating an event raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
D, I, P = C.c_double, C.c_int, C.POINTER(C.c_double)

# include/vah.h constants
VAH_IDEAL, VAH_PIMUNU, VAH_PIMUNU_PI = 0, 1, 2
VAH_EOS_CONFORMAL, VAH_EOS_TABLE = 0, 1
VAH_ZETA_REFERENCE, VAH_ZETA_CROSSOVER = 0, 1
VAH_FP64, VAH_FP32 = 0, 1
VAH_FLUX_PER_CELL, VAH_FLUX_SHARED, VAH_FLUX_PER_CELL_FUSED = 0, 1, 2
VAH_PL_REFERENCE, VAH_PL_ISOTROPIC = 0, 1
NUM_FIELDS = 26
F_E, F_P, F_UT, F_UX, F_UY, F_UN = 16, 17, 18, 19, 20, 21
HBARC = 0.197326938
NUM_VALIDITY = 27  # VAH_NUM_VALIDITY
VALIDITY_NAMES = ["knTaupiT", "knTaupiL", "knTaupi", "knTauPi", "Rpi", "RPi", "Rpi2", "RPi2", "taupi", "dxux", "dyuy",
                  "theta", "stt", "sxx", "syy", "snn", "regulations", "regMag", "regTr", "regU0", "regU1", "regU2",
                  "regU3", "regZ0", "regZ1", "regZ2", "regZ3"]

STATUS = {0: "VAH_OK", -1: "VAH_ERR_ARG", -2: "VAH_ERR_CUDA", -3: "VAH_ERR_NOMEM", -4: "VAH_ERR_NAN",
          -5: "VAH_ERR_NODEVICE", -6: "VAH_ERR_TOO_LARGE"}


class VahError(RuntimeError):
    def __init__(self, where, rc):
        super().__init__(f"{where} failed: {STATUS.get(rc, rc)}")
        self.rc = rc


def check(rc, where):
    if rc != 0:
        raise VahError(where, rc)


class Lattice(C.Structure):
    _fields_ = [("nx", I), ("ny", I), ("nz", I), ("dx", D), ("dy", D), ("dz", D)]


class Hydro(C.Structure):
    _fields_ = [("t0", D), ("eta_over_s", D), ("freezeout_T_GeV", D)]


class Options(C.Structure):
    _fields_ = [("physics", I), ("eos", I), ("zeta", I), ("precision", I), ("flux", I), ("device", I),
                ("stream", C.c_void_p)]


class LaunchChoice(C.Structure):
    _fields_ = [("bx", C.c_int), ("by", C.c_int), ("minb", C.c_int), ("ms_default", C.c_double),
                ("ms_best", C.c_double)]


class TuneReport(C.Structure):
    _fields_ = [("nkinds", C.c_int), ("kind", LaunchChoice * 5)]

    def as_list(self):
        return [{"block": [k.bx, k.by], "minb": k.minb, "ms_default": k.ms_default, "ms_best": k.ms_best}
                for k in self.kind[:self.nkinds]]


class Stats(C.Structure):
    _fields_ = [("face_fallbacks", C.c_longlong), ("cell_fallbacks", C.c_longlong), ("nan_cells", C.c_longlong),
                ("steps", C.c_longlong)]


EXPORTS = ["vah_version", "vah_eos_table_build", "vah_event_create", "vah_event_destroy", "vah_event_set_field",
           "vah_event_get_field", "vah_event_set_conserved", "vah_event_init_from_e", "vah_event_set_ghost_cells",
           "vah_rk2_step", "vah_run", "vah_event_sync", "vah_event_stats", "vah_event_set_timing",
           "vah_event_kernel_time", "vah_rk2_step_host", "vah_ic_optical_glauber", "vah_ic_mc_glauber",
           "vah_ic_longitudinal", "vah_event_autotune", "vah_batch_autotune",
           "vah_batch_freezeout_volume", "vah_batch_fallback_mask", "vah_event_set_validity",
           "vah_event_get_validity", "vah_batch_add_glauber", "vah_ic_mc_glauber_participants",
           "vah_event_track_fallbacks", "vah_event_get_fallback_mask", "vah_fp64_peak", "vah_event_init_glauber",
           "vah_event_init_optical_glauber"]

_lib = None


def lib_path():
    return os.path.join(HERE, "libvah.so")


def library():
    """Load libvah.so (built in-tree by __graft_entry__.build())."""
    global _lib
    if _lib is None:
        path = lib_path()
        if not os.path.exists(path):
            raise RuntimeError(f"libvah.so is not built ({path})")
        L = C.CDLL(path)
        L.vah_version.restype = C.c_char_p
        L.vah_eos_table_build.argtypes = [I, P, C.c_size_t]
        L.vah_event_create.argtypes = [C.POINTER(Lattice), C.POINTER(Hydro), C.POINTER(Options), P,
                                       C.POINTER(C.c_void_p)]
        for name in ("vah_event_destroy", "vah_event_set_ghost_cells", "vah_event_sync"):
            getattr(L, name).argtypes = [C.c_void_p]
        L.vah_event_set_field.argtypes = [C.c_void_p, I, P, I]
        L.vah_event_autotune.argtypes = [C.c_void_p, I, C.POINTER(TuneReport)]
        L.vah_event_get_field.argtypes = [C.c_void_p, I, P, I]
        L.vah_event_set_conserved.argtypes = [C.c_void_p, D, I]
        L.vah_event_init_from_e.argtypes = [C.c_void_p, D, P, I]
        L.vah_rk2_step.argtypes = [C.c_void_p, D, D]
        L.vah_run.argtypes = [C.c_void_p, D, D, I]
        L.vah_event_stats.argtypes = [C.c_void_p, C.POINTER(Stats)]
        L.vah_event_set_timing.argtypes = [C.c_void_p, I]
        L.vah_event_track_fallbacks.argtypes = [C.c_void_p, I]
        L.vah_event_get_fallback_mask.argtypes = [C.c_void_p, I, C.POINTER(C.c_ubyte), I]
        L.vah_event_kernel_time.argtypes = [C.c_void_p, P, C.POINTER(C.c_longlong)]
        L.vah_rk2_step_host.argtypes = [C.c_void_p, D, D, C.POINTER(P)]
        L.vah_ic_optical_glauber.argtypes = [I, I, D, D, D, D, I, D, D, D, D, D, P]
        L.vah_ic_mc_glauber.argtypes = [I, I, D, D, D, D, I, D, D, D, C.c_ulonglong, D, D, P, C.POINTER(I)]
        L.vah_ic_longitudinal.argtypes = [I, D, D, D, P]
        _lib = L
    return _lib


def version():
    return library().vah_version().decode()


def fp64_peak(device=0):
    """Measured FP64 FMA throughput (TFLOP/s) and the timed launch's ms (vah_fp64_peak)."""
    L = library()
    L.vah_fp64_peak.argtypes = [I, C.POINTER(D), C.POINTER(D)]
    tf, ms = D(), D()
    check(L.vah_fp64_peak(device, C.byref(tf), C.byref(ms)), "vah_fp64_peak")
    return tf.value, ms.value


def eos_table(n=4096):
    """The tabulated crossover EoS (vah_eos_table_build)."""
    out = np.zeros(8 + 3 * n)
    check(library().vah_eos_table_build(n, out.ctypes.data_as(P), out.size), "vah_eos_table_build")
    return out


def table_energy_density(tab, T_fm):
    """e(T) by inverting the table's T(e) (bisection in ln e, host side)."""
    n = int(tab[0])
    lne0, dl = tab[1], tab[3]
    Ts = tab[8 + n:8 + 2 * n]
    lne = lne0 + dl * np.arange(n)
    return float(np.exp(np.interp(np.log(T_fm), np.log(Ts), lne)))


def optical_glauber(nx, ny, dx, dy, b=7.0, sigma_nn_fm2=4.2, A=197, R=6.38, a=0.535, x_coll=0.15, e_peak=1.0,
                    e_floor=1e-3):
    out = np.zeros(nx * ny)
    check(library().vah_ic_optical_glauber(nx, ny, dx, dy, b, sigma_nn_fm2, A, R, a, x_coll, e_peak, e_floor,
                                           out.ctypes.data_as(P)), "vah_ic_optical_glauber")
    return out


def mc_glauber(nx, ny, dx, dy, b, seed, sigma_nn_fm2=4.2, A=197, R=6.38, a=0.535, width=0.5, e_peak=1.0,
               e_floor=1e-3):
    out = np.zeros(nx * ny)
    npart = C.c_int()
    check(library().vah_ic_mc_glauber(nx, ny, dx, dy, b, sigma_nn_fm2, A, R, a, width, seed, e_peak, e_floor,
                                      out.ctypes.data_as(P), C.byref(npart)), "vah_ic_mc_glauber")
    return out, npart.value


def longitudinal(nz, dz, eta_flat=1.5, sigma_eta=1.3):
    out = np.zeros(nz)
    check(library().vah_ic_longitudinal(nz, dz, eta_flat, sigma_eta, out.ctypes.data_as(P)), "vah_ic_longitudinal")
    return out


class Event:
    """One hydro event on the GPU, through the C ABI."""

    def __init__(self, nx, ny, nz, dx, dy, dz, eta_over_s, physics=VAH_PIMUNU_PI, eos=VAH_EOS_TABLE,
                 zeta=VAH_ZETA_CROSSOVER, table=None, t0=0.5, precision=VAH_FP64, flux=VAH_FLUX_PER_CELL, device=0,
                 stream=None):
        self.L = library()
        self.nx, self.ny, self.nz = nx, ny, nz
        self.ncell = (nx + 4) * (ny + 4) * (nz + 4)
        self._table = None if table is None else np.ascontiguousarray(table, dtype=np.float64)
        lat = Lattice(nx, ny, nz, dx, dy, dz)
        hyd = Hydro(t0, eta_over_s, 0.155)
        opt = Options(physics, eos, zeta, precision, flux, device, stream)
        self.ev = C.c_void_p()
        tab = self._table.ctypes.data_as(P) if self._table is not None else None
        check(self.L.vah_event_create(C.byref(lat), C.byref(hyd), C.byref(opt), tab, C.byref(self.ev)),
              "vah_event_create")

    def close(self):
        if self.ev:
            self.L.vah_event_destroy(self.ev)
            self.ev = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_field(self, fid, arr, with_ghosts=True):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        check(self.L.vah_event_set_field(self.ev, fid, a.ctypes.data_as(P), int(with_ghosts)), "vah_event_set_field")

    def get_field(self, fid, with_ghosts=True):
        out = np.empty(self.ncell if with_ghosts else self.nx * self.ny * self.nz)
        check(self.L.vah_event_get_field(self.ev, fid, out.ctypes.data_as(P), int(with_ghosts)), "vah_event_get_field")
        return out

    def set_conserved(self, t, pl_from_field):
        check(self.L.vah_event_set_conserved(self.ev, t, int(pl_from_field)), "vah_event_set_conserved")

    def init_from_e(self, t0, e_interior, pl_mode=VAH_PL_ISOTROPIC):
        a = np.ascontiguousarray(e_interior, dtype=np.float64)
        check(self.L.vah_event_init_from_e(self.ev, t0, a.ctypes.data_as(P), pl_mode), "vah_event_init_from_e")

    def init_glauber(self, t0, b, seed, e_peak, e_floor=1e-3, sigma_nn_fm2=4.2, A=197, R=6.38, a=0.535, width=0.5,
                     eta_flat=1.5, sigma_eta=1.3, pl_mode=VAH_PL_ISOTROPIC):
        """MC-Glauber initial state generated on the device (vah_event_init_glauber)."""
        g = Glauber(b, sigma_nn_fm2, A, R, a, width, seed, e_peak, e_floor, eta_flat, sigma_eta)
        self.L.vah_event_init_glauber.argtypes = [C.c_void_p, D, C.POINTER(Glauber), I]
        check(self.L.vah_event_init_glauber(self.ev, t0, C.byref(g), pl_mode), "vah_event_init_glauber")

    def init_optical_glauber(self, t0, b, e_peak, e_floor=1e-3, sigma_nn_fm2=4.2, A=197, R=6.38, a=0.535,
                             x_coll=0.15, eta_flat=1.5, sigma_eta=1.3, pl_mode=VAH_PL_ISOTROPIC):
        """Optical-Glauber initial state generated on the device (vah_event_init_optical_glauber)."""
        o = Optical(b, sigma_nn_fm2, A, R, a, x_coll, e_peak, e_floor, eta_flat, sigma_eta)
        self.L.vah_event_init_optical_glauber.argtypes = [C.c_void_p, D, C.POINTER(Optical), I]
        check(self.L.vah_event_init_optical_glauber(self.ev, t0, C.byref(o), pl_mode),
              "vah_event_init_optical_glauber")

    def set_ghost_cells(self):
        check(self.L.vah_event_set_ghost_cells(self.ev), "vah_event_set_ghost_cells")

    def step(self, t, dt):
        check(self.L.vah_rk2_step(self.ev, t, dt), "vah_rk2_step")

    def run(self, t0, dt, n):
        check(self.L.vah_run(self.ev, t0, dt, n), "vah_run")

    def sync(self):
        check(self.L.vah_event_sync(self.ev), "vah_event_sync")

    def stats(self):
        s = Stats()
        check(self.L.vah_event_stats(self.ev, C.byref(s)), "vah_event_stats")
        return s

    def track_fallbacks(self, on=True):
        check(self.L.vah_event_track_fallbacks(self.ev, int(on)), "vah_event_track_fallbacks")

    def fallback_mask(self, stage, with_ghosts=True):
        """Per cell, 1 where the latest step's stage-`stage` inversion fell back (uint8)."""
        out = np.empty(self.ncell if with_ghosts else self.nx * self.ny * self.nz, dtype=np.uint8)
        check(self.L.vah_event_get_fallback_mask(self.ev, int(stage), out.ctypes.data_as(C.POINTER(C.c_ubyte)),
                                                 int(with_ghosts)), "vah_event_get_fallback_mask")
        return out

    def set_timing(self, on):
        check(self.L.vah_event_set_timing(self.ev, int(on)), "vah_event_set_timing")

    def kernel_time(self):
        ms, n = D(), C.c_longlong()
        check(self.L.vah_event_kernel_time(self.ev, C.byref(ms), C.byref(n)), "vah_event_kernel_time")
        return ms.value, n.value

    def set_validity(self, on):
        """Fill the validity diagnostics (VAH_V_* fields) at every following step."""
        check(self.L.vah_event_set_validity(self.ev, int(on)), "vah_event_set_validity")

    def get_validity(self, vid, with_ghosts=True):
        out = np.empty(self.ncell if with_ghosts else self.nx * self.ny * self.nz)
        check(self.L.vah_event_get_validity(self.ev, vid, out.ctypes.data_as(P), int(with_ghosts)),
              "vah_event_get_validity")
        return out

    def autotune(self, reps=3):
        """Pick the fastest launch configuration per kernel kind (vah_event_autotune); returns the choices."""
        r = TuneReport()
        check(self.L.vah_event_autotune(self.ev, int(reps), C.byref(r)), "vah_event_autotune")
        return r.as_list()

    def step_host(self, t, dt, ptrs):
        """Host-buffer step: ptrs = list of NUM_FIELDS host addresses (0 for unused)."""
        arr = (P * NUM_FIELDS)(*[C.cast(C.c_void_p(p), P) if p else P() for p in ptrs])
        check(self.L.vah_rk2_step_host(self.ev, t, dt, arr), "vah_rk2_step_host")


class EventInfo(C.Structure):
    _fields_ = [("t", D), ("steps", C.c_longlong), ("face_fallbacks", C.c_longlong),
                ("cell_fallbacks", C.c_longlong), ("nan_cells", C.c_longlong), ("bytes", C.c_longlong)]


VAH_ERR_FULL = -7


def _batch_lib():
    L = library()
    if not getattr(L, "_batch_ready", False):
        L.vah_batch_create.argtypes = [C.POINTER(Options), P, C.c_size_t, C.POINTER(C.c_void_p)]
        L.vah_batch_autotune.argtypes = [C.c_void_p, I, C.POINTER(TuneReport)]
        L.vah_batch_add_glauber.argtypes = [C.c_void_p, C.POINTER(Lattice), C.POINTER(Hydro), D, C.POINTER(Glauber), I,
                                            C.POINTER(I)]
        for name in ("vah_batch_destroy", "vah_batch_sync"):
            getattr(L, name).argtypes = [C.c_void_p]
        L.vah_batch_event_bytes.argtypes = [C.c_void_p, C.POINTER(Lattice), C.POINTER(C.c_size_t)]
        L.vah_batch_add.argtypes = [C.c_void_p, C.POINTER(Lattice), C.POINTER(Hydro), D, P, I, C.POINTER(I)]
        L.vah_batch_remove.argtypes = [C.c_void_p, I]
        L.vah_batch_step.argtypes = [C.c_void_p, I]
        L.vah_batch_event_info.argtypes = [C.c_void_p, I, C.POINTER(EventInfo)]
        L.vah_batch_get_field.argtypes = [C.c_void_p, I, I, P, I]
        L.vah_batch_max_energy_density.argtypes = [C.c_void_p, P, I]
        L.vah_batch_observables.argtypes = [C.c_void_p, P, I]
        L.vah_batch_set_timing.argtypes = [C.c_void_p, I]
        L.vah_batch_kernel_time.argtypes = [C.c_void_p, P, C.POINTER(C.c_longlong)]
        L._batch_ready = True
    return L


class Glauber(C.Structure):
    _fields_ = [("b", D), ("sigma_nn_fm2", D), ("A", I), ("ws_R", D), ("ws_a", D), ("width", D),
                ("seed", C.c_ulonglong), ("e_peak", D), ("e_floor", D), ("eta_flat", D), ("sigma_eta", D)]


class Optical(C.Structure):
    _fields_ = [("b", D), ("sigma_nn_fm2", D), ("A", I), ("ws_R", D), ("ws_a", D), ("x_coll", D), ("e_peak", D),
                ("e_floor", D), ("eta_flat", D), ("sigma_eta", D)]


class Batch:
    """Many device-resident events advanced together (vah_batch_*)."""

    def __init__(self, physics=VAH_PIMUNU_PI, eos=VAH_EOS_TABLE, zeta=VAH_ZETA_CROSSOVER, table=None,
                 capacity_bytes=64 << 30, precision=VAH_FP64, flux=VAH_FLUX_PER_CELL, device=0, stream=None):
        self.L = _batch_lib()
        self._table = None if table is None else np.ascontiguousarray(table, dtype=np.float64)
        opt = Options(physics, eos, zeta, precision, flux, device, stream)
        self.b = C.c_void_p()
        tab = self._table.ctypes.data_as(P) if self._table is not None else None
        check(self.L.vah_batch_create(C.byref(opt), tab, capacity_bytes, C.byref(self.b)), "vah_batch_create")
        self.shapes = {}

    def close(self):
        if self.b:
            self.L.vah_batch_destroy(self.b)
            self.b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def event_bytes(self, nx, ny, nz):
        n = C.c_size_t()
        check(self.L.vah_batch_event_bytes(self.b, C.byref(Lattice(nx, ny, nz, 0.1, 0.1, 0.1)), C.byref(n)),
              "vah_batch_event_bytes")
        return n.value

    def add(self, nx, ny, nz, dx, dy, dz, t0, dt, eta_over_s, e_interior, pl_mode=VAH_PL_ISOTROPIC):
        """Returns the slot, or None when the batch is full (VAH_ERR_FULL)."""
        a = np.ascontiguousarray(e_interior, dtype=np.float64)
        slot = C.c_int()
        rc = self.L.vah_batch_add(self.b, C.byref(Lattice(nx, ny, nz, dx, dy, dz)), C.byref(Hydro(t0, eta_over_s, 0.15)),
                                  dt, a.ctypes.data_as(P), pl_mode, C.byref(slot))
        if rc == VAH_ERR_FULL:
            return None
        check(rc, "vah_batch_add")
        self.shapes[slot.value] = (nx, ny, nz)
        return slot.value

    def add_glauber(self, nx, ny, nz, dx, dy, dz, t0, dt, eta_over_s, b, seed, e_peak, e_floor=1e-3, sigma_nn_fm2=4.2,
                    A=197, R=6.38, a=0.535, width=0.5, eta_flat=1.5, sigma_eta=1.3, pl_mode=VAH_PL_ISOTROPIC):
        """An event whose MC-Glauber initial condition is generated on the device; None when full."""
        g = Glauber(b, sigma_nn_fm2, A, R, a, width, seed, e_peak, e_floor, eta_flat, sigma_eta)
        slot = C.c_int()
        rc = self.L.vah_batch_add_glauber(self.b, C.byref(Lattice(nx, ny, nz, dx, dy, dz)),
                                          C.byref(Hydro(t0, eta_over_s, 0.15)), dt, C.byref(g), pl_mode,
                                          C.byref(slot))
        if rc == VAH_ERR_FULL:
            return None
        check(rc, "vah_batch_add_glauber")
        self.shapes[slot.value] = (nx, ny, nz)
        return slot.value

    def remove(self, slot):
        check(self.L.vah_batch_remove(self.b, slot), "vah_batch_remove")
        self.shapes.pop(slot, None)

    def step(self, n=1):
        check(self.L.vah_batch_step(self.b, n), "vah_batch_step")

    def sync(self):
        check(self.L.vah_batch_sync(self.b), "vah_batch_sync")

    def info(self, slot):
        i = EventInfo()
        check(self.L.vah_batch_event_info(self.b, slot, C.byref(i)), "vah_batch_event_info")
        return i

    def get_field(self, slot, fid, with_ghosts=True):
        nx, ny, nz = self.shapes[slot]
        out = np.empty((nx + 4) * (ny + 4) * (nz + 4) if with_ghosts else nx * ny * nz)
        check(self.L.vah_batch_get_field(self.b, slot, fid, out.ctypes.data_as(P), int(with_ghosts)),
              "vah_batch_get_field")
        return out

    def max_energy_density(self, nslots):
        out = np.zeros(nslots)
        check(self.L.vah_batch_max_energy_density(self.b, out.ctypes.data_as(P), nslots),
              "vah_batch_max_energy_density")
        return out

    def observables(self, nslots):
        out = np.zeros(3 * nslots)
        check(self.L.vah_batch_observables(self.b, out.ctypes.data_as(P), nslots), "vah_batch_observables")
        return out.reshape(nslots, 3)

    def freezeout_volume(self, nslots):
        """Per-slot freeze-out surface volume so far (fm^4)."""
        out = np.zeros(nslots)
        check(self.L.vah_batch_freezeout_volume(self.b, out.ctypes.data_as(P), nslots), "vah_batch_freezeout_volume")
        return out

    def fallback_mask(self, slot):
        """Interior cells whose latest inversion fell back (bool array, x fastest)."""
        nx, ny, nz = self.shapes[slot]
        out = np.zeros(nx * ny * nz, np.uint8)
        check(self.L.vah_batch_fallback_mask(self.b, slot, out.ctypes.data_as(C.c_void_p)), "vah_batch_fallback_mask")
        return out.astype(bool)

    def set_timing(self, on):
        check(self.L.vah_batch_set_timing(self.b, int(on)), "vah_batch_set_timing")

    def kernel_time(self):
        ms, n = D(), C.c_longlong()
        check(self.L.vah_batch_kernel_time(self.b, C.byref(ms), C.byref(n)), "vah_batch_kernel_time")
        return ms.value, n.value

    def autotune(self, reps=3):
        """Pick the fastest register-cap variant per launch kind (vah_batch_autotune); returns the choices."""
        r = TuneReport()
        check(self.L.vah_batch_autotune(self.b, int(reps), C.byref(r)), "vah_batch_autotune")
        return r.as_list()


class ServeConfig(C.Structure):
    _fields_ = [("rate", D), ("duration_s", D), ("seed", C.c_ulonglong), ("frac_3d", D), ("side2_min", I),
                ("side2_max", I), ("side3_min", I), ("side3_max", I), ("nz3_min", I), ("nz3_max", I), ("dx", D),
                ("deta", D), ("b_max", D), ("t0", D), ("dt", D), ("eta_over_s", D), ("T0_GeV", D), ("Tf_GeV", D),
                ("t_max", D), ("physics", I), ("eos", I), ("precision", I), ("flux", I), ("device", I),
                ("capacity_bytes", C.c_size_t), ("chunk_steps", I), ("ic_threads", I), ("e_floor", D),
                ("ic_on_device", I)]


class ServeResult(C.Structure):
    _fields_ = [("offered", C.c_longlong), ("completed", C.c_longlong), ("timeouts", C.c_longlong),
                ("rejected", C.c_longlong), ("wall_s", D), ("events_per_s", D), ("p50_s", D), ("p99_s", D),
                ("cell_updates", C.c_longlong), ("cell_updates_per_s", D), ("max_resident", C.c_longlong),
                ("chunks", C.c_longlong), ("failed", C.c_longlong), ("tau_freeze_max", D)]


def serve(**kw):
    """Run the continuous-batching request loop (vah_serve_run); returns (result dict, latencies).

    Defaults: peak temperature 0.4 GeV and an initial floor of 0.01 fm^-4. At a 0.6 GeV peak with the
    reference's 1e-3 floor, lumpy 0.2 fm grids drive most dilute cells into the inversion fallback and
    leave isolated single-cell spikes far above their neighbours, which keep max T above freeze-out."""
    L = library()
    L.vah_serve_run.argtypes = [C.POINTER(ServeConfig), C.POINTER(ServeResult), P, I]
    cfg = dict(rate=50.0, duration_s=10.0, seed=1, frac_3d=0.3, side2_min=61, side2_max=261, side3_min=81,
               side3_max=161, nz3_min=41, nz3_max=81, dx=0.2, deta=0.2, b_max=14.0, t0=0.25, dt=0.02,
               eta_over_s=0.16, T0_GeV=0.4, Tf_GeV=0.150, t_max=100.0, physics=VAH_PIMUNU_PI, eos=VAH_EOS_TABLE,
               precision=VAH_FP64, flux=VAH_FLUX_PER_CELL, device=0, capacity_bytes=120 << 30, chunk_steps=10,
               ic_threads=16, e_floor=1e-2, ic_on_device=1)
    cfg.update(kw)
    c = ServeConfig(**cfg)
    r = ServeResult()
    lat = np.zeros(100000)
    check(L.vah_serve_run(C.byref(c), C.byref(r), lat.ctypes.data_as(P), lat.size), "vah_serve_run")
    out = {k: getattr(r, k) for k, _ in ServeResult._fields_}
    return out, lat[:r.completed].copy()
