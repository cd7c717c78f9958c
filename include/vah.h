/*
 * vah.h -- C ABI of the B200 VAH time step (libvah.so).
 *
 * Drop-in boundary for the anisotropic viscous hydrodynamics step of
 * derekeverett/GPU-VAH. Plain pointers and sizes only; every call returns an
 * int status (VAH_OK = 0, < 0 on error) and never exits or traps. Each entry
 * point names the reference interface it replaces (file:line within the
 * reference project).
 *
 * Data layout (part of the drop-in surface): one array per field, cell
 * (i, j, k) of an nx*ny*nz interior grid with 2 ghost layers per side at
 * i + ncx*(j + ncy*k), nc = n + 4, x fastest
 * (rhic/src/DynamicalVariables.cpp:29-31, rhic/include/LatticeParameters.h:13-15).
 *
 * Threading: calls on one event are not thread-safe; distinct events may be
 * driven from distinct host threads. Work is queued on the event's stream.
 */
#ifndef VAH_H
#define VAH_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define VAH_OK 0
#define VAH_ERR_ARG (-1)        /* invalid argument */
#define VAH_ERR_CUDA (-2)       /* a CUDA runtime call failed */
#define VAH_ERR_NOMEM (-3)      /* device allocation failed */
#define VAH_ERR_NAN (-4)        /* a NaN reached e or u (reference: exit(-1)) */
#define VAH_ERR_NODEVICE (-5)   /* no CUDA device / kernels not loadable */
#define VAH_ERR_TOO_LARGE (-6)  /* request exceeds a stated maximum */
#define VAH_ERR_FULL (-7)       /* batch capacity (bytes or slots) exhausted: retry after a removal */

/* ---- physics variants (reference compile-time macros, DynamicalVariables.h:13-15) ---- */
#define VAH_IDEAL 0       /* N_q = 5:  T^{tau mu}, P_L */
#define VAH_PIMUNU 1      /* N_q = 15: + pi_perp^{mu nu} (-DPIMUNU) */
#define VAH_PIMUNU_PI 2   /* N_q = 16: + bulk Pi (-DPIMUNU -DPI) */

/* ---- equations of state ---- */
#define VAH_EOS_CONFORMAL 0 /* reference EquationOfState.cpp with CONFORMAL_EOS (:78,113,144) */
#define VAH_EOS_TABLE 1     /* tabulated crossover EoS (vah_eos_table_build) */

/* ---- zeta/s ---- */
#define VAH_ZETA_REFERENCE 0 /* SourceTerms.cpp:36-44 */
#define VAH_ZETA_CROSSOVER 1 /* height 0.05 at T = 155 MeV, half-width 50 MeV */

/* ---- storage precision ---- */
#define VAH_FP64 0 /* state stored and updated in FP64 */
#define VAH_FP32 1 /* state, reconstruction, flux and sources in FP32; Newton inversions, closure fits and
                     reductions in FP64; one TMA-tiled launch per RK stage */

/* ---- face-flux evaluation ---- */
#define VAH_FLUX_PER_CELL 0       /* each face evaluated by both neighbouring cells with that cell's
                                     Newton guess and fallback energy, as the reference does
                                     (FullyDiscreteKurganovTadmorScheme.cpp:179,183); face and cell
                                     launches per stage, face fluxes in scratch buffers */
#define VAH_FLUX_SHARED 1         /* each face evaluated once, with the left cell's guess and fallback
                                     energy: equal to the reference up to the Newton tolerance squared
                                     where inversions converge; it does not reproduce the reference's
                                     inversion fallbacks (dilute edges) */
#define VAH_FLUX_PER_CELL_FUSED 2 /* reference face semantics in one fused launch per stage (no face
                                     scratch; fewer launches, lower occupancy) */

/* ---- field ids (order of the reference's CONSERVED_VARIABLES, DynamicalVariables.h:47-75) ---- */
#define VAH_F_TTT 0
#define VAH_F_TTX 1
#define VAH_F_TTY 2
#define VAH_F_TTN 3
#define VAH_F_PL 4
#define VAH_F_PITT 5
#define VAH_F_PITX 6
#define VAH_F_PITY 7
#define VAH_F_PITN 8
#define VAH_F_PIXX 9
#define VAH_F_PIXY 10
#define VAH_F_PIXN 11
#define VAH_F_PIYY 12
#define VAH_F_PIYN 13
#define VAH_F_PINN 14
#define VAH_F_PI 15
#define VAH_F_E 16
#define VAH_F_P 17
#define VAH_F_UT 18
#define VAH_F_UX 19
#define VAH_F_UY 20
#define VAH_F_UN 21
#define VAH_F_UPT 22 /* u at the previous time step ("up", DynamicalVariables.h:120) */
#define VAH_F_UPX 23
#define VAH_F_UPY 24
#define VAH_F_UPN 25
#define VAH_NUM_FIELDS 26

/* ---- EoS table layout ---- */
#define VAH_EOS_TABLE_N 4096
#define VAH_EOS_TABLE_HEADER 8
#define VAH_EOS_TABLE_LEN(n) (VAH_EOS_TABLE_HEADER + 3 * (size_t)(n))

/* Lattice (rhic/include/LatticeParameters.h:17-31; ghost counts implied). */
typedef struct vah_lattice {
    int nx, ny, nz;
    double dx, dy, dz;
} vah_lattice;

/* Hydro parameters (rhic/include/HydroParameters.h:15-21). */
typedef struct vah_hydro {
    double t0;                 /* initialProperTimePoint */
    double eta_over_s;         /* shearViscosityToEntropyDensity */
    double freezeout_T_GeV;    /* freezeoutTemperatureGeV */
} vah_hydro;

typedef struct vah_options {
    int physics;    /* VAH_IDEAL / VAH_PIMUNU / VAH_PIMUNU_PI */
    int eos;        /* VAH_EOS_* */
    int zeta;       /* VAH_ZETA_* */
    int precision;  /* VAH_FP64 / VAH_FP32 */
    int flux;       /* VAH_FLUX_* */
    int device;     /* CUDA device ordinal */
    void *stream;   /* cudaStream_t to queue work on; NULL = library-owned stream */
} vah_options;

typedef struct vah_stats {
    long long face_fallbacks; /* face inversions that took the fallback, since the event was created */
    long long cell_fallbacks; /* cell inversions that took the fallback, since the event was created */
    long long nan_cells;      /* cells where a NaN reached e or u, since the event was created */
    long long steps;          /* steps taken since creation */
} vah_stats;

typedef struct vah_event vah_event;

/* Fill `out` (length VAH_EOS_TABLE_LEN(n)) with the tabulated crossover EoS:
 * n nodes uniform in ln e, each holding p, T, c_s^2 (T in fm^-1, e and p in
 * fm^-4). c_s^2(T) = 1/3 - (1/3 - 0.15)/(1 + (T/155 MeV)^4). No reference
 * counterpart (the reference ships closed-form fits only,
 * EquationOfState.cpp:31-201). */
int vah_eos_table_build(int n, double *out, size_t out_len);

/* Create an event: allocate its device state and bind physics options.
 * Replaces allocateHostMemory/allocateDeviceMemory + the parameter structs
 * (DynamicalVariables.cpp:33-196, DynamicalVariables.cu:202-392). eos_table
 * is copied (VAH_EOS_TABLE only; may be NULL otherwise). */
int vah_event_create(const vah_lattice *lat, const vah_hydro *hydro, const vah_options *opt,
                     const double *eos_table, vah_event **out);
int vah_event_destroy(vah_event *ev);

/* Copy one field between host memory and the event (reference layout;
 * with_ghosts = 1: full nc* array, 0: interior nx*ny*nz only). Replaces the
 * host<->device copies of DynamicalVariables.cu:394-482. On 2+1D lattices the
 * steps leave the eta ghost layers (no stencil reads them); a read with
 * ghosts first fills them with the eta pass of the reference's ghost fill
 * (setGhostCellsKernelK), as vah_batch_get_field and vah_rk2_step_host do. */
int vah_event_set_field(vah_event *ev, int field, const double *host, int with_ghosts);
int vah_event_get_field(vah_event *ev, int field, double *host, int with_ghosts);

/* Primitives currently in the event (e, p, u, pi^{tau mu}, Pi and, if
 * pl_from_field, P_L) -> conserved T^{tau mu}, P_L; up = u.
 * setConservedVariables, DynamicalVariables.cpp:197-287 (pl_from_field = 0
 * keeps its hard-coded P_L = 0.0154483 e). */
int vah_event_set_conserved(vah_event *ev, double t, int pl_from_field);

/* Initial state from an energy density (the reference's init sequence
 * setInitialConditions -> setConservedVariables -> setGhostCells,
 * HydroPlugin.cpp:184-190): e given on the interior (nx*ny*nz, x fastest),
 * p = EoS(e), u = (1,0,0,0), pi^{mu nu} = 0, Pi = 0 (InitialConditions.cpp:
 * 29-52, 122-162), P_L by pl_mode, up = u, then conserved variables and
 * ghost layers. */
#define VAH_PL_REFERENCE 0 /* P_L = 0.0154483 e (DynamicalVariables.cpp:246-248) */
#define VAH_PL_ISOTROPIC 1 /* P_L = p */
int vah_event_init_from_e(vah_event *ev, double t0, const double *e_interior, int pl_mode);

/* Zero-gradient ghost layers (faces) of the current state:
 * setGhostCells, DynamicalVariables.cpp:349-356. */
int vah_event_set_ghost_cells(vah_event *ev);

/* One Heun RK2 step from t with step dt followed by the q <-> Q swap:
 * rungeKutta2 + setCurrentConservedVariables
 * (FullyDiscreteKurganovTadmorScheme.cpp:738-792, DynamicalVariables.cpp:497-499;
 * CUDA: twoStepRungeKutta, FullyDiscreteKurganovTadmorScheme.cu:121-157). */
int vah_rk2_step(vah_event *ev, double t, double dt);

/* nsteps steps from t0 (t_n = t0 + n dt, HydroPlugin.cpp:208-233). */
int vah_run(vah_event *ev, double t0, double dt, int nsteps);

/* Block until the event's queued work is done; reports VAH_ERR_NAN if a
 * step produced a NaN. */
int vah_event_sync(vah_event *ev);
int vah_event_stats(vah_event *ev, vah_stats *out);

/* Which cells took the inversion fallback: vah_event_track_fallbacks(ev, 1)
 * allocates two bytes per ghosted cell and makes every following step record,
 * per cell, whether the cell inversion of stage 1 and of stage 2 fell back to
 * the reference's e = 0.999 e_prev, u = (1,0,0,0) (EnergyMomentumTensor.cpp:
 * 163-172): the fTSolution flags setInferredVariablesKernel writes
 * (EnergyMomentumTensor.cpp:199-268, :255-257); 0 frees them.
 * vah_event_get_fallback_mask copies the flags of the latest step's stage
 * (1 or 2) as bytes (1 = fell back), full ghosted array or interior only. */
int vah_event_track_fallbacks(vah_event *ev, int on);
int vah_event_get_fallback_mask(vah_event *ev, int stage, unsigned char *host, int with_ghosts);

/* Device time (ms) of the stage kernels launched since the last call, and
 * how many launches; enabled by vah_event_set_timing(ev, 1). */
int vah_event_set_timing(vah_event *ev, int on);
int vah_event_kernel_time(vah_event *ev, double *ms, long long *launches);

/* ---- validity diagnostics (HydrodynamicValidity.cpp:47-394) ----
 * The reference computes these at the end of every step
 * (FullyDiscreteKurganovTadmorScheme.cpp:791) from the conserved state at the
 * start of the step, the new e, p, u and the previous u, and the regulator
 * stores its factors (:652-693); nothing in the step reads them, and its
 * outputs of them are commented out (HydroPlugin.cpp:48-105). Here they are
 * off by default. vah_event_set_validity(ev, 1) allocates 27 FP64 fields (and
 * a copy of P_L, pi, Pi taken at the start of each step) and makes every
 * following vah_rk2_step fill them: the regulator maps from the stage-2 cell
 * launch, the rest from one launch after it. Interior cells only; ghost cells
 * read 0. Ids, with the reference's file names in brackets: */
enum {
    VAH_V_KN_TAUPI_T = 0,  /* knudsenNumberTaupiT [knTaupiT]: 5 etabar |theta_T| / T */
    VAH_V_KN_TAUPI_L = 1,  /* knudsenNumberTaupiL [knTaupiL]: 5 etabar |z.D.u| / T */
    VAH_V_KN_TAUPI = 2,    /* knudsenNumberTaupi [knTaupi] */
    VAH_V_KN_TAUPI_BULK = 3, /* knudsenNumberTauPi [knTauPi] (shear + bulk) */
    VAH_V_RPI = 4,         /* Rpi [Rpi]: sqrt|pi.pi| / |P_T hat| */
    VAH_V_RPI_BULK = 5,    /* RPi [RPi]: |Pi| / |P_T hat| (shear + bulk) */
    VAH_V_RPI2 = 6,        /* Rpi2 [Rpi2]: second-order inverse Reynolds number */
    VAH_V_RPI2_BULK = 7,   /* RPi2 [RPi2] (shear + bulk) */
    VAH_V_TAUPI = 8,       /* taupi [taupi] = 5 etabar / T */
    VAH_V_DXUX = 9,        /* dxux [dxux] */
    VAH_V_DYUY = 10,       /* dyuy [dyuy] */
    VAH_V_THETA = 11,      /* theta [theta] = theta_T + z.D.u */
    VAH_V_STT = 12,        /* stt [stt]: the combinations the reference stores last (:197-200) */
    VAH_V_SXX = 13,        /* sxx [sxx] */
    VAH_V_SYY = 14,        /* syy [syy] */
    VAH_V_SNN = 15,        /* snn [snn] */
    VAH_V_REGULATIONS = 16, /* regulations [regulations]: the factor tanh(rho)/rho applied to pi */
    VAH_V_REG_MAG = 17,    /* regMag, regTr, regU0..regU3, regZ0..regZ3: each criterion's own factor */
    VAH_V_REG_TR = 18,
    VAH_V_REG_U0 = 19,
    VAH_V_REG_Z0 = 23,
    VAH_NUM_VALIDITY = 27
};
int vah_event_set_validity(vah_event *ev, int on);
int vah_event_get_validity(vah_event *ev, int id, double *host, int with_ghosts);

/* ---- launch autotuning (no reference counterpart) ----
 * The face/cell kernels come in register-cap variants and take their block
 * shape at run time. vah_event_autotune times every candidate of each launch
 * kind (face x, face y, face z, cell; `reps` timed launches each, after one
 * warm-up) on the event's current state, keeps the fastest for the event's
 * later steps, and reports the choice and its time next to the default's.
 * It writes only stage scratch (the state is unchanged) and synchronises the
 * event's stream. Results do not depend on the choice. The fused flux mode has
 * nothing to tune (nkinds = 0). vah_batch_autotune does the same for a
 * batch's persistent launches (register cap only; tiles stay 32 x 4). */
typedef struct vah_launch_choice {
    int bx, by, minb;   /* block shape and minimum resident blocks per SM the compiler was held to */
    double ms_default;  /* ms per launch of the configuration in use before the call */
    double ms_best;     /* ms per launch of the chosen configuration */
} vah_launch_choice;
typedef struct vah_tune_report {
    int nkinds;
    vah_launch_choice kind[5];
} vah_tune_report;
int vah_event_autotune(vah_event *ev, int reps, vah_tune_report *out);

/* Host-buffer form of the reference CPU step: the caller's host arrays (the
 * reference's process globals q, e, p, u, up; fields ordered by VAH_F_*,
 * full ghosted layout) are copied in, stepped once on the GPU, and copied
 * back. Drop-in for rungeKutta2 on host arrays
 * (FullyDiscreteKurganovTadmorScheme.h:13-15). `fields` holds
 * VAH_NUM_FIELDS pointers; unused physics slots may be NULL. With FP32
 * storage the arrays still cross as FP64 and are narrowed (widened on the
 * way back) by a kernel, through device staging in the host layout that the
 * first such call allocates (one field; every field where the copies
 * overlap).
 * FP64 storage, face/cell split, validity off and nz >= 6: the copies
 * overlap the stages. The lattice is cut into slabs of planes along eta
 * (VAH_HOST_SLAB_PLANES planes each when that environment variable is set to
 * 2 or more, else nz / 6); copy-in of later slabs, the stages of earlier ones
 * and copy-out of finished ones run on three streams (the event's stream and
 * two the first such call creates), with the same results bit for bit.
 * FP32 storage, 3+1D, validity off: the same, in slabs of whole 4-plane tile
 * layers (the thickness above rounded to layers), where that gives at least
 * 3 slabs. The arrays should be pinned (cudaHostAlloc / cudaHostRegister)
 * for the copies to overlap; pageable arrays give the same results, more
 * slowly. */
int vah_rk2_step_host(vah_event *ev, double t, double dt, double *const *fields);

/* ---- batches: many events of uneven size in one launch per kernel kind ----
 * No single reference counterpart: the reference advances one event per
 * process (HydroPlugin.cpp:130-242). A batch keeps every admitted event's
 * state device-resident and advances all of them together: each launch walks
 * a work-list of 32x4-cell tiles over all events in a grid-stride loop, and
 * one RK2 step of the whole batch (face and cell launches of both stages and
 * the per-event clock advance) is replayed from a CUDA graph that is
 * re-captured only when events are added or removed. Every event keeps its
 * own time and dt; all share the batch's physics options (VAH_FLUX_PER_CELL
 * or VAH_FLUX_SHARED). Admission is by device footprint: vah_batch_add
 * returns VAH_ERR_FULL when the event would exceed capacity_bytes. */
typedef struct vah_batch vah_batch;

typedef struct vah_event_info {
    double t;                 /* current proper time */
    long long steps;          /* steps taken */
    long long face_fallbacks; /* inversion fallbacks at faces since admission */
    long long cell_fallbacks;
    long long nan_cells;
    long long bytes;          /* device footprint of the event */
} vah_event_info;

int vah_batch_create(const vah_options *opt, const double *eos_table, size_t capacity_bytes, vah_batch **out);
int vah_batch_destroy(vah_batch *b);
/* Device bytes an event of this lattice occupies in the batch. */
int vah_batch_event_bytes(const vah_batch *b, const vah_lattice *lat, size_t *bytes);
/* Admit an event: e on the interior (nx*ny*nz, x fastest) at hydro->t0, its
 * own step dt; the vah_event_init_from_e initial state. */
int vah_batch_add(vah_batch *b, const vah_lattice *lat, const vah_hydro *hydro, double dt, const double *e_interior,
                  int pl_mode, int *slot);
int vah_batch_remove(vah_batch *b, int slot);
/* An event whose initial energy density is generated on the device (no
 * reference counterpart; the reference builds ICs on the host,
 * InitialConditions.cpp:196-292): the MC-Glauber collision of
 * vah_ic_mc_glauber, computed on the GPU (one block samples both nuclei with
 * the host sampler's random streams and keeps the participants in its order;
 * a grid deposits their Gaussians), e(x, y, eta) = e_peak v(x,y) / max v *
 * f(eta) + e_floor with f vah_ic_longitudinal's profile (1 in 2+1D); then as
 * vah_batch_add. Positions and e agree with the host generator to rounding
 * (the GPU's exp, sin, cos). VAH_ERR_ARG unless 1 <= A <= 256, ws_R > 0, ws_a > 0
 * (finite) and width > 0; also when the rejection sampler runs out of draws
 * (4 million per nucleus, for parameters it cannot sample). */
typedef struct vah_glauber {
    double b, sigma_nn_fm2;
    int A;
    double ws_R, ws_a, width;
    unsigned long long seed;
    double e_peak, e_floor;
    double eta_flat, sigma_eta;
} vah_glauber;
int vah_batch_add_glauber(vah_batch *b, const vah_lattice *lat, const vah_hydro *hydro, double dt,
                          const vah_glauber *g, int pl_mode, int *slot);
/* The same MC-Glauber initial state generated on the device straight into an
 * event (vah_event_init_from_e with the generated e; nothing crosses to or
 * from the host). */
int vah_event_init_glauber(vah_event *ev, double t0, const vah_glauber *g, int pl_mode);
/* The optical Glauber profile of vah_ic_optical_glauber, generated on the
 * device into an event: the Woods-Saxon thickness table by Simpson in z (a
 * thread per radius, 2048 radii), its normalisation to A nucleons, then
 * (1 - x_coll) N_part/2 + x_coll N_coll per transverse cell, e = e_peak v /
 * max v * f(eta) + e_floor with f as above. Where no nucleon pair overlaps
 * (max v = 0) the event holds the flat floor e_floor (the host generator
 * returns VAH_ERR_ARG there). */
typedef struct vah_optical {
    double b, sigma_nn_fm2;
    int A;
    double ws_R, ws_a, x_coll;
    double e_peak, e_floor;
    double eta_flat, sigma_eta;
} vah_optical;
int vah_event_init_optical_glauber(vah_event *ev, double t0, const vah_optical *o, int pl_mode);
/* nsteps RK2 steps of every admitted event (asynchronous). */
int vah_batch_step(vah_batch *b, int nsteps);
int vah_batch_sync(vah_batch *b);
int vah_batch_event_info(vah_batch *b, int slot, vah_event_info *out);
int vah_batch_get_field(vah_batch *b, int slot, int field, double *host, int with_ghosts);
/* Per-slot maximum energy density over the interior cells whose latest
 * inversion converged (the freeze-out test: max T < T_f with T monotone in
 * e; a cell in the reference's inversion fallback holds e = 0.999 e_prev,
 * not a solution, and is left out); out[s] = 0 for free slots. FP64,
 * deterministic. */
int vah_batch_max_energy_density(vah_batch *b, double *out, int nslots);
/* Per-slot observables in FP64 with a fixed summation order (an event's
 * values do not depend on the other events in the batch), over the interior
 * cells whose latest inversion converged: out[3 s + 0] =
 * sum tau T^{tau tau} dx dy deta, out[3 s + 1] = eps_p =
 * sum(T^xx - T^yy)/sum(T^xx + T^yy), out[3 s + 2] = <u_T> = sum e u^tau u_T /
 * sum e u^tau. */
int vah_batch_observables(vah_batch *b, double *out, int nslots);
/* Per-slot freeze-out surface volume so far (fm^4; no reference counterpart,
 * the reference reads freezeoutTemperatureGeV but never uses it,
 * HydroPlugin.cpp:154-158): at the end of every step each cell whose
 * inversion converged and whose e fell through e(T_f) adds tau dx dy deta at
 * the new time, and each that rose through it subtracts the same, so a surface
 * swept once counts once (a cell in the fallback keeps its state). Crossings
 * are integer counts, so the value is deterministic. T_f is the event's
 * vah_hydro.freezeout_T_GeV. out[s] = 0 for free slots. */
int vah_batch_freezeout_volume(vah_batch *b, double *out, int nslots);
/* Interior cells (nx*ny*nz, x fastest) whose latest inversion fell back to
 * the reference's e = 0.999 e_prev, u = (1,0,0,0): 1, else 0. */
int vah_batch_fallback_mask(vah_batch *b, int slot, unsigned char *host);
int vah_batch_set_timing(vah_batch *b, int on);
int vah_batch_kernel_time(vah_batch *b, double *ms, long long *steps);
/* Register-cap autotuning of the batch's launch kinds (face x, y, z, cell
 * 2+1D, cell 3+1D), as vah_event_autotune describes. */
int vah_batch_autotune(vah_batch *b, int reps, vah_tune_report *out);

/* ---- serving: continuous batching of an open-loop request stream ----
 * No reference counterpart (the reference runs one event per process). A
 * seeded Poisson stream of requests (rate per second for duration_s; a
 * fraction frac_3d are 3+1D with side and nz interpolated between the given
 * bounds, the rest 2+1D with side uniform in [side2_min, side2_max]; impact
 * parameter uniform in [0, b_max]; MC-Glauber initial conditions with peak
 * temperature T0_GeV, built on ic_threads host threads at arrival) is served
 * from one vah_batch: requests are admitted in arrival order while the batch
 * has room (capacity_bytes), all resident events advance together in chunks
 * of chunk_steps graph-replayed steps, and an event retires when its maximum
 * temperature falls below Tf_GeV (FP64 device reduction after each chunk) or
 * its time passes t_max (counted in timeouts, not in the latency
 * statistics). Latency = arrival to retirement at freeze-out, wall clock. latencies (optional) receives up to max_latencies
 * values in completion order. */
typedef struct vah_serve_config {
    double rate, duration_s;
    unsigned long long seed;
    double frac_3d;
    int side2_min, side2_max, side3_min, side3_max, nz3_min, nz3_max;
    double dx, deta, b_max;
    double t0, dt, eta_over_s, T0_GeV, Tf_GeV, t_max;
    int physics, eos, precision, flux, device;
    size_t capacity_bytes;
    int chunk_steps, ic_threads;
    double e_floor;  /* energy density added to every initial cell, fm^-4 (the reference adds 1e-3) */
    int ic_on_device; /* 1: admission generates each IC on the GPU (vah_batch_add_glauber); 0: host threads build it */
} vah_serve_config;

typedef struct vah_serve_result {
    long long offered, completed, timeouts, rejected;
    double wall_s, events_per_s, p50_s, p99_s;
    long long cell_updates;
    double cell_updates_per_s;
    long long max_resident, chunks;
    long long failed;       /* events retired because a NaN reached e or u (also in timeouts) */
    double tau_freeze_max;  /* largest event time at freeze-out, fm/c */
} vah_serve_result;

int vah_serve_run(const vah_serve_config *cfg, vah_serve_result *res, double *latencies, int max_latencies);

/* ---- initial energy-density generators (host, deterministic) ----
 * Replace the reference's GSL/libc-rand generators (GlauberModel.cpp:19-108,
 * MonteCarloGlauberModel.cpp:17-108, InitialConditions.cpp:196-292) with the
 * workloads' own definitions. Transverse profiles are nx*ny, x fastest,
 * centred like the reference grid (x_i = (i - (nx-1)/2) dx); each is scaled so
 * its maximum is e_peak, then e_floor is added. */
int vah_ic_optical_glauber(int nx, int ny, double dx, double dy, double b, double sigma_nn_fm2, int A,
                           double ws_R, double ws_a, double x_coll, double e_peak, double e_floor, double *e_xy);
int vah_ic_mc_glauber(int nx, int ny, double dx, double dy, double b, double sigma_nn_fm2, int A, double ws_R,
                      double ws_a, double width, unsigned long long seed, double e_peak, double e_floor,
                      double *e_xy, int *npart_out);
/* The participant positions of vah_ic_mc_glauber's collision (x, y pairs in
 * xy, at most `max`; *n_out is their number, VAH_ERR_TOO_LARGE if above max). */
int vah_ic_mc_glauber_participants(double b, double sigma_nn_fm2, int A, double ws_R, double ws_a,
                                   unsigned long long seed, double *xy, int max, int *n_out);
/* f(eta) = 1 for |eta| < eta_flat, exp(-(|eta|-eta_flat)^2 / (2 sigma_eta^2)) beyond. */
int vah_ic_longitudinal(int nz, double dz, double eta_flat, double sigma_eta, double *f_eta);

/* ---- one RK stage without allocation ----
 * No counterpart in the reference: an entry point for callers that cannot
 * allocate device memory (code inside a framework that owns all device memory
 * through its own pool, work queued where cudaMalloc is not allowed or would
 * synchronise the device, processes whose device footprint must stay fixed).
 * It runs one RK stage -- the face/cell launches with the reference's face
 * semantics, FP64 storage -- on state buffers the caller owns, and keeps the
 * stage's scratch (face fluxes, fallback counters) in a fixed array of
 * VAH_NOALLOC_SCRATCH_BYTES inside the library, held by every GPU that loads
 * libvah.so until exit. It calls no allocator. Limit: 256 +
 * (2 or 3 axes) * N_q * 2 * 8 bytes per ghosted cell must fit, i.e. at most
 * 87,381 ghosted cells for a 3+1D grid with shear + bulk (N_q = 16) and
 * 131,071 for a 2+1D one; larger grids return VAH_ERR_TOO_LARGE.
 * The first call on a device looks up the array's device address (do it
 * before any stream capture); the address is cached per device and context,
 * so the first call after a cudaDeviceReset looks it up again (and should
 * also come before any capture). Calls share the array: calls whose work
 * overlaps on the GPU race on it. Stage 1 then stage 2 with the buffer roles
 * of vah_rk2_step make one time step. The conformal temperature is the
 * correctly rounded fourth root here (the host-libm correction table of the
 * event path needs device memory), so with the conformal EoS the stage
 * departs from the reference at the rounding of the temperature (a few
 * 1e-10 relative on the shear stress after one step on the tested grid). counts_out (host, 3 entries: face
 * fallbacks, cell fallbacks, NaN cells; may be NULL) makes the call wait for
 * the stage and returns VAH_ERR_NAN when a NaN reached e or u. */
#define VAH_NOALLOC_SCRATCH_BYTES (64u << 20)

typedef struct vah_stage_buffers {
    const double *q[16];     /* stage input conserved fields (VAH_F_* order; stage 1: q^n, stage 2: q*) */
    const double *u[4];      /* stage input velocity (stage 1: u^n, stage 2: u*) */
    const double *u_prev[4]; /* previous-stage velocity (stage 1: u^(n-1), stage 2: u^n); Newton guess in stage 2 */
    const double *e, *p;     /* stage input e, p */
    const double *q_avg[16]; /* stage 2: q^n for Q = (q^n + Q*)/2 (may alias q_out); unused in stage 1 */
    double *q_out[16];       /* stage output conserved fields (interior and face ghost layers) */
    double *u_out[4];
    double *e_out, *p_out;
} vah_stage_buffers;

int vah_stage_noalloc(const vah_lattice *lat, double eta_over_s, int physics, int eos, int zeta,
                      const double *d_eos_table, int stage, double t, double dt, const vah_stage_buffers *buf,
                      void *stream, long long *counts_out);

/* Accuracy check of the step's two hand-written device operations: the
 * Newton correction's reciprocal (hardware estimate + one Newton-Raphson
 * step) and 1/sqrt (hardware estimate + two steps), against CUDA's
 * IEEE-rounded reciprocal and square root, on n log-spaced inputs in
 * [lo, hi] (alternating sign for the reciprocal). Writes the largest relative
 * errors (0 where both results are equal, infinities included). Outside
 * |x| in [2^-1000, 2^1001) the Newton correction divides in IEEE arithmetic;
 * 1/sqrt is checked on [2^-1000, 2^1000] only (its callers pass values >= 1).
 * No counterpart in the reference, which divides and takes square roots in
 * IEEE arithmetic on the CPU. */
int vah_math_check(int device, double lo, double hi, int n, double *max_rel_rcp, double *max_rel_rsqrt);

/* FP64 FMA throughput of the device, measured: a persistent grid
 * (8 blocks of 256 threads per SM) in which each thread runs 8 independent
 * chains of dependent fused multiply-adds; best of 5 launches. *tflops =
 * 2 x FMAs / time, *ms the launch's duration. No counterpart in the
 * reference; the benchmark reports the step's FP64 throughput against it. */
int vah_fp64_peak(int device, double *tflops, double *ms);

/* Library version string. */
const char *vah_version(void);

#ifdef __cplusplus
}
#endif
#endif
