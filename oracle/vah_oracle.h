/*
 * oracle/vah_oracle.h -- test infrastructure: the CPU checker's API.
 *
 * A plain-C restatement of the reference CPU time step
 * (old_cpu-vah_code/src, driven as rhic/src/HydroPlugin.cpp:208-233 drives the
 * GPU build). Only tests, the smoke check and the CPU-baseline leg of the
 * benchmark load it; the product never does.
 *
 * Physics variants are chosen at run time instead of the reference's macros:
 *   VO_IDEAL      N_q = 5  (no PIMUNU, no PI: the CPU header's default)
 *   VO_PIMUNU     N_q = 15 (-DPIMUNU)
 *   VO_PIMUNU_PI  N_q = 16 (-DPIMUNU -DPI)
 * W^mu_{perp z} (W_TZ_MU) is off in every reference build and not restated.
 *
 * Arrays use the reference layout: field[i + ncx*(j + ncy*k)] with
 * nc = n + 4 (2 ghost layers per side), DynamicalVariables.cpp:29-31.
 */
#ifndef VAH_ORACLE_H
#define VAH_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { VO_IDEAL = 0, VO_PIMUNU = 1, VO_PIMUNU_PI = 2 };
enum { VO_EOS_CONFORMAL = 0, VO_EOS_TABLE = 1 };
enum { VO_ZETA_REFERENCE = 0, VO_ZETA_CROSSOVER = 1 };

typedef struct {
    int nx, ny, nz;
    double dx, dy, dz;
    double etabar;            /* eta/s */
    int physics;              /* VO_IDEAL / VO_PIMUNU / VO_PIMUNU_PI */
    int eos;                  /* VO_EOS_* */
    int zeta;                 /* VO_ZETA_* */
    const double *eos_table;  /* VO_EOS_TABLE only; layout in vo_eos.h */
} vo_config;

typedef struct vo_state vo_state;

vo_state *vo_create(const vo_config *cfg);
void vo_destroy(vo_state *st);
int vo_num_cells(const vo_state *st);      /* ncx*ncy*ncz */
double *vo_field(vo_state *st, int id);    /* ids as include/vah.h VAH_F_* */
void vo_set_conserved(vo_state *st, double t, int pl_from_field);
void vo_set_ghost_cells(vo_state *st);
void vo_step(vo_state *st, double t, double dt);
double vo_run(vo_state *st, double t0, double dt, int nsteps);
/* counts of inversion fallbacks / NaNs seen during the last step:
 * out[0] face (flux) fallbacks, out[1] cell fallbacks, out[2] NaNs */
void vo_last_step_stats(const vo_state *st, long long out[3]);
/* out[d]: the face fallbacks of the last step along axis d (x, y, eta). In
 * 2+1D the reference still runs the eta sweep, whose fluxes are exact zeros,
 * and its face inversions count here. */
void vo_last_step_face_fallbacks(const vo_state *st, long long out[3]);
/* per ghosted cell, 1 where the cell inversion of stage 1 or 2 of the last
 * step took the reference's fallback (EnergyMomentumTensor.cpp:163-172),
 * else 0; stage outside {1, 2}: NULL */
const unsigned char *vo_fallback_mask(const vo_state *st, int stage);

/* Validity diagnostics (HydrodynamicValidity.cpp:47-394, computed at the end
 * of every step, FullyDiscreteKurganovTadmorScheme.cpp:791) and the regulator
 * maps (same file :652-693), in the order of include/vah.h's VAH_V_* ids.
 * Off until vo_set_validity(st, 1); arrays are ncx*ncy*ncz, interior written. */
#define VO_NUM_VALIDITY 27
void vo_set_validity(vo_state *st, int on);
double *vo_validity_field(vo_state *st, int id);

/* Single-cell operators, for unit tests of the library's pieces. */
int vo_infer(const vo_config *cfg, double t, const double *q, double ePrev, double uT0,
             double *out /* e, p, ut, ux, uy, un */);
double vo_approx_derivative(double qm, double q, double qp);
void vo_eos_eval(const vo_config *cfg, double e, double *out /* p, T, cs2 */);

/* The benchmark workloads' inputs (vo_inputs.c): the tabulated crossover
 * EoS (layout of include/vah.h: n, ln e_0, 1/d ln e, d ln e, e_0, ln e_{n-1},
 * e_{n-1}, 0, then p[n], T[n], c_s^2[n]), a seeded MC-Glauber transverse
 * profile (nx*ny, x fastest) and the longitudinal plateau + Gaussian f(eta).
 * Return 0, or -1 on a bad argument. */
int vo_eos_table_build(int n, double *out, size_t out_len);
int vo_ic_mc_glauber(int nx, int ny, double dx, double dy, double b, double sigma_nn_fm2, int A, double ws_R,
                     double ws_a, double width, unsigned long long seed, double e_peak, double e_floor, double *e_xy,
                     int *npart_out);
int vo_ic_longitudinal(int nz, double dz, double eta_flat, double sigma_eta, double *f_eta);

#ifdef __cplusplus
}
#endif
#endif
