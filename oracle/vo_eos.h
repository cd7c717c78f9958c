/*
 * oracle/vo_eos.h -- test infrastructure (CPU checker), never linked into the
 * product.
 *
 * Equation-of-state and bulk-viscosity closures used by the CPU checkers:
 *   - the reference's conformal EoS, restated with its quirks
 *     (rhic/src/EquationOfState.cpp:31-146 with CONFORMAL_EOS defined,
 *     EquationOfState.h:13-17): p = e/3, c_s^2 = `1/3` evaluated as integer
 *     division (= 0, EquationOfState.cpp:113), T = powf(e/13.8997, 0.25)
 *     in single precision (EquationOfState.cpp:144);
 *   - the reference's zeta/s(T) (SourceTerms.cpp:36-44);
 *   - the tabulated crossover EoS lookup and the crossover zeta/s of the
 *     3+1D workloads. Neither exists in the reference: both are inputs of the
 *     workload definition. The table itself is produced by the library's
 *     table builder and handed to every checker as data; only the lookup rule
 *     (linear interpolation in ln e, power-law continuation outside the table)
 *     is restated here.
 *
 * Table layout (shared with the product, see include/vah.h VAH_EOS_TABLE_*):
 *   tab[0] = n, tab[1] = ln e_0, tab[2] = 1/d(ln e), tab[3] = d(ln e),
 *   tab[4] = e_0, tab[5] = ln e_{n-1}, tab[6] = e_{n-1}, tab[7] = 0,
 *   then p[n], T[n], cs2[n].
 */
#ifndef VO_EOS_H
#define VO_EOS_H

#include <math.h>

#define VO_EOS_HEADER 8
#define VO_HBARC 0.197326938
#define VO_EOS_FACTOR 13.8997

/* EquationOfState.cpp:78 (conformal branch). */
static inline double vo_conf_pressure(double e) { return e / 3; }
/* EquationOfState.cpp:113: `return 1/3;` is integer division, i.e. 0. */
static inline double vo_conf_cs2(double e) { (void)e; return 0.0; }
/* EquationOfState.cpp:144: powf on the float-converted ratio. */
static inline double vo_conf_temperature(double e) {
    return (double)powf((float)(e / VO_EOS_FACTOR), 0.25f);
}

/* SourceTerms.cpp:22-44: the reference zeta/s(T), T in fm^-1. */
static inline double vo_zeta_reference(double T) {
    double x = T / 1.01355;
    if (x > 1.05)
        return 0.9 * exp(-(x - 1) / 0.025) + 0.25 * exp(-(x - 1) / 0.13) + 0.001;
    else if (x < 0.995)
        return 0.9 * exp((x - 1) / 0.0025) + 0.22 * exp((x - 1) / 0.022) + 0.03;
    else
        return -13.77 * x * x + 27.55 * x - 13.45;
}

/* Crossover zeta/s of the 3+1D workloads: a Lorentzian of height 0.05 at
 * T = 155 MeV and half-width 50 MeV (T in fm^-1). Workload definition, no
 * reference counterpart. */
static inline double vo_zeta_crossover(double T) {
    const double tp = 0.155 / VO_HBARC;
    const double w = 0.050 / VO_HBARC;
    double d = (T - tp) / w;
    return 0.05 / (1.0 + d * d);
}

typedef struct {
    double p, T, cs2;
} vo_eos_point;

/* Table lookup: linear interpolation in x = ln e between nodes; below the
 * first node p/e and c_s^2 are frozen and T ~ e^(3/23) (the c_s^2 = 0.15
 * limit of the crossover); above the last node p/e and c_s^2 are frozen and
 * T ~ e^(1/4). */
static inline vo_eos_point vo_table_lookup(const double *tab, double e) {
    vo_eos_point r;
    int n = (int)tab[0];
    const double *P = tab + VO_EOS_HEADER;
    const double *T = P + n;
    const double *C = T + n;
    double lne0 = tab[1], inv = tab[2];
    if (!(e > 0.0)) {
        r.p = e * (P[0] / tab[4]);
        r.T = 0.0;
        r.cs2 = C[0];
        return r;
    }
    double x = log(e);
    double f = (x - lne0) * inv;
    if (f <= 0.0) {
        r.p = e * (P[0] / tab[4]);
        r.T = T[0] * exp((3.0 / 23.0) * (x - lne0));
        r.cs2 = C[0];
        return r;
    }
    if (f >= (double)(n - 1)) {
        r.p = e * (P[n - 1] / tab[6]);
        r.T = T[n - 1] * exp(0.25 * (x - tab[5]));
        r.cs2 = C[n - 1];
        return r;
    }
    int i = (int)f;
    double w = f - (double)i;
    r.p = P[i] + w * (P[i + 1] - P[i]);
    r.T = T[i] + w * (T[i + 1] - T[i]);
    r.cs2 = C[i] + w * (C[i + 1] - C[i]);
    return r;
}

#endif
