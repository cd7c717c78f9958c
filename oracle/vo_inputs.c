/*
 * oracle/vo_inputs.c -- test infrastructure: the benchmark workloads' inputs,
 * generated on the CPU for the reference arm of the benchmark and for tests.
 *
 * The reference builds its initial conditions with GSL quadrature and libc
 * rand (rhic/src/GlauberModel.cpp:19-108, MonteCarloGlauberModel.cpp:17-108,
 * InitialConditions.cpp:196-292) and ships only closed-form EoS fits
 * (EquationOfState.cpp:31-201). The workloads define their own inputs
 * instead -- a tabulated crossover EoS, a seeded MC-Glauber Au+Au collision
 * and a plateau-plus-Gaussian longitudinal profile -- and these functions
 * state those definitions once more, so that a process timing the
 * reference's own CPU step can build the same event without loading the
 * product library. They follow the same evaluation order as the library's
 * host generators, so the arrays agree bit for bit (checked by
 * tests/test_oracle.py).
 *
 * EoS: c_s^2(T) = 1/3 - D/(1 + (T/Tc)^4), D = 1/3 - 0.15, Tc = 155 MeV;
 * s(T) = s_inf tau^3 (tau^4/(tau^4 + a))^(9D/(4a)), tau = T/Tc, a = 1 - 3D,
 * s_inf = (4/3) 13.8997 Tc^3 (the reference's conformal gas, EquationOfState.h:16);
 * p(T) = int s dT (Simpson on ln T pieces of a 2^17-point grid from 1 MeV to
 * 10 GeV, starting from the c_s^2 = 0.15 power law p = 3 T s / 23), e = T s - p;
 * n nodes uniform in ln e between T = 5 MeV and 5 GeV, each holding p, T, c_s^2.
 *
 * MC-Glauber: A nucleons per nucleus from Woods-Saxon (R, a) by rejection
 * sampling of r^2 rho(r) on [0, R + 10 a] with a splitmix64 stream per
 * nucleus (seeds 2 seed + 0x1234567 and 2 seed + 1 + 0x1234567), isotropic
 * directions, nuclei displaced by +-b/2 along x; a nucleon participates when
 * one of the other nucleus lies within sqrt(sigma_NN / pi) transversely; each
 * participant deposits exp(-r^2 / (2 w^2)) within r < 8 w; the sum is scaled
 * to e_peak at its maximum and e_floor is added.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "vah_oracle.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#define VO_HBARC 0.197326938
#define VO_EOS_FACTOR 13.8997

static const double kDelta = 1.0 / 3.0 - 0.15;

static double vo_cs2_of(double T) {
    const double Tc = 0.155 / VO_HBARC;
    double tau = T / Tc;
    double t4 = tau * tau * tau * tau;
    return 1.0 / 3.0 - kDelta / (1.0 + t4);
}

static double vo_s_of(double T) {
    const double kA = 1.0 - 3.0 * kDelta;
    const double expo = 9.0 * kDelta / (4.0 * kA);
    const double Tc = 0.155 / VO_HBARC;
    const double sinf = 4.0 / 3.0 * VO_EOS_FACTOR * Tc * Tc * Tc;
    double tau = T / Tc;
    double t4 = tau * tau * tau * tau;
    return sinf * tau * tau * tau * pow(t4 / (t4 + kA), expo);
}

/* int_{T0}^{T1} s dT, Simpson on ln T over one short interval */
static double vo_simpson_piece(double T0, double T1) {
    double l0 = log(T0), l1 = log(T1), lm = 0.5 * (l0 + l1);
    double Tm = exp(lm);
    return (l1 - l0) / 6.0 * (vo_s_of(T0) * T0 + 4.0 * vo_s_of(Tm) * Tm + vo_s_of(T1) * T1);
}

typedef struct {
    int M;
    double lt0, h;
    double *Tf, *pf, *ef;
} vo_fine;

static double vo_e_at(const vo_fine *g, int k, double T, double *p_out) {
    double p = g->pf[k] + vo_simpson_piece(g->Tf[k], T);
    *p_out = p;
    return T * vo_s_of(T) - p;
}

/* T (and p) where e(T) = e_target: bracketing fine-grid interval, an
 * interpolated start and four Newton steps with de/dT = s / c_s^2 */
static double vo_solve_T(const vo_fine *g, double e_target, double *p_out) {
    int lo = 0, hi = g->M;
    while (hi - lo > 1) {
        int mid = (lo + hi) / 2;
        if (g->ef[mid] <= e_target) lo = mid; else hi = mid;
    }
    double w = (log(e_target) - log(g->ef[lo])) / (log(g->ef[lo + 1]) - log(g->ef[lo]));
    double T = exp(log(g->Tf[lo]) + w * g->h);
    double p = 0.0;
    for (int it = 0; it < 4; ++it) {
        double e = vo_e_at(g, lo, T, &p);
        double dedT = vo_s_of(T) / vo_cs2_of(T);
        T -= (e - e_target) / dedT;
    }
    vo_e_at(g, lo, T, &p);
    *p_out = p;
    return T;
}

int vo_eos_table_build(int n, double *out, size_t out_len) {
    if (n < 16 || !out || out_len < (size_t)(8 + 3 * n)) return -1;
    vo_fine g;
    g.M = 1 << 17;
    g.lt0 = log(0.001 / VO_HBARC);
    const double lt1 = log(10.0 / VO_HBARC);
    g.h = (lt1 - g.lt0) / g.M;
    g.Tf = (double *)malloc((g.M + 1) * sizeof(double));
    g.pf = (double *)malloc((g.M + 1) * sizeof(double));
    g.ef = (double *)malloc((g.M + 1) * sizeof(double));
    if (!g.Tf || !g.pf || !g.ef) {
        free(g.Tf); free(g.pf); free(g.ef);
        return -1;
    }
    for (int k = 0; k <= g.M; ++k) g.Tf[k] = exp(g.lt0 + g.h * k);
    g.pf[0] = 3.0 * g.Tf[0] * vo_s_of(g.Tf[0]) / 23.0;
    for (int k = 0; k < g.M; ++k) g.pf[k + 1] = g.pf[k] + vo_simpson_piece(g.Tf[k], g.Tf[k + 1]);
    for (int k = 0; k <= g.M; ++k) g.ef[k] = g.Tf[k] * vo_s_of(g.Tf[k]) - g.pf[k];

    double ends[2], pend;
    const double Tends[2] = {0.005 / VO_HBARC, 5.0 / VO_HBARC};
    for (int b = 0; b < 2; ++b) {
        int k = (int)floor((log(Tends[b]) - g.lt0) / g.h);
        if (k < 0) k = 0;
        if (k >= g.M) k = g.M - 1;
        ends[b] = log(vo_e_at(&g, k, Tends[b], &pend));
    }
    const double lne0 = ends[0], dl = (ends[1] - ends[0]) / (n - 1);
    double *P = out + 8, *T = P + n, *C = T + n;
    for (int i = 0; i < n; ++i) {
        double et = exp(lne0 + dl * i), p;
        double Ti = vo_solve_T(&g, et, &p);
        P[i] = p;
        T[i] = Ti;
        C[i] = vo_cs2_of(Ti);
    }
    out[0] = (double)n;
    out[1] = lne0;
    out[2] = 1.0 / dl;
    out[3] = dl;
    out[4] = exp(lne0);
    out[5] = lne0 + dl * (n - 1);
    out[6] = exp(out[5]);
    out[7] = 0.0;
    free(g.Tf); free(g.pf); free(g.ef);
    return 0;
}

/* splitmix64 */
static uint64_t vo_next(uint64_t *s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static double vo_uniform(uint64_t *s) { return (double)(vo_next(s) >> 11) * (1.0 / 9007199254740992.0); }

static void vo_sample_nucleus(uint64_t *rng, int A, double R, double a, double xshift, double *x, double *y) {
    const double rmax = R + 10 * a;
    for (int n = 0; n < A; ++n) {
        double r;
        for (;;) {
            r = rmax * vo_uniform(rng);
            const double f = (r * r / (rmax * rmax)) / (1 + exp((r - R) / a));
            if (vo_uniform(rng) < f) break;
        }
        const double cth = 2 * vo_uniform(rng) - 1, phi = 2 * M_PI * vo_uniform(rng);
        const double sth = sqrt(1 - cth * cth);
        x[n] = r * sth * cos(phi) + xshift;
        y[n] = r * sth * sin(phi);
    }
}

int vo_ic_mc_glauber(int nx, int ny, double dx, double dy, double b, double sigma_nn_fm2, int A, double ws_R,
                     double ws_a, double width, unsigned long long seed, double e_peak, double e_floor, double *e_xy,
                     int *npart_out) {
    if (nx < 1 || ny < 1 || !e_xy || !(width > 0) || A < 1) return -1;
    double *xa = malloc(A * sizeof(double)), *ya = malloc(A * sizeof(double));
    double *xb = malloc(A * sizeof(double)), *yb = malloc(A * sizeof(double));
    double *px = malloc(2 * A * sizeof(double)), *py = malloc(2 * A * sizeof(double));
    char *pa = calloc(A, 1), *pb = calloc(A, 1);
    int rc = 0;
    if (!xa || !ya || !xb || !yb || !px || !py || !pa || !pb) {
        rc = -1;
        goto done;
    }
    uint64_t ra = seed * 2 + 0x1234567ull, rb = seed * 2 + 1 + 0x1234567ull;
    vo_sample_nucleus(&ra, A, ws_R, ws_a, +b / 2, xa, ya);
    vo_sample_nucleus(&rb, A, ws_R, ws_a, -b / 2, xb, yb);
    const double d2max = sigma_nn_fm2 / M_PI;
    for (int m = 0; m < A; ++m)
        for (int k = 0; k < A; ++k) {
            const double ddx = xa[m] - xb[k], ddy = ya[m] - yb[k];
            if (ddx * ddx + ddy * ddy < d2max) pa[m] = pb[k] = 1;
        }
    int np = 0;
    for (int m = 0; m < A; ++m)
        if (pa[m]) { px[np] = xa[m]; py[np] = ya[m]; ++np; }
    for (int k = 0; k < A; ++k)
        if (pb[k]) { px[np] = xb[k]; py[np] = yb[k]; ++np; }
    if (npart_out) *npart_out = np;
    const double inv2w2 = 1.0 / (2 * width * width), cut2 = 64 * width * width;
    double emax = 0;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const double x = (i - (nx - 1) / 2.) * dx, y = (j - (ny - 1) / 2.) * dy;
            double v = 0;
            for (int p = 0; p < np; ++p) {
                const double r2 = (x - px[p]) * (x - px[p]) + (y - py[p]) * (y - py[p]);
                if (r2 < cut2) v += exp(-r2 * inv2w2);
            }
            e_xy[i + (size_t)nx * j] = v;
            if (v > emax) emax = v;
        }
    if (!(emax > 0)) {
        for (size_t s = 0; s < (size_t)nx * ny; ++s) e_xy[s] = e_floor;
    } else {
        for (size_t s = 0; s < (size_t)nx * ny; ++s) e_xy[s] = e_peak * e_xy[s] / emax + e_floor;
    }
done:
    free(xa); free(ya); free(xb); free(yb); free(px); free(py); free(pa); free(pb);
    return rc;
}

int vo_ic_longitudinal(int nz, double dz, double eta_flat, double sigma_eta, double *f_eta) {
    if (nz < 1 || !f_eta || !(sigma_eta > 0)) return -1;
    for (int k = 0; k < nz; ++k) {
        const double eta = (k - (nz - 1) / 2.) * dz;
        const double d = fabs(eta) - eta_flat;
        f_eta[k] = d > 0 ? exp(-d * d / (2 * sigma_eta * sigma_eta)) : 1.0;
    }
    return 0;
}
