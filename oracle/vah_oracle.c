/*
 * oracle/vah_oracle.c -- test infrastructure: CPU restatement of the reference
 * time step. Loaded only by tests, the smoke check and the benchmark's
 * CPU-baseline leg (as the checker); never linked into the product.
 *
 * Parity is pinned two ways (tests/test_oracle_*.py): bit-for-bit against the
 * reference's own CPU sources compiled into oracle/_ref (oracle/Makefile), and
 * against the 0+1D conformal Bjorken ODE of python/conformal_bjorken_test.py.
 *
 * Every expression keeps the reference's evaluation order (the last bit
 * depends on it); terms carrying W^mu_{perp z} are dropped because W_TZ_MU
 * is undefined in every reference build (DynamicalVariables.h:14), so those
 * terms are exact zeros added to or subtracted from finite values.
 * Compile with -ffp-contract=off (oracle/Makefile does).
 */
#define _POSIX_C_SOURCE 199309L
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "vah_oracle.h"
#include "vo_closures.h"
#include "vo_eos.h"

#define NQ_MAX 16
#define SLOT_PL 4
#define SLOT_PI 15

struct vo_state {
    vo_config cfg;
    int ncx, ncy, ncz, len, nq;
    double *q[NQ_MAX], *Q[NQ_MAX], *qS[NQ_MAX];
    double *e, *p;
    double *u[4], *up[4], *uS[4];
    long long face_fail, cell_fail, nan_count;
    long long face_fail_axis[3];  /* face_fail split by flux direction */
    unsigned char *fallback[2];  /* per cell, 1 where stage 1 / stage 2's inversion fell back (last step) */
    int validity_on;
    double *vd[VO_NUM_VALIDITY];
};

static int nq_of(int physics) {
    return physics == VO_IDEAL ? 5 : (physics == VO_PIMUNU ? 15 : 16);
}
static int has_pimunu(const vo_config *c) { return c->physics != VO_IDEAL; }
static int has_bulk(const vo_config *c) { return c->physics == VO_PIMUNU_PI; }

/* ------------------------------------------------------------------ EoS -- */
static double eos_p(const vo_config *c, double e) {
    return c->eos == VO_EOS_TABLE ? vo_table_lookup(c->eos_table, e).p : vo_conf_pressure(e);
}
static double eos_T(const vo_config *c, double e) {
    return c->eos == VO_EOS_TABLE ? vo_table_lookup(c->eos_table, e).T : vo_conf_temperature(e);
}
static double eos_cs2(const vo_config *c, double e) {
    return c->eos == VO_EOS_TABLE ? vo_table_lookup(c->eos_table, e).cs2 : vo_conf_cs2(e);
}
static double zeta_over_s(const vo_config *c, double T) {
    return c->zeta == VO_ZETA_CROSSOVER ? vo_zeta_crossover(T) : vo_zeta_reference(T);
}

void vo_eos_eval(const vo_config *cfg, double e, double *out) {
    out[0] = eos_p(cfg, e);
    out[1] = eos_T(cfg, e);
    out[2] = eos_cs2(cfg, e);
}

/* --------------------------------------------------- anisotropic closures -- */
/* a^0 .. a^15 built by repeated multiplication (SourceTerms.cpp:435-449). */
static void powers(double a, double *ap) {
    ap[0] = 1.0;
    ap[1] = a;
    for (int k = 2; k < 16; ++k) ap[k] = ap[k - 1] * a;
}

/* AnisotropicDistributionFunctions.cpp:5-24. */
static double pt_hat(double e, double p, double pl) {
    double ap[16];
    powers(pl / e, ap);
    double rbar0 = VO_RATIO(Rbar0, ap);
    return (e - pl - rbar0 * (e - 3 * p)) / 2;
}

typedef struct {
    double beta_lPi, delta_lPi, lambda_piPi, beta_PiPi, delta_PiPi, lambda_Pipi;
} second_order;

/* AnisotropicDistributionFunctions.cpp:73-190, with the reference's integer
 * divisions kept: 2/9 -> 0 (:93), 3/2 -> 1 (:185), 3/4 -> 0 (:186),
 * 1/3 -> 0 (:189). */
static second_order second_order_z(double e, double p, double pl, double cs2, const double *ap) {
    second_order r;
    double third_minus_cs2 = 1.0 / 3.0 - cs2;
    if (third_minus_cs2 == 0.0) third_minus_cs2 = 1.e-16;
    double meq2 = 36 * third_minus_cs2;
    double z2logz = -2 * (1 - (0.0 * (e - 3 * p)) / (third_minus_cs2 * (e + p)) + 0.02536 * meq2);

    double m2g0m2000 = VO_RATIO(m2g0m2000Z2LogZTerm, ap) * z2logz + VO_RATIO(m2g0m2000Z2Term, ap) * meq2;
    double g0m2040_c = VO_RATIO(g0m2040DividedBym2ConstantTerm, ap);
    double g0m2040_zm2 = VO_RATIO(g0m2040DividedBym2Zm2Term, ap);
    double g0m2040_log = VO_RATIO(g0m2040DividedBym2LogZTerm, ap);
    double g0m2040 = (g0m2040_log * z2logz + g0m2040_zm2) / meq2 + g0m2040_c;
    double g0m2020_c = VO_RATIO(g0m2020ConstantTerm, ap);
    double g0m2020_z2 = VO_RATIO(g0m2020Z2Term, ap);
    double g0m2020_log = VO_RATIO(g0m2020Z2LogZTerm, ap);
    double g0m2020 = g0m2020_c + g0m2020_log * z2logz + g0m2020_z2 * meq2;
    double gg1 = VO_RATIO(G_G1, ap);

    r.beta_lPi = 3 * g0m2040;
    r.delta_lPi = 1 * (g0m2020 + g0m2040);
    r.lambda_piPi = 0 * (m2g0m2000 + 2 * (g0m2020 + 1) + g0m2040);
    r.beta_PiPi = 1 - g0m2020_c;
    r.delta_PiPi = 0.5 * (1 + g0m2020_c);
    r.lambda_Pipi = 3 * gg1 / 5 * (0 - cs2);
    return r;
}

/* ------------------------------------------------------------- limiter -- */
/* FluxLimiter.cpp:15-33 (theta = 1.1, sign(0) = +1). */
static double sgn(double x) { return x < 0.0 ? -1.0 : 1.0; }
static double minmod2(double x, double y) { return (sgn(x) + sgn(y)) * fmin(fabs(x), fabs(y)) / 2; }

double vo_approx_derivative(double x, double y, double z) {
    double l = 1.1 * (y - x);
    double c = (z - x) / 2;
    double r = 1.1 * (z - y);
    return minmod2(l, minmod2(c, r));
}

/* ------------------------------------------------------------ inversion -- */
/* EnergyMomentumTensor.cpp:30-72: Newton for u_T, relative tolerance 1e-7,
 * at most 10^4 iterations. The equilibrium pressure evaluated inside the
 * reference loop is unused there and is not recomputed. */
static int newton_ut(double t, double ut_guess, double mb0, double mbt, double mb3, double pl,
                     double bulk, double ft, double x, double *ut_out) {
    double w = ut_guess;
    double ft2 = ft * ft;
    double bT = x * mbt;
    double bL = x * x * mb0 - ft2 * pl;
    double b = x * x + ft2;
    for (int it = 0; it < 10000; ++it) {
        double e = mb0 - t * ft * mb3 - w / sqrt(1 + w * w) * x * mbt;
        if (e < 0.0) return -1;
        double pt = 0.5 * (e - pl) + 1.5 * bulk;
        double de_dw = -x * mbt / pow(1 + w * w, 1.5);
        double dpt_dw = 0.5 * de_dw;
        double f = w / sqrt(1 + w * w) * (bL + b * pt) - bT;
        double fp = 1 / pow(1 + w * w, 1.5) * (bL + b * pt) + w / sqrt(1 + w * w) * b * dpt_dw;
        if (fabs(fp) == 0.0) fp = 1.e-16;
        double next = w - f / fp;
        *ut_out = next;
        if (isnan(next) || isinf(next) || next < 0 || next > 9.0072e+15) return -1;
        if (fabs(next - w) <= 1.e-7 * fabs(next)) return 0;
        w = next;
    }
    return -1;
}

/* EnergyMomentumTensor.cpp:74-197. Returns 0 (converged), -1 (fallback
 * e = 0.999 ePrev, u = (1,0,0,0)) or 2 (a NaN reached e or u; the reference
 * prints and exits there). */
int vo_infer(const vo_config *cfg, double t, const double *q, double ePrev, double uT0, double *out) {
    double ttt = q[0], ttx = q[1], tty = q[2], ttn = q[3], pl = q[SLOT_PL];
    double pitt = 0, pitx = 0, pity = 0, pitn = 0, bulk = 0;
    if (has_pimunu(cfg)) { pitt = q[5]; pitx = q[6]; pity = q[7]; pitn = q[8]; }
    if (has_bulk(cfg)) bulk = q[SLOT_PI];
    const double w0 = 0.0; /* W^mu_{perp z} components (off) */

    double m0 = ttt - pitt, m1 = ttx - pitx, m2 = tty - pity, m3 = ttn - pitn;
    double m0pl = m0 + pl;
    if (m0pl == 0.0) m0pl = 1.e-16;
    double A = m3 / m0pl;
    double At = t * A;
    double B = w0 / m0pl / t;
    double Bt = t * B;
    double At2 = At * At, Bt2 = Bt * Bt;
    double F = (A - fabs(B) * sqrt(fabs(1 - At2 + Bt2))) / (1 + Bt2);
    double Ft = t * F;
    double Ft2 = Ft * Ft;
    double x = sqrt(fabs(1. - Ft2));
    double mb0 = m0 - 2 * w0 * Ft / x;
    double mb1 = m1 - w0 * Ft / x;
    double mb2 = m2 - w0 * Ft / x;
    double mb3 = m3 - (1 + Ft2) * w0 / t / x;
    double mbt = sqrt(mb1 * mb1 + mb2 * mb2);
    if (mbt == 0.0) mbt = 1.e-16;

    double uT;
    int status = newton_ut(t, uT0, mb0, mbt, mb3, pl, bulk, Ft, x, &uT);
    double e, p, ut, ux, uy, un;
    if (status == 0) {
        double C = sqrt(1.0 + pow(uT, 2.));
        double U = uT / C;
        ux = uT * mb1 / mbt;
        uy = uT * mb2 / mbt;
        un = F * C / x;
        ut = C / x;
        e = mb0 - t * Ft * mb3 - U * x * mbt;
        p = eos_p(cfg, e);
    } else {
        e = ePrev * .999;
        p = eos_p(cfg, e);
        ux = 0.0; uy = 0.0; un = 0.0; ut = 1.0;
    }
    out[0] = e; out[1] = p; out[2] = ut; out[3] = ux; out[4] = uy; out[5] = un;
    if (isnan(e) || isnan(ut) || isnan(ux) || isnan(uy) || isnan(un)) return 2;
    return status;
}

/* --------------------------------------------------------- face fluxes -- */
/* Stencil along one axis: sten[n][m], m = 0..4 <-> offsets -2..+2. */
typedef double stencil_t[NQ_MAX][5];

enum { DIR_X = 0, DIR_Y = 1, DIR_Z = 2 };

/* SemiDiscreteKurganovTadmorScheme.cpp:13-57 with HalfSiteExtrapolation.cpp:
 * 12-26, SpectralRadius.cpp:14-24, LocalPropagationSpeed.cpp:14-22 and
 * FluxFunctions.cpp:15-25. fwd = face at +1/2, else face at -1/2.
 * Returns 0, or the number of the two inversions that fell back. */
static int face_flux(vo_state *st, double t, const stencil_t s, int dir, int fwd, double ePrev,
                     double uT, double *H) {
    const vo_config *c = &st->cfg;
    int nq = st->nq;
    double qR[NQ_MAX] = {0}, qL[NQ_MAX] = {0};
    for (int n = 0; n < nq; ++n) {
        double qmm = s[n][0], qm = s[n][1], q0 = s[n][2], qp = s[n][3], qpp = s[n][4];
        if (fwd) {
            qR[n] = qp - vo_approx_derivative(q0, qp, qpp) / 2;
            qL[n] = q0 + vo_approx_derivative(qm, q0, qp) / 2;
        } else {
            qR[n] = q0 - vo_approx_derivative(qm, q0, qp) / 2;
            qL[n] = qm + vo_approx_derivative(qmm, qm, q0) / 2;
        }
    }
    double vR[6], vL[6];
    int sR = vo_infer(c, t, qR, ePrev, uT, vR);
    int sL = vo_infer(c, t, qL, ePrev, uT, vL);
    if (sR == 2 || sL == 2) st->nan_count++;
    /* velocity component along the axis: ux, uy or un -> out[3 + dir] */
    double udR = vR[3 + dir], udL = vL[3 + dir];
    double a = fmax(fabs(udL / vL[2]), fabs(udR / vR[2]));
    for (int n = 0; n < nq; ++n) {
        double fR = udR * qR[n] / vR[2];
        double fL = udL * qL[n] / vL[2];
        double res = fR + fL - a * (qR[n] - qL[n]);
        res /= 2;
        H[n] = res;
    }
    return (sR != 0) + (sL != 0);
}

/* ------------------------------------------------------------- sources -- */
typedef struct {
    const double *const *cur; /* conserved fields of the stage input */
    double *const *u;         /* velocity of the stage input */
    const double *e, *p;
} stage_in;

/* SourceTerms.cpp:46-176: the pi/Pi gradient terms of the T^{tau mu}
 * equations along one axis, from the same 5-point stencil as the fluxes. */
static void axis_sources(const vo_state *st, const stencil_t s, int dir, double ucomp, double ut,
                         double h, double t, double *S) {
    int pi_on = has_bulk(&st->cfg);
    double fac = 1 / h / 2;
#define D(slot) ((s[slot][3] - s[slot][1]) * fac)
    double v = ucomp / ut;
    if (dir == DIR_X) {
        double d_tt = D(5), d_tx = D(6), d_ty = D(7), d_tn = D(8), d_xx = D(9), d_xy = D(10), d_xn = D(11);
        if (!pi_on) {
            S[0] = d_tt * v - d_tx;
            S[1] = d_tx * v - d_xx;
        } else {
            double dPi = D(SLOT_PI);
            dPi *= 1.5;
            S[0] = d_tt * v - d_tx - v * dPi;
            S[1] = d_tx * v - d_xx - dPi;
        }
        S[2] = d_ty * v - d_xy;
        S[3] = d_tn * v - d_xn;
    } else if (dir == DIR_Y) {
        double d_tt = D(5), d_tx = D(6), d_ty = D(7), d_tn = D(8), d_xy = D(10), d_yy = D(12), d_yn = D(13);
        if (!pi_on) {
            S[0] = d_tt * v - d_ty;
            S[2] = d_ty * v - d_yy;
        } else {
            double dPi = D(SLOT_PI);
            dPi *= 1.5;
            S[0] = d_tt * v - d_ty - v * dPi;
            S[2] = d_ty * v - d_yy - dPi;
        }
        S[1] = d_tx * v - d_xy;
        S[3] = d_tn * v - d_yn;
    } else {
        double d_tt = D(5), d_tx = D(6), d_ty = D(7), d_tn = D(8), d_xn = D(11), d_yn = D(13), d_nn = D(14);
        if (!pi_on) {
            S[0] = d_tt * v - d_tn;
            S[3] = d_tn * v - d_nn;
        } else {
            double dPi = D(SLOT_PI);
            dPi *= 1.5;
            S[0] = d_tt * v - d_tn - v * dPi;
            /* SourceTerms.cpp:172: powf, i.e. t^2 in single precision */
            S[3] = d_tn * v - d_nn - dPi / (double)powf((float)t, 2.0f);
        }
        S[1] = d_tx * v - d_xn;
        S[2] = d_ty * v - d_yn;
    }
#undef D
}

/* SourceTerms.cpp:178-1044: geometric and relaxation sources at one interior
 * cell s. Q = conserved values at s (stage input), (utp..unp) = velocity of
 * the previous stage at s. */
static int cell_sources(const vo_state *st, const stage_in *in, const double *Q, double utp,
                        double uxp, double uyp, double unp, double t, int s, double dt, double *S) {
    const vo_config *c = &st->cfg;
    const int pimunu = has_pimunu(c), bulkon = has_bulk(c);
    const int sx = 1, sy = st->ncx, sz = st->ncx * st->ncy;

    double ttt = Q[0], ttx = Q[1], tty = Q[2], ttn = Q[3], pl = Q[4];
    double pitt = 0, pitx = 0, pity = 0, pitn = 0, pixx = 0, pixy = 0, pixn = 0, piyy = 0, piyn = 0,
           pinn = 0, Pi = 0;
    if (pimunu) {
        pitt = Q[5]; pitx = Q[6]; pity = Q[7]; pitn = Q[8]; pixx = Q[9];
        pixy = Q[10]; pixn = Q[11]; piyy = Q[12]; piyn = Q[13]; pinn = Q[14];
    }
    if (bulkon) Pi = Q[SLOT_PI];

    const double *UT = in->u[0], *UX = in->u[1], *UY = in->u[2], *UN = in->u[3];
    const double *ev = in->e, *pv = in->p, *plv = in->cur[SLOT_PL];
    double e = ev[s], p = pv[s];
    double ut = UT[s], ux = UX[s], uy = UY[s], un = UN[s];

    double facX = 1 / c->dx / 2, facY = 1 / c->dy / 2, facZ = 1 / c->dz / 2;
#define CD(arr, off, fac) (((arr)[s + (off)] - (arr)[s - (off)]) * (fac))
    double dxut = CD(UT, sx, facX), dxux = CD(UX, sx, facX), dxuy = CD(UY, sx, facX), dxun = CD(UN, sx, facX);
    double dyut = CD(UT, sy, facY), dyux = CD(UX, sy, facY), dyuy = CD(UY, sy, facY), dyun = CD(UN, sy, facY);
    double dnut = CD(UT, sz, facZ), dnux = CD(UX, sz, facZ), dnuy = CD(UY, sz, facZ), dnun = CD(UN, sz, facZ);
    double dxp = CD(pv, sx, facX), dyp = CD(pv, sy, facY), dnp = CD(pv, sz, facZ);
    double dxe = CD(ev, sx, facX), dye = CD(ev, sy, facY), dne = CD(ev, sz, facZ);

    double vx = ux / ut, vy = uy / ut, vn = un / ut;
    double dxvx = (dxux - vx * dxut) / ut;
    double dyvy = (dyuy - vy * dyut) / ut;
    double dnvn = (dnun - vn * dnut) / ut;
    double dkvk = dxvx + dyvy + dnvn;

    double t2 = t * t, t3 = t * t2, un2 = un * un, ut2 = ut * ut;

    /* velocity gradients (SourceTerms.cpp:301-334) */
    double dtut = (ut - utp) / dt, dtux = (ux - uxp) / dt, dtuy = (uy - uyp) / dt, dtun = (un - unp) / dt;
    double Dut = ut * dtut + ux * dxut + uy * dyut + un * dnut + t * un * un;
    double Dux = -(ut * dtux + ux * dxux + uy * dyux + un * dnux);
    double Duy = -(ut * dtuy + ux * dxuy + uy * dyuy + un * dnuy);
    double Dun = -t2 * (ut * dtun + ux * dxun + uy * dyun + un * dnun + 2 * ut * un / t);
    double dut = Dut - t * un * un;
    double dux = ut * dtux + ux * dxux + uy * dyux + un * dnux;
    double duy = ut * dtuy + ux * dxuy + uy * dyuy + un * dnuy;
    double dun = ut * dtun + ux * dxun + uy * dyun + un * dnun;
    double theta = ut / t + dtut + dxux + dyuy + dnun;

    double stt = -t * ut * un2 + (dtut - ut * dut) + (ut2 - 1) * theta / 3;
    double stx = -(t * un2 * ux) / 2 + (dtux - dxut) / 2 - (ux * dut + ut * dux) / 2 + ut * ux * theta / 3;
    double sty = -(t * un2 * uy) / 2 + (dtuy - dyut) / 2 - (uy * dut + ut * duy) / 2 + ut * uy * theta / 3;
    double stn = -un * (2 * ut2 + t2 * un2) / (2 * t) + (dtun - dnut / t2) / 2 - (un * dut + ut * dun) / 2 +
                 ut * un * theta / 3;
    double sxx = -(dxux + ux * dux) + (1 + ux * ux) * theta / 3;
    double sxy = -(dxuy + dyux) / 2 - (uy * dux + ux * duy) / 2 + ux * uy * theta / 3;
    double sxn = -ut * ux * un / t - (dxun + dnux / t2) / 2 - (un * dux + ux * dun) / 2 + ux * un * theta / 3;
    double syy = -(dyuy + uy * duy) + (1 + uy * uy) * theta / 3;
    double syn = -ut * uy * un / t - (dyun + dnuy / t2) / 2 - (un * duy + uy * dun) / 2 + uy * un * theta / 3;
    double snn = -ut * (1 + 2 * t2 * un2) / t3 - dnun / t2 - un * dun + (1 / t2 + un2) * theta / 3;

    /* transverse / longitudinal split (SourceTerms.cpp:355-426) */
    double uT2 = ux * ux + uy * uy;
    double uTdtuT = (ux * dtux + uy * dtuy);
    double uTdxuT = (ux * dxux + uy * dxuy);
    double uTdyuT = (ux * dyux + uy * dyuy);
    double uTdnuT = (ux * dnux + uy * dnuy);
    double uTduT = ut * uTdtuT + ux * uTdxuT + uy * uTdyuT + un * uTdnuT;
    double F = 1 + uT2;
    double F2 = F * F;
    double z0 = t * un / sqrt(F);
    double z3 = ut / t / sqrt(F);
    double z02 = z0 * z0, z0z3 = z0 * z3, z32 = z3 * z3;
    double dz0 = (ut * un + t * dun - t * un / F * uTduT) / sqrt(F);
    double dz3 = (-ut2 / t2 + dut / t - ut / t / F * uTduT) / sqrt(F);
    double Dz0 = dz0 + t * un * z3;
    double Dz3 = -t2 * (dz3 + (ut * z3 + un * z0) / t);
    double A = z02 * stt - 2 * t2 * z0z3 * stn + t2 * t2 * z32 * snn;
    double B0 = z0 * stt - t2 * z3 * stn;
    double B1 = z0 * stx - t2 * z3 * sxn;
    double B2 = z0 * sty - t2 * z3 * syn;
    double B3 = z0 * stn - t2 * z3 * snn;
    double thetaT = 2 * theta / 3 + A;
    double zDzu = theta - thetaT;
    double sttT = stt + 2 * z0 * B0 + z02 * A - 0.5 * (1 - ut * ut + z02) * A;
    double stxT = stx + z0 * B1 - 0.5 * (-ut * ux) * A;
    double styT = sty + z0 * B2 - 0.5 * (-ut * uy) * A;
    double stnT = stn + z0 * B3 + z3 * B0 + z0z3 * A - 0.5 * (-ut * un + z0z3) * A;
    double sxxT = sxx - 0.5 * (-1 - ux * ux) * A;
    double sxyT = sxy - 0.5 * (-ux * uy) * A;
    double sxnT = sxn + z3 * B1 - 0.5 * (-ux * un) * A;
    double syyT = syy - 0.5 * (-1 - uy * uy) * A;
    double synT = syn + z3 * B2 - 0.5 * (-uy * un) * A;
    double snnT = snn + 2 * z3 * B3 + z32 * A - 0.5 * (-1 / t2 - un * un + z32) * A;

    /* closures (SourceTerms.cpp:431-481) */
    if (e == 0) e = 1.e-7;
    double T = eos_T(c, e);
    double cs2 = eos_cs2(c, e);
    double ap[16];
    powers(pl / e, ap);
    double a = ap[1];
    double Rtilde = VO_RATIO(Rtilde, ap);
    double Rhat = VO_RATIO(Rhat, ap);
    double Rbar0 = VO_RATIO(Rbar0, ap);
    double Rgamma = VO_RATIO(Rgamma, ap);
    double Rbar0P = VO_RATIO(Rbar0P, ap);
    double R0g1m2031 = VO_RATIO(R0g1m2031, ap);

    double dxpl = CD(plv, sx, facX), dypl = CD(plv, sy, facY), dnpl = CD(plv, sz, facZ);
#undef CD

    double ptHat = pt_hat(e, p, pl);
    double pt = ptHat + 1.5 * Pi;
    double DP = pl - pt;
    double Ltt = DP * t2 * un2 / F;
    double Ltn = DP * ut * un / F;
    double Lnn = DP * ut2 / F / t2;

    double tnn = (e + pt) * un * un + pt / t2 + Lnn + pinn;

    double dxRbar0 = Rbar0P * (dxpl - a * dxe) / e;
    double dyRbar0 = Rbar0P * (dypl - a * dye) / e;
    double dnRbar0 = Rbar0P * (dnpl - a * dne) / e;
    double dxptHat = 0.5 * (dxe - dxpl - Rbar0 * (dxe - 3 * dxp) - (e - 3 * p) * dxRbar0);
    double dyptHat = 0.5 * (dye - dypl - Rbar0 * (dye - 3 * dyp) - (e - 3 * p) * dyRbar0);
    double dnptHat = 0.5 * (dne - dnpl - Rbar0 * (dne - 3 * dnp) - (e - 3 * p) * dnRbar0);
    double dxDP = dxpl - dxptHat, dyDP = dypl - dyptHat, dnDP = dnpl - dnptHat;

    double dxLtt = (2 * DP * dxun * t2 * un) / F + (dxDP * t2 * un2) / F - (2 * DP * uTdxuT * t2 * un2) / F2;
    double dyLtt = (2 * DP * dyun * t2 * un) / F + (dyDP * t2 * un2) / F - (2 * DP * uTdyuT * t2 * un2) / F2;
    double dnLtt = (2 * DP * dnun * t2 * un) / F + (dnDP * t2 * un2) / F - (2 * DP * uTdnuT * t2 * un2) / F2;
    double dxLtn = (DP * dxut * un) / F + (DP * dxun * ut) / F + (dxDP * un * ut) / F - (2 * DP * uTdxuT * un * ut) / F2;
    double dyLtn = (DP * dyut * un) / F + (DP * dyun * ut) / F + (dyDP * un * ut) / F - (2 * DP * uTdyuT * un * ut) / F2;
    double dnLtn = (DP * dnut * un) / F + (DP * dnun * ut) / F + (dnDP * un * ut) / F - (2 * DP * uTdnuT * un * ut) / F2;
    double dnLnn = (2 * DP * dnut * ut) / (F * t2) + (dnDP * ut2) / (F * t2) - (2 * DP * uTdnuT * ut2) / (F2 * t2);

    double zeta_zz = Rtilde * e - 3 * pl;
    double zeta_zT = (Rtilde * e + pl) / 2.;

    second_order so = second_order_z(e, p, pl, cs2, ap);
    double lambda_lpi = Rgamma;
    double delta_pipi = (3 + Rgamma) / 2;
    double tau_pipi = 4 * (delta_pipi - 0) / 3;     /* SourceTerms.cpp:634: 1/2 -> 0 */
    double lambda_pipi = Rgamma - 1;

    double taupiInv = 0.2 * T / c->etabar;

    double psT = pitt * sttT - 2 * pitx * stxT - 2 * pity * styT + pixx * sxxT + 2 * pixy * sxyT + piyy * syyT -
                 2 * pitn * stnT * t2 + 2 * pixn * sxnT * t2 + 2 * piyn * synT * t2 + pinn * snnT * t2 * t2;
    double IL = 0.0 - lambda_lpi * psT;

    double dPL = -(pl - p) * taupiInv + zeta_zz * zDzu - zeta_zT * thetaT - so.beta_lPi * Pi * zDzu -
                 so.delta_lPi * Pi * thetaT + IL;
    S[4] = dPL / ut + dkvk * pl;
    int bad = isnan(S[4]);

    double Htt = Ltt + pitt;
    S[0] = -(ttt / t + t * tnn) + dkvk * (Htt - pt) - vx * dxptHat - vy * dyptHat - vn * dnptHat + vx * dxLtt +
           vy * dyLtt + vn * dnLtt - dnLtn;
    S[1] = -ttx / t - dxptHat + dkvk * pitx;
    S[2] = -tty / t - dyptHat + dkvk * pity;
    /* SourceTerms.cpp:686: the reference writes dnLtn twice */
    S[3] = -3 * ttn / t - dnptHat / t2 + dkvk * (Ltn + pitn) + vx * dxLtn + vy * dyLtn + vn * (dnLtn + dnLtn) - dnLnn;
    bad |= isnan(S[0]);

    double ps = psT;
    if (pimunu) {
        /* SourceTerms.cpp:725-930 (I6/I7 carry W only) */
        double etaBar_TC = ((3 - Rtilde) * e - 2 * pl) / 8;
        double I1Utt = 2 * ut * (pitt * Dut + pitx * Dux + pity * Duy + pitn * Dun);
        double I1Utx = (pitt * ux + pitx * ut) * Dut + (pitx * ux + pixx * ut) * Dux + (pity * ux + pixy * ut) * Duy +
                       (pitn * ux + pixn * ut) * Dun;
        double I1Uty = (pitt * uy + pity * ut) * Dut + (pitx * uy + pixy * ut) * Dux + (pity * uy + piyy * ut) * Duy +
                       (pitn * uy + piyn * ut) * Dun;
        double I1Utn = (pitt * un + pitn * ut) * Dut + (pitx * un + pixn * ut) * Dux + (pity * un + piyn * ut) * Duy +
                       (pitn * un + pinn * ut) * Dun;
        double I1Uxx = 2 * ux * (pitx * Dut + pixx * Dux + pixy * Duy + pixn * Dun);
        double I1Uxy = (pitx * uy + pity * ux) * Dut + (pixx * uy + pixy * ux) * Dux + (pixy * uy + piyy * ux) * Duy +
                       (pixn * uy + piyn * ux) * Dun;
        double I1Uxn = (pitx * un + pitn * ux) * Dut + (pixx * un + pixn * ux) * Dux + (pixy * un + piyn * ux) * Duy +
                       (pixn * un + pinn * ux) * Dun;
        double I1Uyy = 2 * uy * (pity * Dut + pixy * Dux + piyy * Duy + piyn * Dun);
        double I1Uyn = (pity * un + pitn * uy) * Dut + (pixy * un + pixn * uy) * Dux + (piyy * un + piyn * uy) * Duy +
                       (piyn * un + pinn * uy) * Dun;
        double I1Unn = 2 * un * (pitn * Dut + pixn * Dux + piyn * Duy + pinn * Dun);

        double I1Ztt = 2 * z0 * (pitt * Dz0 + pitn * Dz3);
        double I1Ztx = (pitx * z0) * Dz0 + (pitn * ux + pixn * z0) * Dz3;
        double I1Zty = (pity * z0) * Dz0 + (pitn * uy + piyn * z0) * Dz3;
        double I1Ztn = (pitt * z3 + pitn * z0) * Dz0 + (pitn * z3 + pinn * z0) * Dz3;
        double I1Zxn = (pitx * z3) * Dz0 + (pixn * z3) * Dz3;
        double I1Zyn = (pity * z3) * Dz0 + (piyn * z3) * Dz3;
        double I1Znn = 2 * z3 * (pitn * Dz0 + pinn * Dz3);

        double I1tt = I1Utt - I1Ztt, I1tx = I1Utx - I1Ztx, I1ty = I1Uty - I1Zty, I1tn = I1Utn - I1Ztn;
        double I1xx = I1Uxx - 0, I1xy = I1Uxy - 0, I1xn = I1Uxn - I1Zxn, I1yy = I1Uyy - 0;
        double I1yn = I1Uyn - I1Zyn, I1nn = I1Unn - I1Znn;

        double ux2 = ux * ux, uy2 = uy * uy;
        double ps2 = ps / 2;
        double I4tt = (pitt * sttT - pitx * stxT - pity * styT - t2 * pitn * stnT) - (1 - ut2 + z02) * ps2;
        double I4tx = (pitt * stxT + pitx * sttT) / 2 - (pitx * sxxT + pixx * stxT) / 2 - (pity * sxyT + pixy * styT) / 2 -
                      t2 * (pitn * sxnT + pixn * stnT) / 2 + (ut * ux) * ps2;
        double I4ty = (pitt * styT + pity * sttT) / 2 - (pitx * sxyT + pixy * stxT) / 2 - (pity * syyT + piyy * styT) / 2 -
                      t2 * (pitn * synT + piyn * stnT) / 2 + (ut * uy) * ps2;
        double I4tn = (pitt * stnT + pitn * sttT) / 2 - (pitx * sxnT + pixn * stxT) / 2 - (pity * synT + piyn * styT) / 2 -
                      t2 * (pitn * snnT + pinn * stnT) / 2 + (ut * un - z0z3) * ps2;
        double I4xx = (pitx * stxT - pixx * sxxT - pixy * sxyT - t2 * pixn * sxnT) + (1 + ux2) * ps2;
        double I4xy = (pitx * styT + pity * stxT) / 2 - (pixx * sxyT + pixy * sxxT) / 2 - (pixy * syyT + piyy * sxyT) / 2 -
                      t2 * (pixn * synT + piyn * sxnT) / 2 + (ux * uy) * ps2;
        double I4xn = (pitx * stnT + pitn * stxT) / 2 - (pixx * sxnT + pixn * sxxT) / 2 - (pixy * synT + piyn * sxyT) / 2 -
                      t2 * (pixn * snnT + pinn * sxnT) / 2 + (ux * un) * ps2;
        double I4yy = (pity * styT - pixy * sxyT - piyy * syyT - t2 * piyn * synT) + (1 + uy2) * ps2;
        double I4yn = (pity * stnT + pitn * styT) / 2 - (pixy * sxnT + pixn * sxyT) / 2 - (piyy * synT + piyn * syyT) / 2 -
                      t2 * (piyn * snnT + pinn * synT) / 2 + (uy * un) * ps2;
        double I4nn = (pitn * stnT - pixn * sxnT - piyn * synT - t2 * pinn * snnT) + (1 / t2 + un2 - z32) * ps2;

        /* SourceTerms.cpp:899-908: every component subtracts lambda_piPi Pi sttT */
        double lpp = so.lambda_piPi * Pi * sttT;
#define ICOMB(I1, pi, I4) ((I1) - delta_pipi * (thetaT * (pi)) + tau_pipi * (I4) - lambda_pipi * (zDzu * (pi)) - lpp)
        double Itt = ICOMB(I1tt, pitt, I4tt), Itx = ICOMB(I1tx, pitx, I4tx), Ity = ICOMB(I1ty, pity, I4ty);
        double Itn = ICOMB(I1tn, pitn, I4tn), Ixx = ICOMB(I1xx, pixx, I4xx), Ixy = ICOMB(I1xy, pixy, I4xy);
        double Ixn = ICOMB(I1xn, pixn, I4xn), Iyy = ICOMB(I1yy, piyy, I4yy), Iyn = ICOMB(I1yn, piyn, I4yn);
        double Inn = ICOMB(I1nn, pinn, I4nn);
#undef ICOMB
        double dpitt = 2 * etaBar_TC * sttT - pitt * taupiInv - Itt - 2 * un * t * pitn;
        double dpitx = 2 * etaBar_TC * stxT - pitx * taupiInv - Itx - un * t * pixn;
        double dpity = 2 * etaBar_TC * styT - pity * taupiInv - Ity - un * t * piyn;
        double dpitn = 2 * etaBar_TC * stnT - pitn * taupiInv - Itn - un * t * pinn - (ut * pitn + un * pitt) / t;
        double dpixx = 2 * etaBar_TC * sxxT - pixx * taupiInv - Ixx;
        double dpixy = 2 * etaBar_TC * sxyT - pixy * taupiInv - Ixy;
        double dpixn = 2 * etaBar_TC * sxnT - pixn * taupiInv - Ixn - (ut * pixn + un * pitx) / t;
        double dpiyy = 2 * etaBar_TC * syyT - piyy * taupiInv - Iyy;
        double dpiyn = 2 * etaBar_TC * synT - piyn * taupiInv - Iyn - (ut * piyn + un * pity) / t;
        double dpinn = 2 * etaBar_TC * snnT - pinn * taupiInv - Inn - 2 * (ut * pinn + un * pitn) / t;
        S[5] = dpitt / ut + pitt * dkvk;
        S[6] = dpitx / ut + pitx * dkvk;
        S[7] = dpity / ut + pity * dkvk;
        S[8] = dpitn / ut + pitn * dkvk;
        S[9] = dpixx / ut + pixx * dkvk;
        S[10] = dpixy / ut + pixy * dkvk;
        S[11] = dpixn / ut + pixn * dkvk;
        S[12] = dpiyy / ut + piyy * dkvk;
        S[13] = dpiyn / ut + piyn * dkvk;
        S[14] = dpinn / ut + pinn * dkvk;
    }
    if (bulkon) {
        /* SourceTerms.cpp:1030-1042 */
        double b = 1.0 / 3.0 - cs2;
        double b2 = b * b;
        double zetabar = zeta_over_s(c, T);
        double tauPiInv = 15 * b2 * T / zetabar;
        double zeta_z = (Rhat - Rbar0) * (e - 3 * p) / 3;
        double zeta_T = -(Rbar0 + Rhat) * (e - 3 * p) / 6;
        double dPi = -((1 - Rbar0) * (e - 3 * p) / 3 + Pi) * tauPiInv - zeta_z * zDzu - zeta_T * thetaT -
                     so.beta_PiPi * Pi * zDzu - so.delta_PiPi * Pi * thetaT + so.lambda_Pipi * ps;
        S[SLOT_PI] = dPi / ut + Pi * dkvk;
    }
    return bad;
}

/* ------------------------------------------------------------ the step -- */
static int idx(const vo_state *st, int i, int j, int k) { return i + st->ncx * (j + st->ncy * k); }

static void gather(const vo_state *st, const double *const *cur, int s, int stride, stencil_t out) {
    for (int n = 0; n < st->nq; ++n)
        for (int m = 0; m < 5; ++m) out[n][m] = cur[n][s + (m - 2) * stride];
}

/* FullyDiscreteKurganovTadmorScheme.cpp:43-461 fused per cell: the updated
 * value is ((((Q + dt S) + rX) + rY) + rZ), exactly the sequence of the
 * reference's four sweeps at one cell. `up` is the previous velocity. */
static void euler_step(vo_state *st, double t, double dt, double *const *cur, double *const *upd,
                       double *const *u, double *const *up) {
    const vo_config *c = &st->cfg;
    int nq = st->nq, ideal = (c->physics == VO_IDEAL);
    stage_in in = {(const double *const *)cur, u, st->e, st->p};
    double hs[3] = {c->dx, c->dy, c->dz};
    int strides[3] = {1, st->ncx, st->ncx * st->ncy};
    for (int i = 2; i < st->ncx - 2; ++i)
        for (int j = 2; j < st->ncy - 2; ++j)
            for (int k = 2; k < st->ncz - 2; ++k) {
                int s = idx(st, i, j, k);
                double Q[NQ_MAX] = {0}, S[NQ_MAX] = {0}, val[NQ_MAX];
                for (int n = 0; n < nq; ++n) Q[n] = cur[n][s];
                if (cell_sources(st, &in, Q, up[0][s], up[1][s], up[2][s], up[3][s], t, s, dt, S)) st->nan_count++;
                for (int n = 0; n < nq; ++n) val[n] = Q[n] + dt * S[n];
                double uT = sqrt(fabs(u[1][s] * u[1][s] + u[2][s] * u[2][s]));
                for (int dir = 0; dir < 3; ++dir) {
                    stencil_t sten;
                    double Hf[NQ_MAX], Hb[NQ_MAX], Hs[4], r[NQ_MAX];
                    gather(st, (const double *const *)cur, s, strides[dir], sten);
                    const int ff = face_flux(st, t, sten, dir, 1, st->e[s], uT, Hf) +
                                   face_flux(st, t, sten, dir, 0, st->e[s], uT, Hb);
                    st->face_fail += ff;
                    st->face_fail_axis[dir] += ff;
                    for (int n = 0; n < nq; ++n) {
                        r[n] = -Hf[n];
                        r[n] += Hb[n];
                        r[n] /= hs[dir];
                    }
                    if (!ideal) {
                        axis_sources(st, sten, dir, u[1 + dir][s], u[0][s], hs[dir], t, Hs);
                        for (int n = 0; n < 4; ++n) {
                            r[n] += Hs[n];
                            r[n] *= dt;
                        }
                    } else {
                        for (int n = 0; n < 4; ++n) r[n] *= dt;
                    }
                    for (int n = 4; n < nq; ++n) r[n] *= dt;
                    for (int n = 0; n < nq; ++n) val[n] += r[n];
                }
                for (int n = 0; n < nq; ++n) upd[n][s] = val[n];
            }
}

/* EnergyMomentumTensor.cpp:199-268: invert every interior cell of q; the
 * Newton guess is |u_T| of `guess`, e (in place) is the fallback base. */
static void infer_all(vo_state *st, int stage, double t, double *const *q, double *const *guess,
                      double *const *out) {
    for (int i = 2; i < st->ncx - 2; ++i)
        for (int j = 2; j < st->ncy - 2; ++j)
            for (int k = 2; k < st->ncz - 2; ++k) {
                int s = idx(st, i, j, k);
                double qs[NQ_MAX] = {0}, v[6];
                for (int n = 0; n < st->nq; ++n) qs[n] = q[n][s];
                double uT = sqrt(fabs(guess[1][s] * guess[1][s] + guess[2][s] * guess[2][s]));
                int status = vo_infer(&st->cfg, t, qs, st->e[s], uT, v);
                st->fallback[stage][s] = status != 0;
                if (status != 0) st->cell_fail++;
                if (status == 2) st->nan_count++;
                st->e[s] = v[0];
                st->p[s] = v[1];
                for (int m = 0; m < 4; ++m) out[m][s] = v[2 + m];
            }
}

/* FullyDiscreteKurganovTadmorScheme.cpp:524-696: clamp e and P_L, then scale
 * pi^{mu nu} by tanh(rho)/rho (xi0 = 1, rho_max = 1). */
static void regulate(vo_state *st, double t, double *const *q, double *const *u) {
    const int pimunu = has_pimunu(&st->cfg);
    for (int i = 2; i < st->ncx - 2; ++i)
        for (int j = 2; j < st->ncy - 2; ++j)
            for (int k = 2; k < st->ncz - 2; ++k) {
                int s = idx(st, i, j, k);
                if (st->e[s] < 0.0) {
                    st->e[s] = 1.e-7;
                    st->p[s] = 1.e-7;
                }
                if (q[SLOT_PL][s] < 0.0) q[SLOT_PL][s] = 1.e-7;
                if (!pimunu) continue;
                const double xi0 = 1.0, rhomax = 1.0;
                double e_s = st->e[s], pl = q[SLOT_PL][s];
                double ptHat = pt_hat(e_s, st->p[s], pl);
                double pitt = q[5][s], pitx = q[6][s], pity = q[7][s], pitn = q[8][s], pixx = q[9][s];
                double pixy = q[10][s], pixn = q[11][s], piyy = q[12][s], piyn = q[13][s], pinn = q[14][s];
                double ut = u[0][s], ux = u[1][s], uy = u[2][s], un = u[3][s];
                double F = 1 + (ux * ux + uy * uy);
                double z0 = t * un / sqrt(F);
                double z3 = ut / t / sqrt(F);
                double t2 = t * t;
                double TrsTrs = e_s * e_s + pl * pl + 2 * ptHat * ptHat;
                double sTrsTrs = sqrt(fabs(TrsTrs));
                double pipi = pitt * pitt - 2 * pitx * pitx - 2 * pity * pity + pixx * pixx + 2 * pixy * pixy +
                              piyy * piyy - 2 * pitn * pitn * t2 + 2 * pixn * pixn * t2 + 2 * piyn * piyn * t2 +
                              pinn * pinn * t2 * t2;
                double spipi = sqrt(fabs(pipi));
                double cand[10];
                double den = xi0 * rhomax * spipi;
                cand[0] = spipi / rhomax / sTrsTrs;
                cand[1] = (pitt - pixx - piyy - pinn * t * t) / den;
                cand[2] = (-pitn * t2 * un + pitt * ut - pitx * ux - pity * uy) / den;
                cand[3] = (-pixn * t2 * un + pitx * ut - pixx * ux - pixy * uy) / den;
                cand[4] = (-piyn * t2 * un + pity * ut - pixy * ux - piyy * uy) / den;
                cand[5] = (-pinn * t2 * un + pitn * ut - pixn * ux - piyn * uy) / den;
                cand[6] = (z0 * pitt - t2 * z3 * pitn) / den;
                cand[7] = (z0 * pitx - t2 * z3 * pixn) / den;
                cand[8] = (z0 * pity - t2 * z3 * piyn) / den;
                cand[9] = (z0 * pitn - t2 * z3 * pinn) / den;
                double rho = cand[0];
                for (int m = 1; m < 10; ++m)
                    if (cand[m] > rho) rho = cand[m];
                double fac = tanh(rho) / rho;
                if (rho < 1.e-7) fac = 1.0;
                for (int n = 5; n < 15; ++n) q[n][s] *= fac;
                if (st->validity_on) {  /* :666-693: the factor, then each criterion's own factor */
                    st->vd[16][s] = fac;
                    for (int m = 0; m < 10; ++m) {
                        double f = tanh(cand[m]) / cand[m];
                        if (cand[m] < 1.e-7) f = 1.0;
                        st->vd[17 + m][s] = f;
                    }
                }
            }
}

/* HydrodynamicValidity.cpp:47-394 at one interior cell: t = tau + dtau, qn =
 * the conserved state at the start of the step (the reference passes q before
 * it is swapped with Q), e, p, u the new primitives and up the previous u.
 * Shear tensor and its transverse projection as in the source terms; the
 * reference's later assignments of stt..snn (:197-200) are the ones kept. */
static void validity_cell(vo_state *st, double t, double dt, double *const *qn, int s) {
    const vo_config *c = &st->cfg;
    double **v = st->vd;
    const double e_s = st->e[s], p_s = st->p[s];
    const double *U0 = st->u[0], *U1 = st->u[1], *U2 = st->u[2], *U3 = st->u[3];
    const double ut = U0[s], ux = U1[s], uy = U2[s], un = U3[s];
    const double utp = st->up[0][s], uxp = st->up[1][s], uyp = st->up[2][s], unp = st->up[3][s];
    const double fx = 1 / c->dx / 2, fy = 1 / c->dy / 2, fz = 1 / c->dz / 2;
    const int sy = st->ncx, sz = st->ncx * st->ncy;
    const double dxut = (U0[s + 1] - U0[s - 1]) * fx, dxux = (U1[s + 1] - U1[s - 1]) * fx;
    const double dxuy = (U2[s + 1] - U2[s - 1]) * fx, dxun = (U3[s + 1] - U3[s - 1]) * fx;
    const double dyut = (U0[s + sy] - U0[s - sy]) * fy, dyux = (U1[s + sy] - U1[s - sy]) * fy;
    const double dyuy = (U2[s + sy] - U2[s - sy]) * fy, dyun = (U3[s + sy] - U3[s - sy]) * fy;
    const double dnut = (U0[s + sz] - U0[s - sz]) * fz, dnux = (U1[s + sz] - U1[s - sz]) * fz;
    const double dnuy = (U2[s + sz] - U2[s - sz]) * fz, dnun = (U3[s + sz] - U3[s - sz]) * fz;
    const double dtut = (ut - utp) / dt, dtux = (ux - uxp) / dt, dtuy = (uy - uyp) / dt, dtun = (un - unp) / dt;

    const double ut2 = ut * ut, un2 = un * un, t2 = t * t, t3 = t * t2;
    const double Dut = ut * dtut + ux * dxut + uy * dyut + un * dnut + t * un * un;
    const double dut = Dut - t * un * un;
    const double dux = ut * dtux + ux * dxux + uy * dyux + un * dnux;
    const double duy = ut * dtuy + ux * dxuy + uy * dyuy + un * dnuy;
    const double dun = ut * dtun + ux * dxun + uy * dyun + un * dnun;
    const double theta = ut / t + dtut + dxux + dyuy + dnun;
    const double stt = -t * ut * un2 + (dtut - ut * dut) + (ut2 - 1) * theta / 3;
    const double stx = -(t * un2 * ux) / 2 + (dtux - dxut) / 2 - (ux * dut + ut * dux) / 2 + ut * ux * theta / 3;
    const double sty = -(t * un2 * uy) / 2 + (dtuy - dyut) / 2 - (uy * dut + ut * duy) / 2 + ut * uy * theta / 3;
    const double stn = -un * (2 * ut2 + t2 * un2) / (2 * t) + (dtun - dnut / t2) / 2 - (un * dut + ut * dun) / 2 +
                       ut * un * theta / 3;
    const double sxx = -(dxux + ux * dux) + (1 + ux * ux) * theta / 3;
    const double sxy = -(dxuy + dyux) / 2 - (uy * dux + ux * duy) / 2 + ux * uy * theta / 3;
    const double sxn = -ut * ux * un / t - (dxun + dnux / t2) / 2 - (un * dux + ux * dun) / 2 + ux * un * theta / 3;
    const double syy = -(dyuy + uy * duy) + (1 + uy * uy) * theta / 3;
    const double syn = -ut * uy * un / t - (dyun + dnuy / t2) / 2 - (un * duy + uy * dun) / 2 + uy * un * theta / 3;
    const double snn = -ut * (1 + 2 * t2 * un2) / t3 - dnun / t2 - un * dun + (1 / t2 + un2) * theta / 3;

    const double F = 1 + (ux * ux + uy * uy);
    const double z0 = t * un / sqrt(F), z3 = ut / t / sqrt(F);
    const double z02 = z0 * z0, z0z3 = z0 * z3, z32 = z3 * z3;
    const double A = z02 * stt - 2 * t2 * z0z3 * stn + t2 * t2 * z32 * snn;
    const double B0 = z0 * stt - t2 * z3 * stn, B1 = z0 * stx - t2 * z3 * sxn;
    const double B2 = z0 * sty - t2 * z3 * syn, B3 = z0 * stn - t2 * z3 * snn;
    const double thetaT = 2 * theta / 3 + A;  /* the last of the reference's assignments (:183-184) */
    const double zDzu = theta - thetaT;
    const double sttT = stt + 2 * z0 * B0 + z02 * A - 0.5 * (1 - ut * ut + z02) * A;
    const double stxT = stx + z0 * B1 - 0.5 * (-ut * ux) * A;
    const double styT = sty + z0 * B2 - 0.5 * (-ut * uy) * A;
    const double stnT = stn + z0 * B3 + z3 * B0 + z0z3 * A - 0.5 * (-ut * un + z0z3) * A;
    const double sxxT = sxx - 0.5 * (-1 - ux * ux) * A;
    const double sxyT = sxy - 0.5 * (-ux * uy) * A;
    const double sxnT = sxn + z3 * B1 - 0.5 * (-ux * un) * A;
    const double syyT = syy - 0.5 * (-1 - uy * uy) * A;
    const double synT = syn + z3 * B2 - 0.5 * (-uy * un) * A;
    const double snnT = snn + 2 * z3 * B3 + z32 * A - 0.5 * (-1 / t2 - un * un + z32) * A;
    v[12][s] = stt - sxx - syy - t2 * snn;
    v[13][s] = sttT - sxxT - syyT - t2 * snnT;
    v[14][s] = z02 * stt - 2 * t2 * z0z3 * stn + t2 * t2 * z32 * snn;
    v[15][s] = snnT;

    const double Pi = has_bulk(c) ? qn[SLOT_PI][s] : 0.0;
    const double cs2 = eos_cs2(c, e_s);
    const double T = eos_T(c, e_s);
    const double etabar = c->etabar;
    v[0][s] = 5 * etabar * fabs(thetaT) / T;
    v[1][s] = 5 * etabar * fabs(zDzu) / T;
    v[2][s] = 5 * etabar * fabs(theta) / T;
    double pl = 0, ptHat = 0, ps = 0, ap[16];
    if (has_pimunu(c)) {
        pl = qn[SLOT_PL][s];
        const double pitt = qn[5][s], pitx = qn[6][s], pity = qn[7][s], pitn = qn[8][s], pixx = qn[9][s];
        const double pixy = qn[10][s], pixn = qn[11][s], piyy = qn[12][s], piyn = qn[13][s], pinn = qn[14][s];
        const double pipi = pitt * pitt - 2 * pitx * pitx - 2 * pity * pity + pixx * pixx + 2 * pixy * pixy +
                            piyy * piyy - 2 * pitn * pitn * t2 + 2 * pixn * pixn * t2 + 2 * piyn * piyn * t2 +
                            pinn * pinn * t2 * t2;
        ptHat = pt_hat(e_s, p_s, pl);
        v[4][s] = sqrt(fabs(pipi)) / fabs(ptHat);
    }
    if (has_bulk(c)) {
        const double b = 0.333333 - cs2;
        const double tauPiInv = 15 * (b * b) * T / zeta_over_s(c, T);
        v[3][s] = fabs(thetaT + zDzu) / tauPiInv;
        v[5][s] = fabs(Pi) / fabs(ptHat);
    }
    v[8][s] = 5 * etabar / T;
    v[9][s] = dxux;
    v[10][s] = dyuy;
    v[11][s] = thetaT + zDzu;
    if (has_pimunu(c)) {
        powers(pl / e_s, ap);
        const double Rtilde = VO_RATIO(Rtilde, ap), Rhat = VO_RATIO(Rhat, ap);
        const double Rbar0 = VO_RATIO(Rbar0, ap), Rgamma = VO_RATIO(Rgamma, ap);
        const second_order so = second_order_z(e_s, p_s, pl, cs2, ap);
        const double etaBar_TC = ((3 - Rtilde) * e_s - 2 * pl) / 8;
        const double delta_pipi = (3 + Rgamma) / 2;
        const double tau_pipi = 4 * (delta_pipi - 0) / 3;  /* :294, 1/2 -> 0 */
        const double lambda_pipi = Rgamma - 1;
        const double pi[10] = {qn[5][s], qn[6][s], qn[7][s], qn[8][s], qn[9][s],
                               qn[10][s], qn[11][s], qn[12][s], qn[13][s], qn[14][s]};
        const double pitt = pi[0], pitx = pi[1], pity = pi[2], pitn = pi[3], pixx = pi[4];
        const double pixy = pi[5], pixn = pi[6], piyy = pi[7], piyn = pi[8], pinn = pi[9];
        ps = pitt * sttT - 2 * pitx * stxT - 2 * pity * styT + pixx * sxxT + 2 * pixy * sxyT + piyy * syyT -
             2 * pitn * stnT * t2 + 2 * pixn * sxnT * t2 + 2 * piyn * synT * t2 + pinn * snnT * t2 * t2;
        const double ps2 = ps / 2;
        const double I4[10] = {
            (pitt * sttT - pitx * stxT - pity * styT - t2 * pitn * stnT) - (1 - ut2 + z02) * ps2,
            (pitt * stxT + pitx * sttT) / 2 - (pitx * sxxT + pixx * stxT) / 2 - (pity * sxyT + pixy * styT) / 2 -
                t2 * (pitn * sxnT + pixn * stnT) / 2 + (ut * ux) * ps2,
            (pitt * styT + pity * sttT) / 2 - (pitx * sxyT + pixy * stxT) / 2 - (pity * syyT + piyy * styT) / 2 -
                t2 * (pitn * synT + piyn * stnT) / 2 + (ut * uy) * ps2,
            (pitt * stnT + pitn * sttT) / 2 - (pitx * sxnT + pixn * stxT) / 2 - (pity * synT + piyn * styT) / 2 -
                t2 * (pitn * snnT + pinn * stnT) / 2 + (ut * un - z0z3) * ps2,
            (pitx * stxT - pixx * sxxT - pixy * sxyT - t2 * pixn * sxnT) + (1 + ux * ux) * ps2,
            (pitx * styT + pity * stxT) / 2 - (pixx * sxyT + pixy * sxxT) / 2 - (pixy * syyT + piyy * sxyT) / 2 -
                t2 * (pixn * synT + piyn * sxnT) / 2 + (ux * uy) * ps2,
            (pitx * stnT + pitn * stxT) / 2 - (pixx * sxnT + pixn * sxxT) / 2 - (pixy * synT + piyn * sxyT) / 2 -
                t2 * (pixn * snnT + pinn * sxnT) / 2 + (ux * un) * ps2,
            (pity * styT - pixy * sxyT - piyy * syyT - t2 * piyn * synT) + (1 + uy * uy) * ps2,
            (pity * stnT + pitn * styT) / 2 - (pixy * sxnT + pixn * sxyT) / 2 - (piyy * synT + piyn * syyT) / 2 -
                t2 * (piyn * snnT + pinn * synT) / 2 + (uy * un) * ps2,
            (pitn * stnT - pixn * sxnT - piyn * synT - t2 * pinn * snnT) + (1 / t2 + un2 - z32) * ps2};
        /* J = delta I2 + tau I4 - lambda I5 - lambda_piPi Pi sigma^{tt}_T in every component (:335-344) */
        double J[10];
        for (int m = 0; m < 10; ++m)
            J[m] = delta_pipi * (thetaT * pi[m]) + tau_pipi * I4[m] - lambda_pipi * (zDzu * pi[m]) -
                   so.lambda_piPi * Pi * sttT;
        const double ss = sttT * sttT - 2 * stxT * stxT - 2 * styT * styT + sxxT * sxxT + 2 * sxyT * sxyT +
                          syyT * syyT - 2 * stnT * stnT * t2 + 2 * sxnT * sxnT * t2 + 2 * synT * synT * t2 +
                          snnT * snnT * t2 * t2;
        const double JJ = J[0] * J[0] - 2 * J[1] * J[1] - 2 * J[2] * J[2] + J[4] * J[4] + 2 * J[5] * J[5] +
                          J[7] * J[7] - 2 * J[3] * J[3] * t2 + 2 * J[6] * J[6] * t2 + 2 * J[8] * J[8] * t2 +
                          J[9] * J[9] * t2 * t2;
        v[6][s] = sqrt(fabs(JJ / ss)) / 2 / etaBar_TC;
        if (has_bulk(c)) {
            const double zeta_z = (Rhat - Rbar0) * (e_s - 3 * p_s) / 3;
            const double zeta_T = -(Rbar0 + Rhat) * (e_s - 3 * p_s) / 6;
            const double Jb = -so.beta_PiPi * Pi * zDzu - so.delta_PiPi * Pi * thetaT + so.lambda_Pipi * ps;
            v[7][s] = (double)fabsf((float)(Jb / (-zeta_z * zDzu - zeta_T * thetaT)));  /* :391, fabsf */
        }
    }
}

static void check_validity(vo_state *st, double t, double dt, double *const *qn) {
    for (int i = 2; i < st->ncx - 2; ++i)
        for (int j = 2; j < st->ncy - 2; ++j)
            for (int k = 2; k < st->ncz - 2; ++k) validity_cell(st, t, dt, qn, idx(st, i, j, k));
}

void vo_set_validity(vo_state *st, int on) {
    if (on && !st->vd[0])
        for (int m = 0; m < VO_NUM_VALIDITY; ++m) st->vd[m] = (double *)calloc(st->len, sizeof(double));
    st->validity_on = on && st->vd[0] != NULL;
}

double *vo_validity_field(vo_state *st, int id) {
    return (id >= 0 && id < VO_NUM_VALIDITY) ? st->vd[id] : NULL;
}

/* DynamicalVariables.cpp:349-489: zero-gradient ghost layers, I then J then
 * K pass with the reference's loop ranges (which also fix the edges). */
static void ghost_copy(vo_state *st, double *const *q, double *const *u, int s, int sb) {
    st->e[s] = st->e[sb];
    st->p[s] = st->p[sb];
    for (int m = 0; m < 4; ++m) u[m][s] = u[m][sb];
    for (int n = 0; n < st->nq; ++n) q[n][s] = q[n][sb];
}

static void ghosts(vo_state *st, double *const *q, double *const *u) {
    int nx = st->cfg.nx, ny = st->cfg.ny, nz = st->cfg.nz;
    int ncx = st->ncx, ncy = st->ncy, ncz = st->ncz;
    for (int j = 2; j < ncy; ++j)
        for (int k = 2; k < ncz; ++k) {
            for (int i = 0; i <= 1; ++i) ghost_copy(st, q, u, idx(st, i, j, k), idx(st, 2, j, k));
            for (int i = nx + 2; i <= nx + 3; ++i) ghost_copy(st, q, u, idx(st, i, j, k), idx(st, nx + 1, j, k));
        }
    for (int i = 2; i < ncx; ++i)
        for (int k = 2; k < ncz; ++k) {
            for (int j = 0; j <= 1; ++j) ghost_copy(st, q, u, idx(st, i, j, k), idx(st, i, 2, k));
            for (int j = ny + 2; j <= ny + 3; ++j) ghost_copy(st, q, u, idx(st, i, j, k), idx(st, i, ny + 1, k));
        }
    for (int i = 2; i < ncx; ++i)
        for (int j = 2; j < ncy; ++j) {
            for (int k = 0; k <= 1; ++k) ghost_copy(st, q, u, idx(st, i, j, k), idx(st, i, j, 2));
            for (int k = nz + 2; k <= nz + 3; ++k) ghost_copy(st, q, u, idx(st, i, j, k), idx(st, i, j, nz + 1));
        }
}

/* FullyDiscreteKurganovTadmorScheme.cpp:738-792 followed by the caller's
 * q<->Q swap (DynamicalVariables.cpp:497-499). The validity diagnostics
 * (:791) write nothing the step reads and are not restated. */
void vo_step(vo_state *st, double t, double dt) {
    st->face_fail = st->cell_fail = st->nan_count = 0;
    st->face_fail_axis[0] = st->face_fail_axis[1] = st->face_fail_axis[2] = 0;
    euler_step(st, t, dt, st->q, st->qS, st->u, st->up);
    t += dt;
    infer_all(st, 0, t, st->qS, st->u, st->uS);
    regulate(st, t, st->qS, st->uS);
    ghosts(st, st->qS, st->uS);

    euler_step(st, t, dt, st->qS, st->Q, st->uS, st->u);
    for (int i = 2; i < st->ncx - 2; ++i)
        for (int j = 2; j < st->ncy - 2; ++j)
            for (int k = 2; k < st->ncz - 2; ++k) {
                int s = idx(st, i, j, k);
                for (int n = 0; n < st->nq; ++n) {
                    st->Q[n][s] += st->q[n][s];
                    st->Q[n][s] /= 2;
                }
            }
    for (int m = 0; m < 4; ++m) {
        double *tmp = st->up[m];
        st->up[m] = st->u[m];
        st->u[m] = tmp;
    }
    infer_all(st, 1, t, st->Q, st->up, st->u);
    regulate(st, t, st->Q, st->u);
    ghosts(st, st->Q, st->u);
    if (st->validity_on) check_validity(st, t, dt, st->q);  /* :791, before q and Q swap */

    for (int n = 0; n < NQ_MAX; ++n) {
        double *tmp = st->q[n];
        st->q[n] = st->Q[n];
        st->Q[n] = tmp;
    }
}

double vo_run(vo_state *st, double t0, double dt, int nsteps) {
    struct timespec a, b;
    clock_gettime(CLOCK_MONOTONIC, &a);
    for (int n = 0; n < nsteps; ++n) vo_step(st, t0 + n * dt, dt);
    clock_gettime(CLOCK_MONOTONIC, &b);
    return (double)(b.tv_sec - a.tv_sec) + 1e-9 * (double)(b.tv_nsec - a.tv_nsec);
}

void vo_last_step_face_fallbacks(const vo_state *st, long long out[3]) {
    for (int d = 0; d < 3; ++d) out[d] = st->face_fail_axis[d];
}

const unsigned char *vo_fallback_mask(const vo_state *st, int stage) {
    return (stage == 1 || stage == 2) ? st->fallback[stage - 1] : NULL;
}

void vo_last_step_stats(const vo_state *st, long long out[3]) {
    out[0] = st->face_fail;
    out[1] = st->cell_fail;
    out[2] = st->nan_count;
}

/* DynamicalVariables.cpp:197-287: primitives (e, p, u, pi^{tau mu}, Pi) ->
 * conserved T^{tau mu} and P_L, and up = u. pl_from_field = 0 keeps the
 * reference's hard-coded P_L = 0.0154483 e (:246-248); 1 takes P_L from the
 * P_L field as given. */
void vo_set_conserved(vo_state *st, double t, int pl_from_field) {
    const int pimunu = has_pimunu(&st->cfg), bulkon = has_bulk(&st->cfg);
    for (int k = 2; k < st->cfg.nz + 2; ++k)
        for (int j = 2; j < st->cfg.ny + 2; ++j)
            for (int i = 2; i < st->cfg.nx + 2; ++i) {
                int s = idx(st, i, j, k);
                double ux = st->u[1][s], uy = st->u[2][s], un = st->u[3][s], ut = st->u[0][s];
                double eeq = st->e[s];
                double pitt = 0, pitx = 0, pity = 0, pitn = 0, Pi = 0;
                if (pimunu) { pitt = st->q[5][s]; pitx = st->q[6][s]; pity = st->q[7][s]; pitn = st->q[8][s]; }
                if (bulkon) Pi = st->q[SLOT_PI][s];
                double pl = pl_from_field ? st->q[SLOT_PL][s] : 0.0154483 * eeq;
                double ptHat = 0.5 * (eeq - pl);
                double pt = ptHat + 1.5 * Pi;
                double DP = pl - pt;
                double F = 1 + (ux * ux + uy * uy);
                double Ltt = DP * t * t * un * un / F;
                double Ltn = DP * ut * un / F;
                const double Ltx = 0, Lty = 0, W = 0;
                st->q[0][s] = (eeq + pt) * ut * ut - pt + Ltt + W + pitt;
                st->q[1][s] = (eeq + pt) * ut * ux + Ltx + W + pitx;
                st->q[2][s] = (eeq + pt) * ut * uy + Lty + W + pity;
                st->q[3][s] = (eeq + pt) * ut * un + Ltn + W + pitn;
                st->q[SLOT_PL][s] = pl;
                for (int m = 0; m < 4; ++m) st->up[m][s] = st->u[m][s];
            }
}

void vo_set_ghost_cells(vo_state *st) { ghosts(st, st->q, st->u); }

/* ------------------------------------------------------------- storage -- */
vo_state *vo_create(const vo_config *cfg) {
    if (cfg->nx < 1 || cfg->ny < 1 || cfg->nz < 1) return NULL;
    if (cfg->eos == VO_EOS_TABLE && !cfg->eos_table) return NULL;
    vo_state *st = (vo_state *)calloc(1, sizeof(vo_state));
    st->cfg = *cfg;
    st->ncx = cfg->nx + 4;
    st->ncy = cfg->ny + 4;
    st->ncz = cfg->nz + 4;
    st->len = st->ncx * st->ncy * st->ncz;
    st->nq = nq_of(cfg->physics);
    size_t b = sizeof(double);
    for (int n = 0; n < NQ_MAX; ++n) {
        st->q[n] = (double *)calloc(st->len, b);
        st->Q[n] = (double *)calloc(st->len, b);
        st->qS[n] = (double *)calloc(st->len, b);
    }
    st->e = (double *)calloc(st->len, b);
    st->p = (double *)calloc(st->len, b);
    for (int m = 0; m < 4; ++m) {
        st->u[m] = (double *)calloc(st->len, b);
        st->up[m] = (double *)calloc(st->len, b);
        st->uS[m] = (double *)calloc(st->len, b);
    }
    st->fallback[0] = (unsigned char *)calloc(st->len, 1);
    st->fallback[1] = (unsigned char *)calloc(st->len, 1);
    return st;
}

void vo_destroy(vo_state *st) {
    if (!st) return;
    for (int n = 0; n < NQ_MAX; ++n) { free(st->q[n]); free(st->Q[n]); free(st->qS[n]); }
    free(st->e); free(st->p);
    for (int m = 0; m < 4; ++m) { free(st->u[m]); free(st->up[m]); free(st->uS[m]); }
    for (int m = 0; m < VO_NUM_VALIDITY; ++m) free(st->vd[m]);
    free(st->fallback[0]);
    free(st->fallback[1]);
    free(st);
}

int vo_num_cells(const vo_state *st) { return st->len; }

double *vo_field(vo_state *st, int id) {
    if (id >= 0 && id < NQ_MAX) return st->q[id];
    switch (id) {
    case 16: return st->e;
    case 17: return st->p;
    case 18: case 19: case 20: case 21: return st->u[id - 18];
    case 22: case 23: case 24: case 25: return st->up[id - 22];
    default: return NULL;
    }
}
