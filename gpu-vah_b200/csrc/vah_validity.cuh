// vah_validity.cuh -- the validity diagnostics of one cell after a step.
//
// HydrodynamicValidity.cpp:47-394, called at the end of every reference step
// (FullyDiscreteKurganovTadmorScheme.cpp:791) with tau + dtau, the conserved
// state at the START of the step (q is not yet swapped with Q there), the new
// e, p, u and the previous u. Knudsen numbers of the shear and bulk
// relaxation, first- and second-order inverse Reynolds numbers, and the
// shear-tensor combinations the reference stores. Nothing in the step reads
// them. Written once as host/device code so that the CPU build of this file
// is checked against the oracle.
#pragma once

#include "vah_physics.cuh"

namespace vah {

template <typename S>
struct ValidityArgs {
    int nx, ny, nz, ncx, ncy;
    long long plane;
    double t, dt, dx, dy, dz, etabar;
    const S *qn[16];         // conserved state at the start of the step (P_L, pi, Pi are read)
    const S *e, *p;          // new primitives
    const S *u[4], *up[4];   // new velocity, velocity at the start of the step
    Eos eos;
    double *v[16];           // VAH_V_KN_TAUPI_T .. VAH_V_SNN
};

template <typename S, int PHYS>
VAH_HD void validity_cell(const ValidityArgs<S> &a, long long s) {
    constexpr bool PIM = Phys<PHYS>::PIMUNU, BULK = Phys<PHYS>::BULK;
    const double t = a.t, dt = a.dt;
    const double e_s = (double)a.e[s], p_s = (double)a.p[s];
    const S *U0 = a.u[0], *U1 = a.u[1], *U2 = a.u[2], *U3 = a.u[3];
    const double ut = U0[s], ux = U1[s], uy = U2[s], un = U3[s];
    const double utp = a.up[0][s], uxp = a.up[1][s], uyp = a.up[2][s], unp = a.up[3][s];
    const double fx = 1 / a.dx / 2, fy = 1 / a.dy / 2, fz = 1 / a.dz / 2;
    const long long sy = a.ncx, sz = a.plane;
#define VAH_VD(P, off, f) (((double)P[s + (off)] - (double)P[s - (off)]) * (f))
    const double dxut = VAH_VD(U0, 1, fx), dxux = VAH_VD(U1, 1, fx), dxuy = VAH_VD(U2, 1, fx), dxun = VAH_VD(U3, 1, fx);
    const double dyut = VAH_VD(U0, sy, fy), dyux = VAH_VD(U1, sy, fy), dyuy = VAH_VD(U2, sy, fy), dyun = VAH_VD(U3, sy, fy);
    const double dnut = VAH_VD(U0, sz, fz), dnux = VAH_VD(U1, sz, fz), dnuy = VAH_VD(U2, sz, fz), dnun = VAH_VD(U3, sz, fz);
#undef VAH_VD
    const double dtut = (ut - utp) / dt, dtux = (ux - uxp) / dt, dtuy = (uy - uyp) / dt, dtun = (un - unp) / dt;

    // shear tensor in Milne coordinates (:97-130)
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

    // projection transverse to u and z (:152-194)
    const double F = 1 + (ux * ux + uy * uy);
    const double z0 = t * un / sqrt(F), z3 = ut / t / sqrt(F);
    const double z02 = z0 * z0, z0z3 = z0 * z3, z32 = z3 * z3;
    const double A = z02 * stt - 2 * t2 * z0z3 * stn + t2 * t2 * z32 * snn;
    const double B0 = z0 * stt - t2 * z3 * stn, B1 = z0 * stx - t2 * z3 * sxn;
    const double B2 = z0 * sty - t2 * z3 * syn, B3 = z0 * stn - t2 * z3 * snn;
    const double thetaT = 2 * theta / 3 + A;  // the last of the reference's assignments (:183-184)
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
    a.v[12][s] = stt - sxx - syy - t2 * snn;
    a.v[13][s] = sttT - sxxT - syyT - t2 * snnT;
    a.v[14][s] = z02 * stt - 2 * t2 * z0z3 * stn + t2 * t2 * z32 * snn;
    a.v[15][s] = snnT;

    // Knudsen and inverse Reynolds numbers (:204-258)
    const double Pi = BULK ? (double)a.qn[kSlotPi][s] : 0.0;
    double T, cs2;
    eos_T_cs2(a.eos, e_s, &T, &cs2);
    a.v[0][s] = 5 * a.etabar * fabs(thetaT) / T;
    a.v[1][s] = 5 * a.etabar * fabs(zDzu) / T;
    a.v[2][s] = 5 * a.etabar * fabs(theta) / T;
    a.v[8][s] = 5 * a.etabar / T;
    a.v[9][s] = dxux;
    a.v[10][s] = dyuy;
    a.v[11][s] = thetaT + zDzu;
    if (!PIM) return;
    const double pl = a.qn[kSlotPL][s];
    double pi[10];
#pragma unroll
    for (int m = 0; m < 10; ++m) pi[m] = a.qn[5 + m][s];
    const double pitt = pi[0], pitx = pi[1], pity = pi[2], pitn = pi[3], pixx = pi[4];
    const double pixy = pi[5], pixn = pi[6], piyy = pi[7], piyn = pi[8], pinn = pi[9];
    const double pipi = pitt * pitt - 2 * pitx * pitx - 2 * pity * pity + pixx * pixx + 2 * pixy * pixy + piyy * piyy -
                        2 * pitn * pitn * t2 + 2 * pixn * pixn * t2 + 2 * piyn * piyn * t2 + pinn * pinn * t2 * t2;
    double ap[16];
    ap[0] = 1.0;
    ap[1] = pl / e_s;
#pragma unroll
    for (int k = 2; k < 16; ++k) ap[k] = ap[k - 1] * ap[1];
    const double Rtilde = poly::Rtilde(ap), Rhat = poly::Rhat(ap), Rbar0 = poly::Rbar0(ap), Rgamma = poly::Rgamma(ap);
    const double ptHat = (e_s - pl - Rbar0 * (e_s - 3 * p_s)) / 2;
    a.v[4][s] = sqrt(fabs(pipi)) / fabs(ptHat);
    if (BULK) {
        const double b = 0.333333 - cs2;
        const double tauPiInv = 15 * (b * b) * T / zeta_over_s(a.eos, T);
        a.v[3][s] = fabs(thetaT + zDzu) / tauPiInv;
        a.v[5][s] = fabs(Pi) / fabs(ptHat);
    }

    // second-order inverse Reynolds number of the shear (:262-384). The
    // reference's lambda_piPi is 0 (its 1/3 integer division), delta_pipi
    // keeps its 1/2 -> 0.
    const double etaBar_TC = ((3 - Rtilde) * e_s - 2 * pl) / 8;
    const double delta_pipi = (3 + Rgamma) / 2;
    const double tau_pipi = 4 * delta_pipi / 3;
    const double lambda_pipi = Rgamma - 1;
    const double ps = pitt * sttT - 2 * pitx * stxT - 2 * pity * styT + pixx * sxxT + 2 * pixy * sxyT + piyy * syyT -
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
    double J[10];
#pragma unroll
    for (int m = 0; m < 10; ++m) J[m] = delta_pipi * (thetaT * pi[m]) + tau_pipi * I4[m] - lambda_pipi * (zDzu * pi[m]);
    const double ss = sttT * sttT - 2 * stxT * stxT - 2 * styT * styT + sxxT * sxxT + 2 * sxyT * sxyT + syyT * syyT -
                      2 * stnT * stnT * t2 + 2 * sxnT * sxnT * t2 + 2 * synT * synT * t2 + snnT * snnT * t2 * t2;
    const double JJ = J[0] * J[0] - 2 * J[1] * J[1] - 2 * J[2] * J[2] + J[4] * J[4] + 2 * J[5] * J[5] + J[7] * J[7] -
                      2 * J[3] * J[3] * t2 + 2 * J[6] * J[6] * t2 + 2 * J[8] * J[8] * t2 + J[9] * J[9] * t2 * t2;
    a.v[6][s] = sqrt(fabs(JJ / ss)) / 2 / etaBar_TC;

    if (BULK) {
        // second-order inverse Reynolds number of the bulk (:386-392), with the
        // closure coefficients of AnisotropicDistributionFunctions.cpp:73-190
        // (3/2 -> 1, 1/3 -> 0) and the reference's single-precision fabsf
        const double g20c = poly::g0m2020ConstantTerm(ap);
        const double beta_PiPi = 1 - g20c, delta_PiPi = 0.5 * (1 + g20c);
        const double lambda_Pipi = 3 * poly::G_G1(ap) / 5 * (0 - cs2);
        const double zeta_z = (Rhat - Rbar0) * (e_s - 3 * p_s) / 3;
        const double zeta_T = -(Rbar0 + Rhat) * (e_s - 3 * p_s) / 6;
        const double Jb = -beta_PiPi * Pi * zDzu - delta_PiPi * Pi * thetaT + lambda_Pipi * ps;
        a.v[7][s] = (double)fabsf((float)(Jb / (-zeta_z * zDzu - zeta_T * thetaT)));
    }
}

}  // namespace vah
