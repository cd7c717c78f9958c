// vah_physics.cuh -- per-cell physics of the VAH time step.
//
// Everything here is __host__ __device__: the CUDA kernels (vah_kernels.cu)
// call it per thread, and the same code builds for the host so its formulas
// can be checked against the CPU oracle without a GPU. Arithmetic follows the
// reference CPU path (old_cpu-vah_code/src); where a cheaper but equivalent
// form is used (reciprocal square roots, v*q instead of u*q/ut, no W terms),
// results move by rounding only.
#pragma once

#include <math.h>
#include <stdint.h>
#include <string.h>

#ifdef __CUDACC__
#define VAH_HD __host__ __device__ __forceinline__
#else
#define VAH_HD inline
#endif

namespace vah {

// f / d. On the device: the hardware reciprocal estimate (rcp.approx, about
// 20 good bits) refined by one Newton-Raphson step y += y (1 - d y), i.e. to
// about 2^-40 relative (measured: 9.8e-13, vah_math_check), times f -- three
// dependent operations instead of an IEEE division. The estimate flushes
// subnormal inputs and results (.ftz), so outside |d| in [2^-1000, 2^1001)
// -- an exponent test on the integer pipe, essentially never taken -- the
// result is the IEEE quotient (a NaN or infinite d lands there too). On the
// host: the IEEE quotient.
VAH_HD double quotient_fast(double f, double d) {
#ifdef __CUDA_ARCH__
    const unsigned biased = ((unsigned)__double2hiint(d) >> 20) & 0x7ffu;
    if (biased - 23u > 2000u) return f / d;
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d));
    y = fma(y, fma(-d, y, 1.0), y);
    return f * y;
#else
    return f / d;
#endif
}

}  // namespace vah

#include "vah_closure_polys.h"

namespace vah {

constexpr int kIdeal = 0, kPimunu = 1, kPimunuPi = 2;

template <int PHYS>
struct Phys {
    static constexpr int NQ = PHYS == kIdeal ? 5 : (PHYS == kPimunu ? 15 : 16);
    static constexpr bool PIMUNU = PHYS != kIdeal;
    static constexpr bool BULK = PHYS == kPimunuPi;
};

// The FP32 form (R = float) takes closure-fit quotients and the face
// states' divisions through quotient_fast; the FP64 form keeps IEEE divisions.
template <typename R>
constexpr bool kFastQuot = sizeof(R) == 4;

constexpr int kSlotPL = 4;
constexpr int kSlotPi = 15;
constexpr double kEosFactor = 13.8997;  // EquationOfState.h:16
constexpr double kHbarc = 0.197326938;

// ------------------------------------------------------------ math helpers --
// 1/sqrt(x) for x > 0. On the device: the hardware estimate (rsqrt.approx)
// refined by two Newton-Raphson steps for x^-1/2, each y += y (0.5 - (x/2) y y)
// (quadratic convergence: about 2^-20 -> 2^-40 -> rounding level), three
// dependent operations per step. Measured against CUDA's IEEE-rounded
// 1/sqrt: within 2.7e-16 relative (vah_math_check).
VAH_HD double rsqrt_d(double x) {
#ifdef __CUDA_ARCH__
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double h = 0.5 * x;
    y = fma(y, fma(-h * y, y, 0.5), y);
    y = fma(y, fma(-h * y, y, 0.5), y);
    return y;
#else
    return 1.0 / sqrt(x);
#endif
}

// 1/sqrt in the arithmetic type of the caller: rsqrt_d for FP64; in FP32 the
// hardware's single-precision 1/sqrt (about 2 ulp) on the device.
VAH_HD double rsqrt_r(double x) { return rsqrt_d(x); }
VAH_HD float rsqrt_r(float x) {
#ifdef __CUDA_ARCH__
    return rsqrtf(x);
#else
    return 1.0f / sqrtf(x);
#endif
}

VAH_HD uint32_t float_bits(float x) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(x);
#else
    uint32_t u;
    memcpy(&u, &x, 4);
    return u;
#endif
}

template <typename T>
VAH_HD T ldg(const T *p) {
#ifdef __CUDA_ARCH__
    return __ldg(p);
#else
    return *p;
#endif
}

// ------------------------------------------------------------------- EoS --
// Equation of state and zeta/s, passed by value into kernels.
struct Eos {
    int kind;               // 0: conformal (reference quirks), 1: table
    int zeta;               // 0: reference zeta/s, 1: crossover zeta/s
    const double *tab;      // table (layout in include/vah.h)
    const uint32_t *exc;    // conformal T: (input, result) pairs where the
    int nexc;               //   reference libm's powf(x, 0.25f) is not the
                            //   correctly rounded value (see vah_powf_exc.cpp)
};

// Conformal T = powf(e/13.8997, 0.25) in single precision
// (EquationOfState.cpp:144). The fourth root is taken in double and rounded
// once, which gives the correctly rounded single; the reference's libm powf
// differs from that for a small set of inputs, listed in eos.exc as
// (input bits, libm result bits) pairs sorted by input (vah_powf_exc.cpp).
VAH_HD double conformal_T(const Eos &eos, double e) {
    float xf = (float)(e / kEosFactor);
    float r = (float)sqrt(sqrt((double)xf));
    if (eos.nexc > 0) {
        uint32_t key = float_bits(xf);
        int lo = 0, hi = eos.nexc - 1;
        while (lo <= hi) {
            int mid = (lo + hi) >> 1;
            uint32_t v = ldg(eos.exc + 2 * mid);
            if (v == key) {
                uint32_t rb = ldg(eos.exc + 2 * mid + 1);
                memcpy(&r, &rb, 4);
                break;
            }
            if (v < key) lo = mid + 1; else hi = mid - 1;
        }
    }
    return (double)r;
}

template <typename R>
struct EosPoint {
    R p, T, cs2;
};

// Tabulated EoS: linear interpolation in ln e between nodes; power-law
// continuation outside (p/e and c_s^2 frozen, T ~ e^(3/23) below, e^(1/4) above).
// The table is FP64; R is the arithmetic type of the interpolation.
template <bool NEED_P, bool NEED_TC, typename R>
VAH_HD EosPoint<R> table_lookup(const double *tab, R e) {
    EosPoint<R> r{R(0.0), R(0.0), R(0.0)};
    const int n = (int)ldg(tab);
    const double *P = tab + 8, *T = P + n, *C = T + n;
    auto tl = [](const double *q) { return R(ldg(q)); };
    if (!(e > R(0.0))) {
        if (NEED_P) r.p = e * (tl(P) / tl(tab + 4));
        if (NEED_TC) r.cs2 = tl(C);
        return r;
    }
    const R x = log(e);
    const R f = (x - tl(tab + 1)) * tl(tab + 2);
    if (f <= R(0.0)) {
        if (NEED_P) r.p = e * (tl(P) / tl(tab + 4));
        if (NEED_TC) {
            r.T = tl(T) * exp((R(3.0) / R(23.0)) * (x - tl(tab + 1)));
            r.cs2 = tl(C);
        }
        return r;
    }
    if (f >= (R)(n - 1)) {
        if (NEED_P) r.p = e * (tl(P + n - 1) / tl(tab + 6));
        if (NEED_TC) {
            r.T = tl(T + n - 1) * exp(R(0.25) * (x - tl(tab + 5)));
            r.cs2 = tl(C + n - 1);
        }
        return r;
    }
    const int i = (int)f;
    const R w = f - (R)i;
    if (NEED_P) {
        R a = tl(P + i), b = tl(P + i + 1);
        r.p = a + w * (b - a);
    }
    if (NEED_TC) {
        R a = tl(T + i), b = tl(T + i + 1);
        r.T = a + w * (b - a);
        a = tl(C + i);
        b = tl(C + i + 1);
        r.cs2 = a + w * (b - a);
    }
    return r;
}

VAH_HD double eos_pressure(const Eos &eos, double e) {
    if (eos.kind == 0) return e / 3;  // EquationOfState.cpp:78
    return table_lookup<true, false>(eos.tab, e).p;
}

// The same in FP32 arithmetic.
VAH_HD float eos_pressure_f(const Eos &eos, float e) {
    if (eos.kind == 0) return e / 3.0f;
    return table_lookup<true, false>(eos.tab, e).p;
}

// (T, c_s^2); the conformal c_s^2 is the reference's integer `1/3` = 0
// (EquationOfState.cpp:113).
template <typename R>
VAH_HD void eos_T_cs2(const Eos &eos, R e, R *T, R *cs2) {
    if (eos.kind == 0) {
        *T = R(conformal_T(eos, e));
        *cs2 = R(0.0);
        return;
    }
    EosPoint<R> r = table_lookup<false, true>(eos.tab, e);
    *T = r.T;
    *cs2 = r.cs2;
}

// zeta/s(T), T in fm^-1: the reference's parameterisation (SourceTerms.cpp:
// 22-44) or the crossover one (height 0.05 at 155 MeV, half-width 50 MeV).
template <typename R>
VAH_HD R zeta_over_s(const Eos &eos, R T) {
    if (eos.zeta == 1) {
        const R tp = R(0.155) / R(kHbarc), w = R(0.050) / R(kHbarc);
        R d = (T - tp) / w;
        return R(0.05) / (R(1.0) + d * d);
    }
    R x = T / R(1.01355);
    if (x > R(1.05)) return R(0.9) * exp(-(x - 1) / R(0.025)) + R(0.25) * exp(-(x - 1) / R(0.13)) + R(0.001);
    if (x < R(0.995)) return R(0.9) * exp((x - 1) / R(0.0025)) + R(0.22) * exp((x - 1) / R(0.022)) + R(0.03);
    return -R(13.77) * x * x + R(27.55) * x - R(13.45);
}

// --------------------------------------------------------------- limiter --
// FluxLimiter.cpp:28-33, theta = 1.1: minmod(l, minmod(c, r)) with
// minmod(x, y) = (sign x + sign y) min(|x|,|y|) / 2, sign(0) = +1
// (FluxLimiter.cpp:15-22). The centred
// difference c = (z - x)/2 has the sign of l and r whenever those two agree
// (z - x = (y - x) + (z - y), and a rounded difference keeps the exact one's
// sign), so the nested minmod is: l and r of one sign (0 counting as +) ->
// that sign times min(|l|, |c|, |r|), else 0. The same value bit for bit for
// every y that is not NaN (checked exhaustively on edge values and on 5e7
// random triples); a NaN y makes the caller's state NaN either way.
// With l = 1.1 (y - x) and r = 1.1 (z - y), min(|l|, |r|) is 1.1 min(|y - x|,
// |z - y|) rounded once (rounding is monotone), and l, r have the signs of
// y - x, z - y.
template <typename R>
VAH_HD R approx_derivative(R x, R y, R z) {
    const R dl = y - x, dr = z - y;
    const R c = (z - x) * R(0.5);
    const R m = fmin(R(1.1) * fmin(fabs(dl), fabs(dr)), fabs(c));
    const bool neg = dl < R(0.0);
    return neg == (dr < R(0.0)) ? (neg ? -m : m) : R(0.0);
}

// ------------------------------------------------------------- inversion --
// Conserved (T^{tau mu}, P_L, pi^{tau mu}, Pi) -> (e, p, u^mu) by Newton on
// u_T (EnergyMomentumTensor.cpp:30-197): relative tolerance 1e-7, at most
// 10^4 iterations; on failure e = 0.999 ePrev, u = (1,0,0,0).
//
// The guess-independent part (InvSetup) is split from the iteration so that a
// face, inverted from both neighbours' guesses, sets up each state once.
struct InvSetup {
    double pl, bulk, m0, m1, m2, m3, F, x, mbt, bT, bL, b, c0;
    // g(v) = bL + b (0.5 (e(v) - pl) + 1.5 Pi) with e(v) = c0 - v x mbt, expanded:
    // g = G0 - G1 v, and g - 0.5 b bT v = G0 - 2 G1 v (the derivative's factor)
    double G0, G1;
};

template <int PHYS, bool FAST = false>
VAH_HD void invert_setup(double t, const double *q, InvSetup &s) {
    double pitt = 0, pitx = 0, pity = 0, pitn = 0, bulk = 0;
    if (Phys<PHYS>::PIMUNU) {
        pitt = q[5];
        pitx = q[6];
        pity = q[7];
        pitn = q[8];
    }
    if (Phys<PHYS>::BULK) bulk = q[kSlotPi];
    const double pl = q[kSlotPL];
    const double m0 = q[0] - pitt, m1 = q[1] - pitx, m2 = q[2] - pity, m3 = q[3] - pitn;
    double m0pl = m0 + pl;
    if (m0pl == 0.0) m0pl = 1.e-16;
    const double F = FAST ? quotient_fast(m3, m0pl) : m3 / m0pl;  // W off: F = A
    const double Ft = t * F;
    const double Ft2 = Ft * Ft;
    const double x = sqrt(fabs(1. - Ft2));
    double mbt = sqrt(m1 * m1 + m2 * m2);
    if (mbt == 0.0) mbt = 1.e-16;
    s.pl = pl;
    s.bulk = bulk;
    s.m0 = m0;
    s.m1 = m1;
    s.m2 = m2;
    s.m3 = m3;
    s.F = F;
    s.x = x;
    s.mbt = mbt;
    s.bT = x * mbt;
    s.bL = x * x * m0 - Ft2 * pl;
    s.b = x * x + Ft2;
    s.c0 = m0 - t * Ft * m3;
    s.G0 = s.bL + s.b * (0.5 * (s.c0 - pl) + 1.5 * bulk);
    s.G1 = 0.5 * s.b * s.bT;
}

// The Newton correction f / fp through quotient_fast. It only needs to be
// accurate relative to itself: where the iteration stops it is ~1e-7 of u_T,
// so its error (about 1e-12) moves the root by ~1e-19 relative.
VAH_HD double newton_correction(double f, double fp) { return quotient_fast(f, fp); }

// Newton iteration for u_T from the guess uT0 (EnergyMomentumTensor.cpp:30-72).
// Returns 0 with the root in uT, or 1 when the reference falls back.
VAH_HD int newton_uT(const InvSetup &s, double uT0, double &uT) {
    const double x = s.x, mbt = s.mbt, bT = s.bT, c0 = s.c0, G0 = s.G0, G1 = s.G1;
    double w = uT0;
    uT = uT0;
    for (int it = 0; it < 10000; ++it) {
        const double w2 = 1 + w * w;
        const double r = rsqrt_d(w2);
        const double v = w * r;
        const double e = c0 - v * x * mbt;  // the reference's energy, for its exit test
        if (e < 0.0) return 1;
        const double g = G0 - G1 * v;  // bL + b (0.5 (e - pl) + 1.5 Pi), one operation after v
        const double r3 = r * r * r;
        const double f = v * g - bT;
        double fp = r3 * (G0 - 2 * G1 * v);  // r3 g + v b (0.5 (-bT r3))
        if (fabs(fp) == 0.0) fp = 1.e-16;
        const double next = w - newton_correction(f, fp);
        uT = next;
        // NaN, +-inf, negative or above 9.0072e15 (one test: NaN fails both comparisons)
        if (!(next >= 0.0 && next <= 9.0072e+15)) return 1;
        if (fabs(next - w) <= 1.e-7 * fabs(next)) return 0;
        w = next;
    }
    return 1;
}

// One Newton iteration from w, straight-line (the exits are tested after the
// arithmetic, so that two independent iterations can be interleaved by the
// scheduler): 0 = converged to next, 1 = the reference falls back, 2 = go on
// from next. The same operations as newton_uT's loop body.
VAH_HD int newton_step(const InvSetup &s, double w, double &next) {
    const double w2 = 1 + w * w;
    const double r = rsqrt_d(w2);
    const double v = w * r;
    const double e = s.c0 - v * s.x * s.mbt;  // the reference's energy, for its exit test
    const double g = s.G0 - s.G1 * v;          // bL + b (0.5 (e - pl) + 1.5 Pi), one operation after v
    const double r3 = r * r * r;
    const double f = v * g - s.bT;
    double fp = r3 * (s.G0 - 2 * s.G1 * v);   // r3 g + v b (0.5 (-bT r3))
    if (fabs(fp) == 0.0) fp = 1.e-16;
    next = w - newton_correction(f, fp);
    if (e < 0.0) return 1;
    if (!(next >= 0.0 && next <= 9.0072e+15)) return 1;  // NaN, +-inf, negative or too large
    return fabs(next - w) <= 1.e-7 * fabs(next) ? 0 : 2;
}

// Two independent Newton solves in lockstep (same iterates as two newton_uT
// calls, one loop): st = 0 converged (root in u), 1 fallback.
VAH_HD void newton_uT2(const InvSetup &A, const InvSetup &B, double g0, double g1, double &u0, double &u1, int &st0,
                       int &st1) {
    double w0 = g0, w1 = g1;
    st0 = st1 = 2;
    for (int it = 0; it < 10000; ++it) {
        double n0 = w0, n1 = w1;
        const int c0 = newton_step(A, w0, n0);
        const int c1 = newton_step(B, w1, n1);
        if (st0 == 2) {
            st0 = c0;
            w0 = n0;
        }
        if (st1 == 2) {
            st1 = c1;
            w1 = n1;
        }
        if (st0 != 2 && st1 != 2) break;
    }
    if (st0 == 2) st0 = 1;  // 10^4 iterations without convergence
    if (st1 == 2) st1 = 1;
    u0 = w0;
    u1 = w1;
}

// The full inversion. Returns 0 (converged), 1 (fallback) or 2 (a NaN
// reached e or u). out = {e, p, ut, ux, uy, un}. PF32 (the FP32 form): the
// pressure from the EoS in FP32 arithmetic (the form stores p in FP32).
template <int PHYS, bool PF32 = false>
VAH_HD int invert(const Eos &eos, double t, const double *q, double ePrev, double uT0, double *out) {
    InvSetup s;
    invert_setup<PHYS>(t, q, s);
    double uT;
    const int status = newton_uT(s, uT0, uT);
    double e, ut, ux, uy, un;
    if (status == 0) {
        const double C = sqrt(1.0 + uT * uT);
        const double U = uT / C;
        const double inv_mbt = 1.0 / s.mbt, inv_x = 1.0 / s.x;
        ux = uT * s.m1 * inv_mbt;
        uy = uT * s.m2 * inv_mbt;
        un = s.F * C * inv_x;
        ut = C * inv_x;
        e = s.c0 - U * s.x * s.mbt;
    } else {
        e = ePrev * .999;
        ux = 0.0;
        uy = 0.0;
        un = 0.0;
        ut = 1.0;
    }
    out[0] = e;
    out[1] = PF32 ? (double)eos_pressure_f(eos, (float)e) : eos_pressure(eos, e);
    out[2] = ut;
    out[3] = ux;
    out[4] = uy;
    out[5] = un;
    if (isnan(e) || isnan(ut) || isnan(ux) || isnan(uy) || isnan(un)) return 2;
    return status;
}

// What a face needs of an inversion: the velocity v_dir = u^dir / u^tau
// (u^tau = C/x, u^x = uT m1/mbt, u^y = uT m2/mbt, u^eta = F C/x with
// C = sqrt(1 + uT^2), so v_x = uT m1 x / (mbt C), v_eta = F), 0 after a
// fallback (u = (1,0,0,0)). Same statuses as invert; a fallback's NaN check
// is on e = 0.999 ePrev, a converged one's on v and the energy offset.
VAH_HD int face_velocity(const InvSetup &s, double ePrev, double uT0, int dir, double *v) {
    double uT;
    if (newton_uT(s, uT0, uT) != 0) {
        *v = 0.0;
        return isnan(ePrev) ? 2 : 1;
    }
    double vv;
    if (dir == 2) {
        vv = s.F;
    } else {
        // uT m x / (mbt C), C = sqrt(1 + uT^2), with 1/C from rsqrt_d
        vv = uT * (dir == 0 ? s.m1 : s.m2) * s.x * rsqrt_d(1.0 + uT * uT) / s.mbt;
    }
    *v = vv;
    return (isnan(vv) || isnan(s.c0)) ? 2 : 0;
}

// ------------------------------------------------------------ face flux --
// Kurganov-Tadmor central flux at one face from the reconstructed states
// (SemiDiscreteKurganovTadmorScheme.cpp:13-57, SpectralRadius.cpp:14-24,
// LocalPropagationSpeed.cpp:14-22, FluxFunctions.cpp:15-25):
// H = (F(qR) + F(qL) - a (qR - qL)) / 2, F = v_dir q, a = max |v_dir|.
// sR/sL: the inversion set-ups of qR/qL; ePrev, uT: the evaluating cell's
// fallback energy and Newton guess.
// Returns the number of the two inversions that fell back; bit 8 flags a NaN.
// The velocity of a converged solve, as face_velocity (status 0 or 2).
template <bool FAST = false>
VAH_HD int face_velocity_of(const InvSetup &s, double uT, int dir, double *v) {
    double vv;
    if (dir == 2) {
        vv = s.F;
    } else {
        // uT m x / (mbt C), C = sqrt(1 + uT^2), with 1/C from rsqrt_d
        const double num = uT * (dir == 0 ? s.m1 : s.m2) * s.x * rsqrt_d(1.0 + uT * uT);
        vv = FAST ? quotient_fast(num, s.mbt) : num / s.mbt;
    }
    *v = vv;
    return (isnan(vv) || isnan(s.c0)) ? 2 : 0;
}

// The weights of one evaluation, H = wR qR + wL qL (the same statuses).
VAH_HD int face_weights(const InvSetup &sR, const InvSetup &sL, int dir, double ePrev, double uT, double &wR,
                        double &wL) {
    // both states' Newton solves from this guess, in lockstep
    double uR, uL, vR = 0.0, vL = 0.0;
    int nR, nL;
    newton_uT2(sR, sL, uT, uT, uR, uL, nR, nL);
    const int stR = nR != 0 ? (isnan(ePrev) ? 2 : 1) : face_velocity_of(sR, uR, dir, &vR);
    const int stL = nL != 0 ? (isnan(ePrev) ? 2 : 1) : face_velocity_of(sL, uL, dir, &vL);
    const double a = fmax(fabs(vL), fabs(vR));
    // (vR qR + vL qL - a (qR - qL)) / 2 = wR qR + wL qL; the halving is exact
    wR = 0.5 * (vR - a);
    wL = 0.5 * (vL + a);
    return (stR != 0) + (stL != 0) + ((stR == 2 || stL == 2) ? 256 : 0);
}

template <int PHYS>
VAH_HD int face_flux_setup(const InvSetup &sR, const InvSetup &sL, const double *qR, const double *qL, int dir,
                           double ePrev, double uT, double *H) {
    constexpr int NQ = Phys<PHYS>::NQ;
    double wR, wL;
    const int st = face_weights(sR, sL, dir, ePrev, uT, wR, wL);
#pragma unroll
    for (int n = 0; n < NQ; ++n) H[n] = wR * qR[n] + wL * qL[n];
    return st;
}

template <int PHYS>
VAH_HD int face_flux(double t, const double *qR, const double *qL, int dir, double ePrev, double uT, double *H) {
    InvSetup sR, sL;
    invert_setup<PHYS>(t, qR, sR);
    invert_setup<PHYS>(t, qL, sL);
    return face_flux_setup<PHYS>(sR, sL, qR, qL, dir, ePrev, uT, H);
}

// ------------------------------------------------------- axis sources --
// pi/Pi gradient terms of the T^{tau mu} equations along one axis
// (SourceTerms.cpp:46-176). d[n] = (q[+1] - q[-1]) / (2h) for the pi fields.
template <int PHYS, typename R>
VAH_HD void axis_sources(const R *d, int dir, R ucomp, R ut, R t, R *S) {
    const R v = ucomp / ut;
    const R dPi = Phys<PHYS>::BULK ? d[kSlotPi] * R(1.5) : R(0.0);
    if (dir == 0) {
        S[0] = d[5] * v - d[6] - v * dPi;
        S[1] = d[6] * v - d[9] - dPi;
        S[2] = d[7] * v - d[10];
        S[3] = d[8] * v - d[11];
    } else if (dir == 1) {
        S[0] = d[5] * v - d[7] - v * dPi;
        S[2] = d[7] * v - d[12] - dPi;
        S[1] = d[6] * v - d[10];
        S[3] = d[8] * v - d[13];
    } else {
        const float tf = (float)t;  // SourceTerms.cpp:172: powf(t, 2)
        S[0] = d[5] * v - d[8] - v * dPi;
        S[3] = d[8] * v - d[14] - dPi / (R)(tf * tf);
        S[1] = d[6] * v - d[11];
        S[2] = d[7] * v - d[13];
    }
}

// x / d for a constant d with its rounded reciprocal inv_d: the product and
// one FMA correction (q + (x - q d) inv_d), within an ulp of the quotient
// (usually the correctly rounded one), in three operations.
template <typename R>
VAH_HD R div_const(R x, R d, R inv_d) {
    const R q = x * inv_d;
    return fma(fma(-q, d, x), inv_d, q);
}

// ----------------------------------------------------------- cell sources --
// Inputs of the local source terms at one cell: stage-input conserved values,
// primitives, previous-stage velocity and central differences (q(+1)-q(-1))/(2h).
template <typename R>
struct CellGradT {
    R e, p, ut, ux, uy, un;
    R utp, uxp, uyp, unp;
    R dxut, dxux, dxuy, dxun, dyut, dyux, dyuy, dyun, dnut, dnux, dnuy, dnun;
    R dxp, dyp, dnp, dxe, dye, dne, dxpl, dypl, dnpl;
};

// The sources' per-launch constants, formed once per launch with the same
// operations as the per-cell expressions they stand for (bit-identical).
template <typename R>
struct StepConstsT {
    R t, dt, etabar, inv_t, inv_t2, inv_dt;
};

using CellGrad = CellGradT<double>;
using StepConsts = StepConstsT<double>;

template <typename R>
VAH_HD StepConstsT<R> step_consts(R t, R dt, R etabar) {
    StepConstsT<R> k;
    k.t = t;
    k.dt = dt;
    k.etabar = etabar;
    k.inv_t = R(1.0) / t;
    k.inv_t2 = R(1.0) / (t * t);
    k.inv_dt = R(1.0) / dt;
    return k;
}

// Geometric and relaxation sources S[n] (SourceTerms.cpp:178-1044), W off.
template <int PHYS, typename R>
VAH_HD int cell_sources(const Eos &eos, const R *Q, const CellGradT<R> &g, const StepConstsT<R> &k, R *S) {
    const R t = k.t, etabar = k.etabar;
    constexpr bool PIM = Phys<PHYS>::PIMUNU, BULK = Phys<PHYS>::BULK;
    const R ttt = Q[0], ttx = Q[1], tty = Q[2], ttn = Q[3], pl = Q[4];
    R pitt = 0, pitx = 0, pity = 0, pitn = 0, pixx = 0, pixy = 0, pixn = 0, piyy = 0, piyn = 0, pinn = 0,
           Pi = 0;
    if (PIM) {
        pitt = Q[5]; pitx = Q[6]; pity = Q[7]; pitn = Q[8]; pixx = Q[9];
        pixy = Q[10]; pixn = Q[11]; piyy = Q[12]; piyn = Q[13]; pinn = Q[14];
    }
    if (BULK) Pi = Q[kSlotPi];
    R e = g.e;
    const R p = g.p, ut = g.ut, ux = g.ux, uy = g.uy, un = g.un;
    const R dxut = g.dxut, dxux = g.dxux, dxuy = g.dxuy, dxun = g.dxun;
    const R dyut = g.dyut, dyux = g.dyux, dyuy = g.dyuy, dyun = g.dyun;
    const R dnut = g.dnut, dnux = g.dnux, dnuy = g.dnuy, dnun = g.dnun;

    const R inv_ut = R(1.0) / ut, inv_t = k.inv_t;
    const R vx = ux * inv_ut, vy = uy * inv_ut, vn = un * inv_ut;
    const R dkvk = (dxux - vx * dxut) * inv_ut + (dyuy - vy * dyut) * inv_ut + (dnun - vn * dnut) * inv_ut;

    const R t2 = t * t, t3 = t * t2, un2 = un * un, ut2 = ut * ut;
    const R inv_t2 = k.inv_t2;

    // velocity gradients (SourceTerms.cpp:301-334)
    const R inv_dt = k.inv_dt;
    const R dtut = (ut - g.utp) * inv_dt, dtux = (ux - g.uxp) * inv_dt;
    const R dtuy = (uy - g.uyp) * inv_dt, dtun = (un - g.unp) * inv_dt;
    const R dux = ut * dtux + ux * dxux + uy * dyux + un * dnux;
    const R duy = ut * dtuy + ux * dxuy + uy * dyuy + un * dnuy;
    const R dun = ut * dtun + ux * dxun + uy * dyun + un * dnun;
    const R dut = ut * dtut + ux * dxut + uy * dyut + un * dnut;  // = Dut - t un^2
    const R Dut = dut + t * un2;
    const R Dux = -dux, Duy = -duy;
    const R Dun = -t2 * (dun + 2 * ut * un * inv_t);
    const R theta = ut * inv_t + dtut + dxux + dyuy + dnun;
    const R th3 = div_const(theta, R(3.0), R(1.0) / R(3.0));

    const R stt = -t * ut * un2 + (dtut - ut * dut) + (ut2 - 1) * th3;
    const R stx = -(t * un2 * ux) * R(0.5) + (dtux - dxut) * R(0.5) - (ux * dut + ut * dux) * R(0.5) + ut * ux * th3;
    const R sty = -(t * un2 * uy) * R(0.5) + (dtuy - dyut) * R(0.5) - (uy * dut + ut * duy) * R(0.5) + ut * uy * th3;
    const R stn = -un * (2 * ut2 + t2 * un2) * (R(0.5) * inv_t) + (dtun - dnut * inv_t2) * R(0.5) -
                       (un * dut + ut * dun) * R(0.5) + ut * un * th3;
    const R sxx = -(dxux + ux * dux) + (1 + ux * ux) * th3;
    const R sxy = -(dxuy + dyux) * R(0.5) - (uy * dux + ux * duy) * R(0.5) + ux * uy * th3;
    const R sxn = -ut * ux * un * inv_t - (dxun + dnux * inv_t2) * R(0.5) - (un * dux + ux * dun) * R(0.5) + ux * un * th3;
    const R syy = -(dyuy + uy * duy) + (1 + uy * uy) * th3;
    const R syn = -ut * uy * un * inv_t - (dyun + dnuy * inv_t2) * R(0.5) - (un * duy + uy * dun) * R(0.5) + uy * un * th3;
    const R snn = -ut * (1 + 2 * t2 * un2) / t3 - dnun * inv_t2 - un * dun + (inv_t2 + un2) * th3;

    // transverse / longitudinal split (SourceTerms.cpp:355-426)
    const R uT2 = ux * ux + uy * uy;
    const R uTdxuT = ux * dxux + uy * dxuy;
    const R uTdyuT = ux * dyux + uy * dyuy;
    const R uTdnuT = ux * dnux + uy * dnuy;
    const R uTduT = ut * (ux * dtux + uy * dtuy) + ux * uTdxuT + uy * uTdyuT + un * uTdnuT;
    const R F = 1 + uT2;
    const R inv_F = R(1.0) / F;
    const R F2 = F * F;
    const R inv_sF = rsqrt_r(F);
    const R z0 = t * un * inv_sF;
    const R z3 = ut * inv_t * inv_sF;
    const R z02 = z0 * z0, z0z3 = z0 * z3, z32 = z3 * z3;
    const R dz0 = (ut * un + t * dun - t * un * inv_F * uTduT) * inv_sF;
    const R dz3 = (-ut2 * inv_t2 + dut * inv_t - ut * inv_t * inv_F * uTduT) * inv_sF;
    const R Dz0 = dz0 + t * un * z3;
    const R Dz3 = -t2 * (dz3 + (ut * z3 + un * z0) * inv_t);
    const R A = z02 * stt - 2 * t2 * z0z3 * stn + t2 * t2 * z32 * snn;
    const R B0 = z0 * stt - t2 * z3 * stn;
    const R B1 = z0 * stx - t2 * z3 * sxn;
    const R B2 = z0 * sty - t2 * z3 * syn;
    const R B3 = z0 * stn - t2 * z3 * snn;
    const R thetaT = 2 * th3 + A;
    const R zDzu = theta - thetaT;
    const R sttT = stt + 2 * z0 * B0 + z02 * A - R(0.5) * (1 - ut * ut + z02) * A;
    const R stxT = stx + z0 * B1 - R(0.5) * (-ut * ux) * A;
    const R styT = sty + z0 * B2 - R(0.5) * (-ut * uy) * A;
    const R stnT = stn + z0 * B3 + z3 * B0 + z0z3 * A - R(0.5) * (-ut * un + z0z3) * A;
    const R sxxT = sxx - R(0.5) * (-1 - ux * ux) * A;
    const R sxyT = sxy - R(0.5) * (-ux * uy) * A;
    const R sxnT = sxn + z3 * B1 - R(0.5) * (-ux * un) * A;
    const R syyT = syy - R(0.5) * (-1 - uy * uy) * A;
    const R synT = syn + z3 * B2 - R(0.5) * (-uy * un) * A;
    const R snnT = snn + 2 * z3 * B3 + z32 * A - R(0.5) * (-inv_t2 - un * un + z32) * A;

    // closures (SourceTerms.cpp:431-481)
    if (e == 0) e = R(1.e-7);
    R T, cs2;
    eos_T_cs2(eos, e, &T, &cs2);
    const R inv_e = R(1.0) / e;
    // The closure fits are evaluated in FP64 whatever R is: their monomial
    // coefficients (up to ~1e7, alternating in sign) cancel to results of
    // O(1e-3), and in FP32 several lose every digit (Rbar0P turns infinite).
    double ap[16];
    ap[0] = 1.0;
    ap[1] = (double)pl * (double)inv_e;
#pragma unroll
    for (int k = 2; k < 16; ++k) ap[k] = ap[k - 1] * ap[1];
    const R a = R(ap[1]);
    const R Rtilde = R(poly::Rtilde<double, kFastQuot<R>>(ap));
    const R Rbar0 = R(poly::Rbar0<double, kFastQuot<R>>(ap));
    const R Rgamma = R(poly::Rgamma<double, kFastQuot<R>>(ap));
    const R Rbar0P = R(poly::Rbar0P<double, kFastQuot<R>>(ap));

    const R e3p = e - 3 * p;
    const R ptHat = (e - pl - Rbar0 * e3p) * R(0.5);
    const R pt = ptHat + R(1.5) * Pi;
    const R DP = pl - pt;
    const R Ltt = DP * t2 * un2 * inv_F;
    const R Ltn = DP * ut * un * inv_F;
    const R Lnn = DP * ut2 * inv_F * inv_t2;
    const R tnn = (e + pt) * un * un + pt * inv_t2 + Lnn + pinn;

    const R dxRbar0 = Rbar0P * (g.dxpl - a * g.dxe) * inv_e;
    const R dyRbar0 = Rbar0P * (g.dypl - a * g.dye) * inv_e;
    const R dnRbar0 = Rbar0P * (g.dnpl - a * g.dne) * inv_e;
    const R dxptHat = R(0.5) * (g.dxe - g.dxpl - Rbar0 * (g.dxe - 3 * g.dxp) - e3p * dxRbar0);
    const R dyptHat = R(0.5) * (g.dye - g.dypl - Rbar0 * (g.dye - 3 * g.dyp) - e3p * dyRbar0);
    const R dnptHat = R(0.5) * (g.dne - g.dnpl - Rbar0 * (g.dne - 3 * g.dnp) - e3p * dnRbar0);
    const R dxDP = g.dxpl - dxptHat, dyDP = g.dypl - dyptHat, dnDP = g.dnpl - dnptHat;

    const R inv_F2 = inv_F * inv_F;
    const R dxLtt = (2 * DP * dxun * t2 * un) * inv_F + (dxDP * t2 * un2) * inv_F - (2 * DP * uTdxuT * t2 * un2) * inv_F2;
    const R dyLtt = (2 * DP * dyun * t2 * un) * inv_F + (dyDP * t2 * un2) * inv_F - (2 * DP * uTdyuT * t2 * un2) * inv_F2;
    const R dnLtt = (2 * DP * dnun * t2 * un) * inv_F + (dnDP * t2 * un2) * inv_F - (2 * DP * uTdnuT * t2 * un2) * inv_F2;
    const R dxLtn = (DP * dxut * un) * inv_F + (DP * dxun * ut) * inv_F + (dxDP * un * ut) * inv_F -
                         (2 * DP * uTdxuT * un * ut) * inv_F2;
    const R dyLtn = (DP * dyut * un) * inv_F + (DP * dyun * ut) * inv_F + (dyDP * un * ut) * inv_F -
                         (2 * DP * uTdyuT * un * ut) * inv_F2;
    const R dnLtn = (DP * dnut * un) * inv_F + (DP * dnun * ut) * inv_F + (dnDP * un * ut) * inv_F -
                         (2 * DP * uTdnuT * un * ut) * inv_F2;
    const R dnLnn = ((2 * DP * dnut * ut) * inv_F + (dnDP * ut2) * inv_F - (2 * DP * uTdnuT * ut2) * inv_F2) * inv_t2;
    (void)F2;

    const R zeta_zz = Rtilde * e - 3 * pl;
    const R zeta_zT = (Rtilde * e + pl) * R(0.5);
    const R delta_pipi = (3 + Rgamma) * R(0.5);
    const R tau_pipi = div_const(4 * delta_pipi, R(3.0), R(1.0) / R(3.0));  // SourceTerms.cpp:634, 1/2 -> 0
    const R lambda_pipi = Rgamma - 1;
    const R taupiInv = R(0.2) * T / etabar;

    const R psT = pitt * sttT - 2 * pitx * stxT - 2 * pity * styT + pixx * sxxT + 2 * pixy * sxyT + piyy * syyT -
                       2 * pitn * stnT * t2 + 2 * pixn * sxnT * t2 + 2 * piyn * synT * t2 + pinn * snnT * t2 * t2;

    R beta_lPi = 0, delta_lPi = 0, beta_PiPi = 0, delta_PiPi = 0, lambda_Pipi = 0;
    if (BULK) {
        // AnisotropicDistributionFunctions.cpp:73-190 (2/9 -> 0, 3/2 -> 1, 1/3 -> 0)
        R third = R(1.0) / R(3.0) - cs2;
        if (third == R(0.0)) third = R(1.e-16);
        const R meq2 = 36 * third;
        const R z2logz = -2 * (1 + R(0.02536) * meq2);
        const R g40 = (R(poly::g0m2040DividedBym2LogZTerm<double, kFastQuot<R>>(ap)) * z2logz + R(poly::g0m2040DividedBym2Zm2Term<double, kFastQuot<R>>(ap))) /
                          meq2 +
                      R(poly::g0m2040DividedBym2ConstantTerm<double, kFastQuot<R>>(ap));
        const R g20c = R(poly::g0m2020ConstantTerm<double, kFastQuot<R>>(ap));
        const R g20 = g20c + R(poly::g0m2020Z2LogZTerm<double, kFastQuot<R>>(ap)) * z2logz + R(poly::g0m2020Z2Term<double, kFastQuot<R>>(ap)) * meq2;
        beta_lPi = 3 * g40;
        delta_lPi = g20 + g40;
        beta_PiPi = 1 - g20c;
        delta_PiPi = R(0.5) * (1 + g20c);
        lambda_Pipi = div_const(3 * R(poly::G_G1<double, kFastQuot<R>>(ap)), R(5.0), R(1.0) / R(5.0)) * (0 - cs2);
    }

    const R dPL = -(pl - p) * taupiInv + zeta_zz * zDzu - zeta_zT * thetaT - beta_lPi * Pi * zDzu -
                       delta_lPi * Pi * thetaT - Rgamma * psT;
    S[4] = dPL * inv_ut + dkvk * pl;

    S[0] = -(ttt * inv_t + t * tnn) + dkvk * (Ltt + pitt - pt) - vx * dxptHat - vy * dyptHat - vn * dnptHat +
           vx * dxLtt + vy * dyLtt + vn * dnLtt - dnLtn;
    S[1] = -ttx * inv_t - dxptHat + dkvk * pitx;
    S[2] = -tty * inv_t - dyptHat + dkvk * pity;
    // SourceTerms.cpp:686: the reference adds dnLtn twice
    S[3] = -3 * ttn * inv_t - dnptHat * inv_t2 + dkvk * (Ltn + pitn) + vx * dxLtn + vy * dyLtn + vn * (dnLtn + dnLtn) - dnLnn;
    int bad = isnan(S[4]) || isnan(S[0]);

    if (PIM) {
        // SourceTerms.cpp:725-930; the I6/I7 and lambda_piPi terms vanish with W off
        const R etaBar_TC = ((3 - Rtilde) * e - 2 * pl) * R(0.125);
        const R I1tt = 2 * ut * (pitt * Dut + pitx * Dux + pity * Duy + pitn * Dun) - 2 * z0 * (pitt * Dz0 + pitn * Dz3);
        const R I1tx = (pitt * ux + pitx * ut) * Dut + (pitx * ux + pixx * ut) * Dux + (pity * ux + pixy * ut) * Duy +
                            (pitn * ux + pixn * ut) * Dun - ((pitx * z0) * Dz0 + (pitn * ux + pixn * z0) * Dz3);
        const R I1ty = (pitt * uy + pity * ut) * Dut + (pitx * uy + pixy * ut) * Dux + (pity * uy + piyy * ut) * Duy +
                            (pitn * uy + piyn * ut) * Dun - ((pity * z0) * Dz0 + (pitn * uy + piyn * z0) * Dz3);
        const R I1tn = (pitt * un + pitn * ut) * Dut + (pitx * un + pixn * ut) * Dux + (pity * un + piyn * ut) * Duy +
                            (pitn * un + pinn * ut) * Dun - ((pitt * z3 + pitn * z0) * Dz0 + (pitn * z3 + pinn * z0) * Dz3);
        const R I1xx = 2 * ux * (pitx * Dut + pixx * Dux + pixy * Duy + pixn * Dun);
        const R I1xy = (pitx * uy + pity * ux) * Dut + (pixx * uy + pixy * ux) * Dux + (pixy * uy + piyy * ux) * Duy +
                            (pixn * uy + piyn * ux) * Dun;
        const R I1xn = (pitx * un + pitn * ux) * Dut + (pixx * un + pixn * ux) * Dux + (pixy * un + piyn * ux) * Duy +
                            (pixn * un + pinn * ux) * Dun - ((pitx * z3) * Dz0 + (pixn * z3) * Dz3);
        const R I1yy = 2 * uy * (pity * Dut + pixy * Dux + piyy * Duy + piyn * Dun);
        const R I1yn = (pity * un + pitn * uy) * Dut + (pixy * un + pixn * uy) * Dux + (piyy * un + piyn * uy) * Duy +
                            (piyn * un + pinn * uy) * Dun - ((pity * z3) * Dz0 + (piyn * z3) * Dz3);
        const R I1nn = 2 * un * (pitn * Dut + pixn * Dux + piyn * Duy + pinn * Dun) - 2 * z3 * (pitn * Dz0 + pinn * Dz3);

        const R ps2 = psT * R(0.5);
        const R I4tt = (pitt * sttT - pitx * stxT - pity * styT - t2 * pitn * stnT) - (1 - ut2 + z02) * ps2;
        const R I4tx = (pitt * stxT + pitx * sttT) * R(0.5) - (pitx * sxxT + pixx * stxT) * R(0.5) -
                            (pity * sxyT + pixy * styT) * R(0.5) - t2 * (pitn * sxnT + pixn * stnT) * R(0.5) + (ut * ux) * ps2;
        const R I4ty = (pitt * styT + pity * sttT) * R(0.5) - (pitx * sxyT + pixy * stxT) * R(0.5) -
                            (pity * syyT + piyy * styT) * R(0.5) - t2 * (pitn * synT + piyn * stnT) * R(0.5) + (ut * uy) * ps2;
        const R I4tn = (pitt * stnT + pitn * sttT) * R(0.5) - (pitx * sxnT + pixn * stxT) * R(0.5) -
                            (pity * synT + piyn * styT) * R(0.5) - t2 * (pitn * snnT + pinn * stnT) * R(0.5) +
                            (ut * un - z0z3) * ps2;
        const R I4xx = (pitx * stxT - pixx * sxxT - pixy * sxyT - t2 * pixn * sxnT) + (1 + ux * ux) * ps2;
        const R I4xy = (pitx * styT + pity * stxT) * R(0.5) - (pixx * sxyT + pixy * sxxT) * R(0.5) -
                            (pixy * syyT + piyy * sxyT) * R(0.5) - t2 * (pixn * synT + piyn * sxnT) * R(0.5) + (ux * uy) * ps2;
        const R I4xn = (pitx * stnT + pitn * stxT) * R(0.5) - (pixx * sxnT + pixn * sxxT) * R(0.5) -
                            (pixy * synT + piyn * sxyT) * R(0.5) - t2 * (pixn * snnT + pinn * sxnT) * R(0.5) + (ux * un) * ps2;
        const R I4yy = (pity * styT - pixy * sxyT - piyy * syyT - t2 * piyn * synT) + (1 + uy * uy) * ps2;
        const R I4yn = (pity * stnT + pitn * styT) * R(0.5) - (pixy * sxnT + pixn * sxyT) * R(0.5) -
                            (piyy * synT + piyn * syyT) * R(0.5) - t2 * (piyn * snnT + pinn * synT) * R(0.5) + (uy * un) * ps2;
        const R I4nn = (pitn * stnT - pixn * sxnT - piyn * synT - t2 * pinn * snnT) + (inv_t2 + un2 - z32) * ps2;

        const R c2 = delta_pipi * thetaT + lambda_pipi * zDzu;  // I2, I5 both scale pi
        const R two_eta = 2 * etaBar_TC;
        const R dpitt = two_eta * sttT - pitt * taupiInv - (I1tt - c2 * pitt + tau_pipi * I4tt) - 2 * un * t * pitn;
        const R dpitx = two_eta * stxT - pitx * taupiInv - (I1tx - c2 * pitx + tau_pipi * I4tx) - un * t * pixn;
        const R dpity = two_eta * styT - pity * taupiInv - (I1ty - c2 * pity + tau_pipi * I4ty) - un * t * piyn;
        const R dpitn = two_eta * stnT - pitn * taupiInv - (I1tn - c2 * pitn + tau_pipi * I4tn) - un * t * pinn -
                             (ut * pitn + un * pitt) * inv_t;
        const R dpixx = two_eta * sxxT - pixx * taupiInv - (I1xx - c2 * pixx + tau_pipi * I4xx);
        const R dpixy = two_eta * sxyT - pixy * taupiInv - (I1xy - c2 * pixy + tau_pipi * I4xy);
        const R dpixn = two_eta * sxnT - pixn * taupiInv - (I1xn - c2 * pixn + tau_pipi * I4xn) - (ut * pixn + un * pitx) * inv_t;
        const R dpiyy = two_eta * syyT - piyy * taupiInv - (I1yy - c2 * piyy + tau_pipi * I4yy);
        const R dpiyn = two_eta * synT - piyn * taupiInv - (I1yn - c2 * piyn + tau_pipi * I4yn) - (ut * piyn + un * pity) * inv_t;
        const R dpinn = two_eta * snnT - pinn * taupiInv - (I1nn - c2 * pinn + tau_pipi * I4nn) - 2 * (ut * pinn + un * pitn) * inv_t;
        S[5] = dpitt * inv_ut + pitt * dkvk;
        S[6] = dpitx * inv_ut + pitx * dkvk;
        S[7] = dpity * inv_ut + pity * dkvk;
        S[8] = dpitn * inv_ut + pitn * dkvk;
        S[9] = dpixx * inv_ut + pixx * dkvk;
        S[10] = dpixy * inv_ut + pixy * dkvk;
        S[11] = dpixn * inv_ut + pixn * dkvk;
        S[12] = dpiyy * inv_ut + piyy * dkvk;
        S[13] = dpiyn * inv_ut + piyn * dkvk;
        S[14] = dpinn * inv_ut + pinn * dkvk;
    }
    if (BULK) {
        // SourceTerms.cpp:1030-1042
        const R Rhat = R(poly::Rhat<double, kFastQuot<R>>(ap));
        const R bb = R(1.0) / R(3.0) - cs2;
        const R tauPiInv = 15 * bb * bb * T / zeta_over_s(eos, T);
        const R zeta_z = div_const((Rhat - Rbar0) * e3p, R(3.0), R(1.0) / R(3.0));
        const R zeta_T = div_const(-(Rbar0 + Rhat) * e3p, R(6.0), R(1.0) / R(6.0));
        const R dPi = -(div_const((1 - Rbar0) * e3p, R(3.0), R(1.0) / R(3.0)) + Pi) * tauPiInv - zeta_z * zDzu - zeta_T * thetaT -
                           beta_PiPi * Pi * zDzu - delta_PiPi * Pi * thetaT + lambda_Pipi * psT;
        S[kSlotPi] = dPi * inv_ut + Pi * dkvk;
    }
    return bad;
}

// -------------------------------------------------------------- regulator --
// FullyDiscreteKurganovTadmorScheme.cpp:524-696: e < 0 -> e = p = 1e-7,
// P_L < 0 -> 1e-7, then pi^{mu nu} *= tanh(rho)/rho (xi0 = rho_max = 1).
// maps (optional, 11 values, written only with shear): the applied factor and
// each criterion's own factor tanh(a)/a (1 below 1e-7) in the order
// magnitude, trace, u-orthogonality x4, z-orthogonality x4 (:666-693).
template <int PHYS, typename R>
VAH_HD void regulate(R t, R &e, R &p, R *q, const R *u, R *maps = nullptr) {
    if (e < R(0.0)) {
        e = R(1.e-7);
        p = R(1.e-7);
    }
    if (q[kSlotPL] < R(0.0)) q[kSlotPL] = R(1.e-7);
    if (!Phys<PHYS>::PIMUNU) return;
    const R pl = q[kSlotPL];
    double ap[9];  // FP64 closure fit, as in cell_sources
    ap[0] = 1.0;
    ap[1] = kFastQuot<R> ? quotient_fast((double)pl, (double)e) : (double)pl / (double)e;
#pragma unroll
    for (int k = 2; k < 9; ++k) ap[k] = ap[k - 1] * ap[1];
    const R ptHat = (e - pl - R(poly::Rbar0<double, kFastQuot<R>>(ap)) * (e - 3 * p)) * R(0.5);
    const R pitt = q[5], pitx = q[6], pity = q[7], pitn = q[8], pixx = q[9];
    const R pixy = q[10], pixn = q[11], piyy = q[12], piyn = q[13], pinn = q[14];
    const R ut = u[0], ux = u[1], uy = u[2], un = u[3];
    const R inv_sF = rsqrt_r(1 + (ux * ux + uy * uy));
    const R z0 = t * un * inv_sF;
    const R z3 = ut / t * inv_sF;
    const R t2 = t * t;
    const R sTrsTrs = sqrt(fabs(e * e + pl * pl + 2 * ptHat * ptHat));
    const R pipi = pitt * pitt - 2 * pitx * pitx - 2 * pity * pity + pixx * pixx + 2 * pixy * pixy + piyy * piyy -
                        2 * pitn * pitn * t2 + 2 * pixn * pixn * t2 + 2 * piyn * piyn * t2 + pinn * pinn * t2 * t2;
    const R spipi = sqrt(fabs(pipi));
    R rho = spipi / sTrsTrs;
    const R den = spipi;
    const R num[9] = {pitt - pixx - piyy - pinn * t2,
                           -pitn * t2 * un + pitt * ut - pitx * ux - pity * uy,
                           -pixn * t2 * un + pitx * ut - pixx * ux - pixy * uy,
                           -piyn * t2 * un + pity * ut - pixy * ux - piyy * uy,
                           -pinn * t2 * un + pitn * ut - pixn * ux - piyn * uy,
                           z0 * pitt - t2 * z3 * pitn,
                           z0 * pitx - t2 * z3 * pixn,
                           z0 * pity - t2 * z3 * piyn,
                           z0 * pitn - t2 * z3 * pinn};
    R cand[9];
    if (maps) {  // every ratio is reported
#pragma unroll
        for (int m = 0; m < 9; ++m) {
            cand[m] = num[m] / den;
            if (cand[m] > rho) rho = cand[m];
        }
    } else {
        // rho = max(rho, num[m] / den): den = sqrt(|pi.pi|) >= 0 and a rounded
        // division by it is monotone, so the largest ratio is the largest
        // numerator divided once -- the same value bit for bit, NaN ratios
        // (0/0, NaN numerators) ignored as the comparisons ignore them, and
        // den = 0 giving +-inf as the nine quotients would.
        R top = -INFINITY;
#pragma unroll
        for (int m = 0; m < 9; ++m)
            if (num[m] > top) top = num[m];
        const R c = top / den;
        if (c > rho) rho = c;
    }
    R fac = tanh(rho) / rho;
    if (rho < R(1.e-7)) fac = R(1.0);
#pragma unroll
    for (int n = 5; n < 15; ++n) q[n] *= fac;
    if (maps) {
        const R a1 = spipi / sTrsTrs;
        maps[0] = fac;
        maps[1] = a1 < R(1.e-7) ? R(1.0) : tanh(a1) / a1;
        for (int m = 0; m < 9; ++m) maps[2 + m] = cand[m] < R(1.e-7) ? R(1.0) : tanh(cand[m]) / cand[m];
    }
}

}  // namespace vah
