// vah_tile_cell.cuh -- the arithmetic of the FP32 form, shared by the
// TMA-tiled stage kernel (vah_tile.cuh) and its host build (tests/hostcheck):
// the face flux from an accessor of the conserved fields, and the cell update.
// State and arithmetic in FP32; the Newton inversions in FP64.
#pragma once

#include "vah_physics.cuh"

// The face evaluation is inlined: the tile kernel calls it from one place (a
// loop over the face jobs of a tile), so one copy of its code sits in the
// kernel and no call saves registers around it.
#if defined(__CUDACC__)
#define VAH_TILE_FACE __host__ __device__ __forceinline__
#else
#define VAH_TILE_FACE inline
#endif

namespace vah {

// Two FP32 lanes per instruction: sm_100's paired FFMA2 / FMUL2, each lane
// rounded as its scalar operation; on the host one operation per lane.
struct Pair {
    float a, b;
};
VAH_HD Pair pfma(Pair x, Pair y, Pair z) {
#ifdef __CUDA_ARCH__
    const float2 r = __ffma2_rn(make_float2(x.a, x.b), make_float2(y.a, y.b), make_float2(z.a, z.b));
    return {r.x, r.y};
#else
    return {fmaf(x.a, y.a, z.a), fmaf(x.b, y.b, z.b)};
#endif
}
VAH_HD Pair pmul(Pair x, Pair y) {
#ifdef __CUDA_ARCH__
    const float2 r = __fmul2_rn(make_float2(x.a, x.b), make_float2(y.a, y.b));
    return {r.x, r.y};
#else
    return {x.a * y.a, x.b * y.b};
#endif
}
// x - y, rounded once (y times -1 is exact)
VAH_HD Pair psub(Pair x, Pair y) { return pfma(y, Pair{-1.0f, -1.0f}, x); }

// approx_derivative of two fields at once: the differences and products
// paired, the minima and sign tests per lane; the same values bit for bit.
VAH_HD Pair approx_derivative2(Pair x, Pair y, Pair z) {
    const Pair dl = psub(y, x), dr = psub(z, y);
    const Pair c = pmul(psub(z, x), Pair{0.5f, 0.5f});
    const Pair mn = pmul(Pair{1.1f, 1.1f}, Pair{fminf(fabsf(dl.a), fabsf(dr.a)), fminf(fabsf(dl.b), fabsf(dr.b))});
    auto pick = [](float l, float r, float cc, float mm) {
        const float m = fminf(mm, fabsf(cc));
        const bool neg = l < 0.0f;
        return neg == (r < 0.0f) ? (neg ? -m : m) : 0.0f;
    };
    return {pick(dl.a, dr.a, c.a, mn.a), pick(dl.b, dr.b, c.b, mn.b)};
}

// --------------------------------------------- the FP32 form's cell algebra --
// Host-and-device code: the kernel runs it on the shared-memory box, and the
// host build (tests/hostcheck) on plain arrays, through accessors
// q(n, index) of the conserved fields.

// The shared-memory box: field n at n * BOXN.
template <int BOXN>
struct BoxQ {
    const float *s;
    VAH_HD float operator()(int n, long long i) const { return s[n * BOXN + i]; }
};

// One array per field.
struct ArrQ {
    const float *const *f;
    VAH_HD float operator()(int n, long long i) const { return f[n][i]; }
};

// Kurganov-Tadmor flux through the face between cells L and L + st
// (SemiDiscreteKurganovTadmorScheme.cpp:13-57, FluxLimiter.cpp:28-33): the
// states reconstructed in FP32, inverted in FP64 from the guess uT (the left
// cell's |u_T|; the setup's and the velocities' divisions through
// quotient_fast), H[n hs] = wR qR + wL qL in FP32 (hs: the stride of the
// destination, e.g. a shared face buffer). Returns the number of inversions
// that fell back; bit 8 flags a NaN (ePrev: the left cell's e).
template <int PHYS, typename QA>
VAH_TILE_FACE unsigned tile_face(const QA q, long long L, long long st, int dir, double t, double ePrev, double uT,
                                 float *H, int hs) {
    constexpr int NQ = Phys<PHYS>::NQ;
    float qR[NQ], qL[NQ];
#pragma unroll
    for (int n = 0; n + 1 < NQ; n += 2) {  // two fields at a time
        const Pair qm{q(n, L - st), q(n + 1, L - st)}, q0{q(n, L), q(n + 1, L)};
        const Pair qp{q(n, L + st), q(n + 1, L + st)}, qpp{q(n, L + 2 * st), q(n + 1, L + 2 * st)};
        const Pair r = pfma(approx_derivative2(q0, qp, qpp), Pair{-0.5f, -0.5f}, qp);
        const Pair l = pfma(approx_derivative2(qm, q0, qp), Pair{0.5f, 0.5f}, q0);
        qR[n] = r.a;
        qR[n + 1] = r.b;
        qL[n] = l.a;
        qL[n + 1] = l.b;
    }
    if (NQ % 2) {
        constexpr int n = NQ - 1;
        const float qm = q(n, L - st), q0 = q(n, L), qp = q(n, L + st), qpp = q(n, L + 2 * st);
        qR[n] = fmaf(approx_derivative(q0, qp, qpp), -0.5f, qp);
        qL[n] = fmaf(approx_derivative(qm, q0, qp), 0.5f, q0);
    }
    double dR[16], dL[16];
#pragma unroll
    for (int n = 0; n < 16; ++n) {
        dR[n] = n < NQ ? (double)qR[n] : 0.0;
        dL[n] = n < NQ ? (double)qL[n] : 0.0;
    }
    InvSetup sR, sL;
    invert_setup<PHYS, true>(t, dR, sR);
    invert_setup<PHYS, true>(t, dL, sL);
    double uR, uL, vR = 0.0, vL = 0.0;
    int nR, nL;
    newton_uT2(sR, sL, uT, uT, uR, uL, nR, nL);
    const int stR = nR != 0 ? (isnan(ePrev) ? 2 : 1) : face_velocity_of<true>(sR, uR, dir, &vR);
    const int stL = nL != 0 ? (isnan(ePrev) ? 2 : 1) : face_velocity_of<true>(sL, uL, dir, &vL);
    const double a = fmax(fabs(vL), fabs(vR));
    const float wR = (float)(0.5 * (vR - a)), wL = (float)(0.5 * (vL + a));
#pragma unroll
    for (int n = 0; n + 1 < NQ; n += 2) {  // wR qR + wL qL, two fields at a time
        const Pair h = pfma(Pair{wR, wR}, Pair{qR[n], qR[n + 1]}, pmul(Pair{wL, wL}, Pair{qL[n], qL[n + 1]}));
        H[n * hs] = h.a;
        H[(n + 1) * hs] = h.b;
    }
    if (NQ % 2) H[(NQ - 1) * hs] = fmaf(wR, qR[NQ - 1], wL * qL[NQ - 1]);
    return (stR != 0) + (stL != 0) + ((stR == 2 || stL == 2) ? 256u : 0u);
}

// Stage-input primitives: e, p, u read at the cell and its +-1 neighbours
// (index pi, strides psy, psz: the shared-memory box on the device, the
// field arrays on the host), and at the cell only (global index s) the
// previous stage's u and the inversion's guess u.
struct TilePrims {
    const float *E, *P, *U[4];
    long long pi, psy, psz;
    const float *UP[4], *G[4];
};

// The explicit part of a cell's stage (eulerStepKernelSource and the axis
// sources): q: the stage-input conserved fields at box index b (strides bsy,
// bsz); pr: the primitives; s: the cell's global index; flux[n]: the flux
// differences dt/h (H(-1/2) - H(+1/2)) summed over the axes. Writes the
// updated conserved values to val and the cell's e (the inversion's fallback
// energy) to e_prev; sets bad when a source is NaN. The last part of the
// stage that reads q and the primitives around the cell.
template <int PHYS, bool IS3D, typename QA>
VAH_HD void tile_cell_explicit(const QA &q, long long b, long long bsy, long long bsz, const TilePrims &pr,
                               long long s, const float *flux, const Eos &eos, double t_src, double dt, double dx,
                               double dy, double dz, double etabar, float *val, float &e_prev, int &bad) {
    constexpr int NQ = Phys<PHYS>::NQ;
    float qc[NQ];
#pragma unroll
    for (int n = 0; n < NQ; ++n) qc[n] = q(n, b);
    const float fx = (float)(0.5 / dx), fy = (float)(0.5 / dy), fz = (float)(0.5 / dz);
    const float *E = pr.E, *PP = pr.P, *UT = pr.U[0], *UX = pr.U[1], *UY = pr.U[2], *UN = pr.U[3];
    const long long c = pr.pi, sy = pr.psy, sz = pr.psz;
    CellGradT<float> g;
    g.e = E[c];
    g.p = PP[c];
    g.ut = UT[c];
    g.ux = UX[c];
    g.uy = UY[c];
    g.un = UN[c];
    g.utp = pr.UP[0][s];
    g.uxp = pr.UP[1][s];
    g.uyp = pr.UP[2][s];
    g.unp = pr.UP[3][s];
#define VAH_TCD(A, off, f) (((A)[c + (off)] - (A)[c - (off)]) * (f))
    g.dxut = VAH_TCD(UT, 1, fx); g.dxux = VAH_TCD(UX, 1, fx); g.dxuy = VAH_TCD(UY, 1, fx); g.dxun = VAH_TCD(UN, 1, fx);
    g.dyut = VAH_TCD(UT, sy, fy); g.dyux = VAH_TCD(UX, sy, fy); g.dyuy = VAH_TCD(UY, sy, fy); g.dyun = VAH_TCD(UN, sy, fy);
    g.dxp = VAH_TCD(PP, 1, fx); g.dyp = VAH_TCD(PP, sy, fy);
    g.dxe = VAH_TCD(E, 1, fx); g.dye = VAH_TCD(E, sy, fy);
    g.dxpl = (q(kSlotPL, b + 1) - q(kSlotPL, b - 1)) * fx;
    g.dypl = (q(kSlotPL, b + bsy) - q(kSlotPL, b - bsy)) * fy;
    if (IS3D) {
        g.dnut = VAH_TCD(UT, sz, fz); g.dnux = VAH_TCD(UX, sz, fz); g.dnuy = VAH_TCD(UY, sz, fz); g.dnun = VAH_TCD(UN, sz, fz);
        g.dnp = VAH_TCD(PP, sz, fz); g.dne = VAH_TCD(E, sz, fz);
        g.dnpl = (q(kSlotPL, b + bsz) - q(kSlotPL, b - bsz)) * fz;
    } else {
        g.dnut = g.dnux = g.dnuy = g.dnun = 0.0f;
        g.dnp = g.dne = g.dnpl = 0.0f;
    }
#undef VAH_TCD
    const StepConstsT<float> k = step_consts((float)t_src, (float)dt, (float)etabar);
    float Sv[NQ];
    bad = cell_sources<PHYS>(eos, qc, g, k, Sv);
    const float dtf = (float)dt;
#pragma unroll
    for (int n = 0; n < NQ; ++n) val[n] = qc[n] + dtf * Sv[n] + flux[n];
    if (Phys<PHYS>::PIMUNU) {  // pi / Pi gradient sources along each axis (SourceTerms.cpp:46-176)
        const float ucomp[3] = {g.ux, g.uy, g.un};
        const float fh[3] = {fx, fy, fz};
        const long long sts[3] = {1, bsy, bsz};
#pragma unroll
        for (int dir = 0; dir < (IS3D ? 3 : 2); ++dir) {
            float dd[16];
#pragma unroll
            for (int n = 5; n < NQ; ++n) dd[n] = (q(n, b + sts[dir]) - q(n, b - sts[dir])) * fh[dir];
            float Sa[4];
            axis_sources<PHYS>(dd, dir, ucomp[dir], g.ut, (float)t_src, Sa);
#pragma unroll
            for (int n = 0; n < 4; ++n) val[n] += dtf * Sa[n];
        }
    }
    e_prev = g.e;
}

// The rest of the cell's stage ([the convex combination],
// setInferredVariablesKernel, the regulator) from tile_cell_explicit's
// results, reading nothing around the cell: qavg(n, s) = q^n (stage 2), the
// Newton guess from pr.G at s. Writes the new conserved values (val), e, p,
// u; returns the inversion's status (0 converged, 1 fallback, 2 NaN).
template <int PHYS, typename QV>
VAH_HD int tile_cell_invert(const TilePrims &pr, long long s, const QV &qavg, bool stage2, const Eos &eos,
                            double t_inv, float e_prev, float *val, float &e, float &p, float *u, float *rmap) {
    constexpr int NQ = Phys<PHYS>::NQ;
    if (stage2) {  // Q = (q^n + Q*) / 2
#pragma unroll
        for (int n = 0; n < NQ; ++n) val[n] = (val[n] + qavg(n, s)) * 0.5f;
    }
    // FP64 inversion from the previous-stage guess (EnergyMomentumTensor.cpp:74-197);
    // p = EoS(e) in FP32
    const double gx = (double)pr.G[1][s], gy = (double)pr.G[2][s];
    double qd[16], prim[6];
#pragma unroll
    for (int n = 0; n < 16; ++n) qd[n] = n < NQ ? (double)val[n] : 0.0;
    const int st = invert<PHYS, true>(eos, t_inv, qd, (double)e_prev, sqrt(fabs(gx * gx + gy * gy)), prim);
    e = (float)prim[0];
    p = (float)prim[1];
    for (int m = 0; m < 4; ++m) u[m] = (float)prim[2 + m];
    regulate<PHYS>((float)t_inv, e, p, val, u, rmap);
    return st;
}

// The whole cell part of a stage (eulerStepKernelSource, the axis sources,
// [the convex combination], setInferredVariablesKernel, the regulator), as
// the two parts above.
template <int PHYS, bool IS3D, typename QA, typename QV>
VAH_HD int tile_cell(const QA &q, long long b, long long bsy, long long bsz, const TilePrims &pr, long long s,
                     const float *flux, const QV &qavg, bool stage2, const Eos &eos, double t_src, double t_inv,
                     double dt, double dx, double dy, double dz, double etabar, float *val, float &e, float &p,
                     float *u, float *rmap, int &bad) {
    float e_prev;
    tile_cell_explicit<PHYS, IS3D>(q, b, bsy, bsz, pr, s, flux, eos, t_src, dt, dx, dy, dz, etabar, val, e_prev, bad);
    return tile_cell_invert<PHYS>(pr, s, qavg, stage2, eos, t_inv, e_prev, val, e, p, u, rmap);
}


}  // namespace vah
