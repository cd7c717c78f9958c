// vah_stage.cuh -- one RK stage of one interior cell, fused.
//
// The reference runs each RK2 stage as separate full-grid sweeps
// (FullyDiscreteKurganovTadmorScheme.cpp:761-772 and :777-789): source Euler
// step, X/Y/Z flux sweeps, [convex combination], inversion, regulator, ghost
// fill. Every one of them after the flux sweeps reads and writes only its own
// cell, so one thread can carry a cell through the whole stage provided the
// stage inputs (q, u, e, p) and outputs live in different buffers:
//   stage 1: q,  u,  e0,p0 (+ up centre)  ->  qS, uS, e1,p1
//   stage 2: qS, uS, e1,p1 (+ u centre, q centre) -> q (in place), u', e0,p0
// Ghost layers of the outputs are written by the boundary cells themselves
// (faces only: edges and corners are never read by an axis-aligned stencil).
#pragma once

#include "vah_physics.cuh"

namespace vah {

template <typename S>
struct StageArgs {
    int nx, ny, nz;
    int k0, k1;       // face/cell split launches: the interior planes [k0, k1) they update (all: 0, nz)
    int ncx, ncy;
    long long plane;  // ncx * ncy
    double t_src;     // time of the Euler step (stage 1: t, stage 2: t + dt)
    // derived per launch by finish_args: the sources' constants at t_src, dt / h and 1 / (2 h) per axis
    StepConsts ksrc;
    double c_h[3], inv2h[3];
    double t_inv;     // time of the inversion/regulator (t + dt)
    double dt, dx, dy, dz, etabar;
    int stage2;       // 1: convex combination with qavg before inversion
    int shared_faces; // unused by the per-cell path
    int zghosts;      // 1: boundary cells also store the eta ghost layers. On 2+1D lattices no stencil
                      // reads them, so the event and batch paths leave them to a fill when a caller reads
                      // fields with ghosts (and keep them when validity diagnostics, which read them, run)
    const S *qin[16];
    const S *uin[4];
    const S *upin[4];   // previous-stage velocity (centre only)
    const S *guess[4];  // Newton guess of the cell inversion (centre only)
    const S *ein, *pin;
    const S *qavg[16];  // stage 2: q^n (centre only)
    S *qout[16];
    S *uout[4];
    S *eout, *pout;
    Eos eos;
    unsigned long long *counters;  // [face fallbacks, cell fallbacks, NaN cells]
    unsigned char *fallback;       // optional: per ghosted cell, 1 where this stage's inversion fell back
    double *regmap[11];            // optional (validity diagnostics): the regulator's factors per ghosted cell
    // optional freeze-out crossing test at the end of a step (stage 2): per
    // ghosted cell 1 while e > e_freeze; crossings counted [down, up]
    unsigned char *hot;
    double e_freeze;
    unsigned long long *crossings;
    // face/cell split: flux through the face at +1/2 of ghosted cell s along
    // axis d, field n, as cell s evaluates it (H) and as cell s+1 does (HR,
    // reference face semantics only); scratch of ncell entries per field
    S *H[3][16];
    S *HR[3][16];
    // optional (FP64 event launches): the x flux difference of each interior
    // cell, H(-1/2) - H(+1/2) as the cell evaluates both faces, written by the
    // x face launch (face_x_diff_kernel) and read by the cell launch instead of
    // H[0] / HR[0]; null: the cell launch differences H[0] / HR[0] itself
    S *Dx[16];
};

VAH_HD void count_add(unsigned long long *c, unsigned long long v) {
#ifdef __CUDA_ARCH__
    atomicAdd(c, v);
#else
    *c += v;
#endif
}

// The launch constants derived from t_src, dt, etabar and the spacings; to be
// called once the arguments are filled.
template <typename S>
VAH_HD void finish_args(StageArgs<S> &a) {
    a.ksrc = step_consts(a.t_src, a.dt, a.etabar);
    const double h[3] = {a.dx, a.dy, a.dz};
    for (int d = 0; d < 3; ++d) {
        a.c_h[d] = a.dt / h[d];
        a.inv2h[d] = 1 / h[d] / 2;
    }
}

template <typename S>
VAH_HD double ld(const S *p, long long i) {
    return (double)ldg(p + i);
}

// Face values are read once, by the cell launch: loaded with the streaming
// (evict-first) cache policy, so that they do not push the state's neighbour
// reuse out of L1 and L2 (cell launch 3% faster; streaming stores in the face
// launches cost those 2%, so they store normally).
template <typename S>
VAH_HD double ld_stream(const S *p, long long i) {
#ifdef __CUDA_ARCH__
    return (double)__ldcs(p + i);
#else
    return (double)p[i];
#endif
}

// Gradients and centre values the source terms need (SourceTerms.cpp:239-280, 484-486).
template <typename S, bool IS3D>
VAH_HD void load_cell_grad(const StageArgs<S> &a, long long s, CellGrad &g) {
    const long long sx = 1, sy = a.ncx, sz = a.plane;
    const double fx = a.inv2h[0], fy = a.inv2h[1], fz = a.inv2h[2];
    const S *UT = a.uin[0], *UX = a.uin[1], *UY = a.uin[2], *UN = a.uin[3];
    g.e = ld(a.ein, s);
    g.p = ld(a.pin, s);
    g.ut = ld(UT, s);
    g.ux = ld(UX, s);
    g.uy = ld(UY, s);
    g.un = ld(UN, s);
    g.utp = ld(a.upin[0], s);
    g.uxp = ld(a.upin[1], s);
    g.uyp = ld(a.upin[2], s);
    g.unp = ld(a.upin[3], s);
#define VAH_CD(P, off, f) ((ld(P, s + (off)) - ld(P, s - (off))) * (f))
    g.dxut = VAH_CD(UT, sx, fx); g.dxux = VAH_CD(UX, sx, fx); g.dxuy = VAH_CD(UY, sx, fx); g.dxun = VAH_CD(UN, sx, fx);
    g.dyut = VAH_CD(UT, sy, fy); g.dyux = VAH_CD(UX, sy, fy); g.dyuy = VAH_CD(UY, sy, fy); g.dyun = VAH_CD(UN, sy, fy);
    g.dxp = VAH_CD(a.pin, sx, fx); g.dyp = VAH_CD(a.pin, sy, fy);
    g.dxe = VAH_CD(a.ein, sx, fx); g.dye = VAH_CD(a.ein, sy, fy);
    g.dxpl = VAH_CD(a.qin[kSlotPL], sx, fx); g.dypl = VAH_CD(a.qin[kSlotPL], sy, fy);
    if (IS3D) {
        g.dnut = VAH_CD(UT, sz, fz); g.dnux = VAH_CD(UX, sz, fz); g.dnuy = VAH_CD(UY, sz, fz); g.dnun = VAH_CD(UN, sz, fz);
        g.dnp = VAH_CD(a.pin, sz, fz); g.dne = VAH_CD(a.ein, sz, fz); g.dnpl = VAH_CD(a.qin[kSlotPL], sz, fz);
    } else {
        // one eta layer: the ghost layers copy it, so every eta difference is 0
        g.dnut = g.dnux = g.dnuy = g.dnun = 0.0;
        g.dnp = g.dne = g.dnpl = 0.0;
    }
#undef VAH_CD
}

// Flux difference and axis sources along one axis, added to val
// (eulerStepKernelX/Y/Z, FullyDiscreteKurganovTadmorScheme.cpp:124-461):
// val += dt * ((H(-1/2) - H(+1/2)) / h + S_axis).
template <typename S, int PHYS>
VAH_HD unsigned axis_update(const StageArgs<S> &a, long long s, int dir, long long st, double h, const double *qc,
                            double ePrev, double uT, double ucomp, double ut, double *val) {
    constexpr int NQ = Phys<PHYS>::NQ;
    double qR[NQ], qL[NQ], H[NQ];
    unsigned fails = 0;
    const double c = a.dt / h;
    // face at +1/2: right state from cell +1, left state from this cell
#pragma unroll
    for (int n = 0; n < NQ; ++n) {
        const double qm = ld(a.qin[n], s - st), qp = ld(a.qin[n], s + st), qpp = ld(a.qin[n], s + 2 * st);
        qR[n] = qp - approx_derivative(qc[n], qp, qpp) * 0.5;
        qL[n] = qc[n] + approx_derivative(qm, qc[n], qp) * 0.5;
    }
    fails += face_flux<PHYS>(a.t_src, qR, qL, dir, ePrev, uT, H);
#pragma unroll
    for (int n = 0; n < NQ; ++n) val[n] -= c * H[n];
    // face at -1/2: right state from this cell, left state from cell -1
#pragma unroll
    for (int n = 0; n < NQ; ++n) {
        const double qmm = ld(a.qin[n], s - 2 * st), qm = ld(a.qin[n], s - st), qp = ld(a.qin[n], s + st);
        qR[n] = qc[n] - approx_derivative(qm, qc[n], qp) * 0.5;
        qL[n] = qm + approx_derivative(qmm, qm, qc[n]) * 0.5;
    }
    fails += face_flux<PHYS>(a.t_src, qR, qL, dir, ePrev, uT, H);
#pragma unroll
    for (int n = 0; n < NQ; ++n) val[n] += c * H[n];
    if (Phys<PHYS>::PIMUNU) {
        double d[16];
        const double f = 1 / h / 2;
#pragma unroll
        for (int n = 5; n < NQ; ++n) d[n] = (ld(a.qin[n], s + st) - ld(a.qin[n], s - st)) * f;
        double Sa[4];
        axis_sources<PHYS>(d, dir, ucomp, ut, a.t_src, Sa);
#pragma unroll
        for (int n = 0; n < 4; ++n) val[n] += a.dt * Sa[n];
    }
    return fails;
}

template <typename S>
VAH_HD void store_cell(const StageArgs<S> &a, long long s, int NQ, const double *val, const double *u, double e,
                       double p) {
    for (int n = 0; n < NQ; ++n) a.qout[n][s] = (S)val[n];
    for (int m = 0; m < 4; ++m) a.uout[m][s] = (S)u[m];
    a.eout[s] = (S)e;
    a.pout[s] = (S)p;
}

// One interior cell (i, j, k in ghosted coordinates, 2 <= i < nx + 2, ...).
template <typename S, int PHYS, bool IS3D>
VAH_HD void stage_cell(const StageArgs<S> &a, int i, int j, int k) {
    constexpr int NQ = Phys<PHYS>::NQ;
    const long long s = i + (long long)a.ncx * j + a.plane * k;
    double qc[NQ], val[NQ], Sv[NQ];
#pragma unroll
    for (int n = 0; n < NQ; ++n) qc[n] = ld(a.qin[n], s);

    // eulerStepKernelSource: q + dt S (FullyDiscreteKurganovTadmorScheme.cpp:43-122)
    CellGrad g;
    load_cell_grad<S, IS3D>(a, s, g);
    int bad = cell_sources<PHYS>(a.eos, qc, g, a.ksrc, Sv);
#pragma unroll
    for (int n = 0; n < NQ; ++n) val[n] = qc[n] + a.dt * Sv[n];

    // X, Y, Z flux sweeps; Newton guess = |u_T| of this cell, fallback = its e
    const double uT = sqrt(fabs(g.ux * g.ux + g.uy * g.uy));
    unsigned fails = 0;
    fails += axis_update<S, PHYS>(a, s, 0, 1, a.dx, qc, g.e, uT, g.ux, g.ut, val);
    fails += axis_update<S, PHYS>(a, s, 1, a.ncx, a.dy, qc, g.e, uT, g.uy, g.ut, val);
    if (IS3D) fails += axis_update<S, PHYS>(a, s, 2, a.plane, a.dz, qc, g.e, uT, g.un, g.ut, val);

    // stage 2: Q = (q + Q) / 2 (convexCombinationEulerStepKernel, :465-521)
    if (a.stage2) {
#pragma unroll
        for (int n = 0; n < NQ; ++n) val[n] = (val[n] + ld(a.qavg[n], s)) * 0.5;
    }

    // inversion (setInferredVariablesKernel, EnergyMomentumTensor.cpp:199-268)
    const double gx = ld(a.guess[1], s), gy = ld(a.guess[2], s);
    double prim[6];
    double qfull[16];
#pragma unroll
    for (int n = 0; n < 16; ++n) qfull[n] = n < NQ ? val[n] : 0.0;
    const int st = invert<PHYS>(a.eos, a.t_inv, qfull, g.e, sqrt(fabs(gx * gx + gy * gy)), prim);
    double e = prim[0], p = prim[1];
    double u[4] = {prim[2], prim[3], prim[4], prim[5]};
    double rmap[11];
    regulate<PHYS>(a.t_inv, e, p, val, u, a.regmap[0] ? rmap : nullptr);
    if (a.regmap[0] && Phys<PHYS>::PIMUNU)
        for (int m = 0; m < 11; ++m) a.regmap[m][s] = rmap[m];

    if ((fails & 255u) && a.counters) count_add(a.counters + 0, fails & 255u);
    if (st != 0 && a.counters) count_add(a.counters + 1, 1ull);
    if ((bad || st == 2 || (fails >> 8)) && a.counters) count_add(a.counters + 2, 1ull);
    if (a.fallback) a.fallback[s] = st != 0;

    store_cell(a, s, NQ, val, u, e, p);
    // face ghost layers (setGhostCellsKernelI/J/K, DynamicalVariables.cpp:400-489)
    const long long sy = a.ncx, sz = a.plane;
    if (i == 2) { store_cell(a, s - 1, NQ, val, u, e, p); store_cell(a, s - 2, NQ, val, u, e, p); }
    if (i == a.nx + 1) { store_cell(a, s + 1, NQ, val, u, e, p); store_cell(a, s + 2, NQ, val, u, e, p); }
    if (j == 2) { store_cell(a, s - sy, NQ, val, u, e, p); store_cell(a, s - 2 * sy, NQ, val, u, e, p); }
    if (j == a.ny + 1) { store_cell(a, s + sy, NQ, val, u, e, p); store_cell(a, s + 2 * sy, NQ, val, u, e, p); }
    if (a.zghosts) {
        if (k == 2) { store_cell(a, s - sz, NQ, val, u, e, p); store_cell(a, s - 2 * sz, NQ, val, u, e, p); }
        if (k == a.nz + 1) { store_cell(a, s + sz, NQ, val, u, e, p); store_cell(a, s + 2 * sz, NQ, val, u, e, p); }
    }
}

// ------------------------------------------------------- face/cell split --
// The face fluxes of a stage are computed by their own launch (face_compute)
// into scratch buffers, and the cell launch (cell_compute) takes flux
// differences from them. Two face modes:
//   EXACT (reference semantics, VAH_FLUX_PER_CELL): the reference evaluates
//     each face twice, once from each neighbour, with that neighbour's Newton
//     guess and fallback energy (FullyDiscreteKurganovTadmorScheme.cpp:179,183);
//     face_compute does the same, sharing the reconstruction: H[d][n][s] is
//     the face at +1/2 of cell s as cell s evaluates it, HR[d][n][s] as cell
//     s+1 evaluates it.
//   shared (VAH_FLUX_SHARED): one evaluation per face with the left cell's
//     guess and energy. Converged inversions agree with the reference to the
//     solver tolerance squared; where the reference's inversion falls back
//     (dilute edges), shared faces do not reproduce it.

// Face at +1/2 of ghosted cell s along axis dir (stride st). left_in /
// right_in: whether the cells on either side are interior cells. With
// reference faces only interior cells' evaluations are needed (and counted,
// as the reference counts them): the evaluation with a ghost cell's guess at
// the first and last face of a row is skipped.
// The two reconstructed states at the face at +1/2 of ghosted cell s (stride st).
template <typename S, int PHYS>
VAH_HD void face_states(const StageArgs<S> &a, long long s, long long st, double *qR, double *qL) {
    constexpr int NQ = Phys<PHYS>::NQ;
#pragma unroll
    for (int n = 0; n < NQ; ++n) {
        const double qm = ld(a.qin[n], s - st), q0 = ld(a.qin[n], s), qp = ld(a.qin[n], s + st),
                     qpp = ld(a.qin[n], s + 2 * st);
        qR[n] = qp - approx_derivative(q0, qp, qpp) * 0.5;
        qL[n] = q0 + approx_derivative(qm, q0, qp) * 0.5;
    }
}

template <typename S, int PHYS, bool EXACT>
VAH_HD unsigned face_compute(const StageArgs<S> &a, long long s, int dir, long long st, bool left_in = true,
                             bool right_in = true) {
    constexpr int NQ = Phys<PHYS>::NQ;
    double qR[NQ], qL[NQ], H[NQ];
    face_states<S, PHYS>(a, s, st, qR, qL);
    InvSetup sR, sL;  // set up once, inverted from one guess (shared) or both (reference faces)
    invert_setup<PHYS>(a.t_src, qR, sR);
    invert_setup<PHYS>(a.t_src, qL, sL);
    unsigned fails = 0;
    if (!EXACT || left_in) {
        const double ux = ld(a.uin[1], s), uy = ld(a.uin[2], s);
        fails += face_flux_setup<PHYS>(sR, sL, qR, qL, dir, ld(a.ein, s), sqrt(fabs(ux * ux + uy * uy)), H);
#pragma unroll
        for (int n = 0; n < NQ; ++n) a.H[dir][n][s] = (S)H[n];
    }
    if (EXACT && right_in) {
        const double vx = ld(a.uin[1], s + st), vy = ld(a.uin[2], s + st);
        fails += face_flux_setup<PHYS>(sR, sL, qR, qL, dir, ld(a.ein, s + st), sqrt(fabs(vx * vx + vy * vy)), H);
#pragma unroll
        for (int n = 0; n < NQ; ++n) a.HR[dir][n][s] = (S)H[n];
    }
    return fails;
}

// One interior cell of the split path.
template <typename S, int PHYS, bool IS3D, bool EXACT>
VAH_HD void cell_compute(const StageArgs<S> &a, int i, int j, int k) {
    constexpr int NQ = Phys<PHYS>::NQ;
    const long long s = i + (long long)a.ncx * j + a.plane * k;
    double qc[NQ], val[NQ], Sv[NQ];
#pragma unroll
    for (int n = 0; n < NQ; ++n) qc[n] = ld(a.qin[n], s);
    CellGrad g;
    load_cell_grad<S, IS3D>(a, s, g);
    int bad = cell_sources<PHYS>(a.eos, qc, g, a.ksrc, Sv);
#pragma unroll
    for (int n = 0; n < NQ; ++n) val[n] = qc[n] + a.dt * Sv[n];
    const long long strides[3] = {1, a.ncx, a.plane};
    const double hs[3] = {a.dx, a.dy, a.dz};
    const double ucomp[3] = {g.ux, g.uy, g.un};
#pragma unroll
    for (int dir = 0; dir < (IS3D ? 3 : 2); ++dir) {
        const long long st = strides[dir];
        const double c = a.c_h[dir];
        const S *const *Hm = EXACT ? a.HR[dir] : a.H[dir];  // face -1/2 as this cell evaluates it
        if (dir == 0 && a.Dx[0]) {
#pragma unroll
            for (int n = 0; n < NQ; ++n) val[n] += c * ld_stream(a.Dx[n], s);
        } else {
#pragma unroll
            for (int n = 0; n < NQ; ++n) val[n] += c * (ld_stream(Hm[n], s - st) - ld_stream(a.H[dir][n], s));
        }
        if (Phys<PHYS>::PIMUNU) {
            double d[16];
            const double f = a.inv2h[dir];
#pragma unroll
            for (int n = 5; n < NQ; ++n) d[n] = (ld(a.qin[n], s + st) - ld(a.qin[n], s - st)) * f;
            double Sa[4];
            axis_sources<PHYS>(d, dir, ucomp[dir], g.ut, a.t_src, Sa);
#pragma unroll
            for (int n = 0; n < 4; ++n) val[n] += a.dt * Sa[n];
        }
    }
    if (a.stage2) {
#pragma unroll
        for (int n = 0; n < NQ; ++n) val[n] = (val[n] + ld(a.qavg[n], s)) * 0.5;
    }
    const double gx = ld(a.guess[1], s), gy = ld(a.guess[2], s);
    double prim[6], qfull[16];
#pragma unroll
    for (int n = 0; n < 16; ++n) qfull[n] = n < NQ ? val[n] : 0.0;
    const int st = invert<PHYS>(a.eos, a.t_inv, qfull, g.e, sqrt(fabs(gx * gx + gy * gy)), prim);
    double e = prim[0], p = prim[1];
    double u[4] = {prim[2], prim[3], prim[4], prim[5]};
    double rmap[11];
    regulate<PHYS>(a.t_inv, e, p, val, u, a.regmap[0] ? rmap : nullptr);
    if (a.regmap[0] && Phys<PHYS>::PIMUNU)
        for (int m = 0; m < 11; ++m) a.regmap[m][s] = rmap[m];
    if (st != 0 && a.counters) count_add(a.counters + 1, 1ull);
    if ((bad || st == 2) && a.counters) count_add(a.counters + 2, 1ull);
    if (a.fallback) a.fallback[s] = st != 0;
    if (a.hot && a.stage2 && st == 0) {  // the isotherm e = e_freeze passed this (converged) cell during the step
        const unsigned char was = a.hot[s], now = e > a.e_freeze;
        if (was != now) {
            a.hot[s] = now;
            count_add(a.crossings + (was ? 0 : 1), 1ull);
        }
    }
    store_cell(a, s, NQ, val, u, e, p);
    const long long sy = a.ncx, sz = a.plane;
    if (i == 2) { store_cell(a, s - 1, NQ, val, u, e, p); store_cell(a, s - 2, NQ, val, u, e, p); }
    if (i == a.nx + 1) { store_cell(a, s + 1, NQ, val, u, e, p); store_cell(a, s + 2, NQ, val, u, e, p); }
    if (j == 2) { store_cell(a, s - sy, NQ, val, u, e, p); store_cell(a, s - 2 * sy, NQ, val, u, e, p); }
    if (j == a.ny + 1) { store_cell(a, s + sy, NQ, val, u, e, p); store_cell(a, s + 2 * sy, NQ, val, u, e, p); }
    if (a.zghosts) {
        if (k == 2) { store_cell(a, s - sz, NQ, val, u, e, p); store_cell(a, s - 2 * sz, NQ, val, u, e, p); }
        if (k == a.nz + 1) { store_cell(a, s + sz, NQ, val, u, e, p); store_cell(a, s + 2 * sz, NQ, val, u, e, p); }
    }
}

// ------------------------------------------------------------ set-up ops --
// Primitive -> conserved at one interior cell (DynamicalVariables.cpp:197-287,
// W off). pl_from_field = 0: P_L = 0.0154483 e as the reference hard-codes.
template <typename S, int PHYS>
VAH_HD void set_conserved_cell(S *const *q, S *const *u, S *const *up, const S *e, double t, int pl_from_field,
                               long long s) {
    const double ux = (double)u[1][s], uy = (double)u[2][s], un = (double)u[3][s], ut = (double)u[0][s];
    const double eeq = (double)e[s];
    double pitt = 0, pitx = 0, pity = 0, pitn = 0, Pi = 0;
    if (Phys<PHYS>::PIMUNU) {
        pitt = (double)q[5][s];
        pitx = (double)q[6][s];
        pity = (double)q[7][s];
        pitn = (double)q[8][s];
    }
    if (Phys<PHYS>::BULK) Pi = (double)q[kSlotPi][s];
    const double pl = pl_from_field ? (double)q[kSlotPL][s] : 0.0154483 * eeq;
    const double pt = 0.5 * (eeq - pl) + 1.5 * Pi;
    const double DP = pl - pt;
    const double F = 1 + (ux * ux + uy * uy);
    const double Ltt = DP * t * t * un * un / F;
    const double Ltn = DP * ut * un / F;
    q[0][s] = (S)((eeq + pt) * ut * ut - pt + Ltt + pitt);
    q[1][s] = (S)((eeq + pt) * ut * ux + pitx);
    q[2][s] = (S)((eeq + pt) * ut * uy + pity);
    q[3][s] = (S)((eeq + pt) * ut * un + Ltn + pitn);
    q[kSlotPL][s] = (S)pl;
    for (int m = 0; m < 4; ++m) up[m][s] = u[m][s];
}

}  // namespace vah
