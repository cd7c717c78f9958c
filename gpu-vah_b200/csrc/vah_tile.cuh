// vah_tile.cuh -- the FP32 form of the RK stage as one persistent,
// TMA-tiled launch per stage (sm_100a).
//
// Form: the state is stored and updated in FP32 -- reconstruction, minmod
// limiter, Kurganov-Tadmor flux, source terms, convex combination and
// regulator run in single precision -- and only the Newton inversions of
// conserved to primitive variables run in FP64 (ill-conditioned as P_L -> 0
// and u^tau grows). Each face flux is evaluated once, from both reconstructed
// states, with the left cell's Newton guess (the shared-face semantics of
// VAH_FLUX_SHARED), so a cell-stage costs 3 face inversion pairs + 1 cell
// inversion instead of the reference's 6 pairs + 1.
//
// Structure: a persistent grid (2 blocks of 256 threads per SM) takes tiles
// from a work-list through an atomic counter. For each tile one thread issues
// a 4-D TMA load (cp.async.bulk.tensor: x, y, z and all N_q fields) of the
// tile plus a 2-cell halo of the stage-input conserved fields into shared
// memory, and two more of e, p and u^mu with a 1-cell halo, completed on an
// mbarrier. The faces of the tile are then evaluated once each, from one
// inlined call site in a loop over four jobs: the tile's lower boundary faces
// (threads 0-127, into a small shared buffer), then every cell's +1/2 face
// along x (differenced at once with the neighbour cell's through warp
// shuffles), along y and along z (a shared face buffer, differenced after a
// barrier), so that only the flux differences stay live between jobs. Every
// cell then runs its explicit update. Then the next tile's copies are issued, and they land
// while this tile's cells run their FP64 inversions, regulator and stores.
// Face fluxes never leave the SM.
//
// Tiles: 8x8x4 cells for 3+1D events (TMA box 12x12x8 x N_q), 16x16x1 for
// 2+1D (box 20x20x1 x N_q). Buffers use a row pitch padded to 4 floats
// (16 bytes), as the TMA tensor map requires.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "vah_physics.cuh"
#include "vah_tile_cell.cuh"

namespace vah {

constexpr int kTileThreads = 256;

template <bool IS3D>
struct TileShape {
    static constexpr int TX = IS3D ? 8 : 16, TY = IS3D ? 8 : 16, TZ = IS3D ? 4 : 1;
    // box of the conserved fields: halo 2 (2+1D: the one plane)
    static constexpr int BX = TX + 4, BY = TY + 4, BZ = IS3D ? TZ + 4 : 1;
    static constexpr int BOXN = BX * BY * BZ;
    // box of the primitives e, p, u: halo 1 in y and z; x as the conserved box (a 16-byte aligned start)
    static constexpr int PBX = BX, PBY = TY + 2, PBZ = IS3D ? TZ + 2 : 1;
    static constexpr int PBOXN = PBX * PBY * PBZ;
    static constexpr int NBX = TY * TZ, NBY = TX * TZ, NBZ = IS3D ? TX * TY : 0;  // lower boundary faces per axis
    static constexpr int NBXY = NBX + NBY;
    static_assert(TX * TY * TZ == kTileThreads, "one thread per cell");
    static_assert(NBXY + NBZ <= kTileThreads, "boundary faces: one per thread, all in the first face job");
    static_assert((BX * 4) % 16 == 0, "TMA box rows must be a multiple of 16 bytes");
};

// One event in the tile layout, with the buffer roles of vah_rk2_step:
// Q[0] = q (q^n; stage 2 writes q^{n+1} in place), Q[1] = qS (stage 1's
// result), each N_q fields at a stride of fstride floats, so that one rank-4
// tensor map (x, y, z, field) covers a block; ep[0] = (e, p) at t_n (stage 2
// writes t_{n+1}'s), ep[1] = stage 1's; uA / uB = u^n and u^{n-1} in the
// order the clock's parity gives (stage 2 writes u^{n+1} over u^{n-1}, and the
// parity flips); uS = stage 1's u. Cell (i, j, k) of the ghosted grid is at
// i + pitch (j + ncy k), pitch a multiple of 4 floats.
struct alignas(64) TileSlot {
    CUtensorMap tmQ[2];   // over Q[0], Q[1] (N_q fields)
    CUtensorMap tmEP[2];  // over ep[0], ep[1] (e, p: two fields, fstride apart)
    CUtensorMap tmU[3];   // over uA, uB, uS (four fields each, fstride apart)
    float *Q[2];
    float *ep[2][2];
    float *uA[4], *uB[4], *uS[4];
    long long fstride;
    int nx, ny, nz, pitch, ncy, nq;
    int zghosts;                   // 2+1D: 1 to store the eta ghost layers (else filled when read)
    double dx, dy, dz, dt, etabar;
    unsigned long long *counters;  // [face fallbacks, cell fallbacks, NaN cells]
    unsigned char *fallback1, *fallback2;  // optional: per cell, 1 where the stage-1 / stage-2 inversion fell back
    unsigned char *hot;            // optional freeze-out state (1 while e > e_freeze) ...
    double e_freeze;
    unsigned long long *crossings;  // ... and crossings [down, up] of the step
    double *regmap[11];            // optional validity diagnostics (FP64, fstride each)
};

// Per-event clock (the batch's per-slot clock has this layout).
struct TileClock {
    double t;
    int parity;  // 0: u^n in uA, u^{n-1} in uB; 1: swapped
    int active;
    long long steps;
};

struct TileItem {
    int slot, i0, j0, k0;  // tile origin in interior coordinates
};

// Error flags the kernel can raise (bit mask in *err).
constexpr unsigned kTileErrTimeout = 1u;  // an mbarrier wait ran past its iteration limit
constexpr unsigned kTileErrAlign = 2u;    // the shared-memory box was not 128-byte aligned (nothing issued)

#ifdef __CUDACC__

// ------------------------------------------------------------ PTX helpers --
__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: gives up (false) after `limit` polls; each poll blocks for a
// hardware-chosen interval, so the limit bounds the wait to well under a
// second on B200.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, unsigned limit) {
    for (unsigned it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// 4-D tiled TMA load of one box into shared memory, completing on `bar`.
// The x coordinate times 4 bytes must be a multiple of 16 (x % 4 == 0).
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, unsigned long long *bar, int x, int y,
                                            int z, int f) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(f), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void tile_count(unsigned long long *c, unsigned v) {
    // one atomic per warp
    unsigned s = v;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(c, (unsigned long long)s);
}

// flux[n] = c (hm[n] - hp[n]) (ACC: flux[n] += ...) over the N_q fields, two
// at a time.
template <int NQ, bool ACC>
__device__ __forceinline__ void flux_diff(float *flux, float c, const float *hm, const float *hp) {
#pragma unroll
    for (int n = 0; n + 1 < NQ; n += 2) {
        const Pair d = psub(Pair{hm[n], hm[n + 1]}, Pair{hp[n], hp[n + 1]});
        const Pair f = ACC ? pfma(Pair{c, c}, d, Pair{flux[n], flux[n + 1]}) : pmul(Pair{c, c}, d);
        flux[n] = f.a;
        flux[n + 1] = f.b;
    }
    if (NQ % 2) {
        const float d = hm[NQ - 1] - hp[NQ - 1];
        flux[NQ - 1] = ACC ? fmaf(c, d, flux[NQ - 1]) : c * d;
    }
}

// The dynamic shared memory of one block: the TMA boxes (conserved fields,
// then e, p, u), the face buffer of the +1/2 faces along y, then z, the lower
// boundary faces (x and y; z), and the mbarrier and the tile index. 3+1D with
// N_q = 16: 115.6 KB, so that two blocks share an SM's 228 KB.
template <int PHYS, bool IS3D>
struct TileSmem {
    using SH = TileShape<IS3D>;
    static constexpr int NQ = Phys<PHYS>::NQ;
    static constexpr size_t pad32(size_t n) { return (n + 31) / 32 * 32; }  // to 128-byte multiples
    // each TMA destination starts on a 128-byte boundary
    static constexpr size_t box_floats = pad32((size_t)SH::BOXN * NQ);
    static constexpr size_t ep_floats = pad32((size_t)SH::PBOXN * 2);
    static constexpr size_t u_floats = pad32((size_t)SH::PBOXN * 4);
    static constexpr size_t face_floats = (size_t)kTileThreads * NQ;
    static constexpr size_t bnd_floats = (size_t)(SH::NBXY + SH::NBZ) * NQ;
    static constexpr size_t box_bytes = (size_t)SH::BOXN * NQ * 4, ep_bytes = (size_t)SH::PBOXN * 2 * 4,
                            u_bytes = (size_t)SH::PBOXN * 4 * 4;  // what the copies write
    static constexpr size_t bar_offset =
        ((box_floats + ep_floats + u_floats + face_floats + bnd_floats) * 4 + 15) / 16 * 16;
    static constexpr size_t bytes = bar_offset + 16;
};

template <int PHYS, bool IS3D>
__global__ void __launch_bounds__(kTileThreads, 2)
    tile_kernel(const TileSlot *__restrict__ slots, const TileClock *__restrict__ clk, const TileClock clk0,
                const double dt0, const TileItem *__restrict__ items, int nitems, unsigned *next_item, int stage,
                const Eos eos, unsigned *err) {
    using SH = TileShape<IS3D>;
    using SM = TileSmem<PHYS, IS3D>;
    constexpr int NQ = Phys<PHYS>::NQ;
    constexpr int TX = SH::TX, TY = SH::TY, BX = SH::BX, BY = SH::BY, BOXN = SH::BOXN;
    constexpr int PBX = SH::PBX, PBY = SH::PBY, PBOXN = SH::PBOXN;
    constexpr int SY = BX, SZ = BX * BY, PSY = PBX, PSZ = PBX * PBY;
    extern __shared__ __align__(1024) float tile_smem[];
    float *sQ = tile_smem;                     // [NQ][BZ][BY][BX]
    float *sP = sQ + SM::box_floats;           // [2][PBZ][PBY][PBX]: e, p
    float *sU = sP + SM::ep_floats;            // [4][PBZ][PBY][PBX]: ut, ux, uy, un
    float *sF = sU + SM::u_floats;             // [NQ][256]: +1/2 faces along y, then z
    float *sB = sF + SM::face_floats;          // [NQ][NBXY], [NQ][NBZ]: lower boundary faces (x, y; z)
    unsigned long long *bar = (unsigned long long *)((char *)tile_smem + SM::bar_offset);
    int &s_item = *(int *)(bar + 1);
    const float *const sE = sP, *const sPp = sP + PBOXN, *const sUX = sU + PBOXN, *const sUY = sU + 2 * PBOXN;

    const int tid = threadIdx.x;
    const int lx = tid % TX, ly = (tid / TX) % TY, lz = tid / (TX * TY);
    if (smem_u32(sQ) & 127u) {  // the TMA destinations must be 128-byte aligned: report, issue nothing
        if (tid == 0) atomicOr(err, kTileErrAlign);
        return;
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    unsigned phase = 0;

    // the stage inputs of tile w: conserved fields (halo 2), e and p, u (halo 1)
    auto issue = [&](int w) {
        const TileItem it = items[w];
        const TileSlot &d = slots[it.slot];
        const int par = clk ? clk[it.slot].parity : clk0.parity;
        fence_proxy_async_smem();  // the previous tile's generic reads of these buffers come first
        mbar_expect_tx(bar, (unsigned)(SM::box_bytes + SM::ep_bytes + SM::u_bytes));
        const int z0 = IS3D ? it.k0 : 2, pz0 = IS3D ? it.k0 + 1 : 2;
        tma_load_4d(sQ, &d.tmQ[stage == 1 ? 0 : 1], bar, it.i0, it.j0, z0, 0);
        tma_load_4d(sP, &d.tmEP[stage == 1 ? 0 : 1], bar, it.i0, it.j0 + 1, pz0, 0);
        tma_load_4d(sU, &d.tmU[stage == 1 ? par : 2], bar, it.i0, it.j0 + 1, pz0, 0);
    };
    if (tid == 0) {
        s_item = (int)atomicAdd(next_item, 1u);
        if (s_item < nitems) issue(s_item);
    }
    __syncthreads();
    int w = s_item;

    while (w < nitems) {
        const TileItem it = items[w];
        const TileSlot &d = slots[it.slot];
        const TileClock c = clk ? clk[it.slot] : clk0;  // clk0, dt0: a single event's clock and step, by value
        const double dt = clk ? d.dt : dt0;
        const double t_src = stage == 1 ? c.t : c.t + dt;
        const double t_inv = c.t + dt;

        if (!mbar_wait(bar, phase, 1u << 22)) {
            if (tid == 0) atomicOr(err, kTileErrTimeout);
            // wait once more (bounded) so that no copy is left writing this block's memory
            mbar_wait(bar, phase, 1u << 22);
            return;
        }
        phase ^= 1u;

        // this thread's cell, in interior and ghosted coordinates, and in the boxes
        const int ci = it.i0 + lx, cj = it.j0 + ly, ck = it.k0 + lz;
        const bool live = ci < d.nx && cj < d.ny && ck < d.nz;
        const int pitch = d.pitch;
        const long long plane = (long long)pitch * d.ncy;
        const long long s = (ci + 2) + (long long)pitch * (cj + 2) + plane * (ck + 2);
        const int bc = (lx + 2) + BX * ((ly + 2) + BY * (IS3D ? lz + 2 : 0));
        const int pc = (lx + 2) + PBX * ((ly + 1) + PBY * (IS3D ? lz + 1 : 0));
        const BoxQ<BOXN> bq{sQ};
        unsigned ffail = 0, fnan = 0;
        auto count = [&](unsigned f) {
            ffail += f & 255u;
            fnan |= f >> 8;
        };
        // Newton guess and fallback energy of the faces whose left cell is this one
        const double e0 = (double)sE[pc], ux0 = (double)sUX[pc], uy0 = (double)sUY[pc];
        const double uT0 = sqrt(fabs(ux0 * ux0 + uy0 * uy0));

        // ---- faces: one evaluation site, in four jobs --
        //   0: the lower boundary face of the tile that this thread owns
        //      (threads 0 .. NBXY + NBZ - 1: x, y, then z faces) into sB;
        //   1: +1/2 along x, differenced at once through warp shuffles (the
        //      -1/2 face from lane - 1, or from sB at the tile's edge);
        //   2: +1/2 along y into the face buffer, differenced after a barrier;
        //   3: (3+1D) +1/2 along z, the same, reusing the face buffer.
        // Nothing but the flux differences stays live from one job to the next.
        const float cx = (float)(dt / d.dx), cy = (float)(dt / d.dy), cz = (float)(dt / d.dz);
        float flux[NQ];
        constexpr int NB = SH::NBXY + SH::NBZ;
        constexpr int NJOB = IS3D ? 4 : 3;
#pragma unroll 1
        for (int job = 0; job < NJOB; ++job) {
            if (job == 1 || job == 3) __syncthreads();  // 1: boundary faces written; 3: y differences read
            bool act = live, store = true;
            int l = bc, st = 1, dir = job == 2 ? 1 : (job == 3 ? 2 : 0);
            if (job == 2) st = SY;
            if (job == 3) st = SZ;
            double eP = e0, ug = uT0;
            float *dst = sF + tid;
            int ds = kTileThreads;
            if (job == 0) {
                store = tid < NB;
                act = false;
                if (store) {
                    const int bdir = tid < SH::NBX ? 0 : (tid < SH::NBXY ? 1 : 2);
                    const int b = bdir == 0 ? tid : (bdir == 1 ? tid - SH::NBX : tid - SH::NBXY);
                    int bi, bj, bk;  // left cell in the conserved box (in the halo)
                    if (bdir == 0) { bi = 1; bj = 2 + b % TY; bk = IS3D ? 2 + b / TY : 0; }
                    else if (bdir == 1) { bi = 2 + b % TX; bj = 1; bk = IS3D ? 2 + b / TX : 0; }
                    else { bi = 2 + b % TX; bj = 2 + b / TX; bk = 1; }
                    const int ri = it.i0 + bi - 2 + (bdir == 0), rj = it.j0 + bj - 2 + (bdir == 1),
                              rk = it.k0 + (IS3D ? bk - 2 : 0) + (bdir == 2);  // the right cell: the tile's first
                    act = ri < d.nx && rj < d.ny && rk < d.nz;
                    l = bi + BX * (bj + BY * bk);
                    st = bdir == 0 ? 1 : (bdir == 1 ? SY : SZ);
                    dir = bdir;
                    const int pl = bi + PBX * ((bj - 1) + PBY * (IS3D ? bk - 1 : 0));
                    eP = (double)sE[pl];
                    const double ux = (double)sUX[pl], uy = (double)sUY[pl];
                    ug = sqrt(fabs(ux * ux + uy * uy));
                    dst = bdir < 2 ? sB + tid : sB + SH::NBXY * NQ + (tid - SH::NBXY);
                    ds = bdir < 2 ? SH::NBXY : SH::NBZ;
                }
            }
            float Hj[NQ];
            if (act) count(tile_face<PHYS>(bq, l, st, dir, t_src, eP, ug, Hj, 1));
            else
#pragma unroll
                for (int n = 0; n < NQ; ++n) Hj[n] = 0.0f;
            if (job == 1) {  // x: lane - 1 holds the -1/2 face
                float hm[NQ];
#pragma unroll
                for (int n = 0; n < NQ; ++n) {
                    hm[n] = __shfl_up_sync(0xffffffffu, Hj[n], 1, TX);
                    if (lx == 0) hm[n] = sB[n * SH::NBXY + (ly + TY * lz)];
                }
                flux_diff<NQ, false>(flux, cx, hm, Hj);
            } else {
                if (store)
#pragma unroll
                    for (int n = 0; n < NQ; ++n) dst[n * ds] = Hj[n];
                if (job >= 2) {
                    __syncthreads();
                    float hm[NQ], hp[NQ];
                    if (job == 2) {
#pragma unroll
                        for (int n = 0; n < NQ; ++n) {
                            hm[n] = ly > 0 ? sF[n * kTileThreads + tid - TX] : sB[n * SH::NBXY + SH::NBX + lx + TX * lz];
                            hp[n] = sF[n * kTileThreads + tid];
                        }
                        flux_diff<NQ, true>(flux, cy, hm, hp);
                    } else {
                        const float *sBz = sB + SH::NBXY * NQ;
#pragma unroll
                        for (int n = 0; n < NQ; ++n) {
                            hm[n] = lz > 0 ? sF[n * kTileThreads + tid - TX * TY] : sBz[n * SH::NBZ + lx + TX * ly];
                            hp[n] = sF[n * kTileThreads + tid];
                        }
                        flux_diff<NQ, true>(flux, cz, hm, hp);
                    }
                }
            }
        }
        if (d.counters) {
            tile_count(d.counters + 0, ffail);
            tile_count(d.counters + 2, fnan ? 1u : 0u);
        }

        // ---- the cell: the explicit update (the last reads of the boxes) ----
        float *const *u_n = c.parity ? d.uB : d.uA;  // u^n
        float *const *u_p = c.parity ? d.uA : d.uB;  // u^{n-1}
        TilePrims pr;
        pr.E = sE;
        pr.P = sPp;
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            pr.U[m] = sU + m * PBOXN;
            pr.UP[m] = stage == 1 ? u_p[m] : u_n[m];  // previous-stage u (d_tau u)
            pr.G[m] = u_n[m];
        }
        pr.pi = pc;
        pr.psy = PSY;
        pr.psz = PSZ;
        float val[NQ], e_prev = 0.0f;
        int bad = 0;
        if (live)
            tile_cell_explicit<PHYS, IS3D>(bq, bc, SY, SZ, pr, s, flux, eos, t_src, dt, d.dx, d.dy, d.dz, d.etabar, val,
                                           e_prev, bad);

        // after this barrier every read of this tile's boxes is done: the
        // next tile's copies, issued only then, overlap this tile's
        // inversions, regulator and stores
        if (tid == 0) s_item = (int)atomicAdd(next_item, 1u);
        __syncthreads();
        const int w_next = s_item;
        if (tid == 0 && w_next < nitems) issue(w_next);

        // ---- the cell: inversion, regulator, stores (stage outputs:
        // FullyDiscreteKurganovTadmorScheme.cpp:761-789) ----
        if (live) {
            const long long fs = d.fstride;
            struct {
                const float *q;
                long long fs;
                __device__ float operator()(int n, long long i) const { return q[n * fs + i]; }
            } qavg{d.Q[0], fs};
            float e, p, u[4], rmap[11];
            const int st = tile_cell_invert<PHYS>(pr, s, qavg, stage == 2, eos, t_inv, e_prev, val, e, p, u,
                                                  d.regmap[0] ? rmap : nullptr);
            if (d.regmap[0] && Phys<PHYS>::PIMUNU)
                for (int m = 0; m < 11; ++m) d.regmap[m][s] = (double)rmap[m];
            if (d.counters) {
                if (st != 0) atomicAdd(d.counters + 1, 1ull);
                if (bad || st == 2) atomicAdd(d.counters + 2, 1ull);
            }
            unsigned char *fb = stage == 1 ? d.fallback1 : d.fallback2;
            if (fb) fb[s] = st != 0;
            if (d.hot && stage == 2 && st == 0) {
                const unsigned char was = d.hot[s], now = (double)e > d.e_freeze;
                if (was != now) {
                    d.hot[s] = now;
                    atomicAdd(d.crossings + (was ? 0 : 1), 1ull);
                }
            }
            // stores, and the face ghost layers of boundary cells (setGhostCellsKernelI/J/K)
            float *Qout = d.Q[stage == 1 ? 1 : 0];
            float *Eout = d.ep[stage == 1 ? 1 : 0][0], *Pout_p = d.ep[stage == 1 ? 1 : 0][1];
            float *const *Uout = stage == 1 ? d.uS : u_p;
            const long long sy = pitch, sz = plane;
            auto store = [&](long long at) {
#pragma unroll
                for (int n = 0; n < NQ; ++n) Qout[n * fs + at] = val[n];
                Eout[at] = e;
                Pout_p[at] = p;
#pragma unroll
                for (int m = 0; m < 4; ++m) Uout[m][at] = u[m];
            };
            store(s);
            if (ci == 0) { store(s - 1); store(s - 2); }
            if (ci == d.nx - 1) { store(s + 1); store(s + 2); }
            if (cj == 0) { store(s - sy); store(s - 2 * sy); }
            if (cj == d.ny - 1) { store(s + sy); store(s + 2 * sy); }
            if (IS3D || d.zghosts) {
                if (ck == 0) { store(s - sz); store(s - 2 * sz); }
                if (ck == d.nz - 1) { store(s + sz); store(s + 2 * sz); }
            }
        }
        w = w_next;
    }
}

#endif  // __CUDACC__

}  // namespace vah

// ------------------------------------------------------------ host side --
#include <vector>

namespace vah {

// Padded row pitch of the tile layout: nx + 4 rounded up to 4 floats.
inline int tile_pitch(int nx) { return (nx + 4 + 3) / 4 * 4; }

// Rank-4 tensor map (x, y, z, field) over a block of nq fields of float,
// fstride floats apart, with the box of the tile shape. Returns a VAH_* status.
int tile_encode_q(CUtensorMap *tm, const float *base, int nx, int ny, int nz, int pitch, long long fstride, int nq);

// The same over a block of nf primitive fields (e, p or u^mu), with the box of
// the primitives (halo 1 in y and z).
int tile_encode_p(CUtensorMap *tm, const float *base, int nx, int ny, int nz, int pitch, long long fstride, int nf);

// The tiles covering an event's interior, appended to `out`.
void tile_items(std::vector<TileItem> &out, int slot, int nx, int ny, int nz);

// One stage over the given tiles (all 3+1D or all 2+1D): resets the tile
// counter and launches the persistent tile kernel. clk == nullptr: every tile
// uses clk0 and the step dt0 (a single event); else each slot's clock and dt.
cudaError_t tile_launch(const TileSlot *slots, const TileClock *clk, const TileClock &clk0, double dt0,
                        const TileItem *items, int nitems, bool is3d, unsigned *counter, int stage, int physics,
                        const Eos &eos, unsigned *err, cudaStream_t stream);

}  // namespace vah
