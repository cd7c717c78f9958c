// vah_batch.cu -- many events, one persistent launch per kernel kind.
//
// A batch holds up to kMaxSlots events of independent grid sizes. Every
// launch of a step covers all events: a persistent grid of blocks walks a
// work-list of 32x4 tiles (event slot, tile origin), each block a contiguous
// run of it, so events of uneven sizes share one launch and the GPU is filled
// even by many small events.
// The per-event state lives in one device allocation per event (stream-
// ordered, from the batch's memory pool); per-event descriptors (buffer
// pointers, geometry) and clocks (time, u/u_prev parity, step count) live in
// device arrays, so a whole RK2 step -- face and cell launches of both stages
// plus the clock advance -- is captured once as a CUDA graph and replayed.
// The graph is re-captured only when events are added or removed.
// VAH_FP32 batches run the FP32 form on the TMA-tiled stage kernel
// (vah_tile.cuh): one persistent launch per stage and tile shape (2+1D and
// 3+1D events), each slot with a row pitch padded to 4 floats and a tile
// descriptor (tensor maps over its q and qS blocks) admitted with it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "vah.h"
#include "vah_ic_device.cuh"
#include "vah_kernels.cuh"
#include "vah_powf_exc.h"
#include "vah_tile.cuh"

namespace vah {
namespace {

constexpr int kMaxSlots = 4096;
constexpr int kTX = 32, kTY = 4;

template <typename S>
struct SlotDesc {
    int nx, ny, nz, ncx, ncy;
    long long plane;
    double dx, dy, dz, dt, etabar;
    S *q[16], *qS[16], *ep[2][2], *uA[4], *uB[4], *uS[4];
    S *H[3][16], *HR[3][16];
    unsigned char *fallback;  // per ghosted cell: 1 where the latest cell inversion fell back
    unsigned char *hot;       // per ghosted cell: 1 while e > e_freeze (freeze-out crossings)
    double e_freeze;
    unsigned long long *crossings;  // [down, up] during the current step
    unsigned long long *counters;
};

struct SlotClock {
    double t;
    int parity;  // 0: current velocity in uA, previous in uB; 1: swapped
    int active;
    long long steps;
};
// the tile kernel reads the batch's clocks as TileClock
static_assert(sizeof(SlotClock) == sizeof(TileClock) && offsetof(SlotClock, parity) == offsetof(TileClock, parity) &&
                  offsetof(SlotClock, t) == offsetof(TileClock, t),
              "SlotClock and TileClock share a layout");

struct WorkItem {
    int slot, i0, r0, pad;
};

enum { K_FX = 0, K_FY = 1, K_FZ = 2, K_C2 = 3, K_C3 = 4, K_NUM = 5 };

// StageArgs of one slot and stage (the buffer roles of vah_rk2_step).
template <typename S>
__device__ void make_args(StageArgs<S> &a, const SlotDesc<S> &d, const SlotClock &c, int stage, const Eos &eos) {
    a.nx = d.nx;
    a.ny = d.ny;
    a.nz = d.nz;
    a.k0 = 0;
    a.k1 = d.nz;
    a.ncx = d.ncx;
    a.ncy = d.ncy;
    a.plane = d.plane;
    a.dx = d.dx;
    a.dy = d.dy;
    a.dz = d.dz;
    a.dt = d.dt;
    a.etabar = d.etabar;
    a.t_src = stage == 1 ? c.t : c.t + d.dt;
    a.t_inv = c.t + d.dt;
    a.stage2 = stage == 2;
    a.zghosts = d.nz > 1;  // 2+1D: the eta ghost layers are filled when a caller reads them
    a.eos = eos;
    a.counters = d.counters;
    a.fallback = d.fallback;
    for (int m = 0; m < 11; ++m) a.regmap[m] = nullptr;  // validity diagnostics are an event-path option
    a.hot = d.hot;
    a.e_freeze = d.e_freeze;
    a.crossings = d.crossings;
    S *const *u = c.parity ? d.uB : d.uA;
    S *const *up = c.parity ? d.uA : d.uB;
    for (int n = 0; n < 16; ++n) {
        a.qin[n] = stage == 1 ? d.q[n] : d.qS[n];
        a.qout[n] = stage == 1 ? d.qS[n] : d.q[n];
        a.qavg[n] = d.q[n];
    }
    for (int m = 0; m < 4; ++m) {
        a.uin[m] = stage == 1 ? u[m] : d.uS[m];
        a.upin[m] = stage == 1 ? up[m] : u[m];
        a.guess[m] = u[m];
        a.uout[m] = stage == 1 ? d.uS[m] : up[m];
    }
    a.ein = d.ep[stage == 1 ? 0 : 1][0];
    a.pin = d.ep[stage == 1 ? 0 : 1][1];
    a.eout = d.ep[stage == 1 ? 1 : 0][0];
    a.pout = d.ep[stage == 1 ? 1 : 0][1];
    for (int k = 0; k < 3; ++k)
        for (int n = 0; n < 16; ++n) {
            a.H[k][n] = d.H[k][n];
            a.HR[k][n] = d.HR[k][n];
        }
    for (int n = 0; n < 16; ++n) a.Dx[n] = nullptr;  // the batch's cell launch differences H / HR itself
    finish_args(a);
}

// Tiles are taken from the work-list in chunks of kChunk through an atomic
// counter (reset before each launch): blocks that finish early take more,
// so uneven events do not leave a tail; the list runs largest event first.
constexpr int kChunk = 4;

template <typename S, int PHYS, int KIND, bool EXACT, int MINB>
__global__ void __launch_bounds__(kTX *kTY, MINB) batch_kernel(const SlotDesc<S> *__restrict__ descs,
                                                         const SlotClock *__restrict__ clk,
                                                         const WorkItem *__restrict__ work, int nwork, int stage,
                                                         const Eos eos, unsigned *next) {
    __shared__ StageArgs<S> sa;
    __shared__ int sa_slot, s_w0;
    const bool lead = threadIdx.x == 0 && threadIdx.y == 0;
    if (lead) sa_slot = -1;
    for (;;) {
    __syncthreads();  // s_w0 of the previous chunk has been read
    if (lead) s_w0 = (int)atomicAdd(next, (unsigned)kChunk);
    __syncthreads();
    const int w0 = s_w0, w1 = min(nwork, w0 + kChunk);
    if (w0 >= nwork) break;
    // the per-event arguments in shared memory change only at event boundaries
    for (int w = w0; w < w1; ++w) {
        const WorkItem it = work[w];
        __syncthreads();
        if (lead && it.slot != sa_slot) {
            make_args(sa, descs[it.slot], clk[it.slot], stage, eos);
            sa_slot = it.slot;
        }
        __syncthreads();
        const int i = it.i0 + threadIdx.x, r = it.r0 + threadIdx.y;
        if (KIND <= K_FZ) {
            const int ext0 = KIND == K_FX ? sa.nx + 1 : sa.nx;
            const int ext1 = KIND == K_FY ? sa.ny + 1 : sa.ny;
            const int ext2 = KIND == K_FZ ? sa.nz + 1 : sa.nz;
            if (i < ext0 && r < ext1 * ext2) {
                const int j = r % ext1, k = r / ext1;
                const int gi = i + (KIND == K_FX ? 1 : 2), gj = j + (KIND == K_FY ? 1 : 2), gk = k + (KIND == K_FZ ? 1 : 2);
                const long long st = KIND == K_FX ? 1 : (KIND == K_FY ? (long long)sa.ncx : sa.plane);
                const long long s = gi + (long long)sa.ncx * gj + sa.plane * gk;
                const int gl = KIND == K_FX ? gi : (KIND == K_FY ? gj : gk);
                const int n = KIND == K_FX ? sa.nx : (KIND == K_FY ? sa.ny : sa.nz);
                const unsigned fails = face_compute<S, PHYS, EXACT>(sa, s, KIND, st, gl >= 2, gl <= n);
                if (fails & 255u) count_add(sa.counters + 0, fails & 255u);
                if (fails >> 8) count_add(sa.counters + 2, 1ull);
            }
        } else if (i < sa.nx && r < sa.ny * sa.nz) {
            const int j = r % sa.ny, k = r / sa.ny;
            cell_compute<S, PHYS, KIND == K_C3, EXACT>(sa, i + 2, j + 2, k + 2);
        }
    }
    }
}

// End of a step: the clock moves on, and the freeze-out surface volume takes
// the step's net crossings (down - up) times tau dx dy deta at the new time.
__global__ void advance_kernel(SlotClock *clk, const double *dts, int nslots, unsigned long long *cross, double *vol,
                               const double *dv) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nslots && clk[s].active) {
        const double t_new = clk[s].t + dts[s];
        const double net = (double)cross[2 * s] - (double)cross[2 * s + 1];
        if (net != 0.0) vol[s] += t_new * net * dv[s];
        cross[2 * s] = cross[2 * s + 1] = 0;
        clk[s].t = t_new;
        clk[s].parity ^= 1;
        clk[s].steps += 1;
    }
}

// Freeze-out state at admission: 1 where the interior e exceeds e_freeze.
template <typename S>
__global__ void hot_init_kernel(const S *e, unsigned char *hot, double e_freeze, int nx, int ny, int nz, int pitch) {
    const long long n = (long long)nx * ny * nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((long long)nx * ny));
        const long long s = (i + 2) + (long long)pitch * ((j + 2) + (long long)(ny + 4) * (k + 2));
        hot[s] = (double)e[s] > e_freeze;
    }
}

// Per-slot maximum of e over the interior cells whose latest inversion
// converged (positive doubles order like their bit patterns), for the
// freeze-out test. A cell whose inversion fell back holds e = 0.999 e_prev and
// u = (1,0,0,0) instead of a solution, so it does not count. Order-
// independent, so deterministic.
template <typename S>
__global__ void max_e_kernel(const SlotDesc<S> *__restrict__ descs, const WorkItem *__restrict__ work, int nwork,
                             unsigned long long *maxbits, int cur_ep) {
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const WorkItem it = work[w];
        const SlotDesc<S> &d = descs[it.slot];
        const int i = it.i0 + threadIdx.x, r = it.r0 + threadIdx.y;
        double v = 0.0;
        if (i < d.nx && r < d.ny * d.nz) {
            const int j = r % d.ny, k = r / d.ny;
            const long long s = (i + 2) + (long long)d.ncx * (j + 2) + d.plane * (k + 2);
            v = (double)d.ep[cur_ep][0][s];
            if (!(v > 0.0) || d.fallback[s]) v = 0.0;
        }
        unsigned long long b = (unsigned long long)__double_as_longlong(v);
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long x = __shfl_xor_sync(0xffffffffu, b, o);
            b = x > b ? x : b;
        }
        if ((threadIdx.x & 31) == 0) atomicMax(maxbits + it.slot, b);
    }
}

// Per-tile partial sums of the event observables (tau T^tt, T^xx - T^yy,
// T^xx + T^yy, e u^t u_T, e u^t) in FP64 over the cells whose latest
// inversion converged (a fallback cell's state is not a solution), one row
// per cell tile; the host adds the rows of each slot in a fixed order.
template <typename S, int PHYS>
__global__ void observables_kernel(const SlotDesc<S> *__restrict__ descs, const SlotClock *__restrict__ clk,
                                   const WorkItem *__restrict__ work, int nwork, double *partial) {
    __shared__ double red[5][kTX * kTY / 32];
    const int tid = threadIdx.y * kTX + threadIdx.x;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const WorkItem it = work[w];
        const SlotDesc<S> &d = descs[it.slot];
        const SlotClock c = clk[it.slot];
        const int i = it.i0 + threadIdx.x, r = it.r0 + threadIdx.y;
        double acc[5] = {0, 0, 0, 0, 0};
        const bool in = i < d.nx && r < d.ny * d.nz;
        const int j = in ? r % d.ny : 0, k = in ? r / d.ny : 0;
        const long long s = (i + 2) + (long long)d.ncx * (j + 2) + d.plane * (k + 2);
        if (in && !d.fallback[s]) {  // converged cells only
            S *const *u = c.parity ? d.uB : d.uA;
            const double e = (double)d.ep[0][0][s], p = (double)d.ep[0][1][s], pl = (double)d.q[kSlotPL][s];
            const double ut = (double)u[0][s], ux = (double)u[1][s], uy = (double)u[2][s];
            double ap[9];
            ap[0] = 1.0;
            ap[1] = pl / e;
            for (int m = 2; m < 9; ++m) ap[m] = ap[m - 1] * ap[1];
            double pt = 0.5 * (e - pl - poly::Rbar0(ap) * (e - 3 * p));
            double pixx = 0, piyy = 0;
            if (Phys<PHYS>::PIMUNU) {
                pixx = (double)d.q[9][s];
                piyy = (double)d.q[12][s];
            }
            if (Phys<PHYS>::BULK) pt += 1.5 * (double)d.q[kSlotPi][s];
            const double txx = e * ux * ux + pt * (1 + ux * ux) + pixx;
            const double tyy = e * uy * uy + pt * (1 + uy * uy) + piyy;
            acc[0] = c.t * (double)d.q[0][s] * d.dx * d.dy * d.dz;
            acc[1] = txx - tyy;
            acc[2] = txx + tyy;
            acc[3] = e * ut * sqrt(ux * ux + uy * uy);
            acc[4] = e * ut;
        }
        for (int m = 0; m < 5; ++m)
            for (int o = 16; o > 0; o >>= 1) acc[m] += __shfl_xor_sync(0xffffffffu, acc[m], o);
        __syncthreads();
        if ((tid & 31) == 0)
            for (int m = 0; m < 5; ++m) red[m][tid >> 5] = acc[m];
        __syncthreads();
        if (tid < 5) {
            double s = 0;
            for (int q = 0; q < kTX * kTY / 32; ++q) s += red[tid][q];
            partial[(size_t)w * 5 + tid] = s;
        }
    }
}

template <typename S, int PHYS, int KIND, bool EXACT, int MINB>
int blocks_per_sm() {
    static int cached = 0;
    if (!cached) {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel<S, PHYS, KIND, EXACT, MINB>, kTX * kTY,
                                                          0) != cudaSuccess ||
            n < 1)
            n = 1;
        cached = n;
    }
    return cached;
}

// A persistent grid of (SMs x resident blocks) walks the work-list.
template <typename S, int PHYS, int KIND, bool EXACT, int MINB>
cudaError_t launch_minb(const SlotDesc<S> *descs, const SlotClock *clk, const WorkItem *work, int nwork, int stage,
                        const Eos &eos, int sms, unsigned *next, cudaStream_t stream) {
    const int grid = std::min((nwork + kChunk - 1) / kChunk, sms * blocks_per_sm<S, PHYS, KIND, EXACT, MINB>());
    cudaError_t e = cudaMemsetAsync(next, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess) return e;
    batch_kernel<S, PHYS, KIND, EXACT, MINB><<<grid, dim3(kTX, kTY), 0, stream>>>(descs, clk, work, nwork, stage, eos,
                                                                                 next);
    return cudaGetLastError();
}

// minb: the register-cap variant (face kinds 3, 4, 5; cell kinds 2, 3, 4).
template <typename S, int PHYS, int KIND, bool EXACT>
cudaError_t launch_kind(const SlotDesc<S> *descs, const SlotClock *clk, const WorkItem *work, int nwork, int stage,
                        const Eos &eos, int sms, int minb, unsigned *next, cudaStream_t stream) {
    if (nwork <= 0) return cudaSuccess;
    constexpr bool FACE = KIND <= K_FZ;
    switch (minb) {
    case 2:
        if (FACE) break;
        return launch_minb<S, PHYS, KIND, EXACT, 2>(descs, clk, work, nwork, stage, eos, sms, next, stream);
    case 3: return launch_minb<S, PHYS, KIND, EXACT, 3>(descs, clk, work, nwork, stage, eos, sms, next, stream);
    case 4: return launch_minb<S, PHYS, KIND, EXACT, 4>(descs, clk, work, nwork, stage, eos, sms, next, stream);
    case 5:
        if (!FACE) break;
        return launch_minb<S, PHYS, KIND, EXACT, 5>(descs, clk, work, nwork, stage, eos, sms, next, stream);
    default: break;
    }
    return cudaErrorInvalidValue;
}

}  // namespace
}  // namespace vah

using vah::SlotClock;
using vah::SlotDesc;
using vah::WorkItem;

struct vah_batch {
    vah_options opt;
    int nq;
    size_t elem;
    cudaStream_t stream;
    bool own_stream;
    cudaMemPool_t pool;
    size_t capacity, used;
    int sms;
    double *d_tab;
    uint32_t *d_exc;
    int nexc;
    void *d_desc;               // SlotDesc<S>[kMaxSlots]
    SlotClock *d_clk;           // [kMaxSlots]
    double *d_dt;               // [kMaxSlots]
    unsigned long long *d_cross;  // [kMaxSlots * 2] freeze-out crossings of the current step (down, up)
    double *d_vol;              // [kMaxSlots] freeze-out surface volume so far, fm^4
    double *d_dv;               // [kMaxSlots] dx dy deta
    std::vector<double> tab;    // host copy of the EoS table (freeze-out energy densities)
    unsigned long long *d_counters;  // [kMaxSlots * 4]
    unsigned long long *d_maxbits;   // [kMaxSlots]
    struct Slot {
        bool used = false;
        vah_lattice lat{};
        vah_hydro hydro{};
        double dt = 0;
        size_t bytes = 0;
        void *mem = nullptr;
        std::vector<void *> field;  // VAH_F_* -> device array (current roles resolved at query time)
    };
    std::vector<Slot> slots;
    std::vector<unsigned char> desc_host;  // host mirror of the descriptor array
    WorkItem *d_work[vah::K_NUM];
    int minb[vah::K_NUM];  // register-cap variant per launch kind (autotuned)
    // FP32 form: tile descriptors per slot, tile work-lists (2+1D, 3+1D), launch counter and error flags
    bool tile;
    vah::TileSlot *d_tdesc;  // [kMaxSlots]
    vah::TileItem *d_titems[2];
    int ntitems[2], cap_titems[2];
    unsigned *d_tcount;      // [0]: tile counter, [1]: error flags
    unsigned *d_wcount;      // [K_NUM] work-list counters of the face/cell launches
    int nwork[vah::K_NUM], cap_work[vah::K_NUM];
    double *d_partial;
    int cap_partial;
    bool dirty;
    cudaGraphExec_t graph;
    bool has_graph;
    bool timing;
    cudaEvent_t t0, t1;
    double kernel_ms;
    long long kernel_steps;
};

namespace {

int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return VAH_OK;
    if (e == cudaErrorMemoryAllocation) return VAH_ERR_NOMEM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return VAH_ERR_NODEVICE;
    return VAH_ERR_CUDA;
}

#define VAH_TRY(call)                                  \
    do {                                               \
        cudaError_t e_ = (call);                       \
        if (e_ != cudaSuccess) return cuda_status(e_); \
    } while (0)

int nq_of(int physics) { return physics == VAH_IDEAL ? 5 : (physics == VAH_PIMUNU ? 15 : 16); }

// Arrays of one event in its allocation: 16 q, 16 qS, 4 e/p, 4 uA, 4 uB,
// 4 uS, and the face buffers (H, plus HR for reference faces) per axis; then
// one byte per cell of fallback flags and one of freeze-out state.
int arrays_per_event(const vah_batch *b, const vah_lattice *lat) {
    if (b->tile) return 48;  // the tile kernel keeps its face fluxes on chip
    const int ndir = lat->nz > 1 ? 3 : 2;
    const int per_face = b->opt.flux == VAH_FLUX_PER_CELL ? 2 : 1;
    return 48 + ndir * b->nq * per_face;
}

// Row pitch of a slot's arrays: nx + 4, padded to 4 floats for the tile form.
int slot_pitch(const vah_batch *b, int nx) { return b->tile ? vah::tile_pitch(nx) : nx + 4; }

size_t event_bytes(const vah_batch *b, const vah_lattice *lat) {
    const size_t ncell = (size_t)slot_pitch(b, lat->nx) * (lat->ny + 4) * (lat->nz + 4);
    const size_t per = (ncell * b->elem + 255) / 256 * 256;
    return per * arrays_per_event(b, lat) + 2 * ((ncell + 255) / 256 * 256) + 256;
}

vah::Eos batch_eos(const vah_batch *b) {
    vah::Eos eos;
    eos.kind = b->opt.eos == VAH_EOS_TABLE ? 1 : 0;
    eos.zeta = b->opt.zeta == VAH_ZETA_CROSSOVER ? 1 : 0;
    eos.tab = b->d_tab;
    eos.exc = b->d_exc;
    eos.nexc = b->nexc;
    return eos;
}

template <typename S>
SlotDesc<S> *desc_host(vah_batch *b, int slot) {
    return (SlotDesc<S> *)b->desc_host.data() + slot;
}

// Energy density at temperature T (fm^-1): the conformal gas e = 13.8997 T^4
// (EquationOfState.cpp:144 inverted) or the table's monotone T(e), bisected
// in ln e.
double energy_at_temperature(const vah_batch *b, double T) {
    if (b->opt.eos != VAH_EOS_TABLE || b->tab.empty()) return 13.8997 * T * T * T * T;
    const int n = (int)b->tab[0];
    const double *Tt = b->tab.data() + VAH_EOS_TABLE_HEADER + n;
    if (T <= Tt[0]) return b->tab[4];
    if (T >= Tt[n - 1]) return b->tab[6];
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (Tt[mid] < T) lo = mid;
        else hi = mid;
    }
    const double w = (T - Tt[lo]) / (Tt[hi] - Tt[lo]);
    return std::exp(b->tab[1] + b->tab[3] * (lo + w));
}

template <typename S>
int fill_slot(vah_batch *b, int slot) {
    vah_batch::Slot &sl = b->slots[slot];
    SlotDesc<S> d;
    memset(&d, 0, sizeof(d));
    d.nx = sl.lat.nx;
    d.ny = sl.lat.ny;
    d.nz = sl.lat.nz;
    d.ncx = slot_pitch(b, sl.lat.nx);
    d.ncy = sl.lat.ny + 4;
    d.plane = (long long)d.ncx * d.ncy;
    d.dx = sl.lat.dx;
    d.dy = sl.lat.dy;
    d.dz = sl.lat.dz;
    d.dt = sl.dt;
    d.etabar = sl.hydro.eta_over_s;
    d.counters = b->d_counters + 4 * slot;
    const size_t ncell = (size_t)d.ncx * d.ncy * (sl.lat.nz + 4);
    const size_t per = (ncell * b->elem + 255) / 256 * 256;
    char *base = (char *)sl.mem;
    size_t off = 0;
    auto next = [&]() {
        S *p = (S *)(base + off);
        off += per;
        return p;
    };
    for (int n = 0; n < 16; ++n) d.q[n] = next();
    for (int n = 0; n < 16; ++n) d.qS[n] = next();
    for (int x = 0; x < 2; ++x)
        for (int y = 0; y < 2; ++y) d.ep[x][y] = next();
    for (int m = 0; m < 4; ++m) d.uA[m] = next();
    for (int m = 0; m < 4; ++m) d.uB[m] = next();
    for (int m = 0; m < 4; ++m) d.uS[m] = next();
    const int ndir = sl.lat.nz > 1 ? 3 : 2;
    if (!b->tile)
        for (int k = 0; k < ndir; ++k)
            for (int n = 0; n < b->nq; ++n) {
                d.H[k][n] = next();
                if (b->opt.flux == VAH_FLUX_PER_CELL) d.HR[k][n] = next();
            }
    d.fallback = (unsigned char *)(base + off);
    d.hot = (unsigned char *)(base + off + (ncell + 255) / 256 * 256);
    d.e_freeze = energy_at_temperature(b, sl.hydro.freezeout_T_GeV / 0.197326938);
    d.crossings = b->d_cross + 2 * slot;
    *desc_host<S>(b, slot) = d;
    VAH_TRY(cudaMemcpyAsync((char *)b->d_desc + sizeof(SlotDesc<S>) * slot, &d, sizeof(d), cudaMemcpyHostToDevice,
                            b->stream));
    if (b->tile) {  // the FP32 form's tile descriptor: the same buffers, q and qS as blocks of per-byte fields
        vah::TileSlot t;
        memset(&t, 0, sizeof(t));
        t.Q[0] = (float *)d.q[0];
        t.Q[1] = (float *)d.qS[0];
        t.fstride = (long long)(per / sizeof(float));
        for (int bb = 0; bb < 2; ++bb) {
            const int rc = vah::tile_encode_q(&t.tmQ[bb], t.Q[bb], sl.lat.nx, sl.lat.ny, sl.lat.nz, d.ncx, t.fstride,
                                              b->nq);
            if (rc != VAH_OK) return rc;
        }
        for (int x = 0; x < 2; ++x)
            for (int y = 0; y < 2; ++y) t.ep[x][y] = (float *)d.ep[x][y];
        for (int m = 0; m < 4; ++m) {
            t.uA[m] = (float *)d.uA[m];
            t.uB[m] = (float *)d.uB[m];
            t.uS[m] = (float *)d.uS[m];
        }
        // the slot's arrays follow one another `per` bytes apart: (e, p) pairs and u quads are blocks
        for (int bb = 0; bb < 2; ++bb) {
            const int rc = vah::tile_encode_p(&t.tmEP[bb], t.ep[bb][0], sl.lat.nx, sl.lat.ny, sl.lat.nz, d.ncx,
                                              t.fstride, 2);
            if (rc != VAH_OK) return rc;
        }
        float *const *us[3] = {t.uA, t.uB, t.uS};
        for (int bb = 0; bb < 3; ++bb) {
            const int rc = vah::tile_encode_p(&t.tmU[bb], us[bb][0], sl.lat.nx, sl.lat.ny, sl.lat.nz, d.ncx,
                                              t.fstride, 4);
            if (rc != VAH_OK) return rc;
        }
        t.nx = d.nx;
        t.ny = d.ny;
        t.nz = d.nz;
        t.pitch = d.ncx;
        t.ncy = d.ncy;
        t.nq = b->nq;
        t.dx = d.dx;
        t.dy = d.dy;
        t.dz = d.dz;
        t.dt = d.dt;
        t.etabar = d.etabar;
        t.counters = d.counters;
        t.zghosts = d.nz > 1;      // 2+1D: the eta ghost layers are filled when a caller reads them
        t.fallback2 = d.fallback;  // the batch keeps the latest (stage-2) flags
        t.hot = d.hot;
        t.e_freeze = d.e_freeze;
        t.crossings = d.crossings;
        // a pageable source: the copy is staged before the call returns (the slot's next use is stream-ordered)
        VAH_TRY(cudaMemcpy(b->d_tdesc + slot, &t, sizeof(t), cudaMemcpyHostToDevice));
    }
    return VAH_OK;
}

int rebuild_tiles(vah_batch *b) {
    std::vector<vah::TileItem> lists[2];  // 2+1D, 3+1D events
    for (int s = 0; s < (int)b->slots.size(); ++s) {
        const vah_batch::Slot &sl = b->slots[s];
        if (sl.used) vah::tile_items(lists[sl.lat.nz > 1 ? 1 : 0], s, sl.lat.nx, sl.lat.ny, sl.lat.nz);
    }
    for (int k = 0; k < 2; ++k) {
        const int n = (int)lists[k].size();
        if (n > b->cap_titems[k]) {
            if (b->d_titems[k]) VAH_TRY(cudaFreeAsync(b->d_titems[k], b->stream));
            const int cap = std::max(n, 2 * b->cap_titems[k]);
            VAH_TRY(cudaMallocFromPoolAsync((void **)&b->d_titems[k], cap * sizeof(vah::TileItem), b->pool, b->stream));
            b->cap_titems[k] = cap;
        }
        if (n) VAH_TRY(cudaMemcpyAsync(b->d_titems[k], lists[k].data(), n * sizeof(vah::TileItem),
                                       cudaMemcpyHostToDevice, b->stream));
        b->ntitems[k] = n;
    }
    VAH_TRY(cudaStreamSynchronize(b->stream));  // the lists die here
    return VAH_OK;
}

int rebuild_work(vah_batch *b) {
    if (b->tile) {  // the reductions still walk the cell work-lists below
        const int rc = rebuild_tiles(b);
        if (rc != VAH_OK) return rc;
    }
    std::vector<WorkItem> lists[vah::K_NUM];
    std::vector<int> order;  // largest event first: its tiles start first, small ones fill the tail
    for (int s = 0; s < (int)b->slots.size(); ++s)
        if (b->slots[s].used) order.push_back(s);
    auto cells = [&](int s) {
        const vah_lattice &l = b->slots[s].lat;
        return (long long)l.nx * l.ny * l.nz;
    };
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cells(x) > cells(y); });
    for (int s : order) {
        const vah_batch::Slot &sl = b->slots[s];
        const int nx = sl.lat.nx, ny = sl.lat.ny, nz = sl.lat.nz;
        auto add = [&](int kind, int ext0, int rows) {
            for (int r0 = 0; r0 < rows; r0 += vah::kTY)
                for (int i0 = 0; i0 < ext0; i0 += vah::kTX) lists[kind].push_back({s, i0, r0, 0});
        };
        if (!b->tile) {
            add(vah::K_FX, nx + 1, ny * nz);
            add(vah::K_FY, nx, (ny + 1) * nz);
            if (nz > 1) add(vah::K_FZ, nx, ny * (nz + 1));
        }
        add(nz > 1 ? vah::K_C3 : vah::K_C2, nx, ny * nz);
    }
    for (int k = 0; k < vah::K_NUM; ++k) {
        const int n = (int)lists[k].size();
        if (n > b->cap_work[k]) {
            if (b->d_work[k]) VAH_TRY(cudaFreeAsync(b->d_work[k], b->stream));
            const int cap = std::max(n, 2 * b->cap_work[k]);
            VAH_TRY(cudaMallocFromPoolAsync((void **)&b->d_work[k], cap * sizeof(WorkItem), b->pool, b->stream));
            b->cap_work[k] = cap;
        }
        if (n) VAH_TRY(cudaMemcpyAsync(b->d_work[k], lists[k].data(), n * sizeof(WorkItem), cudaMemcpyHostToDevice,
                                       b->stream));
        b->nwork[k] = n;
    }
    const int ncells = b->nwork[vah::K_C2] + b->nwork[vah::K_C3];
    if (ncells > b->cap_partial) {
        if (b->d_partial) VAH_TRY(cudaFreeAsync(b->d_partial, b->stream));
        const int cap = std::max(ncells, 2 * b->cap_partial);
        VAH_TRY(cudaMallocFromPoolAsync((void **)&b->d_partial, (size_t)cap * 5 * sizeof(double), b->pool, b->stream));
        b->cap_partial = cap;
    }
    // the copies above read host vectors that die here
    VAH_TRY(cudaStreamSynchronize(b->stream));
    return VAH_OK;
}

// One launch of a kind known at run time, with the batch's register-cap choice.
template <typename S, int PHYS, bool EXACT>
cudaError_t launch_kind_rt(vah_batch *b, const SlotDesc<S> *descs, int kind, int stage, const vah::Eos &eos) {
    using namespace vah;
    const WorkItem *w = b->d_work[kind];
    const int n = b->nwork[kind], m = b->minb[kind];
    switch (kind) {
    case K_FX: return launch_kind<S, PHYS, K_FX, EXACT>(descs, b->d_clk, w, n, stage, eos, b->sms, m, b->d_wcount + kind, b->stream);
    case K_FY: return launch_kind<S, PHYS, K_FY, EXACT>(descs, b->d_clk, w, n, stage, eos, b->sms, m, b->d_wcount + kind, b->stream);
    case K_FZ: return launch_kind<S, PHYS, K_FZ, EXACT>(descs, b->d_clk, w, n, stage, eos, b->sms, m, b->d_wcount + kind, b->stream);
    case K_C2: return launch_kind<S, PHYS, K_C2, EXACT>(descs, b->d_clk, w, n, stage, eos, b->sms, m, b->d_wcount + kind, b->stream);
    case K_C3: return launch_kind<S, PHYS, K_C3, EXACT>(descs, b->d_clk, w, n, stage, eos, b->sms, m, b->d_wcount + kind, b->stream);
    default: return cudaErrorInvalidValue;
    }
}

template <typename S, int PHYS, bool EXACT>
int enqueue_step(vah_batch *b) {
    using namespace vah;
    const SlotDesc<S> *descs = (const SlotDesc<S> *)b->d_desc;
    const Eos eos = batch_eos(b);
    for (int stage = 1; stage <= 2; ++stage)
        for (int kind = 0; kind < K_NUM; ++kind) VAH_TRY((launch_kind_rt<S, PHYS, EXACT>(b, descs, kind, stage, eos)));
    advance_kernel<<<(kMaxSlots + 255) / 256, 256, 0, b->stream>>>(b->d_clk, b->d_dt, kMaxSlots, b->d_cross, b->d_vol,
                                                                 b->d_dv);
    VAH_TRY(cudaGetLastError());
    return VAH_OK;
}

template <typename S>
int enqueue_step_s(vah_batch *b) {
    const bool exact = b->opt.flux == VAH_FLUX_PER_CELL;
    switch (b->opt.physics) {
    case VAH_IDEAL: return exact ? enqueue_step<S, 0, true>(b) : enqueue_step<S, 0, false>(b);
    case VAH_PIMUNU: return exact ? enqueue_step<S, 1, true>(b) : enqueue_step<S, 1, false>(b);
    default: return exact ? enqueue_step<S, 2, true>(b) : enqueue_step<S, 2, false>(b);
    }
}

// FP32 form: per stage one persistent tile launch per tile shape, then the clocks advance.
int enqueue_tiles(vah_batch *b) {
    using namespace vah;
    const Eos eos = batch_eos(b);
    const TileClock none{0.0, 0, 0, 0};
    for (int stage = 1; stage <= 2; ++stage)
        for (int k = 0; k < 2; ++k)
            VAH_TRY(tile_launch(b->d_tdesc, (const TileClock *)b->d_clk, none, 0.0, b->d_titems[k], b->ntitems[k],
                                k == 1, b->d_tcount, stage, b->opt.physics, eos, b->d_tcount + 1, b->stream));
    advance_kernel<<<(kMaxSlots + 255) / 256, 256, 0, b->stream>>>(b->d_clk, b->d_dt, kMaxSlots, b->d_cross, b->d_vol,
                                                                 b->d_dv);
    VAH_TRY(cudaGetLastError());
    return VAH_OK;
}

int enqueue(vah_batch *b) {
    if (b->tile) return enqueue_tiles(b);
    return b->elem == sizeof(float) ? enqueue_step_s<float>(b) : enqueue_step_s<double>(b);
}

int capture_graph(vah_batch *b) {
    if (b->has_graph) {
        cudaGraphExecDestroy(b->graph);
        b->has_graph = false;
    }
    cudaGraph_t g;
    VAH_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue(b);
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc != VAH_OK) return rc;
    VAH_TRY(e);
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    VAH_TRY(e);
    b->has_graph = true;
    b->dirty = false;
    return VAH_OK;
}

template <typename S>
vah::FieldSet<S> fs(S *const *p, int n) {
    vah::FieldSet<S> f{};
    for (int k = 0; k < n; ++k) f.f[k] = p[k];
    f.n = n;
    return f;
}

// Device-generated initial energy density (vah_batch_add_glauber) into the
// slot's e interior: participants sampled, deposited and normalised on the
// GPU; scratch from the batch's pool, freed in stream order.
template <typename S>
int glauber_slot(vah_batch *b, const SlotDesc<S> &d, const vah_lattice &lat, const vah_glauber &g) {
    if (g.A < 1 || g.A > 256 || !(g.width > 0) || !(g.ws_R > 0) || !(g.ws_a > 0) || !std::isfinite(g.ws_R + g.ws_a) ||
        (lat.nz > 1 && !(g.sigma_eta > 0)))
        return VAH_ERR_ARG;
    const size_t nxy = (size_t)lat.nx * lat.ny;
    const size_t bytes = 256 + sizeof(double) * (4 * (size_t)g.A + nxy);
    char *scratch = nullptr;
    VAH_TRY(cudaMallocFromPoolAsync((void **)&scratch, bytes, b->pool, b->stream));
    unsigned long long *maxbits = (unsigned long long *)scratch;
    int *d_np = (int *)(scratch + 64);
    double *d_pxy = (double *)(scratch + 256), *d_v = d_pxy + 4 * (size_t)g.A;
    VAH_TRY(cudaMemsetAsync(maxbits, 0, sizeof(unsigned long long), b->stream));
    VAH_TRY(vah::ic_participants_device(g.b, g.sigma_nn_fm2, g.A, g.ws_R, g.ws_a, g.seed, d_pxy, d_np, b->stream));
    VAH_TRY(vah::ic_deposit_device(d_pxy, d_np, g.width, lat.nx, lat.ny, lat.dx, lat.dy, d_v, maxbits, b->stream));
    int np = 0;  // the sampler reports -1 when its draws ran out (parameters it cannot sample)
    VAH_TRY(cudaMemcpyAsync(&np, d_np, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    VAH_TRY(cudaStreamSynchronize(b->stream));
    if (np < 0) {
        VAH_TRY(cudaFreeAsync(scratch, b->stream));
        return VAH_ERR_ARG;
    }
    VAH_TRY(vah::ic_fill_device<S>(d_v, maxbits, lat.nx, lat.ny, lat.nz, d.ncx, lat.dz, g.eta_flat, g.sigma_eta,
                                   g.e_peak, g.e_floor, d.ep[0][0], b->stream));
    VAH_TRY(cudaFreeAsync(scratch, b->stream));
    return VAH_OK;
}

// Initial state of a slot: e interior uploaded (or generated on the device),
// p = EoS(e), u = 1, pi = 0, conserved variables, ghost layers (the
// vah_event_init_from_e sequence).
template <typename S>
int init_slot(vah_batch *b, int slot, double t0, const double *e_interior, const vah_glauber *glauber, int pl_mode) {
    vah_batch::Slot &sl = b->slots[slot];
    SlotDesc<S> &d = *desc_host<S>(b, slot);
    const int nx = sl.lat.nx, ny = sl.lat.ny, nz = sl.lat.nz;
    std::vector<S> stage;
    if (glauber) {
        const int rc = glauber_slot<S>(b, d, sl.lat, *glauber);
        if (rc != VAH_OK) return rc;
    } else {
        stage.resize((size_t)nx * ny * nz);
        for (size_t k = 0; k < stage.size(); ++k) stage[k] = (S)e_interior[k];
        for (int k = 0; k < nz; ++k) {
            S *dst = d.ep[0][0] + 2 + (size_t)d.ncx * (2 + (size_t)d.ncy * (k + 2));
            VAH_TRY(cudaMemcpy2DAsync(dst, d.ncx * sizeof(S), stage.data() + (size_t)nx * ny * k, nx * sizeof(S),
                                      nx * sizeof(S), ny, cudaMemcpyHostToDevice, b->stream));
        }
    }
    S *qs[16];
    for (int n = 0; n < 16; ++n) qs[n] = n < b->nq || (n == 15 && b->nq == 16) ? d.q[n] : nullptr;
    VAH_TRY(vah::launch_init_primitives<S>(fs<S>(qs, 16), fs<S>(d.uA, 4), d.ep[0][0], d.ep[0][1], batch_eos(b), nx, ny,
                                           nz, d.ncx, b->stream));
    VAH_TRY(vah::launch_set_conserved<S>(fs<S>(qs, 16), fs<S>(d.uA, 4), fs<S>(d.uB, 4), d.ep[0][0], b->opt.physics,
                                         nx, ny, nz, d.ncx, t0, pl_mode == VAH_PL_ISOTROPIC, b->stream));
    vah::FieldSet<S> g{};
    int m = 0;
    g.f[m++] = d.ep[0][0];
    g.f[m++] = d.ep[0][1];
    for (int k = 0; k < 4; ++k) g.f[m++] = d.uA[k];
    for (int k = 0; k < b->nq; ++k) g.f[m++] = d.q[k];
    g.n = m;
    VAH_TRY(vah::launch_ghosts<S>(g, nx, ny, nz, d.ncx, b->stream));
    SlotClock c{t0, 0, 1, 0};
    VAH_TRY(cudaMemcpyAsync(b->d_clk + slot, &c, sizeof(c), cudaMemcpyHostToDevice, b->stream));
    VAH_TRY(cudaMemcpyAsync(b->d_dt + slot, &sl.dt, sizeof(double), cudaMemcpyHostToDevice, b->stream));
    VAH_TRY(cudaMemsetAsync(b->d_counters + 4 * slot, 0, 4 * sizeof(unsigned long long), b->stream));
    VAH_TRY(cudaMemsetAsync(b->d_cross + 2 * slot, 0, 2 * sizeof(unsigned long long), b->stream));
    VAH_TRY(cudaMemsetAsync(b->d_vol + slot, 0, sizeof(double), b->stream));
    const double dv = sl.lat.dx * sl.lat.dy * sl.lat.dz;
    VAH_TRY(cudaMemcpyAsync(b->d_dv + slot, &dv, sizeof(double), cudaMemcpyHostToDevice, b->stream));
    vah::hot_init_kernel<S><<<std::max(1, std::min(nx * ny * nz / 256 + 1, 148 * 16)), 256, 0, b->stream>>>(
        d.ep[0][0], d.hot, d.e_freeze, nx, ny, nz, d.ncx);
    VAH_TRY(cudaGetLastError());
    VAH_TRY(cudaStreamSynchronize(b->stream));  // the staging vector dies here
    return VAH_OK;
}

// Device array currently holding a field of a slot.
template <typename S>
S *slot_field(vah_batch *b, int slot, int field, int parity) {
    SlotDesc<S> &d = *desc_host<S>(b, slot);
    if (field >= 0 && field < 16) return field < b->nq || (field == 15 && b->nq == 16) ? d.q[field] : nullptr;
    if (field == VAH_F_E) return d.ep[0][0];
    if (field == VAH_F_P) return d.ep[0][1];
    if (field >= VAH_F_UT && field <= VAH_F_UN) return (parity ? d.uB : d.uA)[field - VAH_F_UT];
    if (field >= VAH_F_UPT && field <= VAH_F_UPN) return (parity ? d.uA : d.uB)[field - VAH_F_UPT];
    return nullptr;
}

}  // namespace

extern "C" int vah_batch_create(const vah_options *opt, const double *eos_table, size_t capacity_bytes,
                                vah_batch **out) {
    if (!opt || !out) return VAH_ERR_ARG;
    *out = nullptr;
    if (opt->physics < VAH_IDEAL || opt->physics > VAH_PIMUNU_PI) return VAH_ERR_ARG;
    if (opt->eos == VAH_EOS_TABLE && !eos_table) return VAH_ERR_ARG;
    if (opt->precision != VAH_FP64 && opt->precision != VAH_FP32) return VAH_ERR_ARG;
    if (opt->flux != VAH_FLUX_PER_CELL && opt->flux != VAH_FLUX_SHARED) return VAH_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return VAH_ERR_NODEVICE;
    if (opt->device < 0 || opt->device >= ndev) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(opt->device));
    vah_batch *b = new vah_batch();
    b->opt = *opt;
    b->nq = nq_of(opt->physics);
    b->elem = opt->precision == VAH_FP32 ? sizeof(float) : sizeof(double);
    b->tile = opt->precision == VAH_FP32;
    b->own_stream = opt->stream == nullptr;
    b->capacity = capacity_bytes;
    b->used = 0;
    for (int k = 0; k < vah::K_NUM; ++k) b->minb[k] = k <= vah::K_FZ ? 4 : 3;  // untuned default
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, opt->device);
    int rc = VAH_OK;
    auto chk = [&](cudaError_t e) {
        if (rc == VAH_OK && e != cudaSuccess) rc = cuda_status(e);
    };
    if (b->own_stream) chk(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    else b->stream = (cudaStream_t)opt->stream;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = opt->device;
    chk(cudaMemPoolCreate(&b->pool, &props));
    if (rc == VAH_OK) {
        uint64_t keep = UINT64_MAX;  // keep freed event memory in the pool for the next admission
        cudaMemPoolSetAttribute(b->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    const size_t desc_size = b->elem == sizeof(float) ? sizeof(SlotDesc<float>) : sizeof(SlotDesc<double>);
    b->desc_host.assign(desc_size * vah::kMaxSlots, 0);
    b->slots.resize(vah::kMaxSlots);
    chk(cudaMalloc(&b->d_desc, desc_size * vah::kMaxSlots));
    chk(cudaMalloc((void **)&b->d_clk, sizeof(SlotClock) * vah::kMaxSlots));
    chk(cudaMalloc((void **)&b->d_dt, sizeof(double) * vah::kMaxSlots));
    chk(cudaMalloc((void **)&b->d_cross, sizeof(unsigned long long) * 2 * vah::kMaxSlots));
    chk(cudaMalloc((void **)&b->d_vol, sizeof(double) * vah::kMaxSlots));
    chk(cudaMalloc((void **)&b->d_dv, sizeof(double) * vah::kMaxSlots));
    chk(cudaMalloc((void **)&b->d_counters, sizeof(unsigned long long) * 4 * vah::kMaxSlots));
    chk(cudaMalloc((void **)&b->d_maxbits, sizeof(unsigned long long) * vah::kMaxSlots));
    chk(cudaMalloc((void **)&b->d_wcount, sizeof(unsigned) * vah::K_NUM));
    if (b->tile) {
        chk(cudaMalloc((void **)&b->d_tdesc, sizeof(vah::TileSlot) * vah::kMaxSlots));
        chk(cudaMalloc((void **)&b->d_tcount, 2 * sizeof(unsigned)));
        if (rc == VAH_OK) chk(cudaMemset(b->d_tcount, 0, 2 * sizeof(unsigned)));
    }
    if (rc == VAH_OK) {
        chk(cudaMemset(b->d_clk, 0, sizeof(SlotClock) * vah::kMaxSlots));
        chk(cudaMemset(b->d_dt, 0, sizeof(double) * vah::kMaxSlots));
        chk(cudaMemset(b->d_counters, 0, sizeof(unsigned long long) * 4 * vah::kMaxSlots));
        chk(cudaMemset(b->d_cross, 0, sizeof(unsigned long long) * 2 * vah::kMaxSlots));
        chk(cudaMemset(b->d_vol, 0, sizeof(double) * vah::kMaxSlots));
        chk(cudaMemset(b->d_dv, 0, sizeof(double) * vah::kMaxSlots));
    }
    if (rc == VAH_OK && opt->eos == VAH_EOS_TABLE) {
        const size_t len = VAH_EOS_TABLE_LEN((size_t)eos_table[0]);
        chk(cudaMalloc((void **)&b->d_tab, len * sizeof(double)));
        chk(cudaMemcpy(b->d_tab, eos_table, len * sizeof(double), cudaMemcpyHostToDevice));
        b->tab.assign(eos_table, eos_table + len);
    }
    if (rc == VAH_OK && opt->eos == VAH_EOS_CONFORMAL) {
        const std::vector<uint32_t> &exc = vah::powf_quarter_exceptions();
        b->nexc = (int)(exc.size() / 2);
        if (b->nexc) {
            chk(cudaMalloc((void **)&b->d_exc, exc.size() * sizeof(uint32_t)));
            chk(cudaMemcpy(b->d_exc, exc.data(), exc.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
        }
    }
    chk(cudaEventCreate(&b->t0));
    chk(cudaEventCreate(&b->t1));
    b->dirty = true;
    if (rc != VAH_OK) {
        delete b;  // device resources of a failed create are reclaimed at context teardown
        return rc;
    }
    *out = b;
    return VAH_OK;
}

extern "C" int vah_batch_destroy(vah_batch *b) {
    if (!b) return VAH_ERR_ARG;
    cudaSetDevice(b->opt.device);
    cudaStreamSynchronize(b->stream);
    if (b->has_graph) cudaGraphExecDestroy(b->graph);
    for (auto &sl : b->slots)
        if (sl.mem) cudaFreeAsync(sl.mem, b->stream);
    for (int k = 0; k < vah::K_NUM; ++k)
        if (b->d_work[k]) cudaFreeAsync(b->d_work[k], b->stream);
    for (int k = 0; k < 2; ++k)
        if (b->d_titems[k]) cudaFreeAsync(b->d_titems[k], b->stream);
    if (b->d_partial) cudaFreeAsync(b->d_partial, b->stream);
    cudaStreamSynchronize(b->stream);
    cudaMemPoolDestroy(b->pool);
    cudaFree(b->d_desc);
    cudaFree(b->d_clk);
    cudaFree(b->d_dt);
    cudaFree(b->d_cross);
    cudaFree(b->d_vol);
    cudaFree(b->d_dv);
    cudaFree(b->d_counters);
    cudaFree(b->d_maxbits);
    cudaFree(b->d_wcount);
    cudaFree(b->d_tdesc);
    cudaFree(b->d_tcount);
    cudaFree(b->d_tab);
    cudaFree(b->d_exc);
    cudaEventDestroy(b->t0);
    cudaEventDestroy(b->t1);
    if (b->own_stream) cudaStreamDestroy(b->stream);
    delete b;
    return VAH_OK;
}

extern "C" int vah_batch_event_bytes(const vah_batch *b, const vah_lattice *lat, size_t *bytes) {
    if (!b || !lat || !bytes || lat->nx < 1 || lat->ny < 1 || lat->nz < 1) return VAH_ERR_ARG;
    *bytes = event_bytes(b, lat);
    return VAH_OK;
}

namespace {

// Admission shared by vah_batch_add and vah_batch_add_glauber: footprint
// check, slot memory, descriptors, initial state.
int add_slot(vah_batch *b, const vah_lattice *lat, const vah_hydro *hydro, double dt, const double *e_interior,
             const vah_glauber *glauber, int pl_mode, int *slot_out) {
    if (!b || !lat || !hydro || (!e_interior && !glauber) || !slot_out || !(dt > 0) || !(hydro->t0 > 0))
        return VAH_ERR_ARG;
    if (lat->nx < 1 || lat->ny < 1 || lat->nz < 1 || !(hydro->eta_over_s > 0)) return VAH_ERR_ARG;
    const size_t bytes = event_bytes(b, lat);
    if (b->used + bytes > b->capacity) return VAH_ERR_FULL;
    int slot = -1;
    for (int s = 0; s < vah::kMaxSlots; ++s)
        if (!b->slots[s].used) {
            slot = s;
            break;
        }
    if (slot < 0) return VAH_ERR_FULL;
    VAH_TRY(cudaSetDevice(b->opt.device));
    vah_batch::Slot &sl = b->slots[slot];
    VAH_TRY(cudaMallocFromPoolAsync(&sl.mem, bytes, b->pool, b->stream));
    VAH_TRY(cudaMemsetAsync(sl.mem, 0, bytes, b->stream));
    sl.used = true;
    sl.lat = *lat;
    sl.hydro = *hydro;
    sl.dt = dt;
    sl.bytes = bytes;
    b->used += bytes;
    int rc = b->elem == sizeof(float) ? fill_slot<float>(b, slot) : fill_slot<double>(b, slot);
    if (rc == VAH_OK)
        rc = b->elem == sizeof(float) ? init_slot<float>(b, slot, hydro->t0, e_interior, glauber, pl_mode)
                                      : init_slot<double>(b, slot, hydro->t0, e_interior, glauber, pl_mode);
    if (rc != VAH_OK) {
        vah_batch_remove(b, slot);
        return rc;
    }
    b->dirty = true;
    *slot_out = slot;
    return VAH_OK;
}

}  // namespace

extern "C" int vah_batch_add(vah_batch *b, const vah_lattice *lat, const vah_hydro *hydro, double dt,
                             const double *e_interior, int pl_mode, int *slot_out) {
    if (!e_interior) return VAH_ERR_ARG;
    return add_slot(b, lat, hydro, dt, e_interior, nullptr, pl_mode, slot_out);
}

extern "C" int vah_batch_add_glauber(vah_batch *b, const vah_lattice *lat, const vah_hydro *hydro, double dt,
                                     const vah_glauber *g, int pl_mode, int *slot_out) {
    if (!g || g->A < 1 || !(g->width > 0) || !(g->e_peak > 0) || !(g->e_floor >= 0)) return VAH_ERR_ARG;
    if (lat && lat->nz > 1 && !(g->sigma_eta > 0)) return VAH_ERR_ARG;
    return add_slot(b, lat, hydro, dt, nullptr, g, pl_mode, slot_out);
}

extern "C" int vah_batch_remove(vah_batch *b, int slot) {
    if (!b || slot < 0 || slot >= vah::kMaxSlots || !b->slots[slot].used) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(b->opt.device));
    vah_batch::Slot &sl = b->slots[slot];
    SlotClock c{0.0, 0, 0, 0};
    VAH_TRY(cudaMemcpyAsync(b->d_clk + slot, &c, sizeof(c), cudaMemcpyHostToDevice, b->stream));
    VAH_TRY(cudaFreeAsync(sl.mem, b->stream));
    VAH_TRY(cudaStreamSynchronize(b->stream));
    b->used -= sl.bytes;
    sl = vah_batch::Slot();
    b->dirty = true;
    return VAH_OK;
}

extern "C" int vah_batch_step(vah_batch *b, int nsteps) {
    if (!b || nsteps < 0) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(b->opt.device));
    int rc;
    if (b->dirty) {
        if ((rc = rebuild_work(b)) != VAH_OK) return rc;
        if ((rc = capture_graph(b)) != VAH_OK) return rc;
    }
    if (b->timing) VAH_TRY(cudaEventRecord(b->t0, b->stream));
    for (int n = 0; n < nsteps; ++n) VAH_TRY(cudaGraphLaunch(b->graph, b->stream));
    if (b->timing) {
        VAH_TRY(cudaEventRecord(b->t1, b->stream));
        VAH_TRY(cudaEventSynchronize(b->t1));
        float ms = 0;
        VAH_TRY(cudaEventElapsedTime(&ms, b->t0, b->t1));
        b->kernel_ms += ms;
        b->kernel_steps += nsteps;
    }
    return VAH_OK;
}

extern "C" int vah_batch_sync(vah_batch *b) {
    if (!b) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(b->opt.device));
    VAH_TRY(cudaStreamSynchronize(b->stream));
    return VAH_OK;
}

extern "C" int vah_batch_event_info(vah_batch *b, int slot, vah_event_info *out) {
    if (!b || !out || slot < 0 || slot >= vah::kMaxSlots || !b->slots[slot].used) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(b->opt.device));
    SlotClock c;
    unsigned long long cnt[4];
    VAH_TRY(cudaMemcpyAsync(&c, b->d_clk + slot, sizeof(c), cudaMemcpyDeviceToHost, b->stream));
    VAH_TRY(cudaMemcpyAsync(cnt, b->d_counters + 4 * slot, sizeof(cnt), cudaMemcpyDeviceToHost, b->stream));
    VAH_TRY(cudaStreamSynchronize(b->stream));
    out->t = c.t;
    out->steps = c.steps;
    out->face_fallbacks = (long long)cnt[0];
    out->cell_fallbacks = (long long)cnt[1];
    out->nan_cells = (long long)cnt[2];
    out->bytes = (long long)b->slots[slot].bytes;
    return VAH_OK;
}

template <typename S>
const unsigned char *slot_fallback(vah_batch *b, int slot) {
    return desc_host<S>(b, slot)->fallback;
}

extern "C" int vah_batch_get_field(vah_batch *b, int slot, int field, double *host, int with_ghosts) {
    if (!b || !host || slot < 0 || slot >= vah::kMaxSlots || !b->slots[slot].used) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(b->opt.device));
    SlotClock c;
    VAH_TRY(cudaMemcpyAsync(&c, b->d_clk + slot, sizeof(c), cudaMemcpyDeviceToHost, b->stream));
    VAH_TRY(cudaStreamSynchronize(b->stream));
    const vah_lattice &lat = b->slots[slot].lat;
    const size_t ncx = slot_pitch(b, lat.nx), ncy = lat.ny + 4, hx = lat.nx + 4;
    const size_t ncell = hx * ncy * (lat.nz + 4);  // host layout
    const size_t n = with_ghosts ? ncell : (size_t)lat.nx * lat.ny * lat.nz;
    std::vector<float> f32;
    void *src = b->elem == sizeof(float) ? (void *)slot_field<float>(b, slot, field, c.parity)
                                         : (void *)slot_field<double>(b, slot, field, c.parity);
    if (!src) return VAH_ERR_ARG;
    const size_t es = b->elem;
    if (es == sizeof(float)) f32.resize(n);
    void *dst = es == sizeof(float) ? (void *)f32.data() : (void *)host;
    if (with_ghosts && lat.nz == 1) {  // 2+1D steps leave the eta ghost layers to the reader
        if (es == sizeof(float)) {
            vah::FieldSet<float> f{};
            f.f[0] = (float *)src;
            f.n = 1;
            VAH_TRY(vah::launch_ghost_pass<float>(f, lat.nx, lat.ny, lat.nz, (int)ncx, 2, b->stream));
        } else {
            vah::FieldSet<double> f{};
            f.f[0] = (double *)src;
            f.n = 1;
            VAH_TRY(vah::launch_ghost_pass<double>(f, lat.nx, lat.ny, lat.nz, (int)ncx, 2, b->stream));
        }
    }
    if (with_ghosts) {
        VAH_TRY(cudaMemcpy2DAsync(dst, hx * es, src, ncx * es, hx * es, ncy * (lat.nz + 4), cudaMemcpyDeviceToHost,
                                  b->stream));
    } else {
        for (int k = 0; k < lat.nz; ++k) {
            const char *row = (const char *)src + es * (2 + ncx * (2 + ncy * (k + 2)));
            VAH_TRY(cudaMemcpy2DAsync((char *)dst + es * (size_t)lat.nx * lat.ny * k, lat.nx * es, row, ncx * es,
                                      lat.nx * es, lat.ny, cudaMemcpyDeviceToHost, b->stream));
        }
    }
    VAH_TRY(cudaStreamSynchronize(b->stream));
    if (es == sizeof(float))
        for (size_t k = 0; k < n; ++k) host[k] = (double)f32[k];
    return VAH_OK;
}

extern "C" int vah_batch_fallback_mask(vah_batch *b, int slot, unsigned char *host) {
    if (!b || !host || slot < 0 || slot >= vah::kMaxSlots || !b->slots[slot].used) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(b->opt.device));
    const vah_lattice &lat = b->slots[slot].lat;
    const size_t ncx = slot_pitch(b, lat.nx), ncy = lat.ny + 4;
    const unsigned char *src = b->elem == sizeof(float) ? slot_fallback<float>(b, slot) : slot_fallback<double>(b, slot);
    for (int k = 0; k < lat.nz; ++k)
        VAH_TRY(cudaMemcpy2DAsync(host + (size_t)lat.nx * lat.ny * k, lat.nx, src + 2 + ncx * (2 + ncy * (k + 2)), ncx,
                                  lat.nx, lat.ny, cudaMemcpyDeviceToHost, b->stream));
    VAH_TRY(cudaStreamSynchronize(b->stream));
    return VAH_OK;
}

extern "C" int vah_batch_freezeout_volume(vah_batch *b, double *out, int nslots) {
    if (!b || !out || nslots < 0 || nslots > vah::kMaxSlots) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(b->opt.device));
    VAH_TRY(cudaStreamSynchronize(b->stream));
    if (nslots) VAH_TRY(cudaMemcpy(out, b->d_vol, sizeof(double) * nslots, cudaMemcpyDeviceToHost));
    for (int s = 0; s < nslots; ++s)
        if (s >= (int)b->slots.size() || !b->slots[s].used) out[s] = 0.0;
    return VAH_OK;
}

extern "C" int vah_batch_max_energy_density(vah_batch *b, double *out, int nslots) {
    if (!b || !out || nslots < 1) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(b->opt.device));
    int rc;
    if (b->dirty && (rc = rebuild_work(b)) != VAH_OK) return rc;
    VAH_TRY(cudaMemsetAsync(b->d_maxbits, 0, sizeof(unsigned long long) * vah::kMaxSlots, b->stream));
    for (int kind : {vah::K_C2, vah::K_C3}) {
        if (!b->nwork[kind]) continue;
        const int grid = std::min(b->nwork[kind], b->sms * 8);
        if (b->elem == sizeof(float))
            vah::max_e_kernel<float><<<grid, dim3(vah::kTX, vah::kTY), 0, b->stream>>>(
                (const SlotDesc<float> *)b->d_desc, b->d_work[kind], b->nwork[kind], b->d_maxbits, 0);
        else
            vah::max_e_kernel<double><<<grid, dim3(vah::kTX, vah::kTY), 0, b->stream>>>(
                (const SlotDesc<double> *)b->d_desc, b->d_work[kind], b->nwork[kind], b->d_maxbits, 0);
        VAH_TRY(cudaGetLastError());
    }
    std::vector<unsigned long long> bits(vah::kMaxSlots);
    VAH_TRY(cudaMemcpyAsync(bits.data(), b->d_maxbits, bits.size() * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, b->stream));
    VAH_TRY(cudaStreamSynchronize(b->stream));
    for (int s = 0; s < nslots && s < vah::kMaxSlots; ++s) {
        double v;
        memcpy(&v, &bits[s], sizeof(v));
        out[s] = b->slots[s].used ? v : 0.0;
    }
    return VAH_OK;
}

extern "C" int vah_batch_observables(vah_batch *b, double *out, int nslots) {
    if (!b || !out || nslots < 1) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(b->opt.device));
    int rc;
    if (b->dirty && (rc = rebuild_work(b)) != VAH_OK) return rc;
    const int n2 = b->nwork[vah::K_C2], n3 = b->nwork[vah::K_C3];
    auto launch = [&](int kind, double *part) -> cudaError_t {
        const int nw = b->nwork[kind];
        if (!nw) return cudaSuccess;
        const int grid = std::min(nw, b->sms * 8);
        const dim3 blk(vah::kTX, vah::kTY);
        const bool f = b->elem == sizeof(float);
        switch (b->opt.physics) {
        case VAH_IDEAL:
            if (f) vah::observables_kernel<float, 0><<<grid, blk, 0, b->stream>>>((const SlotDesc<float> *)b->d_desc, b->d_clk, b->d_work[kind], nw, part);
            else vah::observables_kernel<double, 0><<<grid, blk, 0, b->stream>>>((const SlotDesc<double> *)b->d_desc, b->d_clk, b->d_work[kind], nw, part);
            break;
        case VAH_PIMUNU:
            if (f) vah::observables_kernel<float, 1><<<grid, blk, 0, b->stream>>>((const SlotDesc<float> *)b->d_desc, b->d_clk, b->d_work[kind], nw, part);
            else vah::observables_kernel<double, 1><<<grid, blk, 0, b->stream>>>((const SlotDesc<double> *)b->d_desc, b->d_clk, b->d_work[kind], nw, part);
            break;
        default:
            if (f) vah::observables_kernel<float, 2><<<grid, blk, 0, b->stream>>>((const SlotDesc<float> *)b->d_desc, b->d_clk, b->d_work[kind], nw, part);
            else vah::observables_kernel<double, 2><<<grid, blk, 0, b->stream>>>((const SlotDesc<double> *)b->d_desc, b->d_clk, b->d_work[kind], nw, part);
        }
        return cudaGetLastError();
    };
    VAH_TRY(launch(vah::K_C2, b->d_partial));
    VAH_TRY(launch(vah::K_C3, b->d_partial + (size_t)n2 * 5));
    std::vector<double> part((size_t)(n2 + n3) * 5);
    std::vector<WorkItem> w2(n2), w3(n3);
    if (n2 + n3) VAH_TRY(cudaMemcpyAsync(part.data(), b->d_partial, part.size() * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    if (n2) VAH_TRY(cudaMemcpyAsync(w2.data(), b->d_work[vah::K_C2], n2 * sizeof(WorkItem), cudaMemcpyDeviceToHost, b->stream));
    if (n3) VAH_TRY(cudaMemcpyAsync(w3.data(), b->d_work[vah::K_C3], n3 * sizeof(WorkItem), cudaMemcpyDeviceToHost, b->stream));
    VAH_TRY(cudaStreamSynchronize(b->stream));
    std::vector<double> acc((size_t)nslots * 5, 0.0);
    auto add = [&](const std::vector<WorkItem> &w, size_t base) {
        for (size_t k = 0; k < w.size(); ++k)
            if (w[k].slot < nslots)
                for (int m = 0; m < 5; ++m) acc[(size_t)w[k].slot * 5 + m] += part[(base + k) * 5 + m];
    };
    add(w2, 0);
    add(w3, n2);
    for (int s = 0; s < nslots; ++s) {
        const double *a = &acc[(size_t)s * 5];
        out[3 * s + 0] = a[0];
        out[3 * s + 1] = a[2] != 0 ? a[1] / a[2] : 0.0;
        out[3 * s + 2] = a[4] != 0 ? a[3] / a[4] : 0.0;
    }
    return VAH_OK;
}

extern "C" int vah_batch_set_timing(vah_batch *b, int on) {
    if (!b) return VAH_ERR_ARG;
    b->timing = on != 0;
    return VAH_OK;
}

extern "C" int vah_batch_kernel_time(vah_batch *b, double *ms, long long *steps) {
    if (!b || !ms || !steps) return VAH_ERR_ARG;
    *ms = b->kernel_ms;
    *steps = b->kernel_steps;
    b->kernel_ms = 0;
    b->kernel_steps = 0;
    return VAH_OK;
}

namespace {

// The batch form of vah_event_autotune: every register-cap variant of each
// launch kind runs over the whole work-list in stage-1 buffer roles (outputs
// are stage scratch), the fastest is kept, the per-slot counters are restored
// and the step graph is re-captured at the next step.
template <typename S, int PHYS, bool EXACT>
int batch_autotune_t(vah_batch *b, int reps, vah_tune_report *out) {
    using namespace vah;
    const SlotDesc<S> *descs = (const SlotDesc<S> *)b->d_desc;
    const Eos eos = batch_eos(b);
    std::vector<unsigned long long> saved((size_t)kMaxSlots * 4);
    VAH_TRY(cudaStreamSynchronize(b->stream));
    VAH_TRY(cudaMemcpy(saved.data(), b->d_counters, saved.size() * sizeof(unsigned long long),
                       cudaMemcpyDeviceToHost));
    cudaEvent_t e0, e1;
    VAH_TRY(cudaEventCreate(&e0));
    VAH_TRY(cudaEventCreate(&e1));
    int rc = VAH_OK;
    out->nkinds = K_NUM;
    for (int kind = 0; kind < K_NUM && rc == VAH_OK; ++kind) {
        vah_launch_choice &r = out->kind[kind];
        const int def = b->minb[kind];
        r = {kTX, kTY, def, 0.0, 0.0};
        if (b->nwork[kind] == 0) continue;
        const int *cand = kind <= K_FZ ? kFaceMinb : kCellMinb;
        double best = 1e300;
        int pick = def;
        for (int c = 0; c < kNumMinb && rc == VAH_OK; ++c) {
            b->minb[kind] = cand[c];
            auto launch = [&]() { return launch_kind_rt<S, PHYS, EXACT>(b, descs, kind, 1, eos); };
            if (launch() != cudaSuccess || cudaEventRecord(e0, b->stream) != cudaSuccess) {
                rc = VAH_ERR_CUDA;
                break;
            }
            for (int k = 0; k < reps && rc == VAH_OK; ++k)
                if (launch() != cudaSuccess) rc = VAH_ERR_CUDA;
            float f = 0;
            if (rc != VAH_OK || cudaEventRecord(e1, b->stream) != cudaSuccess ||
                cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&f, e0, e1) != cudaSuccess) {
                rc = VAH_ERR_CUDA;
                break;
            }
            const double ms = f / reps;
            if (cand[c] == def) r.ms_default = ms;
            if (ms < best) {
                best = ms;
                pick = cand[c];
            }
        }
        b->minb[kind] = pick;
        r = {kTX, kTY, pick, r.ms_default, best};
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (cudaMemcpy(b->d_counters, saved.data(), saved.size() * sizeof(unsigned long long),
                   cudaMemcpyHostToDevice) != cudaSuccess &&
        rc == VAH_OK)
        rc = VAH_ERR_CUDA;
    b->dirty = true;  // the step graph holds the old choice
    return rc;
}

template <typename S>
int batch_autotune_s(vah_batch *b, int reps, vah_tune_report *out) {
    const bool exact = b->opt.flux == VAH_FLUX_PER_CELL;
    switch (b->opt.physics) {
    case VAH_IDEAL: return exact ? batch_autotune_t<S, 0, true>(b, reps, out) : batch_autotune_t<S, 0, false>(b, reps, out);
    case VAH_PIMUNU: return exact ? batch_autotune_t<S, 1, true>(b, reps, out) : batch_autotune_t<S, 1, false>(b, reps, out);
    default: return exact ? batch_autotune_t<S, 2, true>(b, reps, out) : batch_autotune_t<S, 2, false>(b, reps, out);
    }
}

}  // namespace

extern "C" int vah_batch_autotune(vah_batch *b, int reps, vah_tune_report *out) {
    if (!b || !out || reps < 1) return VAH_ERR_ARG;
    memset(out, 0, sizeof(*out));
    if (b->tile) return VAH_OK;  // one persistent tile launch per stage and shape: nothing to tune
    VAH_TRY(cudaSetDevice(b->opt.device));
    if (b->dirty) {  // the work-list must describe the admitted events
        const int rc = rebuild_work(b);
        if (rc != VAH_OK) return rc;
    }
    return b->elem == sizeof(float) ? batch_autotune_s<float>(b, reps, out) : batch_autotune_s<double>(b, reps, out);
}
