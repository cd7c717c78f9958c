// vah_api.cu -- the C ABI of include/vah.h over the CUDA kernels.
//
// An event owns its device state: conserved q (current) and qS (intermediate
// stage), two (e, p) buffers used ping-pong across the two stages, and the
// three velocity sets u (current), up (previous step) and uS (intermediate).
// FP64 storage runs the face/cell split (or fused) kernels on the reference
// layout. VAH_FP32 runs the FP32 form through the TMA-tiled stage kernel
// (vah_tile.cuh): q and qS are then each one block of N_q fields, and every
// field uses a row pitch padded to a multiple of 4 floats; the host-facing
// copies convert to and from the reference layout.
// No call ever exits or traps; failures come back as status codes.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <vector>

#include "vah.h"
#include "vah_ic_device.cuh"
#include "vah_kernels.cuh"
#include "vah_powf_exc.h"
#include "vah_tile.cuh"

using vah::FieldSet;
using vah::StageArgs;
using vah::ValidityArgs;

struct vah_event {
    vah_lattice lat;
    vah_hydro hydro;
    vah_options opt;
    int nq;
    int ncx, ncy, ncz;
    size_t ncell;
    cudaStream_t stream;
    bool own_stream;
    size_t elem;       // bytes per stored value: 8 (VAH_FP64) or 4 (VAH_FP32)
    void *q[16], *qS[16];
    void *ep[2][2];    // [buffer][0 = e, 1 = p]
    int cur;           // current (e, p) buffer
    void *u[4], *up[4], *uS[4];
    void *H[3][16];    // face fluxes as the left cell evaluates them (scratch of a stage)
    void *HR[3][16];   // ... and as the right cell does (reference face semantics)
    double *d_tab;
    uint32_t *d_exc;
    int nexc;
    unsigned long long *d_counters;  // face fallbacks, cell fallbacks, NaN cells
    unsigned char *d_fb;             // optional: per ghosted cell, stage-1 then stage-2 inversion fallback flags
    long long steps;
    double last_t, last_dt;          // time and step of the latest vah_rk2_step (autotuning state)
    double *d_stage64;               // FP32 storage: one FP64 field of staging for the host-buffer step ...
    double *d_stage_all;             // ... and every field, host layout, for its overlapped form (3+1D)
    bool validity;                   // fill the validity diagnostics every step
    double *vd[VAH_NUM_VALIDITY];    // validity fields (FP64, ghosted layout)
    void *vq[16];                    // P_L, pi, Pi at the start of the step (validity input)
    vah::SplitConfig split;          // launch configuration of the face/cell kernels
    bool timing;
    std::vector<cudaEvent_t> tev;  // start/stop pairs of timed launches
    int tev_used;
    double kernel_ms;
    long long kernel_launches;
    cudaStream_t s_in, s_out;         // copy streams of the pipelined host-buffer step (created on first use)
    std::vector<cudaEvent_t> pev;     // its slab events
    // FP32 form (tile layout)
    bool tile;
    void *qblock[2];                  // q and qS: nq fields each, ncell floats apart
    void *pblock;                     // e, p of both buffers, then u, up, uS: 16 fields, ncell floats apart
    vah::TileSlot h_tslot;            // the event's tile descriptor (host copy) ...
    vah::TileSlot *d_tslot;           // ... and on the device
    vah::TileItem *d_titems;
    int ntitems;
    unsigned *d_tcount, *d_terr;      // tile counter of a launch; kernel error flags
    int tparity;                      // 0: u^n in the descriptor's uA; 1: in uB
};

namespace {

int nq_of(int physics) { return physics == VAH_IDEAL ? 5 : (physics == VAH_PIMUNU ? 15 : 16); }

int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return VAH_OK;
    if (e == cudaErrorMemoryAllocation) return VAH_ERR_NOMEM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorNoKernelImageForDevice)
        return VAH_ERR_NODEVICE;
    return VAH_ERR_CUDA;
}

#define VAH_TRY(call)                               \
    do {                                            \
        cudaError_t e_ = (call);                    \
        if (e_ != cudaSuccess) return cuda_status(e_); \
    } while (0)

void *field_ptr(vah_event *ev, int id) {
    if (id >= 0 && id < 16) return ev->q[id];  // null for slots the physics variant lacks
    switch (id) {
    case VAH_F_E: return ev->ep[ev->cur][0];
    case VAH_F_P: return ev->ep[ev->cur][1];
    case VAH_F_UT: case VAH_F_UX: case VAH_F_UY: case VAH_F_UN: return ev->u[id - VAH_F_UT];
    case VAH_F_UPT: case VAH_F_UPX: case VAH_F_UPY: case VAH_F_UPN: return ev->up[id - VAH_F_UPT];
    default: return nullptr;
    }
}

void free_all(vah_event *ev) {
    if (ev->tile) {
        cudaFree(ev->qblock[0]);
        cudaFree(ev->qblock[1]);
        cudaFree(ev->pblock);
        cudaFree(ev->d_tslot);
        cudaFree(ev->d_titems);
        cudaFree(ev->d_tcount);  // d_terr lives in the same allocation
    } else {
        for (int n = 0; n < 16; ++n) {
            cudaFree(ev->q[n]);
            cudaFree(ev->qS[n]);
        }
    }
    if (!ev->tile) {
        for (int b = 0; b < 2; ++b)
            for (int m = 0; m < 2; ++m) cudaFree(ev->ep[b][m]);
        for (int m = 0; m < 4; ++m) {
            cudaFree(ev->u[m]);
            cudaFree(ev->up[m]);
            cudaFree(ev->uS[m]);
        }
    }
    for (int d = 0; d < 3; ++d)
        for (int n = 0; n < 16; ++n) {
            cudaFree(ev->H[d][n]);
            cudaFree(ev->HR[d][n]);
        }
    cudaFree(ev->d_tab);
    cudaFree(ev->d_exc);
    cudaFree(ev->d_counters);
    cudaFree(ev->d_fb);
    cudaFree(ev->d_stage64);
    cudaFree(ev->d_stage_all);
    for (int m = 0; m < VAH_NUM_VALIDITY; ++m) cudaFree(ev->vd[m]);
    for (int n = 0; n < 16; ++n) cudaFree(ev->vq[n]);
    for (cudaEvent_t e : ev->tev) cudaEventDestroy(e);
    for (cudaEvent_t e : ev->pev) cudaEventDestroy(e);
    if (ev->s_in) cudaStreamDestroy(ev->s_in);
    if (ev->s_out) cudaStreamDestroy(ev->s_out);
    if (ev->own_stream && ev->stream) cudaStreamDestroy(ev->stream);
}

vah::Eos make_eos(const vah_event *ev) {
    vah::Eos eos;
    eos.kind = ev->opt.eos == VAH_EOS_TABLE ? 1 : 0;
    eos.zeta = ev->opt.zeta == VAH_ZETA_CROSSOVER ? 1 : 0;
    eos.tab = ev->d_tab;
    eos.exc = ev->d_exc;
    eos.nexc = ev->nexc;
    return eos;
}

// Whether the steps store the eta ghost layers (3+1D, or validity
// diagnostics, which read them); else they are filled when read.
bool zghosts_eager(const vah_event *ev) { return ev->lat.nz > 1 || ev->validity; }

template <typename S>
void fill_common(const vah_event *ev, StageArgs<S> &a) {
    memset(&a, 0, sizeof(a));
    a.nx = ev->lat.nx;
    a.ny = ev->lat.ny;
    a.nz = ev->lat.nz;
    a.k0 = 0;
    a.k1 = ev->lat.nz;
    a.ncx = ev->ncx;
    a.ncy = ev->ncy;
    a.plane = (long long)ev->ncx * ev->ncy;
    a.dx = ev->lat.dx;
    a.dy = ev->lat.dy;
    a.dz = ev->lat.dz;
    a.etabar = ev->hydro.eta_over_s;
    a.eos = make_eos(ev);
    a.zghosts = zghosts_eager(ev);
    a.counters = ev->d_counters;
    for (int d = 0; d < 3; ++d)
        for (int n = 0; n < 16; ++n) {
            a.H[d][n] = (S *)ev->H[d][n];
            a.HR[d][n] = (S *)ev->HR[d][n];
        }
    // FP64 face/cell split: the x face launch writes each cell's x flux
    // difference into the x face scratch, and the cell launch reads that
    if (sizeof(S) == sizeof(double) && ev->opt.flux != VAH_FLUX_PER_CELL_FUSED)
        for (int n = 0; n < 16; ++n) a.Dx[n] = (S *)ev->H[0][n];
    if (ev->validity)
        for (int m = 0; m < 11; ++m) a.regmap[m] = ev->vd[VAH_V_REGULATIONS + m];
}

// Run `launch` (the launches of one stage), bracketed by CUDA events on the
// event's stream when timing is on.
template <typename F>
int timed(vah_event *ev, F launch) {
    cudaEvent_t *pair = nullptr;
    if (ev->timing) {
        if ((size_t)(ev->tev_used + 2) > ev->tev.size()) {
            for (int k = 0; k < 256; ++k) {
                cudaEvent_t e;
                VAH_TRY(cudaEventCreate(&e));
                ev->tev.push_back(e);
            }
        }
        pair = &ev->tev[ev->tev_used];
        ev->tev_used += 2;
        VAH_TRY(cudaEventRecord(pair[0], ev->stream));
    }
    VAH_TRY(launch());
    if (pair) VAH_TRY(cudaEventRecord(pair[1], ev->stream));
    return VAH_OK;
}

template <typename S>
int timed_launch(vah_event *ev, const StageArgs<S> &a) {
    return timed(ev, [&]() {
        if (ev->opt.flux == VAH_FLUX_PER_CELL_FUSED) return vah::launch_stage<S>(a, ev->opt.physics, ev->stream);
        return vah::launch_stage_split<S>(a, ev->opt.physics, ev->opt.flux == VAH_FLUX_PER_CELL, ev->split,
                                          ev->stream);
    });
}

// One stage of the FP32 form: the persistent tile launch over the event's tiles.
int tile_stage(vah_event *ev, int stage, double t, double dt) {
    const vah::TileClock clk0{t, ev->tparity, 1, ev->steps};
    const vah::Eos eos = make_eos(ev);
    return timed(ev, [&]() {
        return vah::tile_launch(ev->d_tslot, nullptr, clk0, dt, ev->d_titems, ev->ntitems, ev->lat.nz > 1,
                                ev->d_tcount, stage, ev->opt.physics, eos, ev->d_terr, ev->stream);
    });
}

}  // namespace

namespace {

// Copy the host tile descriptor to the device (after a buffer role changes).
int tile_sync_desc(vah_event *ev) {
    VAH_TRY(cudaMemcpyAsync(ev->d_tslot, &ev->h_tslot, sizeof(vah::TileSlot), cudaMemcpyHostToDevice, ev->stream));
    VAH_TRY(cudaStreamSynchronize(ev->stream));  // the host copy may change again
    return VAH_OK;
}

// The tile descriptor, tensor maps and work-list of an FP32 event.
int tile_setup(vah_event *ev) {
    vah::TileSlot &d = ev->h_tslot;
    memset(&d, 0, sizeof(d));
    for (int b = 0; b < 2; ++b) {
        d.Q[b] = (float *)ev->qblock[b];
        const int rc = vah::tile_encode_q(&d.tmQ[b], d.Q[b], ev->lat.nx, ev->lat.ny, ev->lat.nz, ev->ncx,
                                          (long long)ev->ncell, ev->nq);
        if (rc != VAH_OK) return rc;
    }
    for (int b = 0; b < 2; ++b)
        for (int m = 0; m < 2; ++m) d.ep[b][m] = (float *)ev->ep[b == 0 ? ev->cur : 1 - ev->cur][m];
    for (int m = 0; m < 4; ++m) {
        d.uA[m] = (float *)ev->u[m];
        d.uB[m] = (float *)ev->up[m];
        d.uS[m] = (float *)ev->uS[m];
    }
    const int nx = ev->lat.nx, ny = ev->lat.ny, nz = ev->lat.nz;
    const long long fs = (long long)ev->ncell;
    for (int b = 0; b < 2; ++b) {
        const int rc = vah::tile_encode_p(&d.tmEP[b], d.ep[b][0], nx, ny, nz, ev->ncx, fs, 2);
        if (rc != VAH_OK) return rc;
    }
    float *const *us[3] = {d.uA, d.uB, d.uS};
    for (int b = 0; b < 3; ++b) {
        const int rc = vah::tile_encode_p(&d.tmU[b], us[b][0], nx, ny, nz, ev->ncx, fs, 4);
        if (rc != VAH_OK) return rc;
    }
    d.fstride = (long long)ev->ncell;
    d.nx = ev->lat.nx;
    d.ny = ev->lat.ny;
    d.nz = ev->lat.nz;
    d.pitch = ev->ncx;
    d.ncy = ev->ncy;
    d.nq = ev->nq;
    d.dx = ev->lat.dx;
    d.dy = ev->lat.dy;
    d.dz = ev->lat.dz;
    d.dt = 0.0;  // events pass their step with each launch
    d.etabar = ev->hydro.eta_over_s;
    d.counters = ev->d_counters;
    d.zghosts = zghosts_eager(ev);
    VAH_TRY(cudaMalloc((void **)&ev->d_tslot, sizeof(vah::TileSlot)));
    std::vector<vah::TileItem> items;
    vah::tile_items(items, 0, ev->lat.nx, ev->lat.ny, ev->lat.nz);
    ev->ntitems = (int)items.size();
    VAH_TRY(cudaMalloc((void **)&ev->d_titems, items.size() * sizeof(vah::TileItem)));
    VAH_TRY(cudaMemcpy(ev->d_titems, items.data(), items.size() * sizeof(vah::TileItem), cudaMemcpyHostToDevice));
    VAH_TRY(cudaMalloc((void **)&ev->d_tcount, 2 * sizeof(unsigned)));
    ev->d_terr = ev->d_tcount + 1;
    VAH_TRY(cudaMemset(ev->d_tcount, 0, 2 * sizeof(unsigned)));
    return tile_sync_desc(ev);
}

}  // namespace

extern "C" const char *vah_version(void) { return "vah-b200 0.1 (sm_100a)"; }

namespace {

// Per input: relative error of the Newton correction's reciprocal and of
// rsqrt_d against CUDA's IEEE-rounded operations.
__global__ void math_check_kernel(const double *x, double *err, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double v = x[i];
        const double r_ref = __drcp_rn(v), r = vah::newton_correction(1.0, v);
        err[2 * i] = r == r_ref ? 0.0 : fabs(r - r_ref) / fabs(r_ref);  // equal infinities included
        // rsqrt_d's callers pass 1 + (a sum of squares) >= 1; it is checked on [2^-1000, 2^1000]
        const double a = fabs(v), s_ref = 1.0 / __dsqrt_rn(a);
        err[2 * i + 1] = (a >= 0x1p-1000 && a <= 0x1p1000) ? fabs(vah::rsqrt_d(a) - s_ref) / s_ref : 0.0;
    }
}

}  // namespace

extern "C" int vah_math_check(int device, double lo, double hi, int n, double *max_rel_rcp, double *max_rel_rsqrt) {
    if (!max_rel_rcp || !max_rel_rsqrt || n < 2 || !(lo > 0) || !(hi > lo)) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(device));
    std::vector<double> x(n), err(2 * (size_t)n);
    const double l0 = std::log(lo), l1 = std::log(hi);
    for (int i = 0; i < n; ++i) x[i] = (i & 1 ? -1.0 : 1.0) * std::exp(l0 + (l1 - l0) * i / (n - 1));
    double *d_x = nullptr, *d_err = nullptr;
    int rc = VAH_OK;
    if (cudaMalloc((void **)&d_x, n * sizeof(double)) != cudaSuccess ||
        cudaMalloc((void **)&d_err, 2 * (size_t)n * sizeof(double)) != cudaSuccess)
        rc = VAH_ERR_NOMEM;
    if (rc == VAH_OK && cudaMemcpy(d_x, x.data(), n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        rc = VAH_ERR_CUDA;
    if (rc == VAH_OK) {
        math_check_kernel<<<148 * 4, 256>>>(d_x, d_err, n);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpy(err.data(), d_err, err.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = VAH_ERR_CUDA;
    }
    cudaFree(d_x);
    cudaFree(d_err);
    if (rc != VAH_OK) return rc;
    double m0 = 0, m1 = 0;
    for (int i = 0; i < n; ++i) {  // a NaN error counts as infinite
        m0 = std::max(m0, err[2 * i] == err[2 * i] ? err[2 * i] : INFINITY);
        m1 = std::max(m1, err[2 * i + 1] == err[2 * i + 1] ? err[2 * i + 1] : INFINITY);
    }
    *max_rel_rcp = m0;
    *max_rel_rsqrt = m1;
    return VAH_OK;
}

namespace {

// FP64 FMA throughput: every thread runs 8 independent chains of `iters`
// dependent FMAs (enough independent work to hide the FMA latency at full
// occupancy); the result is folded into one store so the chains stay live.
__global__ void __launch_bounds__(256) fp64_fma_kernel(double *out, int iters, double a, double b) {
    double x[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) x[c] = (threadIdx.x + blockIdx.x * 7 + c) * 1e-3;
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int c = 0; c < 8; ++c) x[c] = fma(x[c], a, b);
    double s = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) s += x[c];
    if (s == 12345.678) out[0] = s;  // practically never: keeps the chains from being removed
}

}  // namespace

extern "C" int vah_fp64_peak(int device, double *tflops, double *ms) {
    if (!tflops || !ms) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(device));
    int sms = 0;
    VAH_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    double *d_out = nullptr;
    VAH_TRY(cudaMalloc((void **)&d_out, sizeof(double)));
    cudaEvent_t e0, e1;
    int rc = VAH_OK;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) rc = VAH_ERR_CUDA;
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;
    if (rc == VAH_OK) {
        fp64_fma_kernel<<<blocks, threads>>>(d_out, iters / 16, 0.999999, 1e-7);  // warm-up
        double best = 1e30;
        for (int r = 0; r < 5 && rc == VAH_OK; ++r) {
            float m = 0;
            if (cudaEventRecord(e0) != cudaSuccess) rc = VAH_ERR_CUDA;
            fp64_fma_kernel<<<blocks, threads>>>(d_out, iters, 0.999999, 1e-7);
            if (cudaEventRecord(e1) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                cudaEventElapsedTime(&m, e0, e1) != cudaSuccess)
                rc = VAH_ERR_CUDA;
            best = std::min(best, (double)m);
        }
        if (rc == VAH_OK) {
            *ms = best;
            *tflops = 2.0 * 8.0 * iters * (double)blocks * threads / (best * 1e-3) / 1e12;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d_out);
    return rc;
}

extern "C" int vah_event_create(const vah_lattice *lat, const vah_hydro *hydro, const vah_options *opt,
                                const double *eos_table, vah_event **out) {
    if (!lat || !hydro || !opt || !out) return VAH_ERR_ARG;
    *out = nullptr;
    if (lat->nx < 1 || lat->ny < 1 || lat->nz < 1) return VAH_ERR_ARG;
    if (!(lat->dx > 0) || !(lat->dy > 0) || !(lat->dz > 0) || !(hydro->eta_over_s > 0)) return VAH_ERR_ARG;
    if (opt->physics < VAH_IDEAL || opt->physics > VAH_PIMUNU_PI) return VAH_ERR_ARG;
    if (opt->eos != VAH_EOS_CONFORMAL && opt->eos != VAH_EOS_TABLE) return VAH_ERR_ARG;
    if (opt->eos == VAH_EOS_TABLE && !eos_table) return VAH_ERR_ARG;
    if (opt->precision != VAH_FP64 && opt->precision != VAH_FP32) return VAH_ERR_ARG;
    if (opt->flux != VAH_FLUX_PER_CELL && opt->flux != VAH_FLUX_SHARED && opt->flux != VAH_FLUX_PER_CELL_FUSED)
        return VAH_ERR_ARG;

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return VAH_ERR_NODEVICE;
    if (opt->device < 0 || opt->device >= ndev) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(opt->device));

    vah_event *ev = new vah_event();
    memset(ev->q, 0, sizeof(ev->q));
    ev->lat = *lat;
    ev->hydro = *hydro;
    ev->opt = *opt;
    ev->nq = nq_of(opt->physics);
    ev->tile = opt->precision == VAH_FP32;
    ev->ncx = ev->tile ? vah::tile_pitch(lat->nx) : lat->nx + 4;  // row pitch of the device arrays
    ev->ncy = lat->ny + 4;
    ev->ncz = lat->nz + 4;
    ev->ncell = (size_t)ev->ncx * ev->ncy * ev->ncz;
    ev->elem = opt->precision == VAH_FP32 ? sizeof(float) : sizeof(double);
    ev->cur = 0;
    ev->tev_used = 0;
    ev->kernel_ms = 0;
    ev->kernel_launches = 0;
    ev->timing = false;
    ev->steps = 0;
    ev->last_t = hydro->t0;
    ev->d_stage64 = nullptr;
    ev->d_stage_all = nullptr;
    ev->d_fb = nullptr;
    ev->s_in = nullptr;
    ev->s_out = nullptr;
    ev->validity = false;
    memset(ev->vd, 0, sizeof(ev->vd));
    memset(ev->vq, 0, sizeof(ev->vq));
    ev->last_dt = 0.005;
    ev->split = vah::default_split_config();
    ev->nexc = 0;
    ev->qblock[0] = ev->qblock[1] = nullptr;
    ev->pblock = nullptr;
    ev->d_tslot = nullptr;
    ev->d_titems = nullptr;
    ev->d_tcount = ev->d_terr = nullptr;
    ev->ntitems = 0;
    ev->tparity = 0;
    ev->own_stream = opt->stream == nullptr;
    int rc = VAH_OK;
    auto alloc = [&](void **p) {
        if (rc != VAH_OK) return;
        cudaError_t e = cudaMalloc(p, ev->ncell * ev->elem);
        if (e == cudaSuccess) e = cudaMemset(*p, 0, ev->ncell * ev->elem);
        if (e != cudaSuccess) rc = cuda_status(e);
    };
    if (ev->own_stream) {
        if (cudaStreamCreateWithFlags(&ev->stream, cudaStreamNonBlocking) != cudaSuccess) rc = VAH_ERR_CUDA;
    } else {
        ev->stream = (cudaStream_t)opt->stream;
    }
    if (ev->tile) {  // q and qS as blocks of nq fields (one tensor map each)
        for (int b = 0; b < 2 && rc == VAH_OK; ++b) {
            cudaError_t e = cudaMalloc(&ev->qblock[b], ev->nq * ev->ncell * sizeof(float));
            if (e == cudaSuccess) e = cudaMemset(ev->qblock[b], 0, ev->nq * ev->ncell * sizeof(float));
            if (e != cudaSuccess) rc = cuda_status(e);
        }
        if (rc == VAH_OK)
            for (int n = 0; n < ev->nq; ++n) {
                ev->q[n] = (float *)ev->qblock[0] + n * ev->ncell;
                ev->qS[n] = (float *)ev->qblock[1] + n * ev->ncell;
            }
    } else {
        for (int n = 0; n < 16; ++n)
            if (n < ev->nq || (n == VAH_F_PI && ev->nq == 16)) {
                alloc(&ev->q[n]);
                alloc(&ev->qS[n]);
            }
    }
    if (ev->tile) {  // the primitives as one block: (e, p) pairs and u quads are TMA boxes
        if (rc == VAH_OK) {
            cudaError_t e = cudaMalloc(&ev->pblock, 16 * ev->ncell * sizeof(float));
            if (e == cudaSuccess) e = cudaMemset(ev->pblock, 0, 16 * ev->ncell * sizeof(float));
            if (e != cudaSuccess) rc = cuda_status(e);
        }
        if (rc == VAH_OK) {
            float *pb = (float *)ev->pblock;
            for (int b = 0; b < 2; ++b)
                for (int m = 0; m < 2; ++m) ev->ep[b][m] = pb + (2 * b + m) * ev->ncell;
            for (int m = 0; m < 4; ++m) {
                ev->u[m] = pb + (4 + m) * ev->ncell;
                ev->up[m] = pb + (8 + m) * ev->ncell;
                ev->uS[m] = pb + (12 + m) * ev->ncell;
            }
        }
    } else {
        for (int b = 0; b < 2; ++b)
            for (int m = 0; m < 2; ++m) alloc(&ev->ep[b][m]);
        for (int m = 0; m < 4; ++m) {
            alloc(&ev->u[m]);
            alloc(&ev->up[m]);
            alloc(&ev->uS[m]);
        }
    }
    if (opt->flux != VAH_FLUX_PER_CELL_FUSED && !ev->tile)
        for (int d = 0; d < (lat->nz > 1 ? 3 : 2); ++d)
            for (int n = 0; n < ev->nq; ++n) {
                alloc(&ev->H[d][n]);
                if (opt->flux == VAH_FLUX_PER_CELL) alloc(&ev->HR[d][n]);
            }
    if (rc == VAH_OK && cudaMalloc((void **)&ev->d_counters, 4 * sizeof(unsigned long long)) != cudaSuccess)
        rc = VAH_ERR_NOMEM;
    if (rc == VAH_OK) cudaMemset(ev->d_counters, 0, 4 * sizeof(unsigned long long));
    if (rc == VAH_OK && opt->eos == VAH_EOS_TABLE) {
        const size_t len = VAH_EOS_TABLE_LEN((size_t)eos_table[0]);
        if (cudaMalloc((void **)&ev->d_tab, len * sizeof(double)) != cudaSuccess) rc = VAH_ERR_NOMEM;
        else if (cudaMemcpy(ev->d_tab, eos_table, len * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
            rc = VAH_ERR_CUDA;
    }
    if (rc == VAH_OK && opt->eos == VAH_EOS_CONFORMAL) {
        const std::vector<uint32_t> &exc = vah::powf_quarter_exceptions();
        ev->nexc = (int)(exc.size() / 2);
        if (ev->nexc > 0) {
            if (cudaMalloc((void **)&ev->d_exc, exc.size() * sizeof(uint32_t)) != cudaSuccess) rc = VAH_ERR_NOMEM;
            else if (cudaMemcpy(ev->d_exc, exc.data(), exc.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) !=
                     cudaSuccess)
                rc = VAH_ERR_CUDA;
        }
    }
    if (rc == VAH_OK && ev->tile) rc = tile_setup(ev);
    if (rc != VAH_OK) {
        free_all(ev);
        delete ev;
        return rc;
    }
    *out = ev;
    return VAH_OK;
}

extern "C" int vah_event_destroy(vah_event *ev) {
    if (!ev) return VAH_ERR_ARG;
    cudaSetDevice(ev->opt.device);
    cudaStreamSynchronize(ev->stream);
    free_all(ev);
    delete ev;
    return VAH_OK;
}

namespace {

// Copy interior or full arrays between double host memory and the event's
// storage type; FP32 storage converts through a host staging buffer.
int copy_field(vah_event *ev, void *d, double *host_out, const double *host_in, int with_ghosts) {
    const int nx = ev->lat.nx, ny = ev->lat.ny, nz = ev->lat.nz;
    const size_t full = (size_t)(nx + 4) * ev->ncy * ev->ncz, inner = (size_t)nx * ny * nz;  // host layouts
    const size_t n = with_ghosts ? full : inner;
    const bool to_dev = host_in != nullptr;
    std::vector<float> stage;
    if (ev->elem == sizeof(float)) {
        stage.resize(n);
        if (to_dev)
            for (size_t k = 0; k < n; ++k) stage[k] = (float)host_in[k];
    }
    const void *src_h = ev->elem == sizeof(float) ? (const void *)stage.data() : (const void *)host_in;
    void *dst_h = ev->elem == sizeof(float) ? (void *)stage.data() : (void *)host_out;
    const size_t es = ev->elem;
    if (with_ghosts) {  // rows of nx + 4 on the host, of the device pitch on the device
        const size_t w = (size_t)(nx + 4) * es, rows = (size_t)ev->ncy * ev->ncz;
        if (to_dev)
            VAH_TRY(cudaMemcpy2DAsync(d, ev->ncx * es, src_h, w, w, rows, cudaMemcpyHostToDevice, ev->stream));
        else
            VAH_TRY(cudaMemcpy2DAsync(dst_h, w, d, ev->ncx * es, w, rows, cudaMemcpyDeviceToHost, ev->stream));
    } else {
        for (int k = 0; k < nz; ++k) {
            char *dev_row = (char *)d + es * (2 + (size_t)ev->ncx * (2 + (size_t)ev->ncy * (k + 2)));
            const size_t off = es * (size_t)nx * ny * k;
            if (to_dev)
                VAH_TRY(cudaMemcpy2DAsync(dev_row, ev->ncx * es, (const char *)src_h + off, nx * es, nx * es, ny,
                                          cudaMemcpyHostToDevice, ev->stream));
            else
                VAH_TRY(cudaMemcpy2DAsync((char *)dst_h + off, nx * es, dev_row, ev->ncx * es, nx * es, ny,
                                          cudaMemcpyDeviceToHost, ev->stream));
        }
    }
    VAH_TRY(cudaStreamSynchronize(ev->stream));
    if (!to_dev && ev->elem == sizeof(float))
        for (size_t k = 0; k < n; ++k) host_out[k] = (double)stage[k];
    return VAH_OK;
}

}  // namespace

extern "C" int vah_event_set_field(vah_event *ev, int field, const double *host, int with_ghosts) {
    if (!ev || !host) return VAH_ERR_ARG;
    void *d = field_ptr(ev, field);
    if (!d) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(ev->opt.device));
    return copy_field(ev, d, nullptr, host, with_ghosts);
}

namespace {

template <typename S>
int fill_zghosts_t(vah_event *ev, const int *ids, int n) {
    vah::FieldSet<S> f{};
    for (int k = 0; k < n; ++k) {
        // u^{n-1} is a former u buffer once a step has run; before that it is the caller's, which
        // the reference's ghost fill does not touch (setGhostCellVars, DynamicalVariables.cpp:358-389)
        void *d = ids[k] >= VAH_F_UPT && ev->steps == 0 ? nullptr : field_ptr(ev, ids[k]);
        if (d) f.f[f.n++] = (S *)d;
        if (f.n == 32 || (k == n - 1 && f.n)) {
            VAH_TRY(vah::launch_ghost_pass<S>(f, ev->lat.nx, ev->lat.ny, ev->lat.nz, ev->ncx, 2, ev->stream));
            f.n = 0;
        }
    }
    return VAH_OK;
}

// 2+1D events whose steps leave the eta ghost layers (no stencil reads them):
// the eta pass of the reference's ghost fill (setGhostCellsKernelK) over the
// given fields, before a caller reads them with ghosts. Stream-ordered.
int fill_zghosts(vah_event *ev, const int *ids, int n) {
    if (zghosts_eager(ev) || n <= 0) return VAH_OK;
    return ev->elem == sizeof(float) ? fill_zghosts_t<float>(ev, ids, n) : fill_zghosts_t<double>(ev, ids, n);
}

}  // namespace

extern "C" int vah_event_get_field(vah_event *ev, int field, double *host, int with_ghosts) {
    if (!ev || !host) return VAH_ERR_ARG;
    void *d = field_ptr(ev, field);
    if (!d) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(ev->opt.device));
    if (with_ghosts) {
        const int rc = fill_zghosts(ev, &field, 1);
        if (rc != VAH_OK) return rc;
    }
    return copy_field(ev, d, host, nullptr, with_ghosts);
}

namespace {

template <typename S>
FieldSet<S> field_set(void *const *p, int n) {
    FieldSet<S> f{};
    for (int k = 0; k < n; ++k) f.f[k] = (S *)p[k];
    f.n = n;
    return f;
}

template <typename S>
int set_conserved_t(vah_event *ev, double t, int pl_from_field) {
    VAH_TRY(vah::launch_set_conserved<S>(field_set<S>(ev->q, 16), field_set<S>(ev->u, 4), field_set<S>(ev->up, 4),
                                         (const S *)ev->ep[ev->cur][0], ev->opt.physics, ev->lat.nx, ev->lat.ny,
                                         ev->lat.nz, ev->ncx, t, pl_from_field, ev->stream));
    VAH_TRY(cudaStreamSynchronize(ev->stream));
    return VAH_OK;
}

template <typename S>
int ghosts_t(vah_event *ev) {
    FieldSet<S> f{};
    int n = 0;
    f.f[n++] = (S *)ev->ep[ev->cur][0];
    f.f[n++] = (S *)ev->ep[ev->cur][1];
    for (int m = 0; m < 4; ++m) f.f[n++] = (S *)ev->u[m];
    for (int k = 0; k < 16; ++k)
        if (ev->q[k]) f.f[n++] = (S *)ev->q[k];
    f.n = n;
    VAH_TRY(vah::launch_ghosts<S>(f, ev->lat.nx, ev->lat.ny, ev->lat.nz, ev->ncx, ev->stream));
    VAH_TRY(cudaStreamSynchronize(ev->stream));
    return VAH_OK;
}

template <typename S>
int init_primitives_t(vah_event *ev) {
    VAH_TRY(vah::launch_init_primitives<S>(field_set<S>(ev->q, 16), field_set<S>(ev->u, 4),
                                           (const S *)ev->ep[ev->cur][0], (S *)ev->ep[ev->cur][1], make_eos(ev),
                                           ev->lat.nx, ev->lat.ny, ev->lat.nz, ev->ncx, ev->stream));
    return VAH_OK;
}

}  // namespace

extern "C" int vah_event_set_conserved(vah_event *ev, double t, int pl_from_field) {
    if (!ev) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(ev->opt.device));
    return ev->elem == sizeof(float) ? set_conserved_t<float>(ev, t, pl_from_field)
                                     : set_conserved_t<double>(ev, t, pl_from_field);
}

extern "C" int vah_event_init_from_e(vah_event *ev, double t0, const double *e_interior, int pl_mode) {
    if (!ev || !e_interior || (pl_mode != VAH_PL_REFERENCE && pl_mode != VAH_PL_ISOTROPIC)) return VAH_ERR_ARG;
    int rc = vah_event_set_field(ev, VAH_F_E, e_interior, 0);
    if (rc != VAH_OK) return rc;
    rc = ev->elem == sizeof(float) ? init_primitives_t<float>(ev) : init_primitives_t<double>(ev);
    if (rc != VAH_OK) return rc;
    rc = vah_event_set_conserved(ev, t0, pl_mode == VAH_PL_ISOTROPIC);
    if (rc != VAH_OK) return rc;
    return vah_event_set_ghost_cells(ev);
}

namespace {

// The e interior generated on the device (MC-Glauber when g is given, else
// the optical Glauber profile o), then the vah_event_init_from_e sequence.
int init_device_ic(vah_event *ev, double t0, const vah_glauber *g, const vah_optical *o, int pl_mode) {
    if (!ev || (pl_mode != VAH_PL_REFERENCE && pl_mode != VAH_PL_ISOTROPIC)) return VAH_ERR_ARG;
    const vah_lattice &lat = ev->lat;
    const int A = g ? g->A : o->A;
    const double eta_flat = g ? g->eta_flat : o->eta_flat, sigma_eta = g ? g->sigma_eta : o->sigma_eta;
    if (A < 1 || (lat.nz > 1 && !(sigma_eta > 0))) return VAH_ERR_ARG;
    const double R = g ? g->ws_R : o->ws_R, a = g ? g->ws_a : o->ws_a;
    if (!(R > 0) || !(a > 0) || !std::isfinite(R + a)) return VAH_ERR_ARG;
    if (g && (A > 256 || !(g->width > 0))) return VAH_ERR_ARG;
    if (o && !(o->sigma_nn_fm2 > 0)) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(ev->opt.device));
    const size_t nxy = (size_t)lat.nx * lat.ny;
    const size_t aux = g ? 4 * (size_t)A : (size_t)vah::kThicknessPoints + 1;
    char *scratch = nullptr;
    VAH_TRY(cudaMallocAsync((void **)&scratch, 256 + sizeof(double) * (aux + nxy), ev->stream));
    unsigned long long *maxbits = (unsigned long long *)scratch;
    double *d_aux = (double *)(scratch + 256), *d_v = d_aux + aux;
    cudaError_t err = cudaMemsetAsync(maxbits, 0, sizeof(unsigned long long), ev->stream);
    if (err == cudaSuccess && g) {
        int *d_np = (int *)(scratch + 64);
        err = vah::ic_participants_device(g->b, g->sigma_nn_fm2, A, g->ws_R, g->ws_a, g->seed, d_aux, d_np, ev->stream);
        if (err == cudaSuccess)
            err = vah::ic_deposit_device(d_aux, d_np, g->width, lat.nx, lat.ny, lat.dx, lat.dy, d_v, maxbits,
                                         ev->stream);
    } else if (err == cudaSuccess) {
        err = vah::ic_optical_device(lat.nx, lat.ny, lat.dx, lat.dy, o->b, o->sigma_nn_fm2, A, o->ws_R, o->ws_a,
                                     o->x_coll, d_aux, d_v, maxbits, ev->stream);
    }
    int np = 0;  // the sampler reports -1 when its draws ran out (parameters it cannot sample)
    if (err == cudaSuccess && g) err = cudaMemcpyAsync(&np, scratch + 64, sizeof(int), cudaMemcpyDeviceToHost, ev->stream);
    if (err == cudaSuccess && g) err = cudaStreamSynchronize(ev->stream);
    if (err == cudaSuccess && np < 0) {
        VAH_TRY(cudaFreeAsync(scratch, ev->stream));
        return VAH_ERR_ARG;
    }
    const double e_peak = g ? g->e_peak : o->e_peak, e_floor = g ? g->e_floor : o->e_floor;
    if (err == cudaSuccess)
        err = ev->elem == sizeof(float)
                  ? vah::ic_fill_device<float>(d_v, maxbits, lat.nx, lat.ny, lat.nz, ev->ncx, lat.dz, eta_flat,
                                               sigma_eta, e_peak, e_floor, (float *)ev->ep[ev->cur][0], ev->stream)
                  : vah::ic_fill_device<double>(d_v, maxbits, lat.nx, lat.ny, lat.nz, ev->ncx, lat.dz, eta_flat,
                                                sigma_eta, e_peak, e_floor, (double *)ev->ep[ev->cur][0], ev->stream);
    const cudaError_t ferr = cudaFreeAsync(scratch, ev->stream);
    VAH_TRY(err);
    VAH_TRY(ferr);
    int rc = ev->elem == sizeof(float) ? init_primitives_t<float>(ev) : init_primitives_t<double>(ev);
    if (rc != VAH_OK) return rc;
    rc = vah_event_set_conserved(ev, t0, pl_mode == VAH_PL_ISOTROPIC);
    if (rc != VAH_OK) return rc;
    return vah_event_set_ghost_cells(ev);
}

}  // namespace

extern "C" int vah_event_init_glauber(vah_event *ev, double t0, const vah_glauber *g, int pl_mode) {
    if (!g) return VAH_ERR_ARG;
    return init_device_ic(ev, t0, g, nullptr, pl_mode);
}

extern "C" int vah_event_init_optical_glauber(vah_event *ev, double t0, const vah_optical *o, int pl_mode) {
    if (!o) return VAH_ERR_ARG;
    return init_device_ic(ev, t0, nullptr, o, pl_mode);
}

extern "C" int vah_event_set_ghost_cells(vah_event *ev) {
    if (!ev) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(ev->opt.device));
    return ev->elem == sizeof(float) ? ghosts_t<float>(ev) : ghosts_t<double>(ev);
}

namespace {

// Stage-1 arguments: q, u, (e, p)[cur], up -> qS, uS, (e, p)[1 - cur].
template <typename S>
void stage1_args(const vah_event *ev, double t, double dt, StageArgs<S> &a) {
    const int c = ev->cur, o = 1 - ev->cur;
    fill_common(ev, a);
    a.t_src = t;
    a.t_inv = t + dt;
    a.dt = dt;
    a.stage2 = 0;
    for (int n = 0; n < 16; ++n) {
        a.qin[n] = (const S *)ev->q[n];
        a.qout[n] = (S *)ev->qS[n];
    }
    for (int m = 0; m < 4; ++m) {
        a.uin[m] = (const S *)ev->u[m];
        a.upin[m] = (const S *)ev->up[m];
        a.guess[m] = (const S *)ev->u[m];
        a.uout[m] = (S *)ev->uS[m];
    }
    a.ein = (const S *)ev->ep[c][0];
    a.pin = (const S *)ev->ep[c][1];
    a.eout = (S *)ev->ep[o][0];
    a.pout = (S *)ev->ep[o][1];
    a.fallback = ev->d_fb;
    finish_args(a);
}

// Stage 2: qS, uS, (e, p)[o], u -> q (in place, with the convex
// combination), up buffer (becomes u^{n+1}), (e, p)[c].
template <typename S>
void stage2_args(const vah_event *ev, double t, double dt, StageArgs<S> &a) {
    const int c = ev->cur, o = 1 - ev->cur;
    fill_common(ev, a);
    a.t_src = t + dt;
    a.t_inv = t + dt;
    a.dt = dt;
    a.stage2 = 1;
    for (int n = 0; n < 16; ++n) {
        a.qin[n] = (const S *)ev->qS[n];
        a.qavg[n] = (const S *)ev->q[n];
        a.qout[n] = (S *)ev->q[n];
    }
    for (int m = 0; m < 4; ++m) {
        a.uin[m] = (const S *)ev->uS[m];
        a.upin[m] = (const S *)ev->u[m];
        a.guess[m] = (const S *)ev->u[m];
        a.uout[m] = (S *)ev->up[m];
    }
    a.ein = (const S *)ev->ep[o][0];
    a.pin = (const S *)ev->ep[o][1];
    a.eout = (S *)ev->ep[c][0];
    a.pout = (S *)ev->ep[c][1];
    a.fallback = ev->d_fb ? ev->d_fb + ev->ncell : nullptr;
    finish_args(a);
}

template <typename S>
int rk2_step_t(vah_event *ev, double t, double dt) {
    const int c = ev->cur;
    if (ev->validity)  // the diagnostics read P_L, pi, Pi as they are at the start of the step
        for (int n = VAH_F_PL; n < ev->nq; ++n)
            VAH_TRY(cudaMemcpyAsync(ev->vq[n], ev->q[n], ev->ncell * sizeof(S), cudaMemcpyDeviceToDevice, ev->stream));
    int rc;
    if (ev->tile) {
        rc = tile_stage(ev, 1, t, dt);
        if (rc == VAH_OK) rc = tile_stage(ev, 2, t, dt);
    } else {
        StageArgs<S> a;
        stage1_args(ev, t, dt, a);
        rc = timed_launch(ev, a);
        if (rc != VAH_OK) return rc;
        stage2_args(ev, t, dt, a);
        rc = timed_launch(ev, a);
    }
    if (rc != VAH_OK || !ev->validity) return rc;
    ValidityArgs<S> v;
    memset(&v, 0, sizeof(v));
    v.nx = ev->lat.nx;
    v.ny = ev->lat.ny;
    v.nz = ev->lat.nz;
    v.ncx = ev->ncx;
    v.ncy = ev->ncy;
    v.plane = (long long)ev->ncx * ev->ncy;
    v.t = t + dt;
    v.dt = dt;
    v.dx = ev->lat.dx;
    v.dy = ev->lat.dy;
    v.dz = ev->lat.dz;
    v.etabar = ev->hydro.eta_over_s;
    for (int n = 0; n < 16; ++n) v.qn[n] = (const S *)ev->vq[n];
    v.e = (const S *)ev->ep[c][0];
    v.p = (const S *)ev->ep[c][1];
    for (int m = 0; m < 4; ++m) {
        v.u[m] = (const S *)ev->up[m];  // the new velocity (the buffers swap after this call)
        v.up[m] = (const S *)ev->u[m];
    }
    v.eos = make_eos(ev);
    for (int m = 0; m < 16; ++m) v.v[m] = ev->vd[m];
    return cuda_status(vah::launch_validity<S>(v, ev->opt.physics, ev->stream));
}

}  // namespace

extern "C" int vah_rk2_step(vah_event *ev, double t, double dt) {
    if (!ev || !(dt > 0) || !(t > 0)) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(ev->opt.device));
    int rc = ev->elem == sizeof(float) ? rk2_step_t<float>(ev, t, dt) : rk2_step_t<double>(ev, t, dt);
    if (rc != VAH_OK) return rc;
    // swapFluidVelocity(&up, &u) (FullyDiscreteKurganovTadmorScheme.cpp:784)
    for (int m = 0; m < 4; ++m) {
        void *tmp = ev->u[m];
        ev->u[m] = ev->up[m];
        ev->up[m] = tmp;
    }
    ev->tparity ^= 1;  // the tile descriptor keeps its buffers; the parity follows the swap
    ev->steps++;
    ev->last_t = t + dt;
    ev->last_dt = dt;
    return VAH_OK;
}

namespace {

// Time every candidate launch configuration of each split kind on the
// event's current state, in stage-1 buffer roles (their outputs -- the face
// buffers, qS, uS and the other (e, p) pair -- are scratch that the next step
// rewrites), and keep the fastest. The device counters are restored after.
template <typename S>
int autotune_t(vah_event *ev, int reps, vah_tune_report *out) {
    StageArgs<S> a;
    stage1_args(ev, ev->last_t, ev->last_dt, a);
    const bool exact = ev->opt.flux == VAH_FLUX_PER_CELL;
    unsigned long long saved[4];
    VAH_TRY(cudaStreamSynchronize(ev->stream));
    VAH_TRY(cudaMemcpy(saved, ev->d_counters, sizeof(saved), cudaMemcpyDeviceToHost));
    cudaEvent_t e0, e1;
    VAH_TRY(cudaEventCreate(&e0));
    VAH_TRY(cudaEventCreate(&e1));
    int rc = VAH_OK;
    auto launch = [&](int kind, const vah::KindConfig &c) {
        return vah::launch_split_kind<S>(a, ev->opt.physics, exact, kind, c, ev->stream);
    };
    auto time_one = [&](int kind, const vah::KindConfig &c, double *ms) -> int {
        if (launch(kind, c) != cudaSuccess) return VAH_ERR_CUDA;  // warm-up
        if (cudaEventRecord(e0, ev->stream) != cudaSuccess) return VAH_ERR_CUDA;
        for (int r = 0; r < reps; ++r)
            if (launch(kind, c) != cudaSuccess) return VAH_ERR_CUDA;
        if (cudaEventRecord(e1, ev->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess)
            return VAH_ERR_CUDA;
        float f = 0;
        if (cudaEventElapsedTime(&f, e0, e1) != cudaSuccess) return VAH_ERR_CUDA;
        *ms = f / reps;
        return VAH_OK;
    };
    out->nkinds = vah::kNumSplitKinds;
    for (int kind = 0; kind < vah::kNumSplitKinds && rc == VAH_OK; ++kind) {
        vah_launch_choice &r = out->kind[kind];
        const vah::KindConfig def = ev->split.k[kind];
        r = {def.bx, def.by, def.minb, 0.0, 0.0};
        if (kind == vah::kFaceZ && ev->lat.nz == 1) continue;  // no eta faces in 2+1D
        vah::KindConfig cand[16];
        const int n = vah::split_candidates(kind, cand, 16);
        double best = 1e300;
        for (int i = 0; i < n && rc == VAH_OK; ++i) {
            double ms = 0;
            rc = time_one(kind, cand[i], &ms);
            if (rc != VAH_OK) break;
            if (cand[i].bx == def.bx && cand[i].by == def.by && cand[i].minb == def.minb) r.ms_default = ms;
            if (ms < best) {
                best = ms;
                ev->split.k[kind] = cand[i];
            }
        }
        const vah::KindConfig &b = ev->split.k[kind];
        r = {b.bx, b.by, b.minb, r.ms_default, best};
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (cudaMemcpy(ev->d_counters, saved, sizeof(saved), cudaMemcpyHostToDevice) != cudaSuccess && rc == VAH_OK)
        rc = VAH_ERR_CUDA;
    return rc;
}

}  // namespace

extern "C" int vah_event_autotune(vah_event *ev, int reps, vah_tune_report *out) {
    if (!ev || !out || reps < 1) return VAH_ERR_ARG;
    memset(out, 0, sizeof(*out));
    if (ev->opt.flux == VAH_FLUX_PER_CELL_FUSED || ev->tile) return VAH_OK;  // one launch shape: nothing to tune
    VAH_TRY(cudaSetDevice(ev->opt.device));
    return ev->elem == sizeof(float) ? autotune_t<float>(ev, reps, out) : autotune_t<double>(ev, reps, out);
}

extern "C" int vah_event_set_validity(vah_event *ev, int on) {
    if (!ev) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(ev->opt.device));
    if (on && !ev->vd[0]) {
        for (int m = 0; m < VAH_NUM_VALIDITY; ++m) {
            cudaError_t e = cudaMalloc((void **)&ev->vd[m], ev->ncell * sizeof(double));
            if (e == cudaSuccess) e = cudaMemsetAsync(ev->vd[m], 0, ev->ncell * sizeof(double), ev->stream);
            if (e != cudaSuccess) return cuda_status(e);
        }
        for (int n = VAH_F_PL; n < ev->nq; ++n) {
            cudaError_t e = cudaMalloc(&ev->vq[n], ev->ncell * ev->elem);
            if (e == cudaSuccess) e = cudaMemsetAsync(ev->vq[n], 0, ev->ncell * ev->elem, ev->stream);
            if (e != cudaSuccess) return cuda_status(e);
        }
    }
    if (on && !ev->validity && ev->lat.nz == 1) {  // the diagnostics read the eta ghost layers: fill them now
        int ids[VAH_NUM_FIELDS];
        for (int id = 0; id < VAH_NUM_FIELDS; ++id) ids[id] = id;
        const int rc = fill_zghosts(ev, ids, VAH_NUM_FIELDS);
        if (rc != VAH_OK) return rc;
    }
    ev->validity = on != 0;
    if (ev->tile) {  // the tile kernel writes the regulator maps through its descriptor
        for (int m = 0; m < 11; ++m) ev->h_tslot.regmap[m] = ev->validity ? ev->vd[VAH_V_REGULATIONS + m] : nullptr;
        ev->h_tslot.zghosts = zghosts_eager(ev);
        return tile_sync_desc(ev);
    }
    return VAH_OK;
}

extern "C" int vah_event_get_validity(vah_event *ev, int id, double *host, int with_ghosts) {
    if (!ev || !host || id < 0 || id >= VAH_NUM_VALIDITY || !ev->vd[id]) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(ev->opt.device));
    VAH_TRY(cudaStreamSynchronize(ev->stream));
    const size_t es = sizeof(double);
    if (with_ghosts) {
        const size_t w = (size_t)(ev->lat.nx + 4) * es;
        VAH_TRY(cudaMemcpy2D(host, w, ev->vd[id], ev->ncx * es, w, (size_t)ev->ncy * ev->ncz, cudaMemcpyDeviceToHost));
        return VAH_OK;
    }
    const int nx = ev->lat.nx, ny = ev->lat.ny, nz = ev->lat.nz;
    for (int k = 0; k < nz; ++k) {
        const double *row = ev->vd[id] + 2 + (size_t)ev->ncx * (2 + (size_t)ev->ncy * (k + 2));
        VAH_TRY(cudaMemcpy2D(host + (size_t)nx * ny * k, nx * es, row, ev->ncx * es, nx * es, ny,
                             cudaMemcpyDeviceToHost));
    }
    return VAH_OK;
}

extern "C" int vah_run(vah_event *ev, double t0, double dt, int nsteps) {
    if (!ev || nsteps < 0) return VAH_ERR_ARG;
    for (int n = 0; n < nsteps; ++n) {
        int rc = vah_rk2_step(ev, t0 + n * dt, dt);
        if (rc != VAH_OK) return rc;
    }
    return VAH_OK;
}

extern "C" int vah_event_sync(vah_event *ev) {
    if (!ev) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(ev->opt.device));
    VAH_TRY(cudaStreamSynchronize(ev->stream));
    unsigned long long c[4];
    VAH_TRY(cudaMemcpy(c, ev->d_counters, sizeof(c), cudaMemcpyDeviceToHost));
    if (ev->tile) {  // a tile launch that gave up waiting for its copy (never expected)
        unsigned err = 0;
        VAH_TRY(cudaMemcpy(&err, ev->d_terr, sizeof(err), cudaMemcpyDeviceToHost));
        if (err) return VAH_ERR_CUDA;
    }
    return c[2] ? VAH_ERR_NAN : VAH_OK;
}

extern "C" int vah_event_stats(vah_event *ev, vah_stats *out) {
    if (!ev || !out) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(ev->opt.device));
    VAH_TRY(cudaStreamSynchronize(ev->stream));
    unsigned long long c[4];
    VAH_TRY(cudaMemcpy(c, ev->d_counters, sizeof(c), cudaMemcpyDeviceToHost));
    out->face_fallbacks = (long long)c[0];
    out->cell_fallbacks = (long long)c[1];
    out->nan_cells = (long long)c[2];
    out->steps = ev->steps;
    return VAH_OK;
}

extern "C" int vah_event_track_fallbacks(vah_event *ev, int on) {
    if (!ev) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(ev->opt.device));
    if (on && !ev->d_fb) {
        VAH_TRY(cudaMalloc((void **)&ev->d_fb, 2 * ev->ncell));
        VAH_TRY(cudaMemsetAsync(ev->d_fb, 0, 2 * ev->ncell, ev->stream));
    } else if (!on && ev->d_fb) {
        VAH_TRY(cudaStreamSynchronize(ev->stream));
        VAH_TRY(cudaFree(ev->d_fb));
        ev->d_fb = nullptr;
    }
    if (ev->tile) {
        ev->h_tslot.fallback1 = ev->d_fb;
        ev->h_tslot.fallback2 = ev->d_fb ? ev->d_fb + ev->ncell : nullptr;
        return tile_sync_desc(ev);
    }
    return VAH_OK;
}

extern "C" int vah_event_get_fallback_mask(vah_event *ev, int stage, unsigned char *host, int with_ghosts) {
    if (!ev || !host || (stage != 1 && stage != 2) || !ev->d_fb) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(ev->opt.device));
    VAH_TRY(cudaStreamSynchronize(ev->stream));
    const unsigned char *src = ev->d_fb + (stage - 1) * ev->ncell;
    if (with_ghosts) {
        const size_t w = (size_t)(ev->lat.nx + 4);
        VAH_TRY(cudaMemcpy2D(host, w, src, ev->ncx, w, (size_t)ev->ncy * ev->ncz, cudaMemcpyDeviceToHost));
        return VAH_OK;
    }
    const int nx = ev->lat.nx, ny = ev->lat.ny, nz = ev->lat.nz;
    for (int k = 0; k < nz; ++k) {
        const unsigned char *row = src + 2 + (size_t)ev->ncx * (2 + (size_t)ev->ncy * (k + 2));
        VAH_TRY(cudaMemcpy2D(host + (size_t)nx * ny * k, nx, row, ev->ncx, nx, ny, cudaMemcpyDeviceToHost));
    }
    return VAH_OK;
}

extern "C" int vah_event_set_timing(vah_event *ev, int on) {
    if (!ev) return VAH_ERR_ARG;
    ev->timing = on != 0;
    return VAH_OK;
}

extern "C" int vah_event_kernel_time(vah_event *ev, double *ms, long long *launches) {
    if (!ev || !ms || !launches) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(ev->opt.device));
    VAH_TRY(cudaStreamSynchronize(ev->stream));
    double total = 0;
    for (int k = 0; k + 1 < ev->tev_used; k += 2) {
        float m = 0;
        VAH_TRY(cudaEventElapsedTime(&m, ev->tev[k], ev->tev[k + 1]));
        total += m;
    }
    *ms = total;
    *launches = ev->tev_used / 2;
    ev->tev_used = 0;
    return VAH_OK;
}

namespace {

// The eta ghost layers of the fields a host-buffer step returns (2+1D).
int fill_host_zghosts(vah_event *ev, double *const *fields) {
    int ids[VAH_NUM_FIELDS], n = 0;
    for (int id = 0; id < VAH_NUM_FIELDS; ++id)
        if (fields[id]) ids[n++] = id;
    return fill_zghosts(ev, ids, n);
}

// FP64 host rows of hx values <-> FP32 device rows of the padded pitch.
__global__ void widen_kernel(const float *__restrict__ src, double *__restrict__ dst, int hx, int pitch, size_t rows) {
    const size_t n = (size_t)hx * rows;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        dst[k] = (double)src[(k / hx) * pitch + k % hx];
}

__global__ void narrow_kernel(const double *__restrict__ src, float *__restrict__ dst, int hx, int pitch, size_t rows) {
    const size_t n = (size_t)hx * rows;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        dst[(k / hx) * pitch + k % hx] = (float)src[k];
}

// FP32 storage: the caller's FP64 host arrays cross PCIe as FP64, one
// contiguous copy per field into device staging in the host layout, and are
// narrowed into the padded device rows (widened on the way out) by a kernel,
// all in stream order, with one synchronisation at the end.
int step_host_fp32(vah_event *ev, double t, double dt, double *const *fields) {
    const int hx = ev->lat.nx + 4;
    const size_t rows = (size_t)ev->ncy * ev->ncz, hn = (size_t)hx * rows;  // host layout
    if (!ev->d_stage64) VAH_TRY(cudaMalloc((void **)&ev->d_stage64, ev->ncell * sizeof(double)));
    const int block = 256, grid = (int)std::min<size_t>((hn + block - 1) / block, 148 * 16);
    for (int id = 0; id < VAH_NUM_FIELDS; ++id) {
        float *d = (float *)field_ptr(ev, id);
        if (!d || !fields[id]) continue;
        VAH_TRY(cudaMemcpyAsync(ev->d_stage64, fields[id], hn * sizeof(double), cudaMemcpyHostToDevice, ev->stream));
        narrow_kernel<<<grid, block, 0, ev->stream>>>(ev->d_stage64, d, hx, ev->ncx, rows);
        VAH_TRY(cudaGetLastError());
    }
    int rc = vah_rk2_step(ev, t, dt);
    if (rc != VAH_OK) return rc;
    if ((rc = fill_host_zghosts(ev, fields)) != VAH_OK) return rc;
    for (int id = 0; id < VAH_NUM_FIELDS; ++id) {  // pointers after the u <-> up swap
        const float *d = (const float *)field_ptr(ev, id);
        if (!d || !fields[id]) continue;
        widen_kernel<<<grid, block, 0, ev->stream>>>(d, ev->d_stage64, hx, ev->ncx, rows);
        VAH_TRY(cudaGetLastError());
        VAH_TRY(cudaMemcpyAsync(fields[id], ev->d_stage64, hn * sizeof(double), cudaMemcpyDeviceToHost, ev->stream));
    }
    return vah_event_sync(ev);
}

// Slab boundaries along eta for the overlapped host-buffer step: nz / thick
// slabs (at least one) of as equal a thickness as nz allows, each of at least
// `thick` >= 2 planes. (Thinner first and last slabs shorten the pipeline's
// fill and drain but make more, smaller copies, which cost more than they
// save on PCIe: measured on the 121x121x81 event.)
std::vector<int> slab_bounds(int nz, int thick) {
    thick = std::max(2, thick);
    const int n = std::max(1, nz / thick);
    std::vector<int> b = {0};
    for (int m = 0; m < n; ++m) b.push_back(b.back() + nz / n + (m < nz % n ? 1 : 0));
    return b;
}

// Host-buffer step (FP64 storage, face/cell split) with its copies
// overlapped: the lattice is cut into slabs of planes along eta; the
// host-to-device copy of later slabs, the stages of earlier ones and the
// device-to-host copy of finished ones run on three streams. Slab m (interior
// planes [lo, hi)) may start stage 1 once the input planes up to hi + 2
// (ghosted) are on the device; its stage 2 follows stage 1 of slab m + 1
// (which writes the stage-1 planes hi, hi + 1 that it reads); stage 1 of slab
// m + 1 runs before stage 2 of slab m overwrites q, e and p in place under it.
// Host planes are read (copy-in) before they are written back (copy-out):
// each copy-out covers planes that the copy-ins before the slab's stage 1
// have read. One compute stream keeps the face buffers' reuse in order.
int step_host_pipelined(vah_event *ev, double t, double dt, double *const *fields, int thick) {
    const int nz = ev->lat.nz;
    const std::vector<int> bound = slab_bounds(nz, thick);
    const int nslab = (int)bound.size() - 1;
    const size_t pbytes = (size_t)ev->ncx * ev->ncy * sizeof(double);
    if (!ev->s_in) VAH_TRY(cudaStreamCreateWithFlags(&ev->s_in, cudaStreamNonBlocking));
    if (!ev->s_out) VAH_TRY(cudaStreamCreateWithFlags(&ev->s_out, cudaStreamNonBlocking));
    while (ev->pev.size() < (size_t)(2 * nslab + 2)) {
        cudaEvent_t e;
        VAH_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ev->pev.push_back(e);
    }
    cudaEvent_t start = ev->pev[0], end = ev->pev[1], *in_ready = &ev->pev[2], *done = &ev->pev[2 + nslab];
    // device buffers by field id: what the step reads, and what holds the field after it
    void *din[VAH_NUM_FIELDS], *dout[VAH_NUM_FIELDS];
    for (int id = 0; id < VAH_NUM_FIELDS; ++id) din[id] = dout[id] = fields[id] ? field_ptr(ev, id) : nullptr;
    for (int m = 0; m < 4; ++m) {  // stage 2 writes u^{n+1} into the up buffer; u^n becomes up
        if (fields[VAH_F_UT + m]) dout[VAH_F_UT + m] = ev->up[m];
        if (fields[VAH_F_UPT + m]) dout[VAH_F_UPT + m] = ev->u[m];
    }
    auto copy_planes = [&](bool to_device, size_t p0, size_t p1, cudaStream_t s) -> int {
        if (p1 <= p0) return VAH_OK;
        for (int id = 0; id < VAH_NUM_FIELDS; ++id) {
            if (!din[id]) continue;
            char *h = (char *)fields[id] + p0 * pbytes;
            if (to_device)
                VAH_TRY(cudaMemcpyAsync((char *)din[id] + p0 * pbytes, h, (p1 - p0) * pbytes, cudaMemcpyHostToDevice, s));
            else
                VAH_TRY(cudaMemcpyAsync(h, (char *)dout[id] + p0 * pbytes, (p1 - p0) * pbytes, cudaMemcpyDeviceToHost, s));
        }
        return VAH_OK;
    };
    StageArgs<double> a1, a2;
    stage1_args(ev, t, dt, a1);
    stage2_args(ev, t, dt, a2);
    const bool exact = ev->opt.flux == VAH_FLUX_PER_CELL;
    VAH_TRY(cudaEventRecord(start, ev->stream));  // after the work queued before this step
    VAH_TRY(cudaStreamWaitEvent(ev->s_in, start, 0));
    VAH_TRY(cudaStreamWaitEvent(ev->s_out, start, 0));
    size_t loaded = 0;  // ghosted planes [0, loaded) queued for copy-in
    int rc = VAH_OK;
    for (int m = 0; m <= nslab && rc == VAH_OK; ++m) {
        if (m < nslab) {
            const int hi = bound[m + 1];
            const size_t need = m == nslab - 1 ? (size_t)nz + 4 : (size_t)hi + 4;
            rc = copy_planes(true, loaded, need, ev->s_in);
            if (rc != VAH_OK) break;
            loaded = need;
            VAH_TRY(cudaEventRecord(in_ready[m], ev->s_in));
            VAH_TRY(cudaStreamWaitEvent(ev->stream, in_ready[m], 0));
            a1.k0 = bound[m];
            a1.k1 = hi;
            VAH_TRY(vah::launch_stage_split<double>(a1, ev->opt.physics, exact, ev->split, ev->stream));
        }
        if (m >= 1) {
            const int k = m - 1, lo = bound[k], hi = bound[k + 1];
            a2.k0 = lo;
            a2.k1 = hi;
            VAH_TRY(vah::launch_stage_split<double>(a2, ev->opt.physics, exact, ev->split, ev->stream));
            VAH_TRY(cudaEventRecord(done[k], ev->stream));
            VAH_TRY(cudaStreamWaitEvent(ev->s_out, done[k], 0));
            const size_t p0 = k == 0 ? 0 : (size_t)lo + 2, p1 = k == nslab - 1 ? (size_t)nz + 4 : (size_t)hi + 2;
            rc = copy_planes(false, p0, p1, ev->s_out);
        }
    }
    // join the copy streams back into the event's stream, also on an error
    if (cudaEventRecord(end, ev->s_out) == cudaSuccess) cudaStreamWaitEvent(ev->stream, end, 0);
    if (cudaEventRecord(end, ev->s_in) == cudaSuccess) cudaStreamWaitEvent(ev->stream, end, 0);
    if (rc != VAH_OK) return rc;
    for (int m = 0; m < 4; ++m) {  // as vah_rk2_step
        void *tmp = ev->u[m];
        ev->u[m] = ev->up[m];
        ev->up[m] = tmp;
    }
    ev->steps++;
    ev->last_t = t + dt;
    ev->last_dt = dt;
    return vah_event_sync(ev);
}

// Every field of a host-buffer step at once (blockIdx.y: the field): FP64
// host-layout rows [r0, r0 + rows) of hx values <-> FP32 device rows of the
// padded pitch.
struct FieldRows {
    const void *src[VAH_NUM_FIELDS];
    void *dst[VAH_NUM_FIELDS];
};

__global__ void narrow_rows_kernel(FieldRows f, int hx, int pitch, size_t r0, size_t rows) {
    const double *src = (const double *)f.src[blockIdx.y] + r0 * hx;
    float *dst = (float *)f.dst[blockIdx.y] + r0 * pitch;
    const size_t n = (size_t)hx * rows;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        dst[(k / hx) * pitch + k % hx] = (float)src[k];
}

__global__ void widen_rows_kernel(FieldRows f, int hx, int pitch, size_t r0, size_t rows) {
    const float *src = (const float *)f.src[blockIdx.y] + r0 * pitch;
    double *dst = (double *)f.dst[blockIdx.y] + r0 * hx;
    const size_t n = (size_t)hx * rows;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        dst[k] = (double)src[(k / hx) * pitch + k % hx];
}

// Slabs of whole tile layers along eta for the FP32 form's overlapped
// host-buffer step: about `thick` planes each (rounded to tile layers, at
// least one), as in slab_bounds. Returns the bounds in tile layers.
std::vector<int> tile_slab_layers(int nz, int thick) {
    constexpr int TZ = vah::TileShape<true>::TZ;
    const int nlayer = (nz + TZ - 1) / TZ, per = std::max(1, (thick + TZ / 2) / TZ);
    const int n = std::max(1, nlayer / per);
    std::vector<int> b = {0};
    for (int m = 0; m < n; ++m) b.push_back(b.back() + nlayer / n + (m < nlayer % n ? 1 : 0));
    return b;
}

// Host-buffer step of the FP32 form (3+1D) with its copies overlapped, in the
// slab order of step_host_pipelined. A slab is a run of whole tile layers, so
// its tiles are one run of the k-major work-list, and its stage 1 or 2 is one
// tile launch over that run. Its FP64 planes cross PCIe into a device copy of
// the host layout (d_stage_all) and are narrowed into the FP32 fields on the
// event's stream before its stage 1; after its stage 2 they are widened there
// and copied back. Every slab but possibly the last has at least 4 planes, so
// the 2-plane stencil halo of a slab lies in its neighbours, which is what the
// order relies on.
int step_host_fp32_pipelined(vah_event *ev, double t, double dt, double *const *fields, int thick) {
    constexpr int TZ = vah::TileShape<true>::TZ, TX = vah::TileShape<true>::TX, TY = vah::TileShape<true>::TY;
    const int nx = ev->lat.nx, ny = ev->lat.ny, nz = ev->lat.nz, hx = nx + 4;
    const std::vector<int> lb = tile_slab_layers(nz, thick);
    const int nslab = (int)lb.size() - 1, per_layer = ((nx + TX - 1) / TX) * ((ny + TY - 1) / TY);
    auto plane_of = [&](int layer) { return std::min(layer * TZ, nz); };  // interior plane of a slab bound
    const size_t hplane = (size_t)hx * ev->ncy, hn = hplane * ev->ncz;  // doubles per host plane, field
    if (!ev->d_stage_all) VAH_TRY(cudaMalloc((void **)&ev->d_stage_all, VAH_NUM_FIELDS * hn * sizeof(double)));
    if (!ev->s_in) VAH_TRY(cudaStreamCreateWithFlags(&ev->s_in, cudaStreamNonBlocking));
    if (!ev->s_out) VAH_TRY(cudaStreamCreateWithFlags(&ev->s_out, cudaStreamNonBlocking));
    while (ev->pev.size() < (size_t)(2 * nslab + 2)) {
        cudaEvent_t e;
        VAH_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ev->pev.push_back(e);
    }
    cudaEvent_t start = ev->pev[0], end = ev->pev[1], *in_ready = &ev->pev[2], *done = &ev->pev[2 + nslab];
    // per field: the host array, its staging copy, the device field the step
    // reads (narrowed into) and the one that holds it after the step (widened)
    FieldRows in{}, out{};
    double *host[VAH_NUM_FIELDS], *stg[VAH_NUM_FIELDS];
    int nf = 0;
    for (int id = 0; id < VAH_NUM_FIELDS; ++id) {
        void *d = field_ptr(ev, id);
        if (!d || !fields[id]) continue;
        void *after = d;  // stage 2 writes u^{n+1} into the up buffer; u^n becomes up
        if (id >= VAH_F_UT && id < VAH_F_UT + 4) after = ev->up[id - VAH_F_UT];
        if (id >= VAH_F_UPT && id < VAH_F_UPT + 4) after = ev->u[id - VAH_F_UPT];
        host[nf] = fields[id];
        stg[nf] = ev->d_stage_all + (size_t)id * hn;
        in.src[nf] = stg[nf];
        in.dst[nf] = d;
        out.src[nf] = after;
        out.dst[nf] = stg[nf];
        ++nf;
    }
    auto copy_planes = [&](bool to_device, size_t p0, size_t p1, cudaStream_t s) -> int {
        if (p1 <= p0) return VAH_OK;
        const size_t off = p0 * hplane, bytes = (p1 - p0) * hplane * sizeof(double);
        for (int f = 0; f < nf; ++f) {
            if (to_device)
                VAH_TRY(cudaMemcpyAsync(stg[f] + off, host[f] + off, bytes, cudaMemcpyHostToDevice, s));
            else
                VAH_TRY(cudaMemcpyAsync(host[f] + off, stg[f] + off, bytes, cudaMemcpyDeviceToHost, s));
        }
        return VAH_OK;
    };
    auto convert = [&](bool narrow, size_t p0, size_t p1) -> int {
        if (p1 <= p0 || nf == 0) return VAH_OK;
        const size_t r0 = p0 * ev->ncy, rows = (p1 - p0) * ev->ncy;
        const dim3 grid((unsigned)std::min<size_t>((rows * hx + 255) / 256, 148 * 4), (unsigned)nf);
        if (narrow)
            narrow_rows_kernel<<<grid, 256, 0, ev->stream>>>(in, hx, ev->ncx, r0, rows);
        else
            widen_rows_kernel<<<grid, 256, 0, ev->stream>>>(out, hx, ev->ncx, r0, rows);
        VAH_TRY(cudaGetLastError());
        return VAH_OK;
    };
    const vah::TileClock clk0{t, ev->tparity, 1, ev->steps};
    const vah::Eos eos = make_eos(ev);
    auto stage = [&](int st, int m) {
        return vah::tile_launch(ev->d_tslot, nullptr, clk0, dt, ev->d_titems + (size_t)lb[m] * per_layer,
                                (lb[m + 1] - lb[m]) * per_layer, true, ev->d_tcount, st, ev->opt.physics, eos,
                                ev->d_terr, ev->stream);
    };
    VAH_TRY(cudaEventRecord(start, ev->stream));  // after the work queued before this step
    VAH_TRY(cudaStreamWaitEvent(ev->s_in, start, 0));
    VAH_TRY(cudaStreamWaitEvent(ev->s_out, start, 0));
    size_t loaded = 0;  // ghosted planes [0, loaded) queued for copy-in and narrowed
    int rc = VAH_OK;
    for (int m = 0; m <= nslab && rc == VAH_OK; ++m) {
        if (m < nslab) {
            const size_t need = m == nslab - 1 ? (size_t)nz + 4 : (size_t)plane_of(lb[m + 1]) + 4;
            rc = copy_planes(true, loaded, need, ev->s_in);
            if (rc != VAH_OK) break;
            VAH_TRY(cudaEventRecord(in_ready[m], ev->s_in));
            VAH_TRY(cudaStreamWaitEvent(ev->stream, in_ready[m], 0));
            rc = convert(true, loaded, need);
            if (rc != VAH_OK) break;
            loaded = need;
            VAH_TRY(stage(1, m));
        }
        if (m >= 1) {
            const int k = m - 1, lo = plane_of(lb[k]), hi = plane_of(lb[k + 1]);
            VAH_TRY(stage(2, k));
            const size_t p0 = k == 0 ? 0 : (size_t)lo + 2, p1 = k == nslab - 1 ? (size_t)nz + 4 : (size_t)hi + 2;
            rc = convert(false, p0, p1);
            if (rc != VAH_OK) break;
            VAH_TRY(cudaEventRecord(done[k], ev->stream));
            VAH_TRY(cudaStreamWaitEvent(ev->s_out, done[k], 0));
            rc = copy_planes(false, p0, p1, ev->s_out);
        }
    }
    // join the copy streams back into the event's stream, also on an error
    if (cudaEventRecord(end, ev->s_out) == cudaSuccess) cudaStreamWaitEvent(ev->stream, end, 0);
    if (cudaEventRecord(end, ev->s_in) == cudaSuccess) cudaStreamWaitEvent(ev->stream, end, 0);
    if (rc != VAH_OK) return rc;
    for (int m = 0; m < 4; ++m) {  // as vah_rk2_step
        void *tmp = ev->u[m];
        ev->u[m] = ev->up[m];
        ev->up[m] = tmp;
    }
    ev->tparity ^= 1;
    ev->steps++;
    ev->last_t = t + dt;
    ev->last_dt = dt;
    return vah_event_sync(ev);
}

}  // namespace

extern "C" int vah_rk2_step_host(vah_event *ev, double t, double dt, double *const *fields) {
    if (!ev || !fields) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(ev->opt.device));
    int rc;
    // overlapped copies where the lattice has enough planes along eta (at
    // least 3 slabs); slab thickness from VAH_HOST_SLAB_PLANES (>= 2) when
    // set, else nz / 6 (6 slabs: the best of 3 to 40 on the 121x121x81 event;
    // the FP32 form rounds it to whole tile layers)
    static const int slab_env = [] {
        const char *v = getenv("VAH_HOST_SLAB_PLANES");
        return v ? atoi(v) : 0;
    }();
    const int slab = slab_env >= 2 ? slab_env : std::max(2, ev->lat.nz / 6);
    if (ev->elem != sizeof(double)) {
        if (ev->lat.nz > 1 && !ev->validity && tile_slab_layers(ev->lat.nz, slab).size() >= 4) {
            if (!(dt > 0) || !(t > 0)) return VAH_ERR_ARG;
            return step_host_fp32_pipelined(ev, t, dt, fields, slab);
        }
        return step_host_fp32(ev, t, dt, fields);
    }
    if (ev->opt.flux != VAH_FLUX_PER_CELL_FUSED && !ev->validity && ev->lat.nz >= 3 * slab) {
        if (!(dt > 0) || !(t > 0)) return VAH_ERR_ARG;
        return step_host_pipelined(ev, t, dt, fields, slab);
    }
    const size_t bytes = ev->ncell * sizeof(double);
    // all copies are queued on the event's stream; one synchronisation at the end
    for (int id = 0; id < VAH_NUM_FIELDS; ++id) {
        void *d = field_ptr(ev, id);
        if (d && fields[id]) VAH_TRY(cudaMemcpyAsync(d, fields[id], bytes, cudaMemcpyHostToDevice, ev->stream));
    }
    rc = vah_rk2_step(ev, t, dt);
    if (rc != VAH_OK) return rc;
    if ((rc = fill_host_zghosts(ev, fields)) != VAH_OK) return rc;
    for (int id = 0; id < VAH_NUM_FIELDS; ++id) {  // pointers after the u <-> up swap
        void *d = field_ptr(ev, id);
        if (d && fields[id]) VAH_TRY(cudaMemcpyAsync(fields[id], d, bytes, cudaMemcpyDeviceToHost, ev->stream));
    }
    return vah_event_sync(ev);
}
