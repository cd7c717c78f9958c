// vah_noalloc.cu -- one RK stage that allocates nothing.
//
// Some callers cannot allocate device memory: code running inside a host
// framework that owns all device memory through its own pool, callers that
// queue work from a context where cudaMalloc is forbidden or would
// synchronise the device, and processes that must keep their device
// footprint fixed after start-up. vah_stage_noalloc serves them. It runs one
// RK stage of the face/cell split (reference face semantics, FP64 storage)
// on state buffers the caller owns, and keeps the stage's scratch -- the face
// fluxes as each neighbour evaluates them, plus the fallback/NaN counters --
// in the file-scope array below instead of allocating it.
//
// The array is a fixed part of the library's device image: every GPU that
// loads libvah.so holds its VAH_NOALLOC_SCRATCH_BYTES until the process
// exits. Host code cannot use the array's name as a device address (on the
// host the name denotes a host-side stand-in), so the first call on each
// device looks the address up with cudaGetSymbolAddress while that device is
// current and caches it; that first call should therefore come before any
// stream capture. The cache is keyed on the device's context as well (its
// driver-assigned unique id): after the caller resets the device
// (cudaDeviceReset) the module may load at another address, and the next
// call looks it up again -- so the first call after a reset should also come
// before any capture. All calls share the array and it keeps the last call's
// contents: the counters are cleared at the start of every call, and calls
// whose work overlaps on the GPU (two streams, two host threads) race on it.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "vah.h"
#include "vah_kernels.cuh"

namespace {

constexpr size_t kCounterBytes = 256;  // 3 counters, padded to the alignment
static_assert(VAH_NOALLOC_SCRATCH_BYTES % 256 == 0, "scratch size must be 256-byte aligned");

static __device__ __align__(256) unsigned char g_noalloc_scratch[VAH_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char *g_scratch_ptr[kMaxDevices] = {nullptr};
unsigned long long g_scratch_ctx[kMaxDevices] = {0};  // context id the cached address belongs to

// The two driver calls that identify the current context, resolved through
// the runtime (the library does not link the driver library directly).
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

// Unique id of the calling thread's current context (the device's primary
// context after cudaSetDevice); called with g_setup_mutex held.
int current_context_id(unsigned long long *id) {
    if (!g_ctx_get_current || !g_ctx_get_id) {
        cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", (void **)&g_ctx_get_current, 12000,
                                             cudaEnableDefault, &q1) != cudaSuccess ||
            cudaGetDriverEntryPointByVersion("cuCtxGetId", (void **)&g_ctx_get_id, 12000, cudaEnableDefault, &q2) !=
                cudaSuccess ||
            q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess) {
            g_ctx_get_current = nullptr;
            g_ctx_get_id = nullptr;
            return VAH_ERR_CUDA;
        }
    }
    CUcontext ctx = nullptr;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return VAH_ERR_CUDA;
    if (g_ctx_get_id(ctx, id) != CUDA_SUCCESS) return VAH_ERR_CUDA;
    return VAH_OK;
}

// Device address of the scratch array on the current device: looked up on
// the first call in each context of the device (set-up), cached after.
int scratch_address(int device, unsigned char **out) {
    if (device < 0 || device >= kMaxDevices) return VAH_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return VAH_ERR_CUDA;  // makes the primary context current
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    unsigned long long ctx = 0;
    int rc = current_context_id(&ctx);
    if (rc != VAH_OK) return rc;
    if (!g_scratch_ptr[device] || g_scratch_ctx[device] != ctx) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) return VAH_ERR_CUDA;
        g_scratch_ptr[device] = (unsigned char *)p;
        g_scratch_ctx[device] = ctx;
    }
    *out = g_scratch_ptr[device];
    return VAH_OK;
}

int nq_of(int physics) { return physics == VAH_IDEAL ? 5 : (physics == VAH_PIMUNU ? 15 : 16); }

}  // namespace

extern "C" int vah_stage_noalloc(const vah_lattice *lat, double eta_over_s, int physics, int eos, int zeta,
                                 const double *d_eos_table, int stage, double t, double dt,
                                 const vah_stage_buffers *buf, void *stream, long long *counts_out) {
    if (!lat || !buf || (stage != 1 && stage != 2) || !(dt > 0) || !(t > 0) || !(eta_over_s > 0)) return VAH_ERR_ARG;
    if (lat->nx < 1 || lat->ny < 1 || lat->nz < 1) return VAH_ERR_ARG;
    if (!(lat->dx > 0) || !(lat->dy > 0) || !(lat->dz > 0)) return VAH_ERR_ARG;
    if (physics < VAH_IDEAL || physics > VAH_PIMUNU_PI) return VAH_ERR_ARG;
    if (eos != VAH_EOS_CONFORMAL && eos != VAH_EOS_TABLE) return VAH_ERR_ARG;
    if (eos == VAH_EOS_TABLE && !d_eos_table) return VAH_ERR_ARG;
    const int nq = nq_of(physics);
    for (int n = 0; n < nq; ++n)
        if (!buf->q[n] || !buf->q_out[n] || (stage == 2 && !buf->q_avg[n])) return VAH_ERR_ARG;
    for (int m = 0; m < 4; ++m)
        if (!buf->u[m] || !buf->u_prev[m] || !buf->u_out[m]) return VAH_ERR_ARG;
    if (!buf->e || !buf->p || !buf->e_out || !buf->p_out) return VAH_ERR_ARG;

    const size_t ncell = (size_t)(lat->nx + 4) * (lat->ny + 4) * (lat->nz + 4);
    const int ndir = lat->nz > 1 ? 3 : 2;
    const size_t need = kCounterBytes + (size_t)ndir * nq * 2 * ncell * sizeof(double);
    if (need > VAH_NOALLOC_SCRATCH_BYTES) return VAH_ERR_TOO_LARGE;

    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return VAH_ERR_NODEVICE;
    unsigned char *base = nullptr;
    int rc = scratch_address(device, &base);
    if (rc != VAH_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;

    vah::StageArgs<double> a;
    memset(&a, 0, sizeof(a));
    a.nx = lat->nx;
    a.ny = lat->ny;
    a.nz = lat->nz;
    a.k0 = 0;
    a.k1 = lat->nz;
    a.ncx = lat->nx + 4;
    a.ncy = lat->ny + 4;
    a.plane = (long long)a.ncx * a.ncy;
    a.dx = lat->dx;
    a.dy = lat->dy;
    a.dz = lat->dz;
    a.dt = dt;
    a.etabar = eta_over_s;
    a.t_src = stage == 1 ? t : t + dt;
    a.t_inv = t + dt;
    a.stage2 = stage == 2;
    a.zghosts = 1;  // the caller's buffers come back with every ghost layer a stage writes
    a.eos.kind = eos == VAH_EOS_TABLE ? 1 : 0;
    a.eos.zeta = zeta == VAH_ZETA_CROSSOVER ? 1 : 0;
    a.eos.tab = d_eos_table;
    a.eos.exc = nullptr;  // conformal T: the correctly rounded fourth root (no libm table here)
    a.eos.nexc = 0;
    for (int n = 0; n < nq; ++n) {
        a.qin[n] = buf->q[n];
        a.qout[n] = buf->q_out[n];
        a.qavg[n] = buf->q_avg[n];
    }
    for (int m = 0; m < 4; ++m) {
        a.uin[m] = buf->u[m];
        a.upin[m] = buf->u_prev[m];
        a.guess[m] = stage == 1 ? buf->u[m] : buf->u_prev[m];
        a.uout[m] = buf->u_out[m];
    }
    a.ein = buf->e;
    a.pin = buf->p;
    a.eout = buf->e_out;
    a.pout = buf->p_out;
    a.counters = (unsigned long long *)base;
    double *faces = (double *)(base + kCounterBytes);
    for (int d = 0; d < ndir; ++d)
        for (int n = 0; n < nq; ++n) {
            a.H[d][n] = faces + ((size_t)(d * nq + n) * 2) * ncell;
            a.HR[d][n] = faces + ((size_t)(d * nq + n) * 2 + 1) * ncell;
        }

    vah::finish_args(a);
    if (cudaMemsetAsync(base, 0, kCounterBytes, s) != cudaSuccess) return VAH_ERR_CUDA;
    if (vah::launch_stage_split<double>(a, physics, true, s) != cudaSuccess) return VAH_ERR_CUDA;
    if (counts_out) {
        unsigned long long c[3];
        if (cudaMemcpyAsync(c, base, sizeof(c), cudaMemcpyDeviceToHost, s) != cudaSuccess) return VAH_ERR_CUDA;
        if (cudaStreamSynchronize(s) != cudaSuccess) return VAH_ERR_CUDA;
        for (int k = 0; k < 3; ++k) counts_out[k] = (long long)c[k];
        if (c[2]) return VAH_ERR_NAN;
    }
    return VAH_OK;
}
