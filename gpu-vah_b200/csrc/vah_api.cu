// vah_api.cu -- the C ABI of include/vah.h over the CUDA kernels.
//
// An event owns its device state: conserved q (current) and qS (intermediate
// stage), two (e, p) buffers used ping-pong across the two stages, and the
// three velocity sets u (current), up (previous step) and uS (intermediate).
// No call ever exits or traps; failures come back as status codes.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "vah.h"
#include "vah_kernels.cuh"
#include "vah_powf_exc.h"

using vah::FieldSet;
using vah::StageArgs;

struct vah_event {
    vah_lattice lat;
    vah_hydro hydro;
    vah_options opt;
    int nq;
    int ncx, ncy, ncz;
    size_t ncell;
    cudaStream_t stream;
    bool own_stream;
    double *q[16], *qS[16];
    double *ep[2][2];  // [buffer][0 = e, 1 = p]
    int cur;           // current (e, p) buffer
    double *u[4], *up[4], *uS[4];
    double *H[3][16];  // face fluxes (VAH_FLUX_SHARED): scratch of the stage launches
    double *HR[3][16];
    double *d_tab;
    uint32_t *d_exc;
    int nexc;
    unsigned long long *d_counters;  // face fallbacks, cell fallbacks, NaN cells
    long long steps;
    bool timing;
    std::vector<cudaEvent_t> tev;  // start/stop pairs of timed launches
    int tev_used;
    double kernel_ms;
    long long kernel_launches;
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

double *field_ptr(vah_event *ev, int id) {
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
    for (int n = 0; n < 16; ++n) {
        cudaFree(ev->q[n]);
        cudaFree(ev->qS[n]);
    }
    for (int b = 0; b < 2; ++b)
        for (int m = 0; m < 2; ++m) cudaFree(ev->ep[b][m]);
    for (int m = 0; m < 4; ++m) {
        cudaFree(ev->u[m]);
        cudaFree(ev->up[m]);
        cudaFree(ev->uS[m]);
    }
    for (int d = 0; d < 3; ++d)
        for (int n = 0; n < 16; ++n) {
            cudaFree(ev->H[d][n]);
            cudaFree(ev->HR[d][n]);
        }
    cudaFree(ev->d_tab);
    cudaFree(ev->d_exc);
    cudaFree(ev->d_counters);
    for (cudaEvent_t e : ev->tev) cudaEventDestroy(e);
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

void fill_common(const vah_event *ev, StageArgs<double> &a) {
    memset(&a, 0, sizeof(a));
    a.nx = ev->lat.nx;
    a.ny = ev->lat.ny;
    a.nz = ev->lat.nz;
    a.ncx = ev->ncx;
    a.ncy = ev->ncy;
    a.plane = (long long)ev->ncx * ev->ncy;
    a.dx = ev->lat.dx;
    a.dy = ev->lat.dy;
    a.dz = ev->lat.dz;
    a.etabar = ev->hydro.eta_over_s;
    a.eos = make_eos(ev);
    a.counters = ev->d_counters;
    for (int d = 0; d < 3; ++d)
        for (int n = 0; n < 16; ++n) {
            a.H[d][n] = ev->H[d][n];
            a.HR[d][n] = ev->HR[d][n];
        }
}

int timed_launch(vah_event *ev, const StageArgs<double> &a) {
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
    if (ev->opt.flux == VAH_FLUX_PER_CELL_FUSED)
        VAH_TRY(vah::launch_stage<double>(a, ev->opt.physics, ev->stream));
    else
        VAH_TRY(vah::launch_stage_split<double>(a, ev->opt.physics, ev->opt.flux == VAH_FLUX_PER_CELL, ev->stream));
    if (pair) VAH_TRY(cudaEventRecord(pair[1], ev->stream));
    return VAH_OK;
}

}  // namespace

extern "C" const char *vah_version(void) { return "vah-b200 0.1 (sm_100a)"; }

extern "C" int vah_event_create(const vah_lattice *lat, const vah_hydro *hydro, const vah_options *opt,
                                const double *eos_table, vah_event **out) {
    if (!lat || !hydro || !opt || !out) return VAH_ERR_ARG;
    *out = nullptr;
    if (lat->nx < 1 || lat->ny < 1 || lat->nz < 1) return VAH_ERR_ARG;
    if (!(lat->dx > 0) || !(lat->dy > 0) || !(lat->dz > 0) || !(hydro->eta_over_s > 0)) return VAH_ERR_ARG;
    if (opt->physics < VAH_IDEAL || opt->physics > VAH_PIMUNU_PI) return VAH_ERR_ARG;
    if (opt->eos != VAH_EOS_CONFORMAL && opt->eos != VAH_EOS_TABLE) return VAH_ERR_ARG;
    if (opt->eos == VAH_EOS_TABLE && !eos_table) return VAH_ERR_ARG;
    if (opt->precision != VAH_FP64) return VAH_ERR_ARG;  // FP32 storage: separate entry
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
    ev->ncx = lat->nx + 4;
    ev->ncy = lat->ny + 4;
    ev->ncz = lat->nz + 4;
    ev->ncell = (size_t)ev->ncx * ev->ncy * ev->ncz;
    ev->cur = 0;
    ev->tev_used = 0;
    ev->kernel_ms = 0;
    ev->kernel_launches = 0;
    ev->timing = false;
    ev->steps = 0;
    ev->nexc = 0;
    ev->own_stream = opt->stream == nullptr;
    int rc = VAH_OK;
    auto alloc = [&](double **p) {
        if (rc != VAH_OK) return;
        cudaError_t e = cudaMalloc((void **)p, ev->ncell * sizeof(double));
        if (e == cudaSuccess) e = cudaMemset(*p, 0, ev->ncell * sizeof(double));
        if (e != cudaSuccess) rc = cuda_status(e);
    };
    if (ev->own_stream) {
        if (cudaStreamCreateWithFlags(&ev->stream, cudaStreamNonBlocking) != cudaSuccess) rc = VAH_ERR_CUDA;
    } else {
        ev->stream = (cudaStream_t)opt->stream;
    }
    for (int n = 0; n < 16; ++n)
        if (n < ev->nq || (n == VAH_F_PI && ev->nq == 16)) {
            alloc(&ev->q[n]);
            alloc(&ev->qS[n]);
        }
    for (int b = 0; b < 2; ++b)
        for (int m = 0; m < 2; ++m) alloc(&ev->ep[b][m]);
    for (int m = 0; m < 4; ++m) {
        alloc(&ev->u[m]);
        alloc(&ev->up[m]);
        alloc(&ev->uS[m]);
    }
    if (opt->flux != VAH_FLUX_PER_CELL_FUSED)
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

extern "C" int vah_event_set_field(vah_event *ev, int field, const double *host, int with_ghosts) {
    if (!ev || !host) return VAH_ERR_ARG;
    double *d = field_ptr(ev, field);
    if (!d) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(ev->opt.device));
    if (with_ghosts) {
        VAH_TRY(cudaMemcpyAsync(d, host, ev->ncell * sizeof(double), cudaMemcpyHostToDevice, ev->stream));
        VAH_TRY(cudaStreamSynchronize(ev->stream));
        return VAH_OK;
    }
    // interior rows: one 2D copy per eta layer
    const int nx = ev->lat.nx, ny = ev->lat.ny, nz = ev->lat.nz;
    for (int k = 0; k < nz; ++k) {
        double *dst = d + 2 + (size_t)ev->ncx * (2 + (size_t)ev->ncy * (k + 2));
        const double *src = host + (size_t)nx * ny * k;
        VAH_TRY(cudaMemcpy2DAsync(dst, ev->ncx * sizeof(double), src, nx * sizeof(double), nx * sizeof(double), ny,
                                  cudaMemcpyHostToDevice, ev->stream));
    }
    VAH_TRY(cudaStreamSynchronize(ev->stream));
    return VAH_OK;
}

extern "C" int vah_event_get_field(vah_event *ev, int field, double *host, int with_ghosts) {
    if (!ev || !host) return VAH_ERR_ARG;
    double *d = field_ptr(ev, field);
    if (!d) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(ev->opt.device));
    if (with_ghosts) {
        VAH_TRY(cudaMemcpyAsync(host, d, ev->ncell * sizeof(double), cudaMemcpyDeviceToHost, ev->stream));
    } else {
        const int nx = ev->lat.nx, ny = ev->lat.ny, nz = ev->lat.nz;
        for (int k = 0; k < nz; ++k) {
            const double *src = d + 2 + (size_t)ev->ncx * (2 + (size_t)ev->ncy * (k + 2));
            double *dst = host + (size_t)nx * ny * k;
            VAH_TRY(cudaMemcpy2DAsync(dst, nx * sizeof(double), src, ev->ncx * sizeof(double), nx * sizeof(double), ny,
                                      cudaMemcpyDeviceToHost, ev->stream));
        }
    }
    VAH_TRY(cudaStreamSynchronize(ev->stream));
    return VAH_OK;
}

extern "C" int vah_event_set_conserved(vah_event *ev, double t, int pl_from_field) {
    if (!ev) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(ev->opt.device));
    FieldSet<double> q{}, u{}, up{};
    for (int n = 0; n < 16; ++n) q.f[n] = ev->q[n];
    q.n = 16;
    for (int m = 0; m < 4; ++m) {
        u.f[m] = ev->u[m];
        up.f[m] = ev->up[m];
    }
    u.n = up.n = 4;
    VAH_TRY(vah::launch_set_conserved<double>(q, u, up, ev->ep[ev->cur][0], ev->opt.physics, ev->lat.nx, ev->lat.ny,
                                              ev->lat.nz, t, pl_from_field, ev->stream));
    VAH_TRY(cudaStreamSynchronize(ev->stream));
    return VAH_OK;
}

extern "C" int vah_event_init_from_e(vah_event *ev, double t0, const double *e_interior, int pl_mode) {
    if (!ev || !e_interior || (pl_mode != VAH_PL_REFERENCE && pl_mode != VAH_PL_ISOTROPIC)) return VAH_ERR_ARG;
    int rc = vah_event_set_field(ev, VAH_F_E, e_interior, 0);
    if (rc != VAH_OK) return rc;
    FieldSet<double> q{}, u{};
    for (int n = 0; n < 16; ++n) q.f[n] = ev->q[n];
    q.n = 16;
    for (int m = 0; m < 4; ++m) u.f[m] = ev->u[m];
    u.n = 4;
    VAH_TRY(vah::launch_init_primitives<double>(q, u, ev->ep[ev->cur][0], ev->ep[ev->cur][1], make_eos(ev),
                                                ev->lat.nx, ev->lat.ny, ev->lat.nz, ev->stream));
    rc = vah_event_set_conserved(ev, t0, pl_mode == VAH_PL_ISOTROPIC);
    if (rc != VAH_OK) return rc;
    return vah_event_set_ghost_cells(ev);
}

extern "C" int vah_event_set_ghost_cells(vah_event *ev) {
    if (!ev) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(ev->opt.device));
    FieldSet<double> f{};
    int n = 0;
    f.f[n++] = ev->ep[ev->cur][0];
    f.f[n++] = ev->ep[ev->cur][1];
    for (int m = 0; m < 4; ++m) f.f[n++] = ev->u[m];
    for (int k = 0; k < 16; ++k)
        if (ev->q[k]) f.f[n++] = ev->q[k];
    f.n = n;
    VAH_TRY(vah::launch_ghosts<double>(f, ev->lat.nx, ev->lat.ny, ev->lat.nz, ev->stream));
    VAH_TRY(cudaStreamSynchronize(ev->stream));
    return VAH_OK;
}

extern "C" int vah_rk2_step(vah_event *ev, double t, double dt) {
    if (!ev || !(dt > 0) || !(t > 0)) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(ev->opt.device));
    const int c = ev->cur, o = 1 - ev->cur;
    StageArgs<double> a;
    // stage 1: q, u, (e, p)[c], up -> qS, uS, (e, p)[o]
    fill_common(ev, a);
    a.t_src = t;
    a.t_inv = t + dt;
    a.dt = dt;
    a.stage2 = 0;
    for (int n = 0; n < 16; ++n) {
        a.qin[n] = ev->q[n];
        a.qout[n] = ev->qS[n];
    }
    for (int m = 0; m < 4; ++m) {
        a.uin[m] = ev->u[m];
        a.upin[m] = ev->up[m];
        a.guess[m] = ev->u[m];
        a.uout[m] = ev->uS[m];
    }
    a.ein = ev->ep[c][0];
    a.pin = ev->ep[c][1];
    a.eout = ev->ep[o][0];
    a.pout = ev->ep[o][1];
    int rc = timed_launch(ev, a);
    if (rc != VAH_OK) return rc;
    // stage 2: qS, uS, (e, p)[o], u -> q (in place, with the convex
    // combination), up buffer (becomes u^{n+1}), (e, p)[c]
    fill_common(ev, a);
    a.t_src = t + dt;
    a.t_inv = t + dt;
    a.dt = dt;
    a.stage2 = 1;
    for (int n = 0; n < 16; ++n) {
        a.qin[n] = ev->qS[n];
        a.qavg[n] = ev->q[n];
        a.qout[n] = ev->q[n];
    }
    for (int m = 0; m < 4; ++m) {
        a.uin[m] = ev->uS[m];
        a.upin[m] = ev->u[m];
        a.guess[m] = ev->u[m];
        a.uout[m] = ev->up[m];
    }
    a.ein = ev->ep[o][0];
    a.pin = ev->ep[o][1];
    a.eout = ev->ep[c][0];
    a.pout = ev->ep[c][1];
    rc = timed_launch(ev, a);
    if (rc != VAH_OK) return rc;
    // swapFluidVelocity(&up, &u) (FullyDiscreteKurganovTadmorScheme.cpp:784)
    for (int m = 0; m < 4; ++m) {
        double *tmp = ev->u[m];
        ev->u[m] = ev->up[m];
        ev->up[m] = tmp;
    }
    ev->steps++;
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

extern "C" int vah_rk2_step_host(vah_event *ev, double t, double dt, double *const *fields) {
    if (!ev || !fields) return VAH_ERR_ARG;
    VAH_TRY(cudaSetDevice(ev->opt.device));
    const size_t bytes = ev->ncell * sizeof(double);
    // all copies are queued on the event's stream; one synchronisation at the end
    for (int id = 0; id < VAH_NUM_FIELDS; ++id) {
        double *d = field_ptr(ev, id);
        if (d && fields[id]) VAH_TRY(cudaMemcpyAsync(d, fields[id], bytes, cudaMemcpyHostToDevice, ev->stream));
    }
    int rc = vah_rk2_step(ev, t, dt);
    if (rc != VAH_OK) return rc;
    for (int id = 0; id < VAH_NUM_FIELDS; ++id) {  // pointers after the u <-> up swap
        double *d = field_ptr(ev, id);
        if (d && fields[id]) VAH_TRY(cudaMemcpyAsync(fields[id], d, bytes, cudaMemcpyDeviceToHost, ev->stream));
    }
    return vah_event_sync(ev);
}
