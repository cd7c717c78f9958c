// tests/hostcheck/vah_hostcheck.cpp -- test harness: the library's per-cell
// stage code (gpu-vah_b200/csrc/vah_stage.cuh) compiled for the host and driven
// cell by cell with the same buffer rotation as vah_rk2_step in vah_api.cu.
// It lets the tests check the device formulas against the CPU oracle without
// a GPU. Not part of the library, and never loaded by it.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "vah.h"
#include "vah_powf_exc.h"
#include "vah_stage.cuh"
#include "vah_validity.cuh"

namespace {

struct HostEvent {
    int nx, ny, nz, ncx, ncy, ncz, nq, physics;
    size_t ncell;
    double dx, dy, dz, etabar;
    std::vector<double> store;
    double *q[16], *qS[16], *ep[2][2], *u[4], *up[4], *uS[4];
    int cur;
    int shared;  // VAH_FLUX_SHARED: faces once, then cells
    std::vector<double> hstore;
    double *H[3][16], *HR[3][16];
    vah::Eos eos;
    std::vector<double> tab;
    unsigned long long counters[4];
    bool validity = false;
    std::vector<double> vstore, vqstore;  // 27 validity fields; P_L, pi, Pi at the start of the step
};

template <int PHYS>
void run_stage(const vah::StageArgs<double> &a) {
    for (int k = 0; k < a.nz; ++k)
        for (int j = 0; j < a.ny; ++j)
            for (int i = 0; i < a.nx; ++i) {
                if (a.nz > 1) vah::stage_cell<double, PHYS, true>(a, i + 2, j + 2, k + 2);
                else vah::stage_cell<double, PHYS, false>(a, i + 2, j + 2, k + 2);
            }
}

template <int PHYS, bool EXACT>
void run_stage_split(const vah::StageArgs<double> &a) {
    const long long strides[3] = {1, a.ncx, a.plane};
    for (int dir = 0; dir < (a.nz > 1 ? 3 : 2); ++dir)
        for (int k = (dir == 2 ? 1 : 2); k < a.nz + 2; ++k)
            for (int j = (dir == 1 ? 1 : 2); j < a.ny + 2; ++j)
                for (int i = (dir == 0 ? 1 : 2); i < a.nx + 2; ++i) {
                    const int gl = dir == 0 ? i : (dir == 1 ? j : k), n = dir == 0 ? a.nx : (dir == 1 ? a.ny : a.nz);
                    unsigned f = vah::face_compute<double, PHYS, EXACT>(a, i + (long long)a.ncx * j + a.plane * k,
                                                                          dir, strides[dir], gl >= 2, gl <= n);
                    a.counters[0] += f & 255u;
                }
    for (int k = 0; k < a.nz; ++k)
        for (int j = 0; j < a.ny; ++j)
            for (int i = 0; i < a.nx; ++i) {
                if (a.nz > 1) vah::cell_compute<double, PHYS, true, EXACT>(a, i + 2, j + 2, k + 2);
                else vah::cell_compute<double, PHYS, false, EXACT>(a, i + 2, j + 2, k + 2);
            }
}

template <int PHYS>
void run_split(int mode, const vah::StageArgs<double> &a) {
    if (mode == 1) run_stage_split<PHYS, true>(a);
    else run_stage_split<PHYS, false>(a);
}

void stage(HostEvent *h, const vah::StageArgs<double> &a) {
    if (h->shared) {  // 1: split with reference faces, 2: split with shared faces
        if (h->physics == 0) run_split<0>(h->shared, a);
        else if (h->physics == 1) run_split<1>(h->shared, a);
        else run_split<2>(h->shared, a);
        return;
    }
    if (h->physics == 0) run_stage<0>(a);
    else if (h->physics == 1) run_stage<1>(a);
    else run_stage<2>(a);
}

void common(HostEvent *h, vah::StageArgs<double> &a) {
    std::memset(&a, 0, sizeof(a));
    a.nx = h->nx; a.ny = h->ny; a.nz = h->nz; a.ncx = h->ncx; a.ncy = h->ncy;
    a.k0 = 0; a.k1 = h->nz;
    a.plane = (long long)h->ncx * h->ncy;
    a.dx = h->dx; a.dy = h->dy; a.dz = h->dz; a.etabar = h->etabar;
    a.eos = h->eos;
    a.zghosts = 1;  // every ghost layer the stage writes, as the oracle's arrays hold them
    a.counters = h->counters;
    for (int d = 0; d < 3; ++d)
        for (int n = 0; n < 16; ++n) {
            a.H[d][n] = h->H[d][n];
            a.HR[d][n] = h->HR[d][n];
        }
}

void set_regmap(HostEvent *h, vah::StageArgs<double> &a) {
    if (h->validity)
        for (int m = 0; m < 11; ++m) a.regmap[m] = h->vstore.data() + h->ncell * (VAH_V_REGULATIONS + m);
}

template <int PHYS>
void run_validity(const vah::ValidityArgs<double> &v) {
    for (int k = 0; k < v.nz; ++k)
        for (int j = 0; j < v.ny; ++j)
            for (int i = 0; i < v.nx; ++i)
                vah::validity_cell<double, PHYS>(v, (i + 2) + (long long)v.ncx * (j + 2) + v.plane * (k + 2));
}

}  // namespace

extern "C" {

void *hc_create(int nx, int ny, int nz, double dx, double dy, double dz, double etabar, int physics, int eos,
                int zeta, const double *tab, const unsigned *exc, int nexc) {
    HostEvent *h = new HostEvent();
    h->nx = nx; h->ny = ny; h->nz = nz; h->ncx = nx + 4; h->ncy = ny + 4; h->ncz = nz + 4;
    h->ncell = (size_t)h->ncx * h->ncy * h->ncz;
    h->physics = physics;
    h->nq = physics == 0 ? 5 : (physics == 1 ? 15 : 16);
    h->dx = dx; h->dy = dy; h->dz = dz; h->etabar = etabar;
    h->store.assign(h->ncell * (32 + 4 + 12), 0.0);
    double *p = h->store.data();
    for (int n = 0; n < 16; ++n) { h->q[n] = p; p += h->ncell; h->qS[n] = p; p += h->ncell; }
    for (int b = 0; b < 2; ++b) for (int m = 0; m < 2; ++m) { h->ep[b][m] = p; p += h->ncell; }
    for (int m = 0; m < 4; ++m) { h->u[m] = p; p += h->ncell; h->up[m] = p; p += h->ncell; h->uS[m] = p; p += h->ncell; }
    h->cur = 0;
    h->shared = 0;
    h->hstore.assign(h->ncell * 96, 0.0);
    for (int d = 0; d < 3; ++d)
        for (int n = 0; n < 16; ++n) {
            h->H[d][n] = h->hstore.data() + h->ncell * (16 * d + n);
            h->HR[d][n] = h->hstore.data() + h->ncell * (48 + 16 * d + n);
        }
    h->eos.kind = eos;
    h->eos.zeta = zeta;
    if (tab) {
        int n = (int)tab[0];
        h->tab.assign(tab, tab + VAH_EOS_TABLE_LEN(n));
        h->eos.tab = h->tab.data();
    } else {
        h->eos.tab = nullptr;
    }
    if (nexc < 0) {  // use the library's libm-exception table
        const std::vector<uint32_t> &t = vah::powf_quarter_exceptions();
        h->eos.exc = t.data();
        h->eos.nexc = (int)(t.size() / 2);
    } else {
        h->eos.exc = (const uint32_t *)exc;
        h->eos.nexc = nexc;
    }
    std::memset(h->counters, 0, sizeof(h->counters));
    return h;
}

void hc_destroy(void *p) { delete (HostEvent *)p; }

void hc_set_split(void *p, int mode) { ((HostEvent *)p)->shared = mode; }

double *hc_field(void *p, int id) {
    HostEvent *h = (HostEvent *)p;
    if (id < 16) return h->q[id];
    if (id == VAH_F_E) return h->ep[h->cur][0];
    if (id == VAH_F_P) return h->ep[h->cur][1];
    if (id >= VAH_F_UT && id <= VAH_F_UN) return h->u[id - VAH_F_UT];
    if (id >= VAH_F_UPT && id <= VAH_F_UPN) return h->up[id - VAH_F_UPT];
    return nullptr;
}

void hc_set_conserved(void *p, double t, int pl_from_field) {
    HostEvent *h = (HostEvent *)p;
    for (int k = 0; k < h->nz; ++k)
        for (int j = 0; j < h->ny; ++j)
            for (int i = 0; i < h->nx; ++i) {
                long long s = (i + 2) + (long long)h->ncx * ((j + 2) + (long long)h->ncy * (k + 2));
                if (h->physics == 0) vah::set_conserved_cell<double, 0>(h->q, h->u, h->up, h->ep[h->cur][0], t, pl_from_field, s);
                else if (h->physics == 1) vah::set_conserved_cell<double, 1>(h->q, h->u, h->up, h->ep[h->cur][0], t, pl_from_field, s);
                else vah::set_conserved_cell<double, 2>(h->q, h->u, h->up, h->ep[h->cur][0], t, pl_from_field, s);
            }
}

void hc_set_validity(void *p, int on) {
    HostEvent *h = (HostEvent *)p;
    if (on && h->vstore.empty()) {
        h->vstore.assign(h->ncell * VAH_NUM_VALIDITY, 0.0);
        h->vqstore.assign(h->ncell * 16, 0.0);
    }
    h->validity = on != 0;
}

double *hc_validity_field(void *p, int id) {
    HostEvent *h = (HostEvent *)p;
    return h->vstore.empty() ? nullptr : h->vstore.data() + h->ncell * id;
}

void hc_step(void *p, double t, double dt) {
    HostEvent *h = (HostEvent *)p;
    const int c = h->cur, o = 1 - c;
    if (h->validity)
        for (int n = 4; n < h->nq; ++n)
            std::memcpy(h->vqstore.data() + h->ncell * n, h->q[n], h->ncell * sizeof(double));
    vah::StageArgs<double> a;
    common(h, a);
    set_regmap(h, a);
    a.t_src = t; a.t_inv = t + dt; a.dt = dt; a.stage2 = 0;
    for (int n = 0; n < 16; ++n) { a.qin[n] = h->q[n]; a.qout[n] = h->qS[n]; }
    for (int m = 0; m < 4; ++m) { a.uin[m] = h->u[m]; a.upin[m] = h->up[m]; a.guess[m] = h->u[m]; a.uout[m] = h->uS[m]; }
    a.ein = h->ep[c][0]; a.pin = h->ep[c][1]; a.eout = h->ep[o][0]; a.pout = h->ep[o][1];
    vah::finish_args(a);
    stage(h, a);
    common(h, a);
    set_regmap(h, a);
    a.t_src = t + dt; a.t_inv = t + dt; a.dt = dt; a.stage2 = 1;
    for (int n = 0; n < 16; ++n) { a.qin[n] = h->qS[n]; a.qavg[n] = h->q[n]; a.qout[n] = h->q[n]; }
    for (int m = 0; m < 4; ++m) { a.uin[m] = h->uS[m]; a.upin[m] = h->u[m]; a.guess[m] = h->u[m]; a.uout[m] = h->up[m]; }
    a.ein = h->ep[o][0]; a.pin = h->ep[o][1]; a.eout = h->ep[c][0]; a.pout = h->ep[c][1];
    vah::finish_args(a);
    stage(h, a);
    if (h->validity) {
        vah::ValidityArgs<double> v;
        std::memset(&v, 0, sizeof(v));
        v.nx = h->nx; v.ny = h->ny; v.nz = h->nz; v.ncx = h->ncx; v.ncy = h->ncy;
        v.plane = (long long)h->ncx * h->ncy;
        v.t = t + dt; v.dt = dt; v.dx = h->dx; v.dy = h->dy; v.dz = h->dz; v.etabar = h->etabar;
        for (int n = 0; n < 16; ++n) v.qn[n] = h->vqstore.data() + h->ncell * n;
        v.e = h->ep[c][0]; v.p = h->ep[c][1];
        for (int m = 0; m < 4; ++m) { v.u[m] = h->up[m]; v.up[m] = h->u[m]; }
        v.eos = h->eos;
        for (int m = 0; m < 16; ++m) v.v[m] = h->vstore.data() + h->ncell * m;
        if (h->physics == 0) run_validity<0>(v);
        else if (h->physics == 1) run_validity<1>(v);
        else run_validity<2>(v);
    }
    for (int m = 0; m < 4; ++m) { double *tmp = h->u[m]; h->u[m] = h->up[m]; h->up[m] = tmp; }
}

void hc_counters(void *p, unsigned long long *out) {
    HostEvent *h = (HostEvent *)p;
    for (int k = 0; k < 3; ++k) out[k] = h->counters[k];
}

// The device regulator on one cell (shear + bulk): q[16] and u[4] in, q out;
// with_maps selects the path that also reports the nine ratios.
void hc_regulate(double t, double e, double p, double *q, const double *u, int with_maps) {
    double maps[11];
    vah::regulate<2>(t, e, p, q, u, with_maps ? maps : nullptr);
}

// The limiter of the device code over arrays of (x, y, z) triples.
void hc_approx_derivative(const double *x, const double *y, const double *z, double *out, long long n) {
    for (long long i = 0; i < n; ++i) out[i] = vah::approx_derivative(x[i], y[i], z[i]);
}

}  // extern "C"
