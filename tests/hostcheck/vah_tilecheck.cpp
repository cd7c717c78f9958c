// tests/hostcheck/vah_tilecheck.cpp -- test harness: the FP32 form of the
// stage (gpu-vah_b200/csrc/vah_tile_cell.cuh, the arithmetic the TMA-tiled
// kernel runs) compiled for the host and driven face by face and cell by cell
// with the buffer roles of vah_rk2_step. The tests compare it with the FP64
// forms on the CPU and with the tile kernel on the GPU. Not part of the
// library, and never loaded by it.
#include <cmath>
#include <cstring>
#include <vector>

#include "vah.h"
#include "vah_powf_exc.h"
#include "vah_stage.cuh"
#include "vah_tile_cell.cuh"

namespace {

struct TileHost {
    int nx, ny, nz, ncx, ncy, ncz, nq, physics;
    size_t ncell;
    double dx, dy, dz, etabar;
    std::vector<float> store, hstore;
    float *q[16], *qS[16], *ep[2][2], *u[4], *up[4], *uS[4];
    float *H[3][16];  // face at +1/2 of cell s along each axis
    vah::Eos eos;
    std::vector<double> tab;
    unsigned long long counters[3];
};

template <int PHYS, bool IS3D>
void tile_stage(TileHost *h, int stage, double t, double dt) {
    constexpr int NQ = vah::Phys<PHYS>::NQ;
    const long long sy = h->ncx, sz = (long long)h->ncx * h->ncy;
    const long long strides[3] = {1, sy, sz};
    const double hs[3] = {h->dx, h->dy, h->dz};
    float *const *qin = stage == 1 ? h->q : h->qS;
    float *const *qout = stage == 1 ? h->qS : h->q;
    const float *Ein = h->ep[stage == 1 ? 0 : 1][0], *Pin = h->ep[stage == 1 ? 0 : 1][1];
    float *Eout = h->ep[stage == 1 ? 1 : 0][0], *Pout = h->ep[stage == 1 ? 1 : 0][1];
    float *const *Uin = stage == 1 ? h->u : h->uS;
    float *const *Uup = stage == 1 ? h->up : h->u;
    float *const *Uout = stage == 1 ? h->uS : h->up;
    const double t_src = stage == 1 ? t : t + dt, t_inv = t + dt;
    const vah::ArrQ qa{(const float *const *)qin};
    // faces at +1/2 of the cells 1 .. n + 1 along each axis, interior across
    for (int d = 0; d < (IS3D ? 3 : 2); ++d)
        for (int k = (d == 2 ? 1 : 2); k < h->nz + 2; ++k)
            for (int j = (d == 1 ? 1 : 2); j < h->ny + 2; ++j)
                for (int i = (d == 0 ? 1 : 2); i < h->nx + 2; ++i) {
                    const long long s = i + sy * j + sz * k;
                    const double ux = Uin[1][s], uy = Uin[2][s];
                    float H[NQ];
                    const unsigned f = vah::tile_face<PHYS>(qa, s, strides[d], d, t_src, (double)Ein[s],
                                                            std::sqrt(std::fabs(ux * ux + uy * uy)), H, 1);
                    h->counters[0] += f & 255u;
                    for (int n = 0; n < NQ; ++n) h->H[d][n][s] = H[n];
                }
    vah::TilePrims pr;
    pr.E = Ein;
    pr.P = Pin;
    pr.psy = sy;
    pr.psz = sz;
    for (int m = 0; m < 4; ++m) {
        pr.U[m] = Uin[m];
        pr.UP[m] = Uup[m];
        pr.G[m] = h->u[m];
    }
    const vah::ArrQ qavg{(const float *const *)h->q};
    std::vector<float> outv((size_t)NQ * h->ncell), oute(h->ncell), outp(h->ncell), outu(4 * h->ncell);
    for (int k = 2; k < h->nz + 2; ++k)
        for (int j = 2; j < h->ny + 2; ++j)
            for (int i = 2; i < h->nx + 2; ++i) {
                const long long s = i + sy * j + sz * k;
                float flux[NQ];
                for (int n = 0; n < NQ; ++n) flux[n] = 0.0f;
                for (int d = 0; d < (IS3D ? 3 : 2); ++d) {
                    const float c = (float)(dt / hs[d]);
                    for (int n = 0; n < NQ; ++n) flux[n] += c * (h->H[d][n][s - strides[d]] - h->H[d][n][s]);
                }
                float val[NQ], e, p, u[4];
                int bad = 0;
                pr.pi = s;
                const int st = vah::tile_cell<PHYS, IS3D>(qa, s, sy, sz, pr, s, flux, qavg, stage == 2, h->eos, t_src,
                                                         t_inv, dt, h->dx, h->dy, h->dz, h->etabar, val, e, p, u,
                                                         nullptr, bad);
                if (st != 0) h->counters[1]++;
                if (bad || st == 2) h->counters[2]++;
                for (int n = 0; n < NQ; ++n) outv[n * h->ncell + s] = val[n];
                oute[s] = e;
                outp[s] = p;
                for (int m = 0; m < 4; ++m) outu[m * h->ncell + s] = u[m];
            }
    // stores after every cell has read its inputs (stage 2 writes q in place)
    auto store = [&](long long s, long long at) {
        for (int n = 0; n < NQ; ++n) qout[n][at] = outv[n * h->ncell + s];
        Eout[at] = oute[s];
        Pout[at] = outp[s];
        for (int m = 0; m < 4; ++m) Uout[m][at] = outu[m * h->ncell + s];
    };
    for (int k = 2; k < h->nz + 2; ++k)
        for (int j = 2; j < h->ny + 2; ++j)
            for (int i = 2; i < h->nx + 2; ++i) {
                const long long s = i + sy * j + sz * k;
                store(s, s);
                if (i == 2) { store(s, s - 1); store(s, s - 2); }
                if (i == h->nx + 1) { store(s, s + 1); store(s, s + 2); }
                if (j == 2) { store(s, s - sy); store(s, s - 2 * sy); }
                if (j == h->ny + 1) { store(s, s + sy); store(s, s + 2 * sy); }
                if (k == 2) { store(s, s - sz); store(s, s - 2 * sz); }
                if (k == h->nz + 1) { store(s, s + sz); store(s, s + 2 * sz); }
            }
}

template <bool IS3D>
void stage_any(TileHost *h, int stage, double t, double dt) {
    switch (h->physics) {
    case 0: tile_stage<0, IS3D>(h, stage, t, dt); break;
    case 1: tile_stage<1, IS3D>(h, stage, t, dt); break;
    default: tile_stage<2, IS3D>(h, stage, t, dt); break;
    }
}

}  // namespace

extern "C" {

void *tc_create(int nx, int ny, int nz, double dx, double dy, double dz, double etabar, int physics, int eos, int zeta,
                const double *tab) {
    TileHost *h = new TileHost();
    h->nx = nx; h->ny = ny; h->nz = nz; h->ncx = nx + 4; h->ncy = ny + 4; h->ncz = nz + 4;
    h->ncell = (size_t)h->ncx * h->ncy * h->ncz;
    h->physics = physics;
    h->nq = physics == 0 ? 5 : (physics == 1 ? 15 : 16);
    h->dx = dx; h->dy = dy; h->dz = dz; h->etabar = etabar;
    h->store.assign(h->ncell * 48, 0.0f);
    float *p = h->store.data();
    for (int n = 0; n < 16; ++n) { h->q[n] = p; p += h->ncell; h->qS[n] = p; p += h->ncell; }
    for (int b = 0; b < 2; ++b) for (int m = 0; m < 2; ++m) { h->ep[b][m] = p; p += h->ncell; }
    for (int m = 0; m < 4; ++m) { h->u[m] = p; p += h->ncell; h->up[m] = p; p += h->ncell; h->uS[m] = p; p += h->ncell; }
    h->hstore.assign(h->ncell * 48, 0.0f);
    for (int d = 0; d < 3; ++d)
        for (int n = 0; n < 16; ++n) h->H[d][n] = h->hstore.data() + h->ncell * (16 * d + n);
    h->eos.kind = eos;
    h->eos.zeta = zeta;
    h->eos.tab = nullptr;
    if (tab) {
        h->tab.assign(tab, tab + VAH_EOS_TABLE_LEN((int)tab[0]));
        h->eos.tab = h->tab.data();
    }
    const std::vector<uint32_t> &t = vah::powf_quarter_exceptions();  // the library's libm table
    h->eos.exc = t.data();
    h->eos.nexc = (int)(t.size() / 2);
    std::memset(h->counters, 0, sizeof(h->counters));
    return h;
}

void tc_destroy(void *p) { delete (TileHost *)p; }

// Field VAH_F_* in its current role (float, ghosted reference layout).
float *tc_field(void *p, int id) {
    TileHost *h = (TileHost *)p;
    if (id >= 0 && id < 16) return id < h->nq ? h->q[id] : nullptr;
    if (id == VAH_F_E) return h->ep[0][0];
    if (id == VAH_F_P) return h->ep[0][1];
    if (id >= VAH_F_UT && id <= VAH_F_UN) return h->u[id - VAH_F_UT];
    if (id >= VAH_F_UPT && id <= VAH_F_UPN) return h->up[id - VAH_F_UPT];
    return nullptr;
}

void tc_step(void *p, double t, double dt) {
    TileHost *h = (TileHost *)p;
    if (h->nz > 1) {
        stage_any<true>(h, 1, t, dt);
        stage_any<true>(h, 2, t, dt);
    } else {
        stage_any<false>(h, 1, t, dt);
        stage_any<false>(h, 2, t, dt);
    }
    for (int m = 0; m < 4; ++m) std::swap(h->u[m], h->up[m]);
}

void tc_counters(void *p, unsigned long long *out) { std::memcpy(out, ((TileHost *)p)->counters, 3 * 8); }

}  // extern "C"
