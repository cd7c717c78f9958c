// vah_ic.cpp -- initial energy-density profiles of the benchmark workloads.
//
// The reference builds its Glauber profiles with GSL quadrature and libc rand
// (rhic/src/GlauberModel.cpp:19-108, MonteCarloGlauberModel.cpp:17-108,
// InitialConditions.cpp:196-292). The workloads define their own generators
// (Au+Au, Woods-Saxon R = 6.38 fm, a = 0.535 fm); these are written here
// without GSL, with a counter-based RNG so that an event is a pure function of
// its seed:
//   optical Glauber: e ~ (1-x) N_part/2 + x N_coll with x = 0.15, normalised
//                    to a given peak;
//   MC Glauber:      nucleons sampled from Woods-Saxon, a pair collides when
//                    its transverse distance is below sqrt(sigma_NN/pi), each
//                    participant deposits a 2D Gaussian of width w;
//   longitudinal:    flat for |eta| < eta_flat, Gaussian tails of width sigma_eta.
#include <cmath>
#include <cstdint>
#include <vector>

#include "vah.h"

namespace {

// Woods-Saxon thickness T(r_perp) = int rho dz, rho normalised to A nucleons.
struct Thickness {
    double R, a, rmax, dr;
    std::vector<double> tab;

    Thickness(int A, double R_, double a_) : R(R_), a(a_) {
        rmax = R + 12 * a;
        const int nr = 2048, nz = 2048;
        dr = rmax / (nr - 1);
        tab.assign(nr, 0.0);
        const double zmax = rmax, hz = 2 * zmax / nz;
        for (int ir = 0; ir < nr; ++ir) {
            const double r = ir * dr;
            double s = 0;
            for (int iz = 0; iz <= nz; ++iz) {  // Simpson in z
                const double z = -zmax + iz * hz;
                const double w = (iz == 0 || iz == nz) ? 1 : ((iz & 1) ? 4 : 2);
                s += w / (1 + std::exp((std::sqrt(r * r + z * z) - R) / a));
            }
            tab[ir] = s * hz / 3;
        }
        // normalisation: int T d^2r = A  (trapezoid in r)
        double norm = 0;
        for (int ir = 1; ir < nr; ++ir) {
            const double r0 = (ir - 1) * dr, r1 = ir * dr;
            norm += 0.5 * (tab[ir - 1] * r0 + tab[ir] * r1) * dr;
        }
        norm *= 2 * M_PI;
        for (double &v : tab) v *= A / norm;
    }

    double operator()(double r) const {
        const double f = r / dr;
        const int i = (int)f;
        if (i >= (int)tab.size() - 1) return 0.0;
        const double w = f - i;
        return tab[i] + w * (tab[i + 1] - tab[i]);
    }
};

// splitmix64: counter-based stream, one per (seed, nucleus).
struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
};

void sample_nucleus(Rng &rng, int A, double R, double a, double xshift, std::vector<double> &x,
                    std::vector<double> &y) {
    const double rmax = R + 10 * a;
    for (int n = 0; n < A; ++n) {
        double r;
        for (;;) {  // rejection sampling of r^2 rho(r)
            r = rmax * rng.uniform();
            const double f = (r * r / (rmax * rmax)) / (1 + std::exp((r - R) / a));
            if (rng.uniform() < f) break;
        }
        const double cth = 2 * rng.uniform() - 1, phi = 2 * M_PI * rng.uniform();
        const double sth = std::sqrt(1 - cth * cth);
        x.push_back(r * sth * std::cos(phi) + xshift);
        y.push_back(r * sth * std::sin(phi));
    }
}

}  // namespace

extern "C" int vah_ic_optical_glauber(int nx, int ny, double dx, double dy, double b, double sigma_nn_fm2, int A,
                                      double ws_R, double ws_a, double x_coll, double e_peak, double e_floor,
                                      double *e_xy) {
    if (nx < 1 || ny < 1 || !e_xy || !(sigma_nn_fm2 > 0) || A < 1) return VAH_ERR_ARG;
    const Thickness T(A, ws_R, ws_a);
    double emax = 0;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const double x = (i - (nx - 1) / 2.) * dx, y = (j - (ny - 1) / 2.) * dy;
            const double ta = T(std::hypot(x - b / 2, y)), tb = T(std::hypot(x + b / 2, y));
            const double npart = ta * (1 - std::pow(1 - sigma_nn_fm2 * tb / A, A)) +
                                 tb * (1 - std::pow(1 - sigma_nn_fm2 * ta / A, A));
            const double ncoll = sigma_nn_fm2 * ta * tb;
            const double v = (1 - x_coll) * npart / 2 + x_coll * ncoll;
            e_xy[i + (size_t)nx * j] = v;
            if (v > emax) emax = v;
        }
    if (!(emax > 0)) return VAH_ERR_ARG;
    for (size_t s = 0; s < (size_t)nx * ny; ++s) e_xy[s] = e_peak * e_xy[s] / emax + e_floor;
    return VAH_OK;
}

namespace {

// Participant positions of one seeded MC-Glauber collision: nucleons drawn from
// the two Woods-Saxon nuclei displaced by +-b/2 along x; a nucleon
// participates if some nucleon of the other nucleus lies within
// sqrt(sigma_NN / pi) in the transverse plane.
void participants(double b, double sigma_nn_fm2, int A, double ws_R, double ws_a, unsigned long long seed,
                  std::vector<double> &px, std::vector<double> &py) {
    std::vector<double> xa, ya, xb, yb;
    Rng ra(seed * 2 + 0x1234567ull), rb(seed * 2 + 1 + 0x1234567ull);
    sample_nucleus(ra, A, ws_R, ws_a, +b / 2, xa, ya);
    sample_nucleus(rb, A, ws_R, ws_a, -b / 2, xb, yb);
    const double d2max = sigma_nn_fm2 / M_PI;
    std::vector<char> pa(A, 0), pb(A, 0);
    for (int m = 0; m < A; ++m)
        for (int n = 0; n < A; ++n) {
            const double ddx = xa[m] - xb[n], ddy = ya[m] - yb[n];
            if (ddx * ddx + ddy * ddy < d2max) pa[m] = pb[n] = 1;
        }
    px.clear();
    py.clear();
    for (int m = 0; m < A; ++m) if (pa[m]) { px.push_back(xa[m]); py.push_back(ya[m]); }
    for (int n = 0; n < A; ++n) if (pb[n]) { px.push_back(xb[n]); py.push_back(yb[n]); }
}

}  // namespace

extern "C" int vah_ic_mc_glauber_participants(double b, double sigma_nn_fm2, int A, double ws_R, double ws_a,
                                              unsigned long long seed, double *xy, int max, int *n_out) {
    if (!xy || !n_out || A < 1 || max < 0) return VAH_ERR_ARG;
    std::vector<double> px, py;
    participants(b, sigma_nn_fm2, A, ws_R, ws_a, seed, px, py);
    *n_out = (int)px.size();
    if ((int)px.size() > max) return VAH_ERR_TOO_LARGE;
    for (size_t p = 0; p < px.size(); ++p) {
        xy[2 * p] = px[p];
        xy[2 * p + 1] = py[p];
    }
    return VAH_OK;
}

extern "C" int vah_ic_mc_glauber(int nx, int ny, double dx, double dy, double b, double sigma_nn_fm2, int A,
                                 double ws_R, double ws_a, double width, unsigned long long seed, double e_peak,
                                 double e_floor, double *e_xy, int *npart_out) {
    if (nx < 1 || ny < 1 || !e_xy || !(width > 0) || A < 1) return VAH_ERR_ARG;
    std::vector<double> px, py;
    participants(b, sigma_nn_fm2, A, ws_R, ws_a, seed, px, py);
    if (npart_out) *npart_out = (int)px.size();
    const double inv2w2 = 1.0 / (2 * width * width), cut2 = 64 * width * width;
    double emax = 0;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const double x = (i - (nx - 1) / 2.) * dx, y = (j - (ny - 1) / 2.) * dy;
            double v = 0;
            for (size_t p = 0; p < px.size(); ++p) {
                const double r2 = (x - px[p]) * (x - px[p]) + (y - py[p]) * (y - py[p]);
                if (r2 < cut2) v += std::exp(-r2 * inv2w2);
            }
            e_xy[i + (size_t)nx * j] = v;
            if (v > emax) emax = v;
        }
    if (!(emax > 0)) {  // no collision: a flat floor
        for (size_t s = 0; s < (size_t)nx * ny; ++s) e_xy[s] = e_floor;
        return VAH_OK;
    }
    for (size_t s = 0; s < (size_t)nx * ny; ++s) e_xy[s] = e_peak * e_xy[s] / emax + e_floor;
    return VAH_OK;
}

extern "C" int vah_ic_longitudinal(int nz, double dz, double eta_flat, double sigma_eta, double *f_eta) {
    if (nz < 1 || !f_eta || !(sigma_eta > 0)) return VAH_ERR_ARG;
    for (int k = 0; k < nz; ++k) {
        const double eta = (k - (nz - 1) / 2.) * dz;
        const double d = std::fabs(eta) - eta_flat;
        f_eta[k] = d > 0 ? std::exp(-d * d / (2 * sigma_eta * sigma_eta)) : 1.0;
    }
    return VAH_OK;
}
