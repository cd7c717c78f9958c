// vah_ic_device.cu -- initial energy densities on the GPU (vah_ic_device.cuh).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "vah_ic_device.cuh"

namespace vah {

namespace {

constexpr int kMaxA = 256;           // nucleons per nucleus the sampling block holds
constexpr long long kMaxDraws = 1 << 22;  // rejection-sampling draws per nucleus before the sampler gives up

// splitmix64, as the host generator (vah_ic.cpp)
__device__ __forceinline__ uint64_t sm_next(uint64_t &s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ double sm_uniform(uint64_t &s) { return (sm_next(s) >> 11) * (1.0 / 9007199254740992.0); }

// One block: thread 0 samples nucleus A, thread 1 nucleus B (rejection
// sampling of r^2 rho(r) on [0, R + 10 a], isotropic directions, shifted by
// +-b/2 along x), then every thread flags nucleons with a partner of the
// other nucleus within sqrt(sigma_NN / pi), and a scan writes the
// participants in order (A's, then B's). A nucleus that needs more than
// kMaxDraws draws in all (Au with R = 6.38, a = 0.535 fm takes about 4,000)
// stops the sampler within a fraction of a second: *np = -1.
__global__ void __launch_bounds__(512) participants_kernel(double b, double sigma, int A, double R, double a,
                                                           unsigned long long seed, double *pxy, int *np) {
    __shared__ double x[2][kMaxA], y[2][kMaxA];
    __shared__ int flag[2 * kMaxA], pos[2 * kMaxA];
    __shared__ int failed;
    const int tid = threadIdx.x;
    if (tid == 0) failed = 0;
    __syncthreads();
    if (tid < 2) {
        uint64_t s = seed * 2 + (unsigned long long)tid + 0x1234567ull;
        const double rmax = R + 10 * a, shift = tid == 0 ? +b / 2 : -b / 2;
        long long draws = 0;
        for (int n = 0; n < A; ++n) {
            double r = 0.0;
            bool hit = false;
            for (; draws < kMaxDraws && !hit; ++draws) {
                r = rmax * sm_uniform(s);
                const double f = (r * r / (rmax * rmax)) / (1 + exp((r - R) / a));
                hit = sm_uniform(s) < f;
            }
            if (!hit) {
                atomicExch(&failed, 1);
                break;
            }
            const double cth = 2 * sm_uniform(s) - 1, phi = 2 * M_PI * sm_uniform(s);
            const double sth = sqrt(1 - cth * cth);
            x[tid][n] = r * sth * cos(phi) + shift;
            y[tid][n] = r * sth * sin(phi);
        }
    }
    __syncthreads();
    if (failed) {
        if (tid == 0) *np = -1;
        return;
    }
    const double d2max = sigma / M_PI;
    for (int k = tid; k < 2 * A; k += blockDim.x) {
        const int nu = k < A ? 0 : 1, m = k < A ? k : k - A;
        int hit = 0;
        for (int n = 0; n < A && !hit; ++n) {
            const double ddx = x[nu][m] - x[1 - nu][n], ddy = y[nu][m] - y[1 - nu][n];
            hit = ddx * ddx + ddy * ddy < d2max;
        }
        flag[k] = hit;
    }
    __syncthreads();
    if (tid == 0) {  // scan of 2A flags (a few hundred)
        int c = 0;
        for (int k = 0; k < 2 * A; ++k) {
            pos[k] = c;
            c += flag[k];
        }
        *np = c;
    }
    __syncthreads();
    for (int k = tid; k < 2 * A; k += blockDim.x)
        if (flag[k]) {
            const int nu = k < A ? 0 : 1, m = k < A ? k : k - A;
            pxy[2 * pos[k]] = x[nu][m];
            pxy[2 * pos[k] + 1] = y[nu][m];
        }
}

__global__ void deposit_kernel(const double *__restrict__ pxy, const int *__restrict__ npp, double inv2w2,
                               double cut2, int nx, int ny, double dx, double dy, double *vxy,
                               unsigned long long *maxbits) {
    const int np = *npp;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nx * ny; c += gridDim.x * blockDim.x) {
        const int i = c % nx, j = c / nx;
        const double x = (i - (nx - 1) / 2.) * dx, y = (j - (ny - 1) / 2.) * dy;
        double v = 0;
        for (int p = 0; p < np; ++p) {
            const double rx = x - pxy[2 * p], ry = y - pxy[2 * p + 1];
            const double r2 = rx * rx + ry * ry;
            if (r2 < cut2) v += exp(-r2 * inv2w2);
        }
        vxy[c] = v;
        atomicMax(maxbits, (unsigned long long)__double_as_longlong(v));
    }
}

// T(r_k) = int rho dz over [-rmax, rmax] by Simpson with 2048 intervals, r_k =
// k rmax / (n - 1), rmax = R + 12 a (unnormalised; vah_ic.cpp's table).
__global__ void thickness_kernel(double R, double a, double *tab) {
    const int n = kThicknessPoints, nz = 2048;
    const double rmax = R + 12 * a, dr = rmax / (n - 1), hz = 2 * rmax / nz;
    for (int ir = blockIdx.x * blockDim.x + threadIdx.x; ir < n; ir += gridDim.x * blockDim.x) {
        const double r = ir * dr;
        double s = 0;
        for (int iz = 0; iz <= nz; ++iz) {
            const double z = -rmax + iz * hz;
            const double w = (iz == 0 || iz == nz) ? 1 : ((iz & 1) ? 4 : 2);
            s += w / (1 + exp((sqrt(r * r + z * z) - R) / a));
        }
        tab[ir] = s * hz / 3;
    }
}

// Normalisation int T d^2r = A (trapezoid in r, summed in order by one thread):
// tab[n] = A / norm.
__global__ void thickness_norm_kernel(double R, double a, int A, double *tab) {
    const int n = kThicknessPoints;
    const double dr = (R + 12 * a) / (n - 1);
    double norm = 0;
    for (int ir = 1; ir < n; ++ir) {
        const double r0 = (ir - 1) * dr, r1 = ir * dr;
        norm += 0.5 * (tab[ir - 1] * r0 + tab[ir] * r1) * dr;
    }
    norm *= 2 * M_PI;
    tab[n] = A / norm;
}

__device__ __forceinline__ double thickness_at(const double *tab, double dr, double r) {
    const double f = r / dr;
    const int i = (int)f;
    if (i >= kThicknessPoints - 1) return 0.0;
    const double w = f - i;
    return (tab[i] + w * (tab[i + 1] - tab[i])) * tab[kThicknessPoints];
}

__global__ void optical_kernel(const double *__restrict__ tab, double dr, int nx, int ny, double dx, double dy,
                               double b, double sigma, int A, double x_coll, double *vxy,
                               unsigned long long *maxbits) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nx * ny; c += gridDim.x * blockDim.x) {
        const int i = c % nx, j = c / nx;
        const double x = (i - (nx - 1) / 2.) * dx, y = (j - (ny - 1) / 2.) * dy;
        const double ta = thickness_at(tab, dr, hypot(x - b / 2, y)), tb = thickness_at(tab, dr, hypot(x + b / 2, y));
        const double npart = ta * (1 - pow(1 - sigma * tb / A, A)) + tb * (1 - pow(1 - sigma * ta / A, A));
        const double ncoll = sigma * ta * tb;
        const double v = (1 - x_coll) * npart / 2 + x_coll * ncoll;
        vxy[c] = v;
        atomicMax(maxbits, (unsigned long long)__double_as_longlong(v > 0 ? v : 0.0));
    }
}

template <typename S>
__global__ void fill_kernel(const double *__restrict__ vxy, const unsigned long long *__restrict__ maxbits, int nx,
                            int ny, int nz, int pitch, double dz, double eta_flat, double sigma_eta, double e_peak,
                            double e_floor, S *e) {
    const double vmax = __longlong_as_double((long long)*maxbits);
    const long long n = (long long)nx * ny * nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const long long t = c % ((long long)nx * ny);
        const int k = (int)(c / ((long long)nx * ny)), i = (int)(t % nx), j = (int)(t / nx);
        const double exy = vmax > 0 ? e_peak * vxy[t] / vmax : 0.0;
        double f = 1.0;
        if (nz > 1) {
            const double d = fabs((k - (nz - 1) / 2.) * dz) - eta_flat;
            if (d > 0) f = exp(-d * d / (2 * sigma_eta * sigma_eta));
        }
        e[(i + 2) + (long long)pitch * ((j + 2) + (long long)(ny + 4) * (k + 2))] = (S)(exy * f + e_floor);
    }
}

int grid_of(long long n, int block) {
    long long g = (n + block - 1) / block;
    return (int)(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

}  // namespace

cudaError_t ic_participants_device(double b, double sigma_nn_fm2, int A, double ws_R, double ws_a,
                                   unsigned long long seed, double *d_pxy, int *d_np, cudaStream_t stream) {
    if (A < 1 || A > kMaxA || !(ws_R > 0) || !(ws_a > 0) || !std::isfinite(ws_R + ws_a + b + sigma_nn_fm2))
        return cudaErrorInvalidValue;
    participants_kernel<<<1, 512, 0, stream>>>(b, sigma_nn_fm2, A, ws_R, ws_a, seed, d_pxy, d_np);
    return cudaGetLastError();
}

cudaError_t ic_deposit_device(const double *d_pxy, const int *d_np, double width, int nx, int ny, double dx,
                              double dy, double *d_v, unsigned long long *maxbits, cudaStream_t stream) {
    deposit_kernel<<<grid_of((long long)nx * ny, 128), 128, 0, stream>>>(
        d_pxy, d_np, 1.0 / (2 * width * width), 64 * width * width, nx, ny, dx, dy, d_v, maxbits);
    return cudaGetLastError();
}

cudaError_t ic_optical_device(int nx, int ny, double dx, double dy, double b, double sigma_nn_fm2, int A,
                              double ws_R, double ws_a, double x_coll, double *d_tab, double *d_v,
                              unsigned long long *maxbits, cudaStream_t stream) {
    thickness_kernel<<<kThicknessPoints / 128, 128, 0, stream>>>(ws_R, ws_a, d_tab);
    thickness_norm_kernel<<<1, 1, 0, stream>>>(ws_R, ws_a, A, d_tab);
    const double dr = (ws_R + 12 * ws_a) / (kThicknessPoints - 1);
    optical_kernel<<<grid_of((long long)nx * ny, 128), 128, 0, stream>>>(d_tab, dr, nx, ny, dx, dy, b, sigma_nn_fm2,
                                                                         A, x_coll, d_v, maxbits);
    return cudaGetLastError();
}

template <typename S>
cudaError_t ic_fill_device(const double *d_v, const unsigned long long *maxbits, int nx, int ny, int nz, int pitch,
                           double dz, double eta_flat, double sigma_eta, double e_peak, double e_floor, S *e,
                           cudaStream_t stream) {
    fill_kernel<S><<<grid_of((long long)nx * ny * nz, 128), 128, 0, stream>>>(
        d_v, maxbits, nx, ny, nz, pitch, dz, eta_flat, sigma_eta, e_peak, e_floor, e);
    return cudaGetLastError();
}

template cudaError_t ic_fill_device<double>(const double *, const unsigned long long *, int, int, int, int, double,
                                            double, double, double, double, double *, cudaStream_t);
template cudaError_t ic_fill_device<float>(const double *, const unsigned long long *, int, int, int, int, double,
                                           double, double, double, double, float *, cudaStream_t);

}  // namespace vah
