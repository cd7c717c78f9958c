// vah_kernels_impl.cuh -- CUDA kernels of the VAH time step (sm_100a) and
// their launch dispatch. Compiled once per storage type by vah_kernels_f64.cu
// and vah_kernels_f32.cu (separate translation units build in parallel).
//
// stage_kernel: one thread per interior cell runs the whole RK stage of that
// cell (vah_stage.cuh). face_kernel + cell_kernel: the same stage split into
// per-axis face launches and one cell launch (the default path).
// The step is FP64-arithmetic-bound (13 Newton inversions per cell and stage
// in the reference-faithful flux mode), so launches favour occupancy:
// 128-thread blocks, x fastest so that every load of a field is a coalesced
// row. The split kernels come in register-cap variants (MINB = the minimum
// number of resident 128-thread blocks per SM the compiler must allow) and
// take their block shape at run time; the autotuner picks both per launch
// kind by timing them on the event's own state.
#pragma once

#include "vah_kernels.cuh"

namespace vah {

namespace {

constexpr int kBX = 32, kBY = 4;  // fused stage kernel shape

// Row blocks beyond the grid's y limit (65535) continue along z.
constexpr unsigned kMaxGridY = 65535;

__device__ __forceinline__ int row_block() { return (int)(blockIdx.z * gridDim.y + blockIdx.y); }

dim3 row_grid(long long cols, long long rows, int bx, int by) {
    const unsigned gy = (unsigned)((rows + by - 1) / by);
    const unsigned gz = (gy + kMaxGridY - 1) / kMaxGridY;
    return dim3((unsigned)((cols + bx - 1) / bx), gz > 1 ? kMaxGridY : gy, gz > 1 ? gz : 1);
}

template <typename S, int PHYS, bool IS3D>
__global__ void __launch_bounds__(kBX *kBY) stage_kernel(const StageArgs<S> a) {
    const int i = blockIdx.x * kBX + threadIdx.x;
    const int r = row_block() * kBY + threadIdx.y;  // row index over (j, k)
    if (i >= a.nx || r >= a.ny * a.nz) return;
    const int j = r % a.ny, k = r / a.ny;
    stage_cell<S, PHYS, IS3D>(a, i + 2, j + 2, k + 2);
}

// Faces at +1/2 of the ghosted cells along DIR that bound an interior cell
// of the planes [k0, k1): left cell index 1 .. n along DIR (ghost layer 1
// included), interior across.
template <typename S, int PHYS, int DIR, bool EXACT, int MINB>
__global__ void __launch_bounds__(kSplitThreads, MINB) face_kernel(const StageArgs<S> a) {
    const int ext0 = DIR == 0 ? a.nx + 1 : a.nx;
    const int ext1 = DIR == 1 ? a.ny + 1 : a.ny;
    const int ext2 = DIR == 2 ? a.k1 - a.k0 + 1 : a.k1 - a.k0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = row_block() * blockDim.y + threadIdx.y;
    if (i >= ext0 || r >= ext1 * ext2) return;
    const int j = r % ext1, k = r / ext1 + a.k0;
    const int gi = i + (DIR == 0 ? 1 : 2), gj = j + (DIR == 1 ? 1 : 2), gk = k + (DIR == 2 ? 1 : 2);
    const long long st = DIR == 0 ? 1 : (DIR == 1 ? (long long)a.ncx : a.plane);
    const long long s = gi + (long long)a.ncx * gj + a.plane * gk;
    const int gl = DIR == 0 ? gi : (DIR == 1 ? gj : gk), n = DIR == 0 ? a.nx : (DIR == 1 ? a.ny : a.nz);
    const unsigned fails = face_compute<S, PHYS, EXACT>(a, s, DIR, st, gl >= 2, gl <= n);
    if (a.counters) {
        if (fails & 255u) count_add(a.counters + 0, fails & 255u);
        if (fails >> 8) count_add(a.counters + 2, 1ull);
    }
}

// Faces along x with the x flux differences taken in the launch (a.Dx set):
// blocks of 32 x 4 threads, one warp per row segment. Lane L of warp w in its
// row takes the face at +1/2 of ghosted cell f + 1, f = 31 w + L, so that
// consecutive warps share one face. Each face is evaluated as in face_kernel,
// but only the two evaluations' weights are kept, and each field's two fluxes
// are formed at the exchange: lane L >= 1 owns cell f + 1 (when interior) and
// writes Dx = H(-1/2) - H(+1/2) as that cell evaluates them, the -1/2 value
// from lane L - 1 through a shuffle. The face a warp shares with the previous
// one is evaluated twice and counted once.
template <typename S, int PHYS, bool EXACT, int MINB>
__global__ void __launch_bounds__(kSplitThreads, MINB) face_x_diff_kernel(const StageArgs<S> a) {
    constexpr int NQ = Phys<PHYS>::NQ;
    const int lane = threadIdx.x;  // blockDim.x == 32: a warp is one row segment
    const int r = row_block() * blockDim.y + threadIdx.y;
    if (r >= a.ny * (a.k1 - a.k0)) return;  // whole warps
    const int j = r % a.ny, k = r / a.ny + a.k0;
    const int gi = 31 * blockIdx.x + lane + 1;  // the face at +1/2 of ghosted cell gi
    const bool act = gi <= a.nx + 1;            // faces 1 .. nx + 1 bound the interior cells
    const long long s = gi + (long long)a.ncx * (j + 2) + a.plane * (k + 2);
    double qR[NQ], qL[NQ];
    double wRo = 0.0, wLo = 0.0, wRr = 0.0, wLr = 0.0;  // the left cell's evaluation, the right cell's
    unsigned fails = 0;
    if (act) {
        face_states<S, PHYS>(a, s, 1, qR, qL);
        InvSetup sR, sL;
        invert_setup<PHYS>(a.t_src, qR, sR);
        invert_setup<PHYS>(a.t_src, qL, sL);
        if (!EXACT || gi >= 2) {
            const double ux = ld(a.uin[1], s), uy = ld(a.uin[2], s);
            fails += face_weights(sR, sL, 0, ld(a.ein, s), sqrt(fabs(ux * ux + uy * uy)), wRo, wLo);
        }
        if (EXACT && gi <= a.nx) {
            const double vx = ld(a.uin[1], s + 1), vy = ld(a.uin[2], s + 1);
            fails += face_weights(sR, sL, 0, ld(a.ein, s + 1), sqrt(fabs(vx * vx + vy * vy)), wRr, wLr);
        }
    } else {
#pragma unroll
        for (int n = 0; n < NQ; ++n) qR[n] = qL[n] = 0.0;
    }
    const bool own = act && lane >= 1 && gi >= 2;  // cell gi is interior, and lane - 1 holds its -1/2 face
#pragma unroll
    for (int n = 0; n < NQ; ++n) {
        const double h = wRo * qR[n] + wLo * qL[n];                 // +1/2 as cell gi evaluates it
        const double hr = EXACT ? wRr * qR[n] + wLr * qL[n] : h;   // +1/2 as cell gi + 1 evaluates it
        const double hm = __shfl_up_sync(0xffffffffu, hr, 1);
        if (own) a.Dx[n][s] = (S)(hm - h);
    }
    if (a.counters && act && (lane >= 1 || blockIdx.x == 0)) {
        if (fails & 255u) count_add(a.counters + 0, fails & 255u);
        if (fails >> 8) count_add(a.counters + 2, 1ull);
    }
}

template <typename S, int PHYS, bool IS3D, bool EXACT, int MINB>
__global__ void __launch_bounds__(kSplitThreads, MINB) cell_kernel(const StageArgs<S> a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = row_block() * blockDim.y + threadIdx.y;
    if (i >= a.nx || r >= a.ny * (a.k1 - a.k0)) return;
    const int j = r % a.ny, k = r / a.ny + a.k0;
    cell_compute<S, PHYS, IS3D, EXACT>(a, i + 2, j + 2, k + 2);
}

template <typename S, int PHYS>
__global__ void validity_kernel(const ValidityArgs<S> a) {
    const long long n = (long long)a.nx * a.ny * a.nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % a.nx), j = (int)((c / a.nx) % a.ny), k = (int)(c / ((long long)a.nx * a.ny));
        validity_cell<S, PHYS>(a, (i + 2) + (long long)a.ncx * (j + 2) + a.plane * (k + 2));
    }
}

template <typename S, int PHYS>
__global__ void set_conserved_kernel(const FieldSet<S> q, const FieldSet<S> u, const FieldSet<S> up, const S *e,
                                     int nx, int ny, int nz, int pitch, double t, int pl_from_field) {
    const long long n = (long long)nx * ny * nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((long long)nx * ny));
        const long long s = (i + 2) + (long long)pitch * ((j + 2) + (long long)(ny + 4) * (k + 2));
        set_conserved_cell<S, PHYS>(q.f, u.f, up.f, e, t, pl_from_field, s);
    }
}

template <typename S>
__global__ void init_primitives_kernel(const FieldSet<S> q, const FieldSet<S> u, const S *e, S *p, const Eos eos,
                                       int nx, int ny, int nz, int pitch) {
    const long long n = (long long)nx * ny * nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((long long)nx * ny));
        const long long s = (i + 2) + (long long)pitch * ((j + 2) + (long long)(ny + 4) * (k + 2));
        const double pv = eos_pressure(eos, (double)e[s]);
        p[s] = (S)pv;
        u.f[0][s] = (S)1.0;
        u.f[1][s] = u.f[2][s] = u.f[3][s] = (S)0.0;
        for (int m = 5; m < 16; ++m)
            if (q.f[m]) q.f[m][s] = (S)0.0;
        q.f[kSlotPL][s] = (S)pv;
    }
}

// Pass 0 (I): j in [2, ncy), k in [2, ncz): i = 0,1 <- 2; i = nx+2, nx+3 <- nx+1.
// Pass 1 (J): i in [2, ncx), k in [2, ncz).  Pass 2 (K): i in [2, ncx), j in [2, ncy).
template <typename S>
__global__ void ghost_kernel(const FieldSet<S> f, int nx, int ny, int nz, int pitch, int pass) {
    const int ncx = nx + 4, ncy = ny + 4, ncz = nz + 4;
    const long long plane = (long long)pitch * ncy;
    int na, nb;
    if (pass == 0) { na = ncy - 2; nb = ncz - 2; }
    else if (pass == 1) { na = ncx - 2; nb = ncz - 2; }
    else { na = ncx - 2; nb = ncy - 2; }
    const long long n = (long long)na * nb * 4;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const int slot = (int)(c & 3);
        const long long ab = c >> 2;
        const int A = (int)(ab % na) + 2, B = (int)(ab / na) + 2;
        long long s, sb;
        if (pass == 0) {
            int gi = slot < 2 ? slot : nx + slot, bi = slot < 2 ? 2 : nx + 1;
            s = gi + (long long)pitch * A + plane * B;
            sb = bi + (long long)pitch * A + plane * B;
        } else if (pass == 1) {
            int gj = slot < 2 ? slot : ny + slot, bj = slot < 2 ? 2 : ny + 1;
            s = A + (long long)pitch * gj + plane * B;
            sb = A + (long long)pitch * bj + plane * B;
        } else {
            int gk = slot < 2 ? slot : nz + slot, bk = slot < 2 ? 2 : nz + 1;
            s = A + (long long)pitch * B + plane * gk;
            sb = A + (long long)pitch * B + plane * bk;
        }
        for (int m = 0; m < f.n; ++m) f.f[m][s] = f.f[m][sb];
    }
}

template <typename S, int PHYS>
cudaError_t stage_dispatch(const StageArgs<S> &a, cudaStream_t stream) {
    dim3 block(kBX, kBY);
    const dim3 grid = row_grid(a.nx, (long long)a.ny * a.nz, kBX, kBY);
    if (a.nz > 1)
        stage_kernel<S, PHYS, true><<<grid, block, 0, stream>>>(a);
    else
        stage_kernel<S, PHYS, false><<<grid, block, 0, stream>>>(a);
    return cudaGetLastError();
}

// One launch of a split kernel kind with the given shape and register-cap variant.
template <typename S, int PHYS, bool EXACT, int DIR>
cudaError_t face_launch(const StageArgs<S> &a, const KindConfig &c, cudaStream_t stream) {
    const int ext0 = DIR == 0 ? a.nx + 1 : a.nx;
    const int rows = (DIR == 1 ? a.ny + 1 : a.ny) * (DIR == 2 ? a.k1 - a.k0 + 1 : a.k1 - a.k0);
    const dim3 block(c.bx, c.by), grid = row_grid(ext0, rows, c.bx, c.by);
    switch (c.minb) {
    case 3: face_kernel<S, PHYS, DIR, EXACT, 3><<<grid, block, 0, stream>>>(a); break;
    case 4: face_kernel<S, PHYS, DIR, EXACT, 4><<<grid, block, 0, stream>>>(a); break;
    case 5: face_kernel<S, PHYS, DIR, EXACT, 5><<<grid, block, 0, stream>>>(a); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// The x face launch that also differences (a.Dx set): 32 x 4 blocks whatever
// the tuned shape (a warp must be one row segment); the register cap as tuned.
template <typename S, int PHYS, bool EXACT>
cudaError_t face_x_diff_launch(const StageArgs<S> &a, const KindConfig &c, cudaStream_t stream) {
    const int rows = a.ny * (a.k1 - a.k0);
    const dim3 block(32, kSplitThreads / 32), grid = row_grid((a.nx + 30) / 31, rows, 1, kSplitThreads / 32);
    switch (c.minb) {
    case 3: face_x_diff_kernel<S, PHYS, EXACT, 3><<<grid, block, 0, stream>>>(a); break;
    case 4: face_x_diff_kernel<S, PHYS, EXACT, 4><<<grid, block, 0, stream>>>(a); break;
    case 5: face_x_diff_kernel<S, PHYS, EXACT, 5><<<grid, block, 0, stream>>>(a); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename S, int PHYS, bool EXACT, bool IS3D>
cudaError_t cell_launch(const StageArgs<S> &a, const KindConfig &c, cudaStream_t stream) {
    const dim3 block(c.bx, c.by), grid = row_grid(a.nx, (long long)a.ny * (a.k1 - a.k0), c.bx, c.by);
    switch (c.minb) {
    case 2: cell_kernel<S, PHYS, IS3D, EXACT, 2><<<grid, block, 0, stream>>>(a); break;
    case 3: cell_kernel<S, PHYS, IS3D, EXACT, 3><<<grid, block, 0, stream>>>(a); break;
    case 4: cell_kernel<S, PHYS, IS3D, EXACT, 4><<<grid, block, 0, stream>>>(a); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename S, int PHYS, bool EXACT>
cudaError_t split_kind_dispatch(const StageArgs<S> &a, int kind, const KindConfig &c, cudaStream_t stream) {
    if (a.k0 < 0 || a.k1 > a.nz || a.k0 > a.k1) return cudaErrorInvalidValue;
    if (a.k0 == a.k1) return cudaSuccess;  // no planes
    switch (kind) {
    case kFaceX: return a.Dx[0] ? face_x_diff_launch<S, PHYS, EXACT>(a, c, stream) : face_launch<S, PHYS, EXACT, 0>(a, c, stream);
    case kFaceY: return face_launch<S, PHYS, EXACT, 1>(a, c, stream);
    case kFaceZ: return a.nz > 1 ? face_launch<S, PHYS, EXACT, 2>(a, c, stream) : cudaSuccess;
    case kCell:
        return a.nz > 1 ? cell_launch<S, PHYS, EXACT, true>(a, c, stream) : cell_launch<S, PHYS, EXACT, false>(a, c, stream);
    default: return cudaErrorInvalidValue;
    }
}

int grid_for(long long n, int block) {
    long long g = (n + block - 1) / block;
    if (g > 148 * 64) g = 148 * 64;
    if (g < 1) g = 1;
    return (int)g;
}

}  // namespace

template <typename S>
cudaError_t launch_stage(const StageArgs<S> &a, int physics, cudaStream_t stream) {
    switch (physics) {
    case kIdeal: return stage_dispatch<S, kIdeal>(a, stream);
    case kPimunu: return stage_dispatch<S, kPimunu>(a, stream);
    case kPimunuPi: return stage_dispatch<S, kPimunuPi>(a, stream);
    default: return cudaErrorInvalidValue;
    }
}

template <typename S>
cudaError_t launch_split_kind(const StageArgs<S> &a, int physics, bool exact, int kind, const KindConfig &c,
                              cudaStream_t stream) {
    if (!valid_kind_config(kind, c)) return cudaErrorInvalidValue;
    switch (physics) {
    case kIdeal:
        return exact ? split_kind_dispatch<S, kIdeal, true>(a, kind, c, stream)
                     : split_kind_dispatch<S, kIdeal, false>(a, kind, c, stream);
    case kPimunu:
        return exact ? split_kind_dispatch<S, kPimunu, true>(a, kind, c, stream)
                     : split_kind_dispatch<S, kPimunu, false>(a, kind, c, stream);
    case kPimunuPi:
        return exact ? split_kind_dispatch<S, kPimunuPi, true>(a, kind, c, stream)
                     : split_kind_dispatch<S, kPimunuPi, false>(a, kind, c, stream);
    default: return cudaErrorInvalidValue;
    }
}

template <typename S>
cudaError_t launch_stage_split(const StageArgs<S> &a, int physics, bool exact, const SplitConfig &c,
                               cudaStream_t stream) {
    for (int kind = 0; kind < kNumSplitKinds; ++kind) {
        const cudaError_t e = launch_split_kind<S>(a, physics, exact, kind, c.k[kind], stream);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <typename S>
cudaError_t launch_stage_split(const StageArgs<S> &a, int physics, bool exact, cudaStream_t stream) {
    return launch_stage_split<S>(a, physics, exact, default_split_config(), stream);
}

template <typename S>
cudaError_t launch_validity(const ValidityArgs<S> &a, int physics, cudaStream_t stream) {
    const int block = 128, grid = grid_for((long long)a.nx * a.ny * a.nz, block);
    switch (physics) {
    case kIdeal: validity_kernel<S, kIdeal><<<grid, block, 0, stream>>>(a); break;
    case kPimunu: validity_kernel<S, kPimunu><<<grid, block, 0, stream>>>(a); break;
    case kPimunuPi: validity_kernel<S, kPimunuPi><<<grid, block, 0, stream>>>(a); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename S>
cudaError_t launch_set_conserved(const FieldSet<S> &q, const FieldSet<S> &u, const FieldSet<S> &up, const S *e,
                                 int physics, int nx, int ny, int nz, int pitch, double t, int pl_from_field,
                                 cudaStream_t stream) {
    const int block = 256;
    const int grid = grid_for((long long)nx * ny * nz, block);
    switch (physics) {
    case kIdeal: set_conserved_kernel<S, kIdeal><<<grid, block, 0, stream>>>(q, u, up, e, nx, ny, nz, pitch, t, pl_from_field); break;
    case kPimunu: set_conserved_kernel<S, kPimunu><<<grid, block, 0, stream>>>(q, u, up, e, nx, ny, nz, pitch, t, pl_from_field); break;
    case kPimunuPi: set_conserved_kernel<S, kPimunuPi><<<grid, block, 0, stream>>>(q, u, up, e, nx, ny, nz, pitch, t, pl_from_field); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename S>
cudaError_t launch_init_primitives(const FieldSet<S> &q, const FieldSet<S> &u, const S *e, S *p, const Eos &eos,
                                   int nx, int ny, int nz, int pitch, cudaStream_t stream) {
    const int block = 256;
    init_primitives_kernel<S><<<grid_for((long long)nx * ny * nz, block), block, 0, stream>>>(q, u, e, p, eos, nx, ny,
                                                                                                nz, pitch);
    return cudaGetLastError();
}

template <typename S>
cudaError_t launch_ghosts(const FieldSet<S> &fields, int nx, int ny, int nz, int pitch, cudaStream_t stream) {
    const int block = 256;
    for (int pass = 0; pass < 3; ++pass) {
        long long n;
        if (pass == 0) n = (long long)ny * nz;
        else if (pass == 1) n = (long long)nx * nz;
        else n = (long long)nx * ny;
        n = (n + 4LL * (nx + ny + nz) + 16) * 4;  // the passes also sweep upper ghost rows
        ghost_kernel<S><<<grid_for(n, block), block, 0, stream>>>(fields, nx, ny, nz, pitch, pass);
        cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess) return err;
    }
    return cudaSuccess;
}

// One pass of the ghost fill (0: x, 1: y, 2: eta), as launch_ghosts runs it.
template <typename S>
cudaError_t launch_ghost_pass(const FieldSet<S> &fields, int nx, int ny, int nz, int pitch, int pass,
                              cudaStream_t stream) {
    const int block = 256;
    long long n = pass == 0 ? (long long)ny * nz : (pass == 1 ? (long long)nx * nz : (long long)nx * ny);
    n = (n + 4LL * (nx + ny + nz) + 16) * 4;
    ghost_kernel<S><<<grid_for(n, block), block, 0, stream>>>(fields, nx, ny, nz, pitch, pass);
    return cudaGetLastError();
}

#define VAH_INSTANTIATE(S)                                                                                      \
    template cudaError_t launch_stage<S>(const StageArgs<S> &, int, cudaStream_t);                              \
    template cudaError_t launch_validity<S>(const ValidityArgs<S> &, int, cudaStream_t);                        \
    template cudaError_t launch_split_kind<S>(const StageArgs<S> &, int, bool, int, const KindConfig &,         \
                                              cudaStream_t);                                                    \
    template cudaError_t launch_stage_split<S>(const StageArgs<S> &, int, bool, const SplitConfig &,            \
                                               cudaStream_t);                                                   \
    template cudaError_t launch_stage_split<S>(const StageArgs<S> &, int, bool, cudaStream_t);                  \
    template cudaError_t launch_set_conserved<S>(const FieldSet<S> &, const FieldSet<S> &, const FieldSet<S> &, \
                                                 const S *, int, int, int, int, int, double, int, cudaStream_t); \
    template cudaError_t launch_init_primitives<S>(const FieldSet<S> &, const FieldSet<S> &, const S *, S *,    \
                                                   const Eos &, int, int, int, int, cudaStream_t);             \
    template cudaError_t launch_ghosts<S>(const FieldSet<S> &, int, int, int, int, cudaStream_t);              \
    template cudaError_t launch_ghost_pass<S>(const FieldSet<S> &, int, int, int, int, int, cudaStream_t);

}  // namespace vah
