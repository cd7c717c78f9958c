// vah_tile.cu -- launch side of the TMA-tiled FP32 stage (vah_tile.cuh):
// tensor maps, tile work-lists, the persistent launch.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "vah.h"
#include "vah_tile.cuh"

namespace vah {

namespace {

using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        void *p = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    });
    return fn;
}

template <int PHYS, bool IS3D>
cudaError_t launch_t(const TileSlot *slots, const TileClock *clk, const TileClock &clk0, double dt0,
                     const TileItem *items, int nitems, unsigned *counter, int stage, const Eos &eos, unsigned *err,
                     cudaStream_t stream) {
    using SM = TileSmem<PHYS, IS3D>;
    static int grid_max = 0;  // SMs x resident blocks, found once per instantiation
    if (!grid_max) {
        cudaError_t e = cudaFuncSetAttribute(tile_kernel<PHYS, IS3D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)SM::bytes);
        if (e != cudaSuccess) return e;
        int dev = 0, sms = 0, per = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, tile_kernel<PHYS, IS3D>, kTileThreads,
                                                               SM::bytes)) != cudaSuccess)
            return e;
        grid_max = std::max(1, sms * std::max(per, 1));
    }
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess) return e;
    const int grid = std::min(nitems, grid_max);
    tile_kernel<PHYS, IS3D><<<grid, kTileThreads, SM::bytes, stream>>>(slots, clk, clk0, dt0, items, nitems,
                                                                         counter, stage, eos, err);
    return cudaGetLastError();
}

}  // namespace

int tile_encode_q(CUtensorMap *tm, const float *base, int nx, int ny, int nz, int pitch, long long fstride, int nq) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return VAH_ERR_NODEVICE;
    const bool is3d = nz > 1;
    const int ncy = ny + 4, ncz = nz + 4;
    if (pitch % 4 || fstride % 4 || ((uintptr_t)base & 15)) return VAH_ERR_ARG;
    const cuuint64_t dims[4] = {(cuuint64_t)(nx + 4), (cuuint64_t)ncy, (cuuint64_t)ncz, (cuuint64_t)nq};
    const cuuint64_t strides[3] = {(cuuint64_t)pitch * 4, (cuuint64_t)pitch * ncy * 4, (cuuint64_t)fstride * 4};
    cuuint32_t box[4];
    if (is3d) {
        box[0] = TileShape<true>::BX;
        box[1] = TileShape<true>::BY;
        box[2] = TileShape<true>::BZ;
    } else {
        box[0] = TileShape<false>::BX;
        box[1] = TileShape<false>::BY;
        box[2] = TileShape<false>::BZ;
    }
    box[3] = (cuuint32_t)nq;
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = fn(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void *)base, dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? VAH_OK : VAH_ERR_CUDA;
}

int tile_encode_p(CUtensorMap *tm, const float *base, int nx, int ny, int nz, int pitch, long long fstride, int nf) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return VAH_ERR_NODEVICE;
    const bool is3d = nz > 1;
    const int ncy = ny + 4, ncz = nz + 4;
    if (pitch % 4 || fstride % 4 || ((uintptr_t)base & 15)) return VAH_ERR_ARG;
    const cuuint64_t dims[4] = {(cuuint64_t)(nx + 4), (cuuint64_t)ncy, (cuuint64_t)ncz, (cuuint64_t)nf};
    const cuuint64_t strides[3] = {(cuuint64_t)pitch * 4, (cuuint64_t)pitch * ncy * 4, (cuuint64_t)fstride * 4};
    cuuint32_t box[4];
    if (is3d) {
        box[0] = TileShape<true>::PBX;
        box[1] = TileShape<true>::PBY;
        box[2] = TileShape<true>::PBZ;
    } else {
        box[0] = TileShape<false>::PBX;
        box[1] = TileShape<false>::PBY;
        box[2] = TileShape<false>::PBZ;
    }
    box[3] = (cuuint32_t)nf;
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = fn(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void *)base, dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? VAH_OK : VAH_ERR_CUDA;
}

void tile_items(std::vector<TileItem> &out, int slot, int nx, int ny, int nz) {
    const bool is3d = nz > 1;
    const int tx = is3d ? TileShape<true>::TX : TileShape<false>::TX;
    const int ty = is3d ? TileShape<true>::TY : TileShape<false>::TY;
    const int tz = is3d ? TileShape<true>::TZ : TileShape<false>::TZ;
    for (int k0 = 0; k0 < nz; k0 += tz)
        for (int j0 = 0; j0 < ny; j0 += ty)
            for (int i0 = 0; i0 < nx; i0 += tx) out.push_back({slot, i0, j0, k0});
}

cudaError_t tile_launch(const TileSlot *slots, const TileClock *clk, const TileClock &clk0, double dt0,
                        const TileItem *items, int nitems, bool is3d, unsigned *counter, int stage, int physics,
                        const Eos &eos, unsigned *err, cudaStream_t stream) {
    if (nitems <= 0) return cudaSuccess;
    switch (physics * 2 + (is3d ? 1 : 0)) {
    case 0: return launch_t<kIdeal, false>(slots, clk, clk0, dt0, items, nitems, counter, stage, eos, err, stream);
    case 1: return launch_t<kIdeal, true>(slots, clk, clk0, dt0, items, nitems, counter, stage, eos, err, stream);
    case 2: return launch_t<kPimunu, false>(slots, clk, clk0, dt0, items, nitems, counter, stage, eos, err, stream);
    case 3: return launch_t<kPimunu, true>(slots, clk, clk0, dt0, items, nitems, counter, stage, eos, err, stream);
    case 4: return launch_t<kPimunuPi, false>(slots, clk, clk0, dt0, items, nitems, counter, stage, eos, err, stream);
    case 5: return launch_t<kPimunuPi, true>(slots, clk, clk0, dt0, items, nitems, counter, stage, eos, err, stream);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace vah
