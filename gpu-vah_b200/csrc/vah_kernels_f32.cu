// vah_kernels_f32.cu -- the step kernels with FP32 state storage (FP64 arithmetic).
#include "vah_kernels_impl.cuh"

namespace vah {
VAH_INSTANTIATE(float)
}  // namespace vah
