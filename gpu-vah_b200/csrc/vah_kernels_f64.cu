// vah_kernels_f64.cu -- the step kernels with FP64 state storage.
#include "vah_kernels_impl.cuh"

namespace vah {
VAH_INSTANTIATE(double)
}  // namespace vah
