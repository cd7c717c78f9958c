// vah_powf_exc.h -- inputs on which the host libm's powf(x, 0.25f) is not the
// correctly rounded fourth root.
#pragma once

#include <cstdint>
#include <vector>

namespace vah {

// Sorted (input bits, powf result bits) pairs, flattened, for single-precision
// inputs in [2^-40, 2^24); computed once per process on first use.
const std::vector<uint32_t> &powf_quarter_exceptions();

}  // namespace vah
