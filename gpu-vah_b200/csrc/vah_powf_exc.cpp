// vah_powf_exc.cpp -- where the reference's conformal temperature rounds
// differently from a correctly rounded fourth root.
//
// The reference evaluates T = powf(e/13.8997, 0.25) in single precision
// (rhic/src/EquationOfState.cpp:144). The host libm's powf is not correctly
// rounded: for about 0.06% of inputs it returns the neighbour of the nearest
// single. A one-ulp temperature difference moves P_L by ~1e-9 relative within
// a few hundred steps of the conformal 2+1D workload, so the device reproduces
// the host libm exactly: it rounds the double-precision fourth root once (the
// correctly rounded value) and, for the inputs listed here, substitutes the
// libm result. The list is measured by calling the host libm on every single
// in [2^-40, 2^24) -- e/13.8997 from 1e-12 to 1.7e7 fm^-4 -- split over
// threads; outside that range the device keeps the correctly rounded value.
#include "vah_powf_exc.h"

#include <cmath>
#include <cstring>
#include <mutex>
#include <thread>

namespace vah {

namespace {

uint32_t bits_of(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    return u;
}

float float_of(uint32_t u) {
    float x;
    std::memcpy(&x, &u, 4);
    return x;
}

// powf through a volatile function pointer so the compiler cannot fold or
// substitute it: this must be the same library call the reference makes.
float (*volatile g_powf)(float, float) = powf;

void scan(uint32_t lo, uint32_t hi, std::vector<uint32_t> *out) {
    for (uint32_t u = lo; u < hi; ++u) {
        const float x = float_of(u);
        const float ref = g_powf(x, 0.25f);
        const float cr = (float)std::sqrt(std::sqrt((double)x));
        if (bits_of(ref) != bits_of(cr)) {
            out->push_back(u);
            out->push_back(bits_of(ref));
        }
    }
}

}  // namespace

const std::vector<uint32_t> &powf_quarter_exceptions() {
    static std::vector<uint32_t> table;
    static std::once_flag once;
    std::call_once(once, [] {
        const uint32_t lo = bits_of(std::ldexp(1.0f, -40)), hi = bits_of(std::ldexp(1.0f, 24));
        unsigned nt = std::thread::hardware_concurrency();
        if (nt == 0) nt = 4;
        if (nt > 64) nt = 64;
        std::vector<std::vector<uint32_t>> parts(nt);
        std::vector<std::thread> th;
        const uint32_t span = (hi - lo + nt - 1) / nt;
        for (unsigned k = 0; k < nt; ++k) {
            uint32_t a = lo + k * span, b = a + span;
            if (b > hi || b < a) b = hi;
            if (a >= hi) break;
            th.emplace_back(scan, a, b, &parts[k]);
        }
        for (auto &t : th) t.join();
        for (auto &p : parts) table.insert(table.end(), p.begin(), p.end());
    });
    return table;
}

}  // namespace vah
