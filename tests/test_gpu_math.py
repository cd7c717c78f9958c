"""The step's hand-written device arithmetic against CUDA's IEEE-rounded
operations (vah_math_check): the Newton correction's reciprocal (hardware
estimate + one Newton-Raphson step) and 1/sqrt (estimate + two steps).

Bounds: the reciprocal only scales the Newton correction, which is ~1e-7 of
u_T where the iteration stops, so 1e-11 relative leaves the root untouched at
1e-18; 1/sqrt enters the root directly and must be as good as a correctly
rounded 1/sqrt to a few units in the last place (8 x 2^-53)."""
import ctypes as C

import pytest

import vahlib as V

pytestmark = pytest.mark.gpu


# The last two ranges cross the edges of the reciprocal estimate's band,
# [2^-1000, 2^1001): subnormal and near-overflow inputs, where the Newton
# correction must take the IEEE quotient (equal results, infinities included).
@pytest.mark.parametrize("lo,hi", [(1e-300, 1e300), (1.0, 1e32), (4e-324, 1e-295), (1e295, 1.7e308)])
def test_gpu_fast_reciprocal_and_rsqrt_error_bounds(lo, hi):
    L = V.library()
    L.vah_math_check.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, C.POINTER(C.c_double),
                                 C.POINTER(C.c_double)]
    rcp, rsq = C.c_double(), C.c_double()
    assert L.vah_math_check(0, lo, hi, 1 << 20, C.byref(rcp), C.byref(rsq)) == 0
    print(f"max relative error: reciprocal {rcp.value:.3e}, rsqrt {rsq.value:.3e}")
    assert rcp.value < 1e-11
    assert rsq.value <= 8 * 2.0 ** -53
