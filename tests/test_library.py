"""libvah.so on the CPU: it loads, exports every entry point include/vah.h
declares, and its host-side pieces (EoS table, initial-condition generators)
are consistent. No kernel is launched here."""
import os
import re

import numpy as np

import vahlib as V

HEADER = os.path.join(V.ROOT, "include", "vah.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vah_\w+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    L = V.library()
    names = declared_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(L, name), name
    assert set(V.EXPORTS) <= set(names)


def test_version_string():
    assert "sm_100a" in V.product.version()


def test_eos_table_is_thermodynamically_consistent():
    tab = V.eos_table()
    n = int(tab[0])
    assert n == 4096
    lne = tab[1] + tab[3] * np.arange(n)
    e = np.exp(lne)
    p, T, cs2 = tab[8:8 + n], tab[8 + n:8 + 2 * n], tab[8 + 2 * n:]
    tc = 0.155 / 0.197326938
    # c_s^2(T) = 1/3 - (1/3 - 0.15)/(1 + (T/Tc)^4)
    np.testing.assert_allclose(cs2, 1 / 3 - (1 / 3 - 0.15) / (1 + (T / tc) ** 4), rtol=1e-12)
    # s = (e + p)/T follows the closed form s_inf tau^3 (tau^4/(tau^4+a))^(11/12)
    tau = T / tc
    s_closed = 4 / 3 * 13.8997 * tc ** 3 * tau ** 3 * (tau ** 4 / (tau ** 4 + 0.45)) ** (11 / 12)
    np.testing.assert_allclose((e + p) / T, s_closed, rtol=1e-8)
    # c_s^2 = dp/de along the table
    dp_de = np.gradient(p, e)
    np.testing.assert_allclose(dp_de[5:-5], cs2[5:-5], rtol=2e-4)
    # limits: hadron-gas c_s^2 at the low end, conformal normalisation at the top
    assert abs(cs2[0] - 0.15) < 1e-6 and abs(cs2[-1] - 1 / 3) < 1e-5
    assert abs(e[-1] / (13.8997 * T[-1] ** 4) - 1) < 1e-3
    assert np.all(np.diff(T) > 0) and np.all(np.diff(p) > 0)


def test_eos_table_argument_errors():
    L = V.library()
    out = np.zeros(10)
    assert L.vah_eos_table_build(4096, out.ctypes.data_as(V.P), out.size) == -1


def test_math_check_argument_errors():
    """vah_math_check rejects bad ranges and sizes before touching a device."""
    import ctypes as C
    L = V.library()
    L.vah_math_check.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, C.POINTER(C.c_double),
                                 C.POINTER(C.c_double)]
    a, b = C.c_double(), C.c_double()
    for lo, hi, n in [(0.0, 1.0, 16), (1.0, 1.0, 16), (2.0, 1.0, 16), (1.0, 2.0, 1), (-1.0, 2.0, 16)]:
        assert L.vah_math_check(0, lo, hi, n, C.byref(a), C.byref(b)) == -1
    assert L.vah_math_check(0, 1.0, 2.0, 16, None, C.byref(b)) == -1


def test_initial_condition_generators():
    P = V.product
    e = P.optical_glauber(61, 61, 0.2, 0.2, b=7.0, e_peak=1190.0).reshape(61, 61)
    assert abs(e.max() - 1190.001) < 1e-9
    np.testing.assert_allclose(e, e[::-1, :], rtol=1e-12)   # symmetric in y
    np.testing.assert_allclose(e, e[:, ::-1], rtol=1e-12)   # and in x
    assert e[30, :].argmax() == 30
    assert (e[:, 30] > e[30, :]).sum() > 20                  # b along x: the almond is taller in y
    a, na = P.mc_glauber(81, 81, 0.1, 0.1, 3.0, seed=11, e_peak=50.0)
    b, nb = P.mc_glauber(81, 81, 0.1, 0.1, 3.0, seed=11, e_peak=50.0)
    c, nc = P.mc_glauber(81, 81, 0.1, 0.1, 3.0, seed=12, e_peak=50.0)
    np.testing.assert_array_equal(a, b)
    assert na == nb and 100 < na <= 394
    assert not np.array_equal(a, c)
    f = P.longitudinal(81, 0.1)
    assert f[40] == 1.0 and f[25] == 1.0 and f[0] < 0.2
    np.testing.assert_allclose(f, f[::-1], rtol=0, atol=1e-15)
