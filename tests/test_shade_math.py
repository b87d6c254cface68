"""Host-side pieces of the shading pass: the sine/cosine of AO sample angles (quadrant reduction and
Taylor polynomials, evaluated identically by the library and the oracle) against the error bound of
the method, and the parameter block layout."""
import ctypes as C
import math

import numpy as np


def test_sincos_error_bound(oracle_mod):
    L = oracle_mod.lib()
    s, c = C.c_float(), C.c_float()
    worst = 0.0
    for u in np.linspace(0.0, 1.0, 20001, dtype=np.float32):
        x = float(np.float32(6.2831855) * u)
        L.oracle_sincos(x, C.byref(s), C.byref(c))
        worst = max(worst, abs(s.value - math.sin(x)), abs(c.value - math.cos(x)))
    # Taylor remainders on [-pi/4, pi/4] are below 4e-9; the rest is float rounding of a few terms
    assert worst < 4e-7


def test_shade_params_layout(svdag_lib, oracle_mod):
    assert C.sizeof(svdag_lib.ShadeParams) == 112 == C.sizeof(oracle_mod.ShadeParams)
    p = svdag_lib.shade_params(12, ao_samples=8)
    assert p.flags == svdag_lib.SHADE_SHADOWS | svdag_lib.SHADE_AO and p.ao_ray_length == 4.0
    d = np.array(list(p.sun_direction), dtype=np.float64)
    assert abs(np.linalg.norm(d) - 1.0) < 1e-6 and d[1] > d[2] > d[0] > 0
