"""The mixed form's own small-angle sine and cosine (gp_advance.cuh,
quaternion_step_mixed): the Taylor series of sin and cos about 0, nested in h^2 up to the
h^9 and h^10 terms, used for half angles up to pi/4.  Evaluated here in FP32 with the
device's nesting and single roundings (each fused multiply-add rounded once), it stays
within a few FP32 ulps of the exact values, so the series' truncation (below 3e-9 at
pi/4) is not what limits it; and the incidence angle's sine and cosine taken from the
slip components agree with sin and cos of |atan(syz / b0)|."""
from __future__ import annotations

import numpy as np

f32 = np.float32


def fma32(a, b, c):
    """a*b + c rounded once to FP32 (the exact product and sum fit in FP64 for FP32 inputs
    up to the last bits; the error this leaves is far below the bound checked)."""
    return f32(np.float64(a) * np.float64(b) + np.float64(c))


def mul32(a, b):
    return f32(np.float64(a) * np.float64(b))


def taylor_sincos(h):
    h = f32(h)
    h2 = mul32(h, h)
    ps = fma32(-h2, f32(1.0 / 72.0), f32(1.0))
    ps = fma32(mul32(-h2, f32(1.0 / 42.0)), ps, f32(1.0))
    ps = fma32(mul32(-h2, f32(1.0 / 20.0)), ps, f32(1.0))
    ps = fma32(mul32(-h2, f32(1.0 / 6.0)), ps, f32(1.0))
    s = mul32(h, ps)
    pc = fma32(-h2, f32(1.0 / 90.0), f32(1.0))
    pc = fma32(mul32(-h2, f32(1.0 / 56.0)), pc, f32(1.0))
    pc = fma32(mul32(-h2, f32(1.0 / 30.0)), pc, f32(1.0))
    pc = fma32(mul32(-h2, f32(1.0 / 12.0)), pc, f32(1.0))
    c = fma32(mul32(-h2, f32(0.5)), pc, f32(1.0))
    return s, c


def test_small_angle_sincos_within_fp32_rounding():
    hs = np.concatenate([np.linspace(0.0, 0.785, 4001), np.geomspace(1e-8, 0.785, 2001)])
    worst_s = worst_c = 0.0
    for h in hs:
        s, c = taylor_sincos(h)
        h64 = np.float64(f32(h))
        es, ec = np.sin(h64), np.cos(h64)
        if es > 0:
            worst_s = max(worst_s, abs(np.float64(s) - es) / es)
        worst_c = max(worst_c, abs(np.float64(c) - ec) / ec)
    eps = float(np.finfo(np.float32).eps)
    assert worst_s < 4 * eps, worst_s
    assert worst_c < 4 * eps, worst_c


def test_series_truncation_bound():
    """The first terms left out, h^11/11! and h^12/12!, at the largest half angle taken."""
    import math
    h = 0.785
    assert h ** 11 / math.factorial(11) < 3e-9
    assert h ** 12 / math.factorial(12) < 3e-10


def test_incidence_angle_sine_and_cosine_from_the_slip():
    rng = np.random.default_rng(5)
    b = rng.normal(size=(20000, 3))
    b[:100, 0] = 0.0                                        # phi = pi/2 exactly
    syz = np.sqrt(b[:, 1] ** 2 + b[:, 2] ** 2)
    phi = np.abs(np.arctan2(syz, np.abs(b[:, 0])))
    nb = np.sqrt(b[:, 0] ** 2 + syz ** 2)
    assert np.allclose(syz / nb, np.sin(phi), rtol=0, atol=1e-15)
    assert np.allclose(np.abs(b[:, 0]) / nb, np.cos(phi), rtol=0, atol=1e-15)
