"""The algebraic forms the FP32 arithmetic of the reduced-precision step uses in place of the
reference's expressions (no GPU): they are the same functions, and evaluated in FP32 they stay
within FP32 rounding of the reference's expression in FP64."""
import numpy as np


def test_levermore_chi_rewrite():
    """chi(f) = (3 + 4 f^2) / (5 + 2 sqrt(4 - 3 f^2)) (src/M1Closure.jl:28-33) equals
    (5 - 2 sqrt(4 - 3 f^2)) / 3: multiply numerator and denominator by 5 - 2 sqrt(4 - 3 f^2)."""
    f = np.linspace(0.0, 1.0, 100001)
    s = np.sqrt(4.0 - 3.0 * f * f)
    ref = (3.0 + 4.0 * f * f) / (5.0 + 2.0 * s)
    assert np.max(np.abs((5.0 - 2.0 * s) / 3.0 - ref)) < 4e-16
    f32 = f.astype(np.float32)
    s32 = np.sqrt(np.float32(4.0) - np.float32(3.0) * f32 * f32)
    chi32 = (np.float32(5.0) - np.float32(2.0) * s32) * np.float32(1.0 / 3.0)
    assert chi32.dtype == np.float32
    assert np.max(np.abs(chi32.astype(np.float64) - ref)) < 2e-7


def test_length_and_direction_from_one_reciprocal_root():
    """|f| = s * rsqrt(s) and n = f * rsqrt(s) for s = |f|^2 in FP32's normal range; below it
    the FP32 forms take no direction (n = 0, |f| = 0)."""
    rng = np.random.default_rng(5)
    fr = rng.uniform(-1.5, 1.5, 10000).astype(np.float32)
    fz = rng.uniform(-1.5, 1.5, 10000).astype(np.float32)
    s = fr * fr + fz * fz
    r = (np.float32(1.0) / np.sqrt(s)).astype(np.float32)
    mag = s * r
    ref = np.hypot(fr.astype(np.float64), fz.astype(np.float64))
    assert np.max(np.abs(mag - ref) / ref) < 3e-7
    assert np.max(np.abs(np.hypot(fr * r, fz * r) - 1.0)) < 3e-7
    assert np.float32(1e-20) ** 2 < np.finfo(np.float32).tiny   # such a |f|^2 is subnormal or 0
