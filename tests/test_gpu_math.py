"""Accuracy of the device's FP64 arithmetic helpers (lyd_math_check) against the host's
extended-precision arithmetic: the Newton-refined reciprocal and reciprocal square root the
kernels use in place of IEEE division and square root, the root formed from the latter, and the
closure chi(f) in the form the kernels evaluate, and the table-driven exponential of the
frequency factors."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ULP = 2.0 ** -52


def _run(fn, x):
    from lydion_b200 import _lib
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    _lib.check(_lib.lib().lyd_math_check(fn, x.ctypes.data_as(_lib.P), y.ctypes.data_as(_lib.P), x.size))
    return y


def _args(seed, n=200_000):
    rng = np.random.default_rng(seed)
    wide = np.ldexp(rng.uniform(1.0, 2.0, n), rng.integers(-1020, 1020, n))   # every binade of the normal range
    near = rng.uniform(1.0, 4.0, n)                                           # the closure's root arguments
    return np.concatenate([wide, near, [1.0, 2.0, 4.0, 0.25, np.finfo(np.float64).tiny, 1e300]])


def _rel(got, want):
    want = want.astype(np.longdouble)
    return np.max(np.abs((got.astype(np.longdouble) - want) / want))


def test_reciprocal_square_root():
    x = _args(1)
    assert _rel(_run(0, x), 1 / np.sqrt(x.astype(np.longdouble))) < 1.5 * ULP


def test_reciprocal():
    x = _args(2)
    x = np.concatenate([x, -x[:1000]])
    assert _rel(_run(1, x), 1 / x.astype(np.longdouble)) < 1.5 * ULP


def test_square_root_from_reciprocal_root():
    x = _args(3)
    assert _rel(_run(2, x), np.sqrt(x.astype(np.longdouble))) < 2.0 * ULP


def test_closure_chi():
    # 5 - 2 sqrt(t) loses up to a factor 4 to cancellation at f = 0 (5 - 4): the root's ~1.5 ulp
    # becomes ~3 ulp of chi, plus the rounding of the product by 1/3
    f = np.concatenate([np.linspace(0.0, 1.0, 100_001), np.random.default_rng(4).uniform(0.0, 1.0, 100_000)])
    fl = f.astype(np.longdouble)
    want = (3 + 4 * fl * fl) / (5 + 2 * np.sqrt(4 - 3 * fl * fl))
    assert _rel(_run(3, f), want) < 5.0 * ULP


def test_exponential_of_the_clamped_peclet_range():
    rng = np.random.default_rng(5)
    x = np.concatenate([np.linspace(-40.0, 40.0, 400_001), rng.uniform(-40.0, 40.0, 200_000),
                        rng.uniform(-1e-3, 1e-3, 10_000), [0.0, -0.0, 40.0, -40.0]])
    # half an ulp from the table entry, half from the final rounding, a little from e^r - 1
    assert _rel(_run(4, x), np.exp(x.astype(np.longdouble))) < 1.5 * ULP
