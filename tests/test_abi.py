"""CPU checks of the C ABI: the library loads without a GPU, exports every function the
header declares, and its host-side Voigt tables match the scipy fixture."""
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, ROOT


def _header_functions():
    src = open(os.path.join(ROOT, "include", "lydion_m1.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(lyd_[A-Za-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from lydion_b200 import _lib
    L = _lib.lib()
    names = _header_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n
    # the Python binding declares exactly the header's functions
    assert set(names) == set(_lib.SIGNATURES)


def test_abi_version_and_edge_count():
    from lydion_b200 import _lib
    L = _lib.lib()
    assert L.lyd_abi_version() == 6
    assert L.lyd_edge_count(64, 64) == 62 + 2 * 61


def test_create_rejects_bad_dimensions_without_touching_the_gpu():
    import ctypes as C
    from lydion_b200 import _lib
    L = _lib.lib()
    h = C.c_void_p()
    cfg = _lib.Config(0, 1, 0, 1, 2, 0, 1e-5, 0.0, 0)
    for dims in [(3, 8, 8), (300, 8, 8), (16, 2, 8), (16, 8, 2)]:
        d = _lib.Dims(*dims, 0)
        assert L.lyd_create(C.byref(h), C.byref(d), C.byref(cfg)) == _lib.LYD_ERR_ARG
    bad = _lib.Config(0, 1, 7, 1, 2, 0, 1e-5, 0.0, 0)
    assert L.lyd_create(C.byref(h), C.byref(_lib.Dims(16, 8, 8, 0)), C.byref(bad)) == _lib.LYD_ERR_ARG


def test_device_voigt_tables_match_scipy_fixture():
    from lydion_b200.m1 import voigt_tables
    z = np.load(os.path.join(GOLDEN, "voigt_samples.npz"))
    t = voigt_tables()
    np.testing.assert_allclose(t[0][z["idx"]], z["erf"], rtol=4.5e-16, atol=1e-300)  # libm vs cephes: 1 ulp
    np.testing.assert_allclose(t[1][z["idx"]], z["dawson"], rtol=2e-14, atol=1e-300)
    x = z["x"]
    np.testing.assert_allclose(t[2][z["idx"]], np.exp(-x * x), rtol=1e-15)


def test_dawson_dense_against_scipy():
    from scipy.special import dawsn
    from lydion_b200.m1 import voigt_tables
    t = voigt_tables(n=40001, xmax=100.0)
    x = -100.0 + np.arange(40001) * (200.0 / 40000)
    np.testing.assert_allclose(t[1], dawsn(x), rtol=3e-14, atol=1e-300)
