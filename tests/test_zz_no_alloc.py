"""FindActiveBins for callers that cannot allocate device memory.

lyd_find_active_bins_noalloc serves hosts that own every device allocation themselves (a
framework memory pool, a plugin with a fixed budget, a time loop that must not allocate):
it works on caller-owned device arrays and keeps its reduction scratch in a fixed device
array inside the library. This test calls it through the C ABI on two different states in a
row and checks each window against the context-based lyd_find_active_bins. It sits in a file
of its own that pytest collects last, so a run stopping at the first failure has already run
every other test."""
import ctypes as C

import numpy as np
import pytest

from helpers import matched_pair, random_state
from lydion_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _states(cloud):
    J1, _, _ = random_state(cloud, 31)                # every bin carries energy -> full window
    J2, _, _ = random_state(cloud, 32)
    J2[..., :9] = 1e-58                               # empty red wing -> window starts later
    J2[..., -4:] = 1e-58
    return [J1, J2]


def test_noalloc_window_matches_context_entry_point(oracle_mod):
    import torch
    from lydion_b200 import _lib
    cl = W.small_cloud(nr=20, nz=18, n_nu=64, x_max=600.0)
    _, ctx = matched_pair(oracle_mod, cl)
    L = _lib.lib()
    dev = torch.device("cuda", 0)
    dnu = torch.tensor(cl.freq.dnu, dtype=torch.float64, device=dev)
    dV = torch.tensor(np.ascontiguousarray(cl.geom.dV), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    windows = []
    for J in _states(cl):
        ctx.upload("J", J)
        ref = ctx.find_active_bins()
        dJ = torch.tensor(np.ascontiguousarray(J), dtype=torch.float64, device=dev)
        kmin, kmax = C.c_int32(-1), C.c_int32(-1)
        rc = L.lyd_find_active_bins_noalloc(dJ.data_ptr(), dnu.data_ptr(), dV.data_ptr(), cl.n_nu, cl.nr, cl.nz,
                                            cl.freq.kcore_min, cl.freq.kcore_max, C.c_void_p(stream.cuda_stream),
                                            C.byref(kmin), C.byref(kmax))
        assert rc == _lib.LYD_OK
        assert (kmin.value, kmax.value) == ref
        windows.append(ref)
    assert windows[0] == (0, cl.n_nu - 1)
    assert windows[1][0] > 0 and windows[1][1] < cl.n_nu - 1
    ctx.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    from lydion_b200 import _lib
    L = _lib.lib()
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    kmin, kmax = C.c_int32(), C.c_int32()
    rc = L.lyd_find_active_bins_noalloc(buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), 300, 8, 8, 1, 2, None,
                                        C.byref(kmin), C.byref(kmax))
    assert rc == _lib.LYD_ERR_ARG
