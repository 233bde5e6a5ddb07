"""B200-native Lyman-alpha M1 transport step (LYDION's AdvectJandH / M1Closure /
UpdateLyaJandH / FreqFactors / LymanAlphaDestruction / TridiagonalSolver path).

The compute runs in liblydion_m1.so (hand-written sm_100a CUDA behind the C ABI in
include/lydion_m1.h); this package is its Python front end:

* m1         -- M1Context, a device-resident state wrapping one lyd_ctx;
* lya        -- drop-in functions with the reference's call signatures;
* grid, workloads -- host set-up of geometry, frequency grid and synthetic clouds.
"""
from . import constants, grid, workloads  # noqa: F401

__all__ = ["constants", "grid", "workloads", "m1", "lya", "build"]
