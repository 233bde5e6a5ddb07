"""The C ABI from plain C: tests/c_abi_static_steps.c, compiled here with gcc against
include/lydion_m1.h and the built library, runs the static-cloud steps of a cloud whose inputs
this test writes to a file. Its diagnostics records and final state must be bit for bit those of
the same steps through the Python binding."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from helpers import random_state
from lydion_b200 import _lib
from lydion_b200 import workloads as W

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _record(f, name, values):
    v = np.ascontiguousarray(np.asarray(values, dtype=np.float64).ravel())
    f.write(name.encode().ljust(32, b"\0"))
    f.write(np.int64(v.size).tobytes())
    f.write(v.tobytes())


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_plain_c_caller_matches_python(tmp_path):
    from lydion_b200.m1 import context_for_cloud
    cl = W.small_cloud(nr=20, nz=18, n_nu=32)
    J, Hr, HZ = random_state(cl, 21)
    n = 6
    p = (cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    # the Python path
    ctx = context_for_cloud(cl)
    for name, a in (("J", J), ("H_r", Hr), ("H_Z", HZ)):
        ctx.upload(name, a)
        ctx.upload(name + "_old", a)
    h_py = ctx.static_steps(n, *p)
    s_py = [ctx.download(f) for f in ("J", "H_r", "H_Z")]
    ctx.close()
    # the same inputs for the C program
    g, fq = cl.geom, cl.freq
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as f:
        _record(f, "dims", [cl.n_nu, cl.nr, cl.nz])
        _record(f, "config", [cl.flux_method, int(bool(cl.recoil)), fq.kcore_min, fq.kcore_max, cl.alpha_floor])
        for name in ("r", "Z", "rCoM", "ZCoM", "dV", "inv_dV", "A_r", "A_Z", "inv_r_cell", "dr_L", "dr_R",
                     "inv_dr_i_im1", "inv_dr_ip1_i", "inv_dr_ip2_ip1", "dZ_L", "dZ_R", "inv_dZ_j_jm1",
                     "inv_dZ_jp1_j", "inv_dZ_jp2_jp1"):
            _record(f, name, getattr(g, name))
        _record(f, "dr_bnd", g.dr_b)
        _record(f, "dZ_bnd", g.dZ_b)
        for name in ("nu", "nuC", "dnu", "inv_dnu", "inv_nuC"):
            _record(f, name, getattr(fq, name))
        fields = ["alpha", "alpha_c", "pd", "js", "T", "dur_dr", "dur_dZ", "duZ_dr", "duZ_dZ", "ur_over_r",
                  "u_r_star", "u_Z_star"] + (["alpha_cF"] if np.any(cl.alpha_cF) else [])
        for name in fields:
            _record(f, f"up:{_lib.F[name]}", getattr(cl, name))
        for name, a in (("J", J), ("H_r", Hr), ("H_Z", HZ)):
            _record(f, f"up:{_lib.F[name]}", a)
            _record(f, f"up:{_lib.F[name + '_old']}", a)
        _record(f, "step", list(p) + [n])
    exe = tmp_path / "c_abi_static_steps"
    libdir = os.path.dirname(_lib.LIB_PATH)
    subprocess.run(["gcc", "-O2", "-std=c11", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_abi_static_steps.c"), "-L", libdir, "-llydion_m1",
                    f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), str(inp), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    res = np.fromfile(out, dtype=np.float64)
    h_c = res[:7 * n].reshape(n, 7)
    s_c = res[7 * n:].reshape(3, *s_py[0].shape)
    np.testing.assert_array_equal(h_c, h_py)
    for q in range(3):
        np.testing.assert_array_equal(s_c[q], s_py[q])
