"""Generates the committed golden fixtures that pin the oracle's third-party pieces.

Run from the repository root:  python tests/golden/make_golden.py <path of the LYDION checkout>

The checkout path may also come from the environment variable LYDION_REFERENCE; its data
files are read as text.

* dgtsv_cases.npz -- tridiagonal systems (random, diagonally dominant, pivot-forcing, and
  systems taken from a stiff tau0 = 1e8 cloud) with the solutions and INFO returned by
  scipy.linalg.lapack.dgtsv, i.e. by LAPACK's dgtsv, the routine the reference calls through
  Julia's LinearAlgebra.LAPACK.gtsv! (src/TridiagonalSolver.jl:54).
* voigt_samples.npz -- erf and the Dawson integral from scipy.special at a subset of the
  Voigt look-up-table nodes x_i = -1000 + 0.01 i (src/FastInterpolations.jl:175-197); scipy's
  dawsn and SpecialFunctions.jl's dawson both evaluate the Faddeeva-package algorithm.
* analytic_spectra.npz -- the analytic emergent spectra J_sphere_point / J_sphere_uni of
  src/ConstantsAndFunctions.jl:1018-1049 on an x grid, for physics-level checks, and the
  reference's tabulated analytic force multiplier M_F / (a tau_cl)^(1/3) of a uniform source
  against the dust parameter eps_1 (EscapeFractionTest_StaticCloud/AnalyticalMF_UniformSource.txt,
  read as text; its first rows are the dust-free limit), and its analytic escape fractions of
  dusty point- and uniform-source clouds against eps_1 = 0.4707 (a tau_cl)^(1/3) tau_abs
  (AnalyticalEscapeFraction_{Point,Uniform}Source.txt, stored as -f_esc there), and the
  reference's MCRT comoving spectra of expanding uniform-source clouds with v_max = 10 and
  200 km/s (VelocityGradientsTest/comoving_MCRT_uniform_{10,200}.txt).
"""
import os
import sys

import numpy as np
from scipy.linalg.lapack import dgtsv
from scipy.special import erf, dawsn

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def reference_root():
    """The LYDION checkout whose data files are read as text: the first command-line argument,
    else $LYDION_REFERENCE."""
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LYDION_REFERENCE")
    if not root or not os.path.isdir(root):
        raise SystemExit("usage: python tests/golden/make_golden.py <LYDION checkout> (or set LYDION_REFERENCE)")
    return root


def dgtsv_cases():
    rng = np.random.default_rng(20261203)
    cases = []
    for n in [2, 3, 4, 5, 8, 13, 30, 46, 62, 126]:
        # general random (pivoting likely)
        cases.append((rng.normal(size=n - 1), rng.normal(size=n), rng.normal(size=n - 1), rng.normal(size=n)))
        # diagonally dominant
        dl, du = rng.uniform(0, 1, n - 1), rng.uniform(0, 1, n - 1)
        d = -(2.5 + rng.uniform(0, 1, n))
        cases.append((dl, d, du, rng.normal(size=n)))
        # bin-width-weighted M-matrix like the frequency system (forces interchanges)
        w = 1.3 ** np.arange(n)[::-1]
        F = 10 ** rng.uniform(0, 6, n)
        dl2 = (F[:-1] * w[:-1] / w[1:]) * 0.9
        du2 = F[1:] * 0.1
        d2 = -(F + 1.0)
        cases.append((dl2, d2, du2, -rng.uniform(0, 1, n)))
    # systems from a stiff cloud step, assembled like src/UpdateLyaJandH.jl:200-214
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    from lydion_b200 import workloads as W
    cl = W.static_cloud(8, 8, 64, tau0=1e8, tau_abs=1.0, rs=0.5, umax_kms=200.0)
    st = O.OracleState(cl)
    st.setup_profiles()
    st.run(10)
    st.advect(cl.c_tilde * cl.dt)
    st.emission_absorption(cl.c_tilde, cl.dt)
    O.lib().orc_update_freq_factors(O.C.byref(st.s), O.C.byref(st.v))
    dw = 1.0 / (cl.c_tilde * cl.dt)
    for (j, i) in [(0, 0), (2, 3), (5, 1), (7, 7)]:
        A = st.Fkm[j, i, 1:-1]; B = -(st.Fk[j, i, 1:-1] + dw); Cc = st.Fkp[j, i, 1:-1]; D = -dw * st.J_old[j, i, 1:-1]
        cases.append((A[1:].copy(), B.copy(), Cc[:-1].copy(), D.copy()))
    # a singular system (INFO > 0)
    cases.append((np.array([0.0]), np.array([0.0, 1.0]), np.array([1.0]), np.array([1.0, 2.0])))
    out = {}
    for q, (dl, d, du, b) in enumerate(cases):
        _, _, _, x, info = dgtsv(dl.copy(), d.copy(), du.copy(), b.copy())
        out[f"dl{q}"], out[f"d{q}"], out[f"du{q}"], out[f"b{q}"] = dl, d, du, b
        out[f"x{q}"], out[f"info{q}"] = x, np.array(info)
    out["n"] = np.array(len(cases))
    np.savez_compressed(os.path.join(HERE, "dgtsv_cases.npz"), **out)


def voigt_samples():
    i = np.unique(np.concatenate([np.arange(0, 200001, 997), np.arange(99000, 101001, 7), [0, 100000, 200000]]))
    x = -1000.0 + i * ((1000.0 - -1000.0) / (200001 - 1))
    np.savez_compressed(os.path.join(HERE, "voigt_samples.npz"), idx=i, x=x, erf=erf(x), dawson=dawsn(x))


def analytic_spectra():
    sys.path.insert(0, ROOT)
    from lydion_b200 import constants as K
    x = np.linspace(-80, 80, 321)
    out = {"x": x}
    for T, tau in [(1e4, 1e6), (1e4, 1e7), (1e4, 1e8)]:
        at = K.compute_a(T) * tau
        with np.errstate(over="ignore", divide="ignore", invalid="ignore"):
            pt = np.sqrt(np.pi ** 3 / 24) * (x ** 2 / at) / np.cosh(np.sqrt(np.pi ** 3 / 54) * np.abs(x ** 3) / at) ** 2
            un = -np.sqrt(6 / np.pi) * (x ** 2 / at) * np.log(1 - np.exp(-np.sqrt(2 * np.pi ** 3 / 27) * np.abs(x ** 3) / at))
        out[f"point_T{T:g}_tau{tau:g}"] = np.nan_to_num(pt, nan=0.0)
        out[f"uni_T{T:g}_tau{tau:g}"] = np.nan_to_num(un, nan=0.0)
    ref = reference_root()
    mf = np.loadtxt(os.path.join(ref, "EscapeFractionTest_StaticCloud", "AnalyticalMF_UniformSource.txt"))
    out["mf_uniform_eps1"] = mf[:8, 0]
    out["mf_uniform_over_atau13"] = mf[:8, 1]
    for kind, fn in (("point", "PointSource"), ("uni", "UniformSource")):
        t = np.loadtxt(os.path.join(ref, "EscapeFractionTest_StaticCloud", f"AnalyticalEscapeFraction_{fn}.txt"))
        out[f"fesc_{kind}_eps1"] = t[:, 0]
        out[f"fesc_{kind}"] = -t[:, 1]
    for v in (10, 200):
        t = np.loadtxt(os.path.join(ref, "VelocityGradientsTest", f"comoving_MCRT_uniform_{v}.txt"))
        out[f"mcrt_v{v}_x"] = t[:, 0]
        out[f"mcrt_v{v}"] = t[:, 1]
    np.savez_compressed(os.path.join(HERE, "analytic_spectra.npz"), **out)


if __name__ == "__main__":
    reference_root()
    dgtsv_cases()
    voigt_samples()
    analytic_spectra()
    print("fixtures written to", HERE)
