"""The Cartesian geometry variant of the advection (AdvectJandH_Cartesian!,
src/AdvectJandH.jl:1396-2222) against the oracle: a uniform X-Y grid with no K_phiphi source and
no u_r / r term, the first X interface reflecting or letting flow out (ghost H_X = min(H_X, 0),
:1528-1545), GLF and HLL fluxes, single advection calls and fused static steps; and the adjoint
through the outflowing first interface against central differences."""
import numpy as np
import pytest

from helpers import matched_pair, max_rel, norm_err
from lydion_b200 import workloads as W

pytestmark = pytest.mark.gpu

CASES = [(W.BC_OUTFLOW, W.FLUX_GLF), (W.BC_REFLECT, W.FLUX_GLF), (W.BC_OUTFLOW, W.FLUX_HLL)]


@pytest.mark.parametrize("bc_left,flux", CASES)
def test_cartesian_advect_matches_oracle(oracle_mod, bc_left, flux):
    cl = W.cartesian_cloud(bc_left=bc_left, flux_method=flux)
    st, ctx = matched_pair(oracle_mod, cl, seed=11)
    ctdt = cl.c_tilde * cl.dt
    for _ in range(3):
        km_o = st.advect(ctdt)
        assert ctx.find_active_bins() == km_o
        ctx.advect(ctdt, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top, bc_r_left=cl.bc_r_left)
    for f in ("J", "H_r", "H_Z"):
        e = norm_err(ctx.download(f), getattr(st, f))
        assert e < 1e-12, (f, e)
    ctx.close()


@pytest.mark.parametrize("bc_left,flux", CASES)
def test_cartesian_static_steps_match_oracle(oracle_mod, bc_left, flux):
    cl = W.cartesian_cloud(bc_left=bc_left, flux_method=flux)
    st, ctx = matched_pair(oracle_mod, cl, seed=5)
    n = 30
    d_o = st.run(n)
    d_g = ctx.static_steps(n, cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top)
    np.testing.assert_array_equal(d_g[:, 5:7], d_o[:, 5:7])
    for col in (0, 1, 2):
        assert max_rel(d_g[5:, col], d_o[5:, col]) < 1e-9, col
    for f in ("J", "H_r", "H_Z"):
        assert norm_err(ctx.download(f), getattr(st, f)) < 1e-9, f
    ctx.close()


def test_left_boundary_rule_matters(oracle_mod):
    # the two rules of the first X interface give different states (the outflow case loses
    # the flux that crosses it)
    out = {}
    for bc in (W.BC_OUTFLOW, W.BC_REFLECT):
        cl = W.cartesian_cloud(bc_left=bc)
        _, ctx = matched_pair(oracle_mod, cl, seed=5)
        ctx.static_steps(20, cl.c_tilde, cl.dt, cl.z_center, cl.bc_r_right, cl.bc_z_bot, cl.bc_z_top,
                         history=False)
        out[bc] = ctx.download("J")
        ctx.close()
    assert norm_err(out[W.BC_OUTFLOW], out[W.BC_REFLECT]) > 1e-6


def test_geometry_rules_are_enforced():
    from lydion_b200._lib import LydionError
    from lydion_b200.m1 import M1Context, context_for_cloud
    cl = W.cartesian_cloud()
    ctx = context_for_cloud(cl)
    with pytest.raises(LydionError):
        ctx.upload("ur_over_r", np.ones((cl.nz, cl.nr)))          # no u_r / r on a Cartesian grid
    ctx.close()
    cyl = W.small_cloud()
    ctx = context_for_cloud(cyl)
    with pytest.raises(LydionError):
        ctx.advect(cyl.c_tilde * cyl.dt, bc_r_left=W.BC_OUTFLOW)   # the axis always reflects
    ctx.close()
    with pytest.raises(LydionError):
        fq = cyl.freq
        M1Context(cyl.n_nu, cyl.nr, cyl.nz, fq.kcore_min, fq.kcore_max, cyl.alpha_floor, bc_r_left=W.BC_OUTFLOW)


def test_cartesian_adjoint_through_outflow_boundary():
    """Gradients of the adjoint objective (M_F of the last step + the edge-ring spectrum) with
    respect to the initial J, H_X in the two columns next to the outflowing first interface, and
    to alpha there, against central differences (h = 1e-4 relative)."""
    from helpers import random_state
    from lydion_b200.m1 import context_for_cloud
    cl0 = W.cartesian_cloud(nx=10, ny=9, bc_left=W.BC_OUTFLOW)
    state = random_state(cl0, 7)
    w = np.random.default_rng(1).uniform(0.5, 1.5, cl0.n_nu)
    SS = 1e12
    n = 5
    p = (cl0.c_tilde, cl0.dt, cl0.z_center, cl0.bc_r_right, cl0.bc_z_bot, cl0.bc_z_top)

    def make(mod=None, st=None):
        cl = W.cartesian_cloud(nx=10, ny=9, bc_left=W.BC_OUTFLOW)
        if mod:
            mod(cl)
        ctx = context_for_cloud(cl)
        for name, a in zip(("J", "H_r", "H_Z"), st or state):
            ctx.upload(name, a)
            ctx.upload(name + "_old", a)
        return ctx

    def objective(mod=None, st=None):
        ctx = make(mod, st)
        h = ctx.static_steps(n, *p)
        v = h[-1, 0] + SS * float(np.dot(w, ctx.edge_spectra()[0].mean(0)))
        ctx.close()
        return v

    ctx = make()
    g = ctx.adjoint(n, *p, w_MF=1.0, w_spec=SS * w, checkpoint_every=2)
    ctx.close()
    H = 1e-4
    for (j, i, k) in [(3, 0, 7), (5, 1, 8), (2, 0, 6)]:
        for q, name in enumerate(("grad_J0", "grad_H_r0")):
            x0 = state[q][j, i, k]

            def st(s):
                out = [a.copy() for a in state]
                out[q][j, i, k] = x0 * (1 + s)
                return out
            d = (objective(st=st(H)) - objective(st=st(-H))) / (2 * H)
            adj = g[name][j, i, k] * x0
            if abs(d) < 1e-6:
                assert abs(adj) < 1e-6
                continue
            assert abs(adj - d) <= 1e-5 * abs(d), (name, j, i, k, adj, d)
    for (j, i) in [(3, 0), (4, 1)]:
        a0 = cl0.alpha[j, i]

        def mk(s):
            def m(c):
                c.alpha[j, i] = a0 * (1 + s)
            return m
        d = (objective(mk(H)) - objective(mk(-H))) / (2 * H)
        adj = g["grad_alpha"][j, i] * a0
        assert abs(adj - d) <= 1e-5 * abs(d), ("alpha", j, i, adj, d)
