"""The adjoint of the static-driver loop (lyd_adjoint_run) against central finite differences of
the forward step, on a small seeded cloud.

Objective: w_MF * M_F(last step) + sum_k w_k S_k(final J), S the edge-ring mean spectrum.
Finite differences use h = 1e-4 relative (the perturbation of one input entry), as in the
adjoint configuration this library is specified on. The FP64 step's own rounding (the stiff
frequency solve, ~1e-13 relative) bounds how well a central difference can resolve the
smallest gradients, so each check states its tolerance beside the quantity."""
import numpy as np
import pytest

from helpers import random_state
from lydion_b200 import workloads as W

pytestmark = pytest.mark.gpu

H = 1e-4
SS = 1e12     # scales the spectrum term so that both terms of the objective are O(1)


def _cloud(flux=W.FLUX_GLF):
    return W.small_cloud(nr=10, nz=9, n_nu=16, flux_method=flux)


class Problem:
    def __init__(self, n_steps, flux=W.FLUX_GLF):
        self.flux = flux
        self.cl = _cloud(flux)
        self.n = n_steps
        self.w = np.random.default_rng(1).uniform(0.5, 1.5, self.cl.n_nu)
        self.state = random_state(self.cl, 5)
        c = self.cl
        self.p = (c.c_tilde, c.dt, c.z_center, c.bc_r_right, c.bc_z_bot, c.bc_z_top)

    def ctx(self, mod=None, state=None):
        from lydion_b200.m1 import context_for_cloud
        c = _cloud(self.flux)
        if mod:
            mod(c)
        ctx = context_for_cloud(c)
        for name, a in zip(("J", "H_r", "H_Z"), state or self.state):
            ctx.upload(name, a)
            ctx.upload(name + "_old", a)
        return ctx

    def objective(self, mod=None, state=None):
        ctx = self.ctx(mod, state)
        h = ctx.static_steps(self.n, *self.p)
        v = h[-1, 0] + SS * float(np.dot(self.w, ctx.edge_spectra()[0].mean(0)))
        ctx.close()
        return v

    def adjoint(self, every=2):
        ctx = self.ctx()
        g = ctx.adjoint(self.n, *self.p, w_MF=1.0, w_spec=SS * self.w, checkpoint_every=every)
        return ctx, g

    def fd_field(self, field, idx):
        v0 = getattr(self.cl, field)[idx]

        def mk(s):
            def m(c):
                getattr(c, field)[idx] = v0 * (1 + s)
            return m
        return (self.objective(mk(H)) - self.objective(mk(-H))) / (2 * H), v0

    def fd_state(self, q, idx):
        base = self.state
        x0 = base[q][idx]

        def st(s):
            out = [a.copy() for a in base]
            out[q][idx] = x0 * (1 + s)
            return out
        return (self.objective(state=st(H)) - self.objective(state=st(-H))) / (2 * H), x0


@pytest.fixture(scope="module")
def prob():
    P = Problem(6)
    P.ctx_g = P.adjoint()
    return P


def test_objective_and_final_state(prob):
    ctx, g = prob.ctx_g
    assert abs(g["objective"] - prob.objective()) <= 1e-12 * abs(g["objective"])
    # the context ends in the forward sweep's final state
    ref = prob.ctx()
    ref.static_steps(prob.n, *prob.p, history=False)
    for f in ("J", "H_r", "H_Z"):
        np.testing.assert_array_equal(ctx.download(f), ref.download(f))


CELLS = [(2, 3), (4, 1), (0, 0), (6, 5)]


@pytest.mark.parametrize("field,tol", [("alpha", 1e-5), ("alpha_c", 1e-5), ("T", 1e-5)])
def test_opacity_and_temperature_gradients(prob, field, tol):
    _, g = prob.ctx_g
    for idx in CELLS:
        d, v0 = prob.fd_field(field, idx)
        adj = g["grad_" + field][idx] * v0
        assert abs(adj - d) <= tol * abs(d), (field, idx, adj, d)


@pytest.mark.parametrize("field", ["dur_dr", "duZ_dZ", "ur_over_r"])
def test_velocity_gradient_gradients(prob, field):
    # these gradients are ~1e-6 of the objective: central differences resolve them to ~1e-4
    _, g = prob.ctx_g
    for idx in CELLS[:2]:
        d, v0 = prob.fd_field(field, idx)
        adj = g["grad_" + field][idx] * v0
        assert abs(adj - d) <= 3e-4 * abs(d), (field, idx, adj, d)


def test_face_velocity_gradients(prob):
    _, g = prob.ctx_g
    for (j, i) in CELLS[:3]:
        for field, idx in (("u_r_star", (j, i + 1)), ("u_Z_star", (j + 1, i))):
            d, v0 = prob.fd_field(field, idx)
            if v0 == 0.0:
                continue
            adj = g["grad_" + field][idx] * v0
            assert abs(adj - d) <= 1e-4 * abs(d), (field, idx, adj, d)


def test_initial_state_gradients(prob):
    _, g = prob.ctx_g
    for idx in [(2, 3, 7), (4, 1, 8), (6, 7, 5), (0, 0, 9)]:
        for q, name in enumerate(("grad_J0", "grad_H_r0", "grad_H_Z0")):
            d, x0 = prob.fd_state(q, idx)
            adj = g[name][idx] * x0
            if abs(d) < 1e-6:            # below what the difference resolves
                assert abs(adj) < 1e-6
                continue
            assert abs(adj - d) <= 1e-5 * abs(d), (name, idx, adj, d)


def test_checkpoint_spacing_does_not_change_gradients(prob):
    # the face adjoints scatter with FP64 atomics: equal to rounding, not bitwise. 0 and 1 keep
    # every step's state and tape from the forward sweep; 2 (the fixture), 4 and n recompute
    # segments; -1 is the binomial schedule with 0 (automatic), 1 and 2 extra snapshots
    _, g = prob.ctx_g
    for every, snaps in ((0, 0), (1, 0), (4, 0), (prob.n, 0), (-1, 0), (-1, 1), (-1, 2)):
        ctx = prob.ctx()
        g2 = ctx.adjoint(prob.n, *prob.p, w_MF=1.0, w_spec=SS * prob.w, checkpoint_every=every, snapshots=snaps)
        ctx.close()
        assert g2["objective"] == g["objective"]
        for k in ("grad_alpha", "grad_T", "grad_J0", "grad_u_r_star"):
            np.testing.assert_allclose(g2[k], g[k], rtol=1e-10, atol=1e-11 * np.abs(g[k]).max())


def test_overlapped_recomputation_matches_the_serial_order():
    """With uniform checkpoints and phase timing off, the next segment is recomputed on a second
    stream while the current one is reversed; with timing on the segments run one after the
    other. 30 steps in segments of 4 (8 segments, both state buffers reused several times) give
    the same gradients and the same final state either way."""
    P = Problem(30)
    out, fin = [], []
    for timing in (False, True):
        ctx = P.ctx()
        ctx.set_timing(timing)
        out.append(ctx.adjoint(P.n, *P.p, w_MF=1.0, w_spec=SS * P.w, checkpoint_every=4))
        ctx.set_timing(False)
        fin.append(ctx.download("J"))
        ctx.close()
    assert out[0]["objective"] == out[1]["objective"]
    np.testing.assert_array_equal(fin[0], fin[1])
    for k in ("grad_alpha", "grad_alpha_c", "grad_T", "grad_J0", "grad_H_r0", "grad_u_r_star", "grad_u_Z_star"):
        np.testing.assert_allclose(out[0][k], out[1][k], rtol=1e-10, atol=1e-11 * np.abs(out[1][k]).max())


def test_binomial_schedule_on_a_longer_run():
    """40 steps with 3 extra snapshots (no step advanced more than 4 times) give the gradients of
    the run that keeps every step."""
    P = Problem(40)
    out = []
    for every, snaps in ((1, 0), (-1, 3)):
        ctx = P.ctx()
        out.append(ctx.adjoint(P.n, *P.p, w_MF=1.0, w_spec=SS * P.w, checkpoint_every=every, snapshots=snaps))
        ctx.close()
    for k in ("grad_alpha", "grad_alpha_c", "grad_T", "grad_J0", "grad_u_Z_star"):
        np.testing.assert_allclose(out[1][k], out[0][k], rtol=1e-10, atol=1e-11 * np.abs(out[0][k]).max())


def test_adjoint_rejects_unsupported_forms():
    from lydion_b200._lib import PREC_MIXED, LydionError
    from lydion_b200.m1 import context_for_cloud
    c = _cloud()
    ctx = context_for_cloud(c, precision=PREC_MIXED)
    with pytest.raises(LydionError):
        ctx.adjoint(2, c.c_tilde, c.dt, c.z_center)


@pytest.fixture(scope="module")
def prob_hll():
    P = Problem(6, flux=W.FLUX_HLL)
    P.ctx_g = P.adjoint()
    return P


def test_hll_objective(prob_hll):
    _, g = prob_hll.ctx_g
    assert abs(g["objective"] - prob_hll.objective()) <= 1e-12 * abs(g["objective"])


@pytest.mark.parametrize("field", ["alpha", "alpha_c", "T"])
def test_hll_opacity_and_temperature_gradients(prob_hll, field):
    # the HLL wave speeds depend on the reconstructed f and n: their adjoint enters here
    _, g = prob_hll.ctx_g
    for idx in CELLS:
        d, v0 = prob_hll.fd_field(field, idx)
        adj = g["grad_" + field][idx] * v0
        assert abs(adj - d) <= 1e-5 * abs(d), (field, idx, adj, d)


def test_hll_initial_state_and_face_velocity_gradients(prob_hll):
    _, g = prob_hll.ctx_g
    for idx in [(2, 3, 7), (4, 1, 8), (6, 7, 5)]:
        for q, name in enumerate(("grad_J0", "grad_H_r0", "grad_H_Z0")):
            d, x0 = prob_hll.fd_state(q, idx)
            adj = g[name][idx] * x0
            if abs(d) < 1e-6:
                assert abs(adj) < 1e-6
                continue
            assert abs(adj - d) <= 1e-5 * abs(d), (name, idx, adj, d)
    for (j, i) in CELLS[:2]:
        for field, idx in (("u_r_star", (j, i + 1)), ("u_Z_star", (j + 1, i))):
            d, v0 = prob_hll.fd_field(field, idx)
            if v0 == 0.0:
                continue
            adj = g["grad_" + field][idx] * v0
            assert abs(adj - d) <= 1e-4 * abs(d), (field, idx, adj, d)


@pytest.mark.parametrize("flux", [W.FLUX_GLF, W.FLUX_HLL])
def test_adjoint_matches_forward_mode_oracle(oracle_mod, flux):
    """An independent derivative: the dual-number build of the oracle (forward mode, every
    operation of the restated step differentiated by the chain rule, no hand-written
    derivative) along random directions in alpha, alpha_c, T (with H_voigt(T), phi_nu and
    alpha_F), the face velocities and the initial J, against the hand-written adjoint's gradient
    dotted with the same direction. Both are exact derivatives of the same discrete step; they
    differ by the rounding of two solves of the stiff frequency systems (cyclic reduction on the
    GPU, pivoted elimination in the oracle) and of the two H_voigt tables."""
    P = Problem(6, flux)
    ctx, g = P.adjoint(every=1)
    ctx.close()
    cl = P.cl
    rng = np.random.default_rng(17)
    seeds = {"alpha": rng.normal(size=cl.alpha.shape) * cl.alpha,
             "alpha_c": rng.normal(size=cl.alpha_c.shape) * cl.alpha_c,
             "T": rng.normal(size=cl.T.shape) * cl.T,
             "u_r_star": rng.normal(size=cl.u_r_star.shape) * cl.u_r_star,
             "u_Z_star": rng.normal(size=cl.u_Z_star.shape) * cl.u_Z_star,
             "J0": rng.normal(size=P.state[0].shape) * P.state[0]}
    st = oracle_mod.OracleState(cl)
    for name, a in zip(("J", "H_r", "H_Z"), P.state):
        getattr(st, name)[...] = a
        getattr(st, name + "_old")[...] = a
    st.setup_profiles()
    tol = {"alpha": 1e-8, "alpha_c": 1e-8, "T": 1e-8, "u_r_star": 1e-6, "u_Z_star": 1e-6, "J0": 1e-8}
    for key, sd in seeds.items():
        obj, tan, _, _ = oracle_mod.objective_tangent(st, P.n, 1.0, SS * P.w, {key: sd})
        assert obj == pytest.approx(g["objective"], rel=1e-10)
        adj = float(np.sum(g["grad_" + key] * sd))
        assert adj == pytest.approx(tan, rel=tol[key]), (key, adj, tan)
