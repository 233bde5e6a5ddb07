"""Finite-difference check of the adjoint on the turbulent-cloud workload.

    python -m lydion_b200.adjoint_check [--scale S] [--steps N] [--cells C] [--every K] [--h H]

Objective: M_F of the last step plus the 64-point emergent spectrum (the edge-ring spectrum
linearly interpolated onto 64 points in x), each point weighted by 1 / (64 * its mean value
at the start of the check) so that both terms are O(1). The adjoint gives the gradient with
respect to n_H, T, the dust opacity kappa_d (per cell) and a per-cell velocity scale; C cells
drawn at random inside the cloud are checked against central differences with h = 1e-4
relative. Prints one JSON line with the relative errors.
"""
import argparse
import json
import time

import numpy as np

from . import adjoint as A
from . import constants as K
from . import workloads as W
from .m1 import context_for_cloud


def _params(c):
    return (c.c_tilde, c.dt, c.z_center, c.bc_r_right, c.bc_z_bot, c.bc_z_top)


def run(scale=1, steps=2000, n_cells=64, every=100, h=1e-4, seed=20261207):
    base = W.config_c4(scale)
    n = steps
    M, _ = A.spectrum_resampling(base.freq, 64)

    def objective_of(cloud, w64):
        ctx = context_for_cloud(cloud)
        hist = ctx.static_steps(n, *_params(base))
        s64 = M @ ctx.edge_spectra()[0].mean(0)
        ctx.close()
        return hist[-1, 0] + float(np.dot(w64, s64)), s64

    # weights from a first forward run
    _, s64 = objective_of(W.config_c4(scale), np.zeros(64))
    w64 = 1.0 / (64.0 * np.where(np.abs(s64) > 0, np.abs(s64), 1.0))
    w_MF, w_bins = A.objective_weights(base.freq, 1.0, w64)
    ctx = context_for_cloud(base)
    t0 = time.perf_counter()
    g = ctx.adjoint(n, *_params(base), w_MF=w_MF, w_spec=w_bins, checkpoint_every=every)
    t_adj = time.perf_counter() - t0
    ctx.close()
    phys = A.physical_gradients(base, g)
    gv = A.velocity_scale_gradient(base, g)
    rng = np.random.default_rng(seed)
    inside = np.argwhere(base.alpha > 0)
    pick = inside[rng.choice(len(inside), size=min(n_cells, len(inside)), replace=False)]

    def fresh():
        return W.config_c4(scale)

    def set_nH(c, j, i, s):
        nH = c.n_H[j, i] * (1 + s)
        c.n_H[j, i] = nH
        c.alpha[j, i] = nH * K.compute_sigma0(c.T[j, i])
        c.alpha_c[j, i] = c.kappa_d * 0.01 * nH * K.mH

    def set_T(c, j, i, s):
        T = c.T[j, i] * (1 + s)
        c.T[j, i] = T
        c.alpha[j, i] = c.n_H[j, i] * K.compute_sigma0(T)

    def set_kappa(c, j, i, s):
        c.alpha_c[j, i] *= 1 + s

    def set_v(c, j, i, s):
        A.scale_cell_velocity(c, j, i, s)

    checks = {
        "n_H": (set_nH, lambda j, i: phys["grad_n_H"][j, i] * base.n_H[j, i]),
        "T": (set_T, lambda j, i: phys["grad_T_total"][j, i] * base.T[j, i]),
        "kappa_d": (set_kappa, lambda j, i: phys["grad_kappa_d"][j, i] * base.kappa_d),
        "v": (set_v, lambda j, i: gv[j, i]),
    }
    out = {}
    for name, (setter, adj_of) in checks.items():
        rel = []
        for j, i in pick:
            vals = []
            for s in (h, -h):
                c = fresh()
                setter(c, int(j), int(i), s)
                vals.append(objective_of(c, w64)[0])
            fd = (vals[0] - vals[1]) / (2 * h)
            adj = adj_of(int(j), int(i))
            rel.append(abs(adj - fd) / max(abs(fd), 1e-300))
        rel = np.asarray(rel)
        out[name] = {"median_rel_err": float(np.median(rel)), "max_rel_err": float(rel.max()),
                     "frac_below_1e-3": float(np.mean(rel < 1e-3))}
    return {"workload": f"turbulent cloud {base.nr}x{base.nz}x{base.n_nu}", "steps": n, "checkpoint_every": every,
            "cells": int(len(pick)), "h": h, "objective": g["objective"], "adjoint_wall_s": t_adj, "checks": out}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--cells", type=int, default=64)
    ap.add_argument("--every", type=int, default=100)
    ap.add_argument("--h", type=float, default=1e-4, help="relative finite-difference step")
    a = ap.parse_args()
    print(json.dumps(run(a.scale, a.steps, a.cells, a.every, a.h)), flush=True)


if __name__ == "__main__":
    main()
