"""Radial-column inputs shared by the implicit-solver tests: primitives of a
perturbed isothermal atmosphere with reflected ghosts, an explicit update of
the right scale and the metric values of real cells."""
import numpy as np

from exocubed_b200 import workloads as W

G = 3


def column_problem(oracle_mod, ncol, L, seed):
    """(w [ncol][5][L+6], du [ncol][5][L], colgeo [ncol][4], x1f, x1v, dx1f, cfg)"""
    N = 8
    cfg = W.dry_atmosphere_config(N=N, L=L, rsolver=2)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(W.dry_atmosphere_state(cfg, seed=seed))
    wfull = o.primitive()
    x1f, _, _ = o.mesh(0)
    x1v = 0.5 * (x1f[1:] + x1f[:-1])
    dx1f = np.diff(x1f)
    rng = np.random.default_rng(seed)
    cols = []
    for c in range(ncol):
        p, k, j = rng.integers(6), G + rng.integers(N), G + rng.integers(N)
        cols.append(wfull[p, :, k, j, :])
    w = np.stack(cols)
    scale = np.abs(w[:, :, G:G + L]).mean(axis=(0, 2))
    du = 1e-4 * scale[None, :, None] * rng.standard_normal((ncol, 5, L))
    du[:, 1:4] = 1e-3 * rng.standard_normal((ncol, 3, L))
    cth = 0.5 * rng.uniform(-1, 1, ncol)
    colgeo = np.stack([cth, np.sqrt(1 - cth ** 2),
                       np.pi / 2 / N * rng.uniform(0.8, 1.0, ncol),
                       np.pi / 2 / N * rng.uniform(0.8, 1.0, ncol)], axis=1)
    return w, du, colgeo, x1f, x1v, dx1f, cfg
