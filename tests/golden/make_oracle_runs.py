"""Generates tests/golden/oracle_c2_lmars.npz: a long run of the oracle on the
C2 workload, the FP64 reference that the mixed path's accuracy bar (1e-5
relative L2 after 1000 steps) is measured against (run from the repository
root on the CPU, about half an hour on 8 cores:
python tests/golden/make_oracle_runs.py).

Workload: the exo3 dry ideal-gas atmosphere, 6 panels x 96 x 96 x 64 levels,
WENO5 + LMARS + the 5x5 implicit vertical solve (implicit_flag 9), SSPRK(3,3),
seeded state 0 (isothermal 250 K, 1 K temperature noise, 5 m/s winds).  The
state is generated on the oracle's own mesh.  The oracle takes its first CFL
time step and holds it fixed for the whole run, so a GPU run given the same
dt takes the same steps.

Stored, after 10, 100 and 1000 steps: the primitive variables (rho, v1, v2,
v3, p) at 8192 interior cells drawn uniformly with a seeded generator, the
L2 norm and the largest magnitude of each variable over all interior cells,
the simulated time and the invalid-state flag.  The full state (140 MB) is
not kept; relative errors of a GPU run are estimated on the sampled cells.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from exocubed_b200 import workloads as W  # noqa: E402
from oracle import oracle  # noqa: E402

OUT = os.path.join(HERE, "oracle_c2_lmars.npz")
CHECKPOINTS = (10, 100, 1000)
NSAMPLE = 8192
G = 3


def c2_config():
    return W.dry_atmosphere_config(N=96, L=64, rsolver=1)


def sample_cells(N, L, n=NSAMPLE, seed=20261203):
    """(panel, k, j, i) indices of n distinct interior cells, ghosts offset."""
    rng = np.random.Generator(np.random.PCG64(seed))
    flat = rng.choice(6 * N * N * L, size=n, replace=False)
    p, r = np.divmod(flat, N * N * L)
    k, r = np.divmod(r, N * L)
    j, i = np.divmod(r, L)
    return np.stack([p, k + G, j + G, i + G]).astype(np.int64)


def main():
    cfg = c2_config()
    o = oracle.Oracle(cfg)
    o.set_primitive(W.dry_atmosphere_state(cfg, seed=0, geometry=oracle.cell_geometry))
    dt = o.dt
    idx = sample_cells(cfg["N"], cfg["L"])
    rec = {"N": cfg["N"], "L": cfg["L"], "rsolver": cfg["rsolver"], "seed": 0, "dt": dt,
           "checkpoints": np.array(CHECKPOINTS), "cells": idx}
    done = 0
    t0 = time.time()
    for n in CHECKPOINTS:
        o.step(n - done, dt)
        done = n
        w = o.primitive()[:, :, G:-G, G:-G, G:-G]
        full = o.primitive()
        rec[f"sample_{n}"] = full[idx[0], :, idx[1], idx[2], idx[3]].T.copy()
        rec[f"l2_{n}"] = np.sqrt((w * w).sum(axis=(0, 2, 3, 4)))
        rec[f"max_{n}"] = np.abs(w).max(axis=(0, 2, 3, 4))
        rec[f"time_{n}"] = o.time
        rec[f"invalid_{n}"] = o.invalid()
        print(f"step {n}: t = {o.time:.1f} s, invalid {o.invalid()}, "
              f"{time.time() - t0:.0f} s elapsed", flush=True)
    np.savez_compressed(OUT, **rec)


if __name__ == "__main__":
    main()
