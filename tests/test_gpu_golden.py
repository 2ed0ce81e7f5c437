"""The CUDA path against the frozen oracle outputs of tests/golden/ (the
cases without transcendental functions in the step are bit-exact)."""
import os

import numpy as np
import pytest

from exocubed_b200 import workloads as W
from exocubed_b200.atmosphere import CubedSphereAtmosphere

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_gpu_matches_frozen_outputs():
    frozen = np.load(os.path.join(GOLD, "oracle_small.npz"))
    cfg = W.shallow_water_config(N=8)
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(W.shallow_water_state(cfg, seed=0))
        a.step(5)
        assert np.array_equal(W.interior(a.conserved()), frozen["c1_u"])
        assert a.dt == frozen["c1_dt"][0]
    cfg = W.dry_atmosphere_config(N=8, L=6, rsolver=2, grav=0.0)
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(W.dry_atmosphere_state(cfg, seed=1))
        a.step(2, 50.0)
        assert np.array_equal(W.interior(a.conserved()), frozen["dry_u"])
    cfg = W.hs94_config(N=8, L=20, cfl=0.4)
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(W.hs94_state(cfg, seed=2))
        a.step(2)
        u = W.interior(a.conserved())
    np.testing.assert_allclose([np.linalg.norm(u[:, n]) for n in range(5)],
                               frozen["hs94_norms"], rtol=1e-9)
