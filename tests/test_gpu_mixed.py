"""Mixed precision (FP32 reconstruction, Riemann flux and flux divergence;
FP64 decomposition, implicit solve, equation of state and RK accumulation)
against the FP64 oracle.  Tolerance: relative L2 of density, pressure and
momenta below 1e-6 after a few steps (the configuration target is 1e-5
after 1000 steps, measured at full size by bench.py --accuracy)."""
import numpy as np
import pytest

from exocubed_b200 import workloads as W
from exocubed_b200.atmosphere import CubedSphereAtmosphere

pytestmark = pytest.mark.gpu


def pressure(u, gamma):
    rho = u[:, 0]
    ke = 0.5 * (u[:, 1] ** 2 + u[:, 2] ** 2 + u[:, 3] ** 2) / rho
    return (gamma - 1.0) * (u[:, 4] - ke)


@pytest.mark.parametrize("rsolver", [1, 2])
def test_mixed_dry_atmosphere_close_to_oracle(oracle_mod, rsolver):
    cfg = W.dry_atmosphere_config(N=12, L=16, rsolver=rsolver)
    state = W.dry_atmosphere_state(cfg, seed=31)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(state)
    o.step(4)
    g = CubedSphereAtmosphere(dict(cfg, precision=1))
    g.set_primitive(state)
    g.step(4)
    ug, uo = W.interior(g.conserved()), W.interior(o.conserved())
    rel_rho = np.linalg.norm(ug[:, 0] - uo[:, 0]) / np.linalg.norm(uo[:, 0])
    pg, po = pressure(ug, cfg["gamma"]), pressure(uo, cfg["gamma"])
    rel_p = np.linalg.norm(pg - po) / np.linalg.norm(po)
    assert rel_rho < 1e-6 and rel_p < 1e-6, (rel_rho, rel_p)
    assert g.invalid() == 0
    # FP32 is really used: the mixed result is not the FP64 one
    assert not np.array_equal(ug, uo)


def test_mixed_shallow_water_close_to_oracle(oracle_mod):
    cfg = W.shallow_water_config(N=16)
    state = W.shallow_water_state(cfg, seed=32)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(state)
    o.step(5)
    g = CubedSphereAtmosphere(dict(cfg, precision=1))
    g.set_primitive(state)
    g.step(5)
    ug, uo = W.interior(g.conserved()), W.interior(o.conserved())
    rel = np.linalg.norm(ug[:, 0] - uo[:, 0]) / np.linalg.norm(uo[:, 0])
    assert rel < 1e-6, rel
    assert g.dt == pytest.approx(o.dt, rel=1e-5)
