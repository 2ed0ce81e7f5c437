"""The mixed precisions against the FP64 oracle: EXO_PREC_MIXED (FP32
reconstruction, x2/x3 Riemann fluxes and their divergence; FP64
decomposition, x1 fluxes, implicit solve, equation of state and RK
accumulation) and EXO_PREC_MIXED_F32_SOLVE (the same with FP32 blocks in
the implicit solve).  Tolerance: relative L2 of density and pressure below 1e-6 after a
few steps (the configuration target is 1e-5 after 1000 steps, measured at
full size by bench.py --accuracy).  The implicit solve alone, on the same
inputs as the oracle's SolveImplicit3D: FP64 blocks within 1e-10 relative
L2 (reciprocals and a pivoted LU instead of Gauss-Jordan), FP32 blocks
within 1e-5 and not within 1e-9."""
import numpy as np
import pytest

from exocubed_b200 import _native as nat
from exocubed_b200 import workloads as W
from exocubed_b200.atmosphere import CubedSphereAtmosphere

pytestmark = pytest.mark.gpu


def pressure(u, gamma):
    rho = u[:, 0]
    ke = 0.5 * (u[:, 1] ** 2 + u[:, 2] ** 2 + u[:, 3] ** 2) / rho
    return (gamma - 1.0) * (u[:, 4] - ke)


@pytest.mark.parametrize("L", [16, 32])   # the per-face and the line form of x2/x3
@pytest.mark.parametrize("precision", [nat.EXO_PREC_MIXED, nat.EXO_PREC_MIXED_F32_SOLVE])
@pytest.mark.parametrize("rsolver", [1, 2])
def test_mixed_dry_atmosphere_close_to_oracle(oracle_mod, rsolver, precision, L):
    cfg = W.dry_atmosphere_config(N=12, L=L, rsolver=rsolver)
    state = W.dry_atmosphere_state(cfg, seed=31)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(state)
    o.step(4)
    g = CubedSphereAtmosphere(dict(cfg, precision=precision))
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


@pytest.mark.parametrize("implicit_flag", [1, 9])
def test_mixed_implicit_solve_against_oracle(oracle_mod, implicit_flag):
    cfg = dict(W.dry_atmosphere_config(N=8, L=24, rsolver=1), implicit_flag=implicit_flag)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(W.dry_atmosphere_state(cfg, seed=6))
    w = o.primitive()
    rng = np.random.default_rng(7)
    scale = np.abs(W.interior(w)).mean(axis=(0, 2, 3, 4))
    du = np.zeros_like(w)
    W.interior(du)[...] = 1e-4 * scale[None, :, None, None, None] * \
        rng.standard_normal(W.interior(du).shape)
    want = du.copy()
    o.solve_implicit_3d(want, w, 400.0)
    wi = W.interior(want)
    rel = {}
    for prec in (nat.EXO_PREC_MIXED, nat.EXO_PREC_MIXED_F32_SOLVE):
        got = du.copy()
        with CubedSphereAtmosphere(dict(cfg, precision=prec)) as a:
            a.set_primitive(W.dry_atmosphere_state(cfg, seed=6))
            a.solve_implicit_3d(got, w, 400.0)
        gi = W.interior(got)
        rel[prec] = max(np.linalg.norm(gi[:, n] - wi[:, n]) / np.linalg.norm(wi[:, n])
                        for n in (0, 1, 4))
    assert rel[nat.EXO_PREC_MIXED] < 1e-10, rel
    assert 1e-9 < rel[nat.EXO_PREC_MIXED_F32_SOLVE] < 1e-5, rel


def test_mixed_precisions_differ_only_in_the_implicit_solve():
    """Without the implicit solve the two mixed precisions step the same
    arithmetic (bit-identical); with it they differ."""
    for flag, same in ((0, True), (9, False)):
        cfg = W.dry_atmosphere_config(N=8, L=12, rsolver=1, implicit_flag=flag)
        state = W.dry_atmosphere_state(cfg, seed=12)
        out = []
        for prec in (nat.EXO_PREC_MIXED, nat.EXO_PREC_MIXED_F32_SOLVE):
            with CubedSphereAtmosphere(dict(cfg, precision=prec)) as a:
                a.set_primitive(state)
                a.step(3)
                out.append(a.conserved())
        assert np.array_equal(out[0], out[1]) == same, flag
