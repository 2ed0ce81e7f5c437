"""User sources on the device against the oracle: the Held-Suarez forcing
(examples/2023-Chen-exo3/hs94.cpp:59-155) and CalculateCoriolisForce3
(src/exo3/cubed_sphere.cpp:197-231).

Tolerances as in test_gpu_parity.py: the Coriolis forms use only +, -, *, /
on host-computed tables, so without gravity (no decomposition) the FP64
steps are bit-exact; the Held-Suarez cooling calls log and pow and the
hydrostatic decomposition log, exp and pow, so those steps are compared at
1e-9 relative L2 (FP64) and 1e-6 for density and pressure (mixed)."""
import numpy as np
import pytest

from exocubed_b200 import _native as nat
from exocubed_b200 import workloads as W
from exocubed_b200.atmosphere import CubedSphereAtmosphere
from exocubed_b200.ensemble import Ensemble

pytestmark = pytest.mark.gpu


def _pair(oracle_mod, cfg, state):
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(state)
    g = CubedSphereAtmosphere(cfg)
    g.set_primitive(state)
    return o, g


def test_coriolis3_without_gravity_bitwise(oracle_mod):
    cfg = W.dry_atmosphere_config(N=8, L=10, rsolver=nat.EXO_RS_HLLC, grav=0.0,
                                  coriolis=nat.EXO_CORIOLIS_3D, omega=7.292e-5)
    state = W.dry_atmosphere_state(cfg, seed=9)
    o, g = _pair(oracle_mod, cfg, state)
    o.step(2, 50.0)
    g.step(2, 50.0)
    assert np.array_equal(W.interior(g.conserved()), W.interior(o.conserved()))
    # the source is on: the step differs from one without it
    n = oracle_mod.Oracle(dict(cfg, coriolis=nat.EXO_CORIOLIS_NONE))
    n.set_primitive(state)
    n.step(2, 50.0)
    assert not np.array_equal(W.interior(n.conserved()), W.interior(o.conserved()))


@pytest.mark.parametrize("implicit_flag", [1, 9])
def test_hs94_steps(oracle_mod, implicit_flag):
    cfg = W.hs94_config(N=8, L=20, cfl=0.4, implicit_flag=implicit_flag)
    state = W.hs94_state(cfg, seed=2)
    o, g = _pair(oracle_mod, cfg, state)
    o.step(3)
    g.step(3)
    ug, uo = W.interior(g.conserved()), W.interior(o.conserved())
    for n in range(5):
        rel = np.linalg.norm(ug[:, n] - uo[:, n]) / np.linalg.norm(uo[:, n])
        assert rel < 1e-9, (n, rel)
    assert g.dt == pytest.approx(o.dt, rel=1e-9)
    assert g.invalid() == 0
    n = oracle_mod.Oracle(dict(cfg, forcing=nat.EXO_FORCING_NONE))
    n.set_primitive(state)
    n.step(3)
    assert not np.array_equal(W.interior(n.conserved()), uo)


def test_hs94_mixed_close_to_oracle(oracle_mod):
    cfg = W.hs94_config(N=12, L=16, cfl=0.4)
    state = W.hs94_state(cfg, seed=5)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(state)
    o.step(4)
    g = CubedSphereAtmosphere(dict(cfg, precision=nat.EXO_PREC_MIXED))
    g.set_primitive(state)
    g.step(4)
    ug, uo = W.interior(g.conserved()), W.interior(o.conserved())
    for n in (0, 4):
        rel = np.linalg.norm(ug[:, n] - uo[:, n]) / np.linalg.norm(uo[:, n])
        assert rel < 1e-6, (n, rel)
    assert g.invalid() == 0


@pytest.mark.parametrize("precision", [nat.EXO_PREC_FP64, nat.EXO_PREC_MIXED,
                                       nat.EXO_PREC_MIXED_F32_SOLVE])
def test_forced_and_unforced_members_in_one_batch(precision):
    cfgs = [dict(W.hs94_config(N=8, L=20, cfl=0.4), precision=precision),
            dict(W.dry_atmosphere_config(N=10, L=8, rsolver=nat.EXO_RS_HLLC,
                                         coriolis=nat.EXO_CORIOLIS_3D, omega=7.292e-5),
                 precision=precision),
            dict(W.dry_atmosphere_config(N=6, L=16), precision=precision)]
    states = [W.hs94_state(cfgs[0], seed=1), W.dry_atmosphere_state(cfgs[1], seed=2),
              W.dry_atmosphere_state(cfgs[2], seed=3)]
    alone = []
    for c, s in zip(cfgs, states):
        with CubedSphereAtmosphere(c) as a:
            a.set_primitive(s)
            a.step(3)
            alone.append(a.conserved())
    with Ensemble(precision=precision, capacity=4) as e:
        slots = [e.add(c, s) for c, s in zip(cfgs, states)]
        e.step(3)
        for slot, want in zip(slots, alone):
            assert np.array_equal(e.conserved(slot), want)
            assert e.invalid(slot) == 0


@pytest.mark.parametrize("precision", [nat.EXO_PREC_FP64, nat.EXO_PREC_MIXED])
def test_hs94_at_its_own_size(oracle_mod, precision):
    """The Held-Suarez workload as its input file sets it up (6 x 40 x 40 x
    40, HLLC, implicit_flag 1, CFL 0.9, forcing on), 5 CFL steps against the
    oracle: FP64 every conserved variable to 1e-9 relative L2, mixed density
    and total energy to 1e-6."""
    cfg = W.hs94_config()
    state = W.hs94_state(cfg, seed=0)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(state)
    o.step(5)
    assert o.invalid() == 0
    with CubedSphereAtmosphere(dict(cfg, precision=precision)) as g:
        g.set_primitive(state)
        g.step(5)
        assert g.invalid() == 0
        assert g.dt == pytest.approx(o.dt, rel=1e-9 if precision == nat.EXO_PREC_FP64 else 1e-5)
        ug = W.interior(g.conserved())
    uo = W.interior(o.conserved())
    vars_, tol = ((range(5), 1e-9) if precision == nat.EXO_PREC_FP64 else ((0, 4), 1e-6))
    for n in vars_:
        rel = np.linalg.norm(ug[:, n] - uo[:, n]) / np.linalg.norm(uo[:, n])
        assert rel < tol, (n, rel)
