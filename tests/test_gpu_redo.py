"""The main loop's redo of failed steps (main.cpp.in:126-157,
src/mesh_redo.cpp:12-46) on the device: a step that leaves the state invalid
is taken again from the kept state with half the time step.  No GPU fault
is involved: the failure is an ordinary invalid state (negative pressure
after a step far above the CFL limit), which the context flags and reads
back."""
import numpy as np
import pytest

from exocubed_b200 import _native as nat
from exocubed_b200 import workloads as W
from exocubed_b200.atmosphere import CubedSphereAtmosphere

pytestmark = pytest.mark.gpu


def _cfg(**kw):
    return dict(W.dry_atmosphere_config(N=8, L=12, rsolver=nat.EXO_RS_HLLC), **kw)


PRECISIONS = [nat.EXO_PREC_FP64, nat.EXO_PREC_MIXED, nat.EXO_PREC_MIXED_F32_SOLVE]


@pytest.mark.parametrize("precision", PRECISIONS)
def test_fixed_step_redone_with_half_steps(precision):
    # in the mixed builds the retaken step must also start from the kept FP32
    # primitive copy, not from the failed step's
    cfg = _cfg(precision=precision)
    state = W.dry_atmosphere_state(cfg, seed=3)
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(state)
        dt_big = 16 * a.dt
        a.set_max_redo(10)
        a.step(1, dt_big)
        k = a.redo_count
        assert k >= 1 and a.invalid() == 0
        got, t = a.conserved(), a.time
    with CubedSphereAtmosphere(cfg) as b:
        b.set_primitive(state)
        b.step(1, dt_big / 2 ** k)
        assert np.array_equal(b.conserved(), got)
        assert b.time == t
        assert b.invalid() == 0
    with CubedSphereAtmosphere(cfg) as c:
        # without redo the same step leaves the state flagged invalid
        c.set_primitive(state)
        c.step(1, dt_big)
        assert c.invalid() == 1


@pytest.mark.parametrize("precision", PRECISIONS)
def test_cfl_step_redone_with_half_steps(precision):
    cfg = _cfg(cfl=1.5, precision=precision)
    state = W.dry_atmosphere_state(cfg, seed=3)
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(state)
        dt0 = a.dt
        a.set_max_redo(10)
        a.step(1)
        k = a.redo_count
        assert k >= 1 and a.invalid() == 0
        got = a.conserved()
        assert a.time == dt0 / 2 ** k
        assert 0 < a.dt <= 2 * dt0 / 2 ** k
        a.step(2)
        assert a.invalid() == 0
    with CubedSphereAtmosphere(cfg) as b:
        b.set_primitive(state)
        b.step(1, dt0 / 2 ** k)
        assert np.array_equal(b.conserved(), got)


def test_redo_budget_runs_out():
    cfg = _cfg()
    state = W.dry_atmosphere_state(cfg, seed=3)
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(state)
        before = a.conserved()
        dt_big = 64 * a.dt
        a.set_max_redo(1)
        with pytest.raises(nat.ExoError) as ei:
            a.step(1, dt_big)
        assert ei.value.code == nat.EXO_ERR_NONFINITE
        # the kept state is back in place: the run can go on with smaller steps
        assert np.array_equal(a.conserved(), before)
        assert a.redo_count == 3
        a.set_max_redo(0)
        a.step(1, dt_big / 64)
        assert a.invalid() == 0


def test_redo_rejects_an_invalid_start():
    cfg = _cfg()
    state = W.dry_atmosphere_state(cfg, seed=1)
    state[2, 4, 6, 6, 5] = -5.0
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(state)
        a.set_max_redo(3)
        with pytest.raises(nat.ExoError) as ei:
            a.step(1)
        assert ei.value.code == nat.EXO_ERR_NONFINITE
