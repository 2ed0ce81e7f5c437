"""Batched ensemble (many independent atmospheres in one graph-captured
step): every member's state after k steps must be bitwise equal to the same
configuration advanced alone in its own context, in both precisions, across
membership changes; admission must refuse members beyond the slots or the
memory budget."""
import numpy as np
import pytest

from exocubed_b200 import CubedSphereAtmosphere
from exocubed_b200 import _native as nat
from exocubed_b200 import workloads as W
from exocubed_b200.ensemble import Ensemble, footprint

pytestmark = pytest.mark.gpu


def _members(precision):
    """Uneven members: sizes, levels (32 takes the x2/x3 line form, the
    others the per-face form), solvers, gases and one shallow-water sphere
    (fp64 only: its own equation set and variable count)."""
    out = []
    for n, (N, L, rs) in enumerate([(8, 12, nat.EXO_RS_LMARS), (12, 8, nat.EXO_RS_HLLC),
                                    (6, 32, nat.EXO_RS_LMARS), (10, 16, nat.EXO_RS_HLLC)]):
        cfg = W.dry_atmosphere_config(N=N, L=L, rsolver=rs, T0=200. + 20 * n,
                                      g=5. + 4 * n, gamma=1.3 + 0.1 * n, precision=precision)
        out.append((cfg, W.dry_atmosphere_state(cfg, seed=40 + n)))
    cfg = W.ensemble_member(7, precision=precision)[0]
    cfg.update(N=8, L=10)
    out.append((cfg, W.dry_atmosphere_state(cfg, seed=47)))
    cfg = W.dry_atmosphere_config(N=8, L=12, implicit_flag=0, precision=precision)
    out.append((cfg, W.dry_atmosphere_state(cfg, seed=48)))
    if precision == nat.EXO_PREC_FP64:
        cfg = W.shallow_water_config(N=10)
        out.append((cfg, W.shallow_water_state(cfg, seed=49)))
    return out


def _alone(cfg, w, nsteps):
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(w)
        a.step(nsteps)
        return a.conserved(), a.time


@pytest.mark.parametrize("precision", [nat.EXO_PREC_FP64, nat.EXO_PREC_MIXED,
                                       nat.EXO_PREC_MIXED_F32_SOLVE])
def test_members_equal_alone_and_in_the_mix(precision):
    members = _members(precision)
    ens = Ensemble(precision=precision, capacity=16)
    slots = [ens.add(c, w) for c, w in members]
    ens.step(3)
    ens.synchronize()
    for (c, w), s in zip(members, slots):
        want, t = _alone(c, w, 3)
        got = ens.conserved(s)
        assert np.isfinite(got).all()
        assert np.array_equal(got, want), (c["N"], c["L"], np.abs(got - want).max())
        tm, dt, ncyc = ens.member_time(s)
        assert ncyc == 3 and tm == t
    st = ens.stats()
    assert st["members"] == len(members)
    assert st["bytes"] == sum(footprint(dict(c, precision=precision)) for c, _ in members)
    ens.close()


def test_membership_changes_keep_members_exact():
    prec = nat.EXO_PREC_MIXED
    members = _members(prec)
    ens = Ensemble(precision=prec, capacity=8)
    a = ens.add(*members[0])
    b = ens.add(*members[1])
    ens.step(2)
    ens.remove(a)                      # leaves mid-run
    c = ens.add(*members[2])           # takes the freed slot
    assert c == a
    ens.step(2)
    d = ens.add(*members[3])           # joins late
    ens.step(1)
    ens.synchronize()
    assert np.array_equal(ens.conserved(b), _alone(*members[1], 5)[0])
    assert np.array_equal(ens.conserved(c), _alone(*members[2], 3)[0])
    assert np.array_equal(ens.conserved(d), _alone(*members[3], 1)[0])
    ens.close()


def test_admission_refuses_beyond_slots_and_budget():
    prec = nat.EXO_PREC_FP64
    (c0, w0), (c1, w1) = _members(prec)[:2]
    ens = Ensemble(precision=prec, capacity=1)
    ens.add(c0, w0)
    assert ens.try_add(c1, w1) is None
    with pytest.raises(nat.ExoError) as e:
        ens.add(c1, w1)
    assert e.value.code == 7 and "slot" in str(e.value)
    ens.close()
    ens = Ensemble(precision=prec, capacity=4, budget_bytes=footprint(c0) + footprint(c1) - 1)
    ens.add(c0, w0)
    with pytest.raises(nat.ExoError) as e:
        ens.add(c1, w1)
    assert e.value.code == 7 and "budget" in str(e.value)
    with pytest.raises(nat.ExoError) as e:  # precision differs from the ensemble's
        ens.add(dict(c1, precision=nat.EXO_PREC_MIXED), w1)
    assert e.value.code == 1
    ens.close()
