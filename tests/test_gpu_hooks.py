"""The finer-grained operator hooks of the C ABI: a stage at a time
(DoTaskListOneStage), the boundary exchange with ConservedToPrimitive, and
SolveImplicit3D on caller arrays."""
import numpy as np
import pytest

from exocubed_b200 import CubedSphereAtmosphere
from exocubed_b200 import _native as nat
from exocubed_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [nat.EXO_PREC_FP64, nat.EXO_PREC_MIXED])
@pytest.mark.parametrize("kind", ["dry", "shallow"])
def test_three_stages_equal_one_step(precision, kind):
    if kind == "dry":
        cfg = W.dry_atmosphere_config(N=10, L=16, precision=precision)
        w = W.dry_atmosphere_state(cfg, seed=70)
    else:
        cfg = W.shallow_water_config(N=12, precision=precision)
        w = W.shallow_water_state(cfg, seed=70)
    with CubedSphereAtmosphere(cfg) as a, CubedSphereAtmosphere(cfg) as b:
        a.set_primitive(w)
        b.set_primitive(w)
        a.step(2)
        for _ in range(2):
            for s in range(3):
                b.stage(s)
        assert a.time == b.time and a.dt == b.dt
        assert np.array_equal(a.conserved(), b.conserved())
        assert np.array_equal(a.primitive(), b.primitive())


def test_stage_rejects_bad_index():
    cfg = W.dry_atmosphere_config(N=6, L=8)
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(W.dry_atmosphere_state(cfg, seed=1))
        with pytest.raises(nat.ExoError) as e:
            a.stage(3)
        assert e.value.code == 1


def test_boundary_reproduces_the_primitives():
    cfg = W.dry_atmosphere_config(N=8, L=12)
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(W.dry_atmosphere_state(cfg, seed=2))
        a.step(1)
        w0 = a.primitive()
        a.boundary()
        assert np.array_equal(a.primitive(), w0)


def test_solve_implicit_3d_bitwise_with_oracle(oracle_mod):
    cfg = W.dry_atmosphere_config(N=8, L=20, rsolver=2)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(W.dry_atmosphere_state(cfg, seed=3))
    w = o.primitive()
    rng = np.random.default_rng(4)
    scale = np.abs(W.interior(w)).mean(axis=(0, 2, 3, 4))
    du = np.zeros_like(w)
    W.interior(du)[...] = 1e-4 * scale[None, :, None, None, None] * \
        rng.standard_normal(W.interior(du).shape)
    want = du.copy()
    o.solve_implicit_3d(want, w, 400.0)
    got = du.copy()
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(W.dry_atmosphere_state(cfg, seed=3))
        a.solve_implicit_3d(got, w, 400.0)
    assert np.isfinite(W.interior(got)).all()
    assert np.array_equal(W.interior(got), W.interior(want)), \
        np.abs(W.interior(got) - W.interior(want)).max()
    assert not np.array_equal(W.interior(got), W.interior(du))
