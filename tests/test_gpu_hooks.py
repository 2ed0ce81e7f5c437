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


def test_decomposition_hooks_match_the_oracle(oracle_mod):
    """ChangeToPerturbation / RestoreFromPerturbation on whole arrays: the
    perturbations and restored face states agree with the oracle to 1e-12
    relative (both call log/exp/pow, whose CUDA and glibc results may differ
    in the last bit); the restored cell values are the original ones to the
    bit."""
    cfg = W.dry_atmosphere_config(N=8, L=16)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(W.dry_atmosphere_state(cfg, seed=11))
    w0 = o.primitive()
    rng = np.random.default_rng(12)
    wl0 = np.zeros_like(w0)
    wr0 = np.zeros_like(w0)
    for a in (wl0, wr0):  # perturbation-sized face states, some negative
        a[:, 0] = 0.02 * rng.standard_normal(a[:, 0].shape)
        a[:, 4] = 300.0 * rng.standard_normal(a[:, 4].shape)
    w_o, w_g = w0.copy(), w0.copy()
    o.change_to_perturbation(w_o)
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(W.dry_atmosphere_state(cfg, seed=11))
        a.change_to_perturbation(w_g)
        inner = (slice(None), [0, 4], slice(3, -3), slice(3, -3), slice(None))
        d = np.abs(w_g[inner] - w_o[inner]).max()
        assert d <= 1e-12 * np.abs(w0[inner]).max(), d
        assert not np.array_equal(w_g[inner], w0[inner])
        wl_o, wr_o, wl_g, wr_g = wl0.copy(), wr0.copy(), wl0.copy(), wr0.copy()
        o.restore_from_perturbation(w_o, wl_o, wr_o)
        a.restore_from_perturbation(w_g, wl_g, wr_g)
    assert np.array_equal(w_g[inner], w0[inner]) and np.array_equal(w_o[inner], w0[inner])
    faces = (slice(None), [0, 4], slice(3, -3), slice(3, -3), slice(3, -2))
    for g, r in ((wl_g, wl_o), (wr_g, wr_o)):
        assert np.abs(g[faces] - r[faces]).max() <= 1e-12 * np.abs(r[faces]).max()
        assert (g[faces][:, 1] > 0).all() and (g[faces][:, 0] > 0).all()


def test_restore_needs_a_decomposition_first():
    cfg = W.dry_atmosphere_config(N=6, L=8)
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(W.dry_atmosphere_state(cfg, seed=1))
        w = a.primitive()
        with pytest.raises(nat.ExoError) as e:
            a.restore_from_perturbation(w, w.copy(), w.copy())
        assert e.value.code == 1
