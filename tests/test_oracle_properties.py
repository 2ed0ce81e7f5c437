"""Size-independent properties of the oracle's cubed-sphere step.

These check the restatement itself (no GPU): the mesh, a state at rest,
finite evolution of the configurations' synthetic states, panel symmetry of
the ghost exchange on a uniform field.
"""
import numpy as np
import pytest

from exocubed_b200 import workloads as W

G = 3


def _oracle(oracle_mod, cfg):
    return oracle_mod.Oracle(cfg)


def test_mesh_spans_panel(oracle_mod):
    o = _oracle(oracle_mod, W.shallow_water_config(N=12))
    for p in range(6):
        x1f, x2f, x3f = o.mesh(p)
        assert x2f[G] == pytest.approx(-np.pi / 4, abs=1e-15)
        assert x2f[G + 12] == pytest.approx(np.pi / 4, abs=1e-15)
        assert x3f[G] == pytest.approx(-np.pi / 4, abs=1e-15)
        assert np.all(np.diff(x2f) > 0) and np.all(np.diff(x3f) > 0)
        assert x1f[G] == 6371000. and x1f[G + 3] == 6371001.


def test_uniform_shallow_state_ghosts_and_rest(oracle_mod):
    cfg = W.shallow_water_config(N=12, coriolis=0)
    o = _oracle(oracle_mod, cfg)
    w = np.zeros(o.shape)
    w[:, 0, G:-G, G:-G, G:-G] = 2.94e4
    o.set_primitive(w)
    wp = o.primitive()
    # every ghost band holds the uniform geopotential and no wind
    band = wp[:, 0, G:-G, :G, G:-G]
    np.testing.assert_allclose(band, 2.94e4, rtol=1e-15)
    assert np.abs(wp[:, 2:4, G:-G, :G, G:-G]).max() == 0.0
    u0 = o.conserved()
    o.step(2)
    u1 = o.conserved()
    # a resting, uniform layer stays at rest up to roundoff
    assert np.abs(W.interior(u1)[:, 0] - W.interior(u0)[:, 0]).max() < 1e-8
    assert np.abs(W.interior(u1)[:, 2:4]).max() < 1e-6


def test_shallow_water_config_evolves_finite(oracle_mod):
    cfg = W.shallow_water_config(N=12)
    o = _oracle(oracle_mod, cfg)
    o.set_primitive(W.shallow_water_state(cfg, seed=1))
    dt0 = o.dt
    assert 100. < dt0 < 5000.
    o.step(5)
    u = o.conserved()
    assert np.isfinite(W.interior(u)).all()
    assert o.time > 4 * dt0


@pytest.mark.parametrize("rsolver", [1, 2])
def test_dry_atmosphere_evolves_finite(oracle_mod, rsolver):
    cfg = W.dry_atmosphere_config(N=8, L=12, rsolver=rsolver)
    o = _oracle(oracle_mod, cfg)
    o.set_primitive(W.dry_atmosphere_state(cfg, seed=2))
    o.step(3)
    assert np.isfinite(W.interior(o.conserved())).all()
    assert o.invalid() == 0


def test_hllc_rest_state_balanced(oracle_mod):
    # HLLC projects fluxes to the covariant basis, so an isothermal column at
    # rest stays close to rest; LMARS does not project (lmars.cpp:24-110)
    cfg = W.dry_atmosphere_config(N=8, L=12, rsolver=2)
    o = _oracle(oracle_mod, cfg)
    o.set_primitive(W.dry_atmosphere_state(cfg, seed=0, temp_sigma=0., wind_sigma=0.))
    o.step(2, 600.)
    assert np.abs(W.interior(o.primitive())[:, 2:4]).max() < 1.0


def test_oracle_decomposition_round_trip(oracle_mod):
    """ChangeToPerturbation then RestoreFromPerturbation: the cell values come
    back to the bit, the perturbation pressure is small against the pressure
    (the hydrostatic part is removed) and restored face states stay positive."""
    from exocubed_b200 import workloads as W
    cfg = W.dry_atmosphere_config(N=6, L=12)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(W.dry_atmosphere_state(cfg, seed=2))
    w0 = o.primitive()
    w = w0.copy()
    o.change_to_perturbation(w)
    pi, p0 = W.interior(w)[:, 4], W.interior(w0)[:, 4]
    assert (np.abs(pi) < 0.02 * np.abs(p0)).all()
    wl = np.zeros_like(w)
    wr = np.zeros_like(w)
    wl[:, 4] = -1e9                  # a face state that must fall back to psf
    o.restore_from_perturbation(w, wl, wr)
    assert np.array_equal(W.interior(w), W.interior(w0))
    faces = (slice(None), slice(None), slice(3, -3), slice(3, -3), slice(3, -2))
    assert (wl[faces][:, 4] > 0).all() and (wr[faces][:, 4] > 0).all()
    assert (wl[faces][:, 0] > 0).all()


@pytest.mark.parametrize("case", ["shallow", "dry_lmars", "dry_hllc_partial"])
def test_second_ghost_pass_changes_nothing(oracle_mod, case):
    """The reference syncs the panel ghosts twice per stage and at start-up
    (patches/24.time_integrator.patch:22-28, patches/29.mesh.patch:19-86).
    With one block per panel the second pass reads the same interior cells
    as the first, so the oracle (and the CUDA path) run one pass: running
    both passes leaves every value of the run, ghosts included, unchanged."""
    if case == "shallow":
        cfg = W.shallow_water_config(N=8)
        state, steps = W.shallow_water_state(cfg, seed=2), 4
    else:
        rs, flag = (1, 9) if case == "dry_lmars" else (2, 1)
        cfg = W.dry_atmosphere_config(N=8, L=10, rsolver=rs, implicit_flag=flag)
        state, steps = W.dry_atmosphere_state(cfg, seed=2), 3
    out = []
    for passes in (1, 2):
        o = oracle_mod.Oracle(cfg)
        o.set_ghost_passes(passes)
        o.set_primitive(state)
        o.step(steps)
        out.append((o.conserved(), o.primitive(), o.dt, o.time))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2] and out[0][3] == out[1][3]
