"""implicit_flag = 1: the vertical implicit solve with PartialCorrection, the
3x3 block-tridiagonal system of (rho, m1, E) that the reference's own exo3
inputs select (examples/2023-Chen-exo3/hs94.inp:65, hot_jupiter.inp:64,
polar_dry.inp:59), against the oracle.

Tolerances as in test_gpu_parity.py: the solve itself uses only +, -, *, /
and sqrt, so the column hook, SolveImplicit3D and steps without gravity are
bit-exact in the FP64 build; steps with gravity go through the hydrostatic
decomposition (log, exp, pow) and are compared at 1e-9 relative L2; the
mixed build at 1e-6."""
import numpy as np
import pytest

from _columns import column_problem
from exocubed_b200 import _native as nat
from exocubed_b200 import workloads as W
from exocubed_b200.atmosphere import CubedSphereAtmosphere
from exocubed_b200.ensemble import Ensemble

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ncol,L,dt", [(1, 12, 30.0), (257, 16, 400.0), (1000, 40, 1500.0),
                                       (70, 250, 200.0)])
def test_partial_correction_columns_bitwise(oracle_mod, native, ncol, L, dt):
    torch = pytest.importorskip("torch")
    w, du, colgeo, x1f, x1v, dx1f, cfg = column_problem(oracle_mod, ncol, L, seed=ncol + 1)
    ref = oracle_mod.implicit_columns(w, du, colgeo, x1f, x1v, dx1f, dt, cfg["gamma"],
                                      cfg["grav"], full=False)
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda()
         for k, v in dict(w=w, du=du, g=colgeo, x1f=x1f, x1v=x1v, dx1f=dx1f).items()}
    scratch = torch.empty(ncol * L * 30, dtype=torch.float64, device="cuda")
    rc = native.lib().exo_partial_correction_columns(
        ncol, L, t["w"].data_ptr(), t["du"].data_ptr(), t["g"].data_ptr(), t["x1f"].data_ptr(),
        t["x1v"].data_ptr(), t["dx1f"].data_ptr(), dt, cfg["gamma"], cfg["grav"],
        scratch.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    got = t["du"].cpu().numpy()
    assert np.isfinite(got).all()
    assert np.array_equal(got, ref), np.abs(got - ref).max()
    assert np.array_equal(got[:, 2:4], du[:, 2:4])
    assert np.abs(got - du).max() > 0


def test_partial_correction_rejects_bad_args(native):
    L = native.lib()
    assert L.exo_partial_correction_columns(-1, 4, None, None, None, None, None, None, 1., 1.4,
                                            -9.8, None, None) == 1
    assert L.exo_partial_correction_columns(0, 4, None, None, None, None, None, None, 1., 1.4,
                                            -9.8, None, None) == 0


def test_solve_implicit_3d_partial_bitwise(oracle_mod):
    cfg = dict(W.dry_atmosphere_config(N=8, L=20, rsolver=2), implicit_flag=1)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(W.dry_atmosphere_state(cfg, seed=5))
    w = o.primitive()
    rng = np.random.default_rng(6)
    scale = np.abs(W.interior(w)).mean(axis=(0, 2, 3, 4))
    du = np.zeros_like(w)
    W.interior(du)[...] = 1e-4 * scale[None, :, None, None, None] * \
        rng.standard_normal(W.interior(du).shape)
    want = du.copy()
    o.solve_implicit_3d(want, w, 400.0)
    got = du.copy()
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(W.dry_atmosphere_state(cfg, seed=5))
        a.solve_implicit_3d(got, w, 400.0)
    assert np.array_equal(W.interior(got), W.interior(want)), \
        np.abs(W.interior(got) - W.interior(want)).max()
    assert np.array_equal(W.interior(got)[:, 2:4], W.interior(du)[:, 2:4])
    assert not np.array_equal(W.interior(got), W.interior(du))


def test_partial_steps_without_gravity_bitwise(oracle_mod):
    cfg = dict(W.dry_atmosphere_config(N=8, L=10, rsolver=2, grav=0.0), implicit_flag=1)
    state = W.dry_atmosphere_state(cfg, seed=9)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(state)
    g = CubedSphereAtmosphere(cfg)
    g.set_primitive(state)
    o.step(2, 50.0)
    g.step(2, 50.0)
    assert np.array_equal(W.interior(g.conserved()), W.interior(o.conserved()))


@pytest.mark.parametrize("rsolver", [1, 2])
def test_partial_steps_with_gravity(oracle_mod, rsolver):
    cfg = dict(W.dry_atmosphere_config(N=8, L=12, rsolver=rsolver), implicit_flag=1)
    state = W.dry_atmosphere_state(cfg, seed=8)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(state)
    g = CubedSphereAtmosphere(cfg)
    g.set_primitive(state)
    o.step(3)
    g.step(3)
    ug, uo = W.interior(g.conserved()), W.interior(o.conserved())
    for n in range(5):
        rel = np.linalg.norm(ug[:, n] - uo[:, n]) / np.linalg.norm(uo[:, n])
        assert rel < 1e-9, (n, rel)
    assert g.dt == pytest.approx(o.dt, rel=1e-9)
    assert g.invalid() == 0
    # the partial solve is a different step from the full one
    f = oracle_mod.Oracle(dict(cfg, implicit_flag=9))
    f.set_primitive(state)
    f.step(3)
    assert not np.array_equal(W.interior(f.conserved()), uo)


def test_partial_mixed_close_to_oracle(oracle_mod):
    """Density and pressure within 1e-6 (relative L2) of the FP64 oracle, as
    for the full correction; the momenta of this near-hydrostatic state are
    small, so their FP32 error is judged against the full correction's error
    under the same mixed build."""
    base = W.dry_atmosphere_config(N=12, L=16, rsolver=1)
    state = W.dry_atmosphere_state(base, seed=33)
    err = {}
    for flag in (1, 9):
        cfg = dict(base, implicit_flag=flag)
        o = oracle_mod.Oracle(cfg)
        o.set_primitive(state)
        o.step(4)
        g = CubedSphereAtmosphere(dict(cfg, precision=nat.EXO_PREC_MIXED))
        g.set_primitive(state)
        g.step(4)
        assert g.invalid() == 0
        ug, uo = W.interior(g.conserved()), W.interior(o.conserved())
        err[flag] = [np.linalg.norm(ug[:, n] - uo[:, n]) / np.linalg.norm(uo[:, n])
                     for n in range(5)]
    e1, e9 = err[1], err[9]
    assert e1[0] < 1e-6 and e1[4] < 1e-6, e1
    for n in (1, 2, 3):
        assert e1[n] < 10 * e9[n] + 1e-6, (n, e1, e9)


@pytest.mark.parametrize("precision", [nat.EXO_PREC_FP64, nat.EXO_PREC_MIXED,
                                       nat.EXO_PREC_MIXED_F32_SOLVE])
def test_partial_and_full_members_in_one_batch(precision):
    """A batch may mix members of both corrections: each member's result is
    the one it has alone."""
    cfgs = [dict(W.dry_atmosphere_config(N=8, L=12, rsolver=1), implicit_flag=1,
                 precision=precision),
            dict(W.dry_atmosphere_config(N=10, L=8, rsolver=2), implicit_flag=9,
                 precision=precision),
            dict(W.dry_atmosphere_config(N=6, L=16, rsolver=1), implicit_flag=1,
                 precision=precision)]
    states = [W.dry_atmosphere_state(c, seed=40 + n) for n, c in enumerate(cfgs)]
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
