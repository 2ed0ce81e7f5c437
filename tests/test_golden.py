"""The golden fixtures of tests/golden/ (made by tests/golden/make_golden.py):
the oracle reproduces the reference's known-answer tests as recorded there,
and its outputs on the small seeded cases are the frozen ones."""
import json
import os

import numpy as np
import pytest

from _columns import column_problem
from exocubed_b200 import workloads as W

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def kats():
    with open(os.path.join(GOLD, "reference_kats.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def frozen():
    return np.load(os.path.join(GOLD, "oracle_small.npz"))


def _ulps(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.abs(a.view(np.int64) - b.view(np.int64))


def test_reference_weno_kats(oracle_mod, kats):
    k = kats["interp_weno5"]
    assert abs(oracle_mod.interp_weno5(*k["args"]) - k["expected"]) < k["tol"]
    k = kats["interp_weno3"]
    assert abs(oracle_mod.interp_weno3(*k["args"]) - k["expected"]) < k["tol"]


def test_reference_transform_kats(oracle_mod, kats):
    k = kats["CovariantToContravariant"]
    assert (_ulps(oracle_mod.cov_to_contra(k["w"], k["cth"]), k["expected"]) <= k["ulps"]).all()
    k = kats["ContravariantToCovariant"]
    assert (_ulps(oracle_mod.contra_to_cov(k["w"], k["cth"]), k["expected"]) <= k["ulps"]).all()


def test_oracle_matches_frozen_outputs(oracle_mod, frozen):
    cfg = W.shallow_water_config(N=8)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(W.shallow_water_state(cfg, seed=0))
    o.step(5)
    assert np.array_equal(W.interior(o.conserved()), frozen["c1_u"])
    assert o.dt == frozen["c1_dt"][0]
    cfg = W.dry_atmosphere_config(N=8, L=6, rsolver=2, grav=0.0)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(W.dry_atmosphere_state(cfg, seed=1))
    o.step(2, 50.0)
    assert np.array_equal(W.interior(o.conserved()), frozen["dry_u"])
    cfg = W.hs94_config(N=8, L=20, cfl=0.4)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(W.hs94_state(cfg, seed=2))
    o.step(2)
    u = W.interior(o.conserved())
    # log/exp/pow of the host's libm enter here: equal to rounding
    np.testing.assert_allclose([np.linalg.norm(u[:, n]) for n in range(5)],
                               frozen["hs94_norms"], rtol=1e-12)
    np.testing.assert_allclose(u[0], frozen["hs94_panel0"], rtol=1e-10, atol=1e-12)
    for full in (True, False):
        w, du, colgeo, x1f, x1v, dx1f, c = column_problem(oracle_mod, 4, 8, seed=3)
        out = oracle_mod.implicit_columns(w, du, colgeo, x1f, x1v, dx1f, 300.0, c["gamma"],
                                          c["grav"], full=full)
        assert np.array_equal(out, frozen["columns_full" if full else "columns_partial"])
