"""The MCMC driver's forward models on the GPU: a batch of walkers run as
members of one ensemble gives each walker the values it gets alone on its own
context, so the sampler's chain does not depend on the batching."""
import numpy as np
import pytest

from exocubed_b200 import _native as nat
from exocubed_b200.inversion import (EnsembleForward, SequentialForward, StretchSampler,
                                     profile_problem)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [nat.EXO_PREC_FP64, nat.EXO_PREC_MIXED])
def test_batched_forward_equals_one_at_a_time(precision):
    build, observe, nvalue = profile_problem(N=8, L=12, steps=3)
    theta = np.array([[280., 200.], [300., 180.], [250., 230.], [320., 150.], [270., 260.]])
    fb = EnsembleForward(build, observe, nvalue, 3, precision=precision, capacity=3)
    try:
        got = fb(theta)
    finally:
        fb.close()
    want = SequentialForward(build, observe, nvalue, 3, precision=precision)(theta)
    assert np.isfinite(got).all()
    assert np.array_equal(got, want)
    # the profiles differ between walkers (the parameters matter)
    assert np.abs(got[0] - got[1]).max() > 1.0


def test_chain_does_not_depend_on_batching():
    build, observe, nvalue = profile_problem(N=8, L=12, steps=3)
    seq = SequentialForward(build, observe, nvalue, 3, precision=nat.EXO_PREC_MIXED)
    obs = seq(np.array([[285., 205.]]))[0]

    def log_prob(theta, val):
        Ts, Ttop = theta
        if not (200. < Ts < 350. and 150. < Ttop < Ts) or np.isnan(val).any():
            return -np.inf
        return float(-0.5 * (((val - obs) / 2.0) ** 2).sum())

    rng = np.random.default_rng(0)
    pos = np.stack([280. + 5 * rng.standard_normal(6), 200. + 5 * rng.standard_normal(6)], 1)
    fb = EnsembleForward(build, observe, nvalue, 3, precision=nat.EXO_PREC_MIXED, capacity=8)
    try:
        a = StretchSampler(fb, log_prob, 6, 2, nvalue, seed=11).run(pos, 2)
    finally:
        fb.close()
    b = StretchSampler(SequentialForward(build, observe, nvalue, 3, precision=nat.EXO_PREC_MIXED),
                       log_prob, 6, 2, nvalue, seed=11).run(pos, 2)
    for t in range(3):
        assert np.array_equal(a.par[t], b.par[t])
        assert np.array_equal(a.lnp[t], b.lnp[t])
    assert a.accept == b.accept


@pytest.mark.parametrize("precision", [nat.EXO_PREC_FP64, nat.EXO_PREC_MIXED])
def test_forward_model_against_the_oracle(oracle_mod, precision):
    """A walker's forward model (the profile problem: build the atmosphere
    from the parameters, step it, observe the level-mean temperatures) on the
    GPU against the same model run by the oracle: FP64 to 1e-11 relative,
    mixed to 1e-6."""
    build, observe, nvalue = profile_problem(N=8, L=12, steps=3)
    theta = np.array([[290., 210.], [260., 240.]])
    fb = EnsembleForward(build, observe, nvalue, 3, precision=precision, capacity=2)
    try:
        got = fb(theta)
    finally:
        fb.close()
    for n, p in enumerate(theta):
        cfg, w = build(p)
        o = oracle_mod.Oracle(dict(cfg, precision=0))
        o.set_primitive(w)
        o.step(3)
        assert o.invalid() == 0
        want = observe(cfg, o.primitive())
        rel = np.abs(got[n] - want).max() / np.abs(want).max()
        assert rel < (1e-11 if precision == nat.EXO_PREC_FP64 else 1e-6), (n, rel)
