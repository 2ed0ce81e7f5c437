"""The stretch-move sampler (exocubed_b200.inversion) on the CPU.

* Batched evaluation does not change the chain: a walker-by-walker loop in
  the reference's order (mcmc.cpp:738-782, one forward call per walker, the
  same random numbers per walker) produces the same records bit for bit.
* The sampler recovers a known Gaussian posterior.
* acor (mcmc.cpp:45-120) gives the autocorrelation time of an AR(1) series,
  (1 + phi) / (1 - phi).
* Invalid start points are moved until valid (mcmc_init)."""
import numpy as np
import pytest

from exocubed_b200.inversion import StretchSampler, acor, stretch_proposal

COV = np.array([[1.0, 0.6], [0.6, 2.0]])
ICOV = np.linalg.inv(COV)


def forward(par):
    par = np.atleast_2d(par)
    return np.stack([par[:, 0] + par[:, 1], par[:, 0] - 2 * par[:, 1], par[:, 1] ** 2], axis=1)


def log_prob(par, val):
    return float(-0.5 * par @ ICOV @ par) + 0.0 * val[0]


def reference_loop(pos, nstep, a, seed):
    """mcmc_init + mcmc_advance walker by walker, with the draws the batched
    sampler takes from the same stream."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nw, nd = pos.shape
    par = [pos.copy()]
    val = [np.stack([forward(pos[k])[0] for k in range(nw)])]
    lnp = [np.array([log_prob(pos[k], val[0][k]) for k in range(nw)])]
    for _ in range(nstep):
        r = rng.random(nw)
        j = rng.integers(0, nw - 1, nw)
        u = None
        p0, v0, l0 = par[-1], val[-1], lnp[-1]
        p1, v1, l1 = p0.copy(), v0.copy(), l0.copy()
        props = []
        for k in range(nw):
            y, z = stretch_proposal(p0, k, r[k], j[k], a)
            vy = forward(y)[0]
            props.append((y, z, vy, log_prob(y, vy)))
        u = rng.random(nw)
        for k in range(nw):
            y, z, vy, ly = props[k]
            if (nd - 1.) * np.log(z) + ly - l0[k] > np.log(u[k]):
                p1[k], v1[k], l1[k] = y, vy, ly
        par.append(p1)
        val.append(v1)
        lnp.append(l1)
    return par, val, lnp


def test_batched_chain_equals_walker_by_walker_loop():
    rng = np.random.default_rng(1)
    pos = rng.standard_normal((10, 2))
    s = StretchSampler(forward, log_prob, 10, 2, 3, a=2.0, seed=5)
    rec = s.run(pos, 25)
    par, val, lnp = reference_loop(pos, 25, 2.0, 5)
    assert rec.cur == 26
    for t in range(26):
        assert np.array_equal(rec.par[t], par[t])
        assert np.array_equal(rec.val[t], val[t])
        assert np.array_equal(rec.lnp[t], lnp[t])
    assert s.evaluations == 10 * 26


def test_gaussian_posterior_is_recovered():
    rng = np.random.default_rng(2)
    s = StretchSampler(forward, log_prob, 64, 2, 3, seed=3)
    rec = s.run(0.1 * rng.standard_normal((64, 2)), 600)
    samples = np.concatenate(rec.par[100:])
    assert np.abs(samples.mean(axis=0)).max() < 0.15
    assert np.allclose(np.cov(samples.T), COV, rtol=0.15, atol=0.1)
    assert 0.2 < rec.acceptance_fraction() < 0.9
    st = s.statistics()
    # the walker-averaged chain: its mean, and a positive autocorrelation time
    # where the series is long enough for acor's window (-1 otherwise)
    assert np.abs(st["mean"]).max() < 0.15
    assert ((st["tau"] > 0) | (st["tau"] == -1)).all()
    assert rec.opt_lnp <= 0 and rec.opt_lnp > -0.1


def test_acor_of_an_ar1_series():
    rng = np.random.default_rng(4)
    phi, n = 0.5, 200000
    x = np.empty(n)
    x[0] = 0.
    e = rng.standard_normal(n)
    for i in range(1, n):
        x[i] = phi * x[i - 1] + e[i]
    mean, sigma, tau = acor(x)
    assert tau == pytest.approx((1 + phi) / (1 - phi), rel=0.1)
    assert abs(mean) < 0.05 and sigma > 0
    assert acor(x[:20])[2] == -1.0


def test_invalid_start_points_are_moved():
    def fwd(par):
        par = np.atleast_2d(par)
        out = forward(par)
        out[np.abs(par[:, 0] - 1.6) < 0.1] = np.nan  # a band of invalid points
        return out

    def lp(par, val):
        return np.nan if np.isnan(val).any() else log_prob(par, val)

    rng = np.random.default_rng(6)
    pos = 0.1 * rng.standard_normal((8, 2))
    pos[[1, 4], 0] = 1.6
    s = StretchSampler(fwd, lp, 8, 2, 3, seed=7)
    s.init(pos)
    assert np.isfinite(s.recs.lnp[0]).all()
    assert (np.abs(s.recs.par[0][:, 0] - 1.6) >= 0.1).all()
    assert s.evaluations > 8
    s.advance()
    assert np.isfinite(s.recs.lnp[1]).all()
