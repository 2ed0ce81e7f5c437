"""Ensemble MCMC over batched forward models.

The reference's inversion (src/inversion/mcmc.cpp, mcmc_init.cpp,
mcmc_step.cpp) samples a posterior with the affine-invariant stretch move of
Goodman & Weare (2010): every walker k proposes

    z = ((a - 1) r + 1)^2 / a,   r ~ U[0, 1]
    y = (1 - z) X_j + z X_k,     j ~ U{walkers other than k}

from the positions of the previous iteration, evaluates its forward model at
y and accepts with probability min(1, z^(ndim-1) p(y) / p(X_k))
(mcmc.cpp:738-825).  The reference runs the walkers' forward models one
after another (mcmc_advance; profile_inversion.cpp:112-120 puts them in the
k-slices of one block).  Since every proposal of an iteration is built from
the previous iteration's positions, the proposals are independent: here
they are drawn first and all forward models of the iteration run together
as members of one batched ensemble (one launch per kernel per step); the
accept/reject pass then follows in walker order.  The chain is the one the
walker-by-walker loop produces from the same random numbers
(tests/test_inversion_host.py checks it bit for bit).

Random numbers: one seeded PCG64 stream, per iteration the pairs (r, j) of
all walkers, then the acceptance draws u.  (The reference seeds rand_r with
time(NULL) on every call, mcmc.cpp:747,805, so its draws are not
reproducible and repeat within a second.)
"""
import dataclasses

import numpy as np

from . import _native as nat


# ------------------------------------------------------------ sampler ----
@dataclasses.dataclass
class ChainRecords:
    """mcmc_recs (mcmc.hpp:50-72): positions, forward values and log
    probabilities of every walker at every iteration, and the best point."""
    nwalker: int
    ndim: int
    nvalue: int
    par: list = dataclasses.field(default_factory=list)       # [iteration] -> (nwalker, ndim)
    val: list = dataclasses.field(default_factory=list)       # [iteration] -> (nwalker, nvalue)
    lnp: list = dataclasses.field(default_factory=list)       # [iteration] -> (nwalker,)
    newstate: list = dataclasses.field(default_factory=list)  # [iteration] -> (nwalker,) 0/1
    accept: int = 0
    opt_lnp: float = -1.0e10
    opt_par: np.ndarray = None
    opt_val: np.ndarray = None

    @property
    def cur(self):
        return len(self.par)

    def acceptance_fraction(self):
        return self.accept / max(1, self.cur * self.nwalker)


def stretch_proposal(pos, k, r, j_draw, a):
    """mcmc_stretch_move (mcmc.cpp:784-825) for walker k with the uniform
    draw r and the walker draw j_draw in [0, nwalker - 2]: returns (y, z)."""
    z = ((a - 1.) * r + 1.) * ((a - 1.) * r + 1.) / a
    j = j_draw + 1 if j_draw >= k else j_draw
    return (1. - z) * pos[j] + z * pos[k], z


def acor(x):
    """Integrated autocorrelation time of a series by Goodman's acor
    (the _acor of mcmc.cpp:45-120): autocovariances up to lag 10, the
    self-consistent window 5 tau, and pairwise coarsening while tau is too
    long for that window.  Returns (mean, sigma, tau); tau = -1 when the
    series is shorter than 50."""
    TAUMAX, WINMULT, MINFAC = 2, 5, 5
    MAXLAG = TAUMAX * WINMULT

    def run(X):
        L = len(X)
        mean = X.sum() / L
        X = X - mean
        if L < MINFAC * MAXLAG:
            return mean, None, None
        iMax = L - MAXLAG
        C = np.array([np.dot(X[:iMax], X[s:s + iMax]) for s in range(MAXLAG + 1)]) / iMax
        D = C[0] + 2 * C[1:].sum()
        sigma = np.sqrt(D / L)
        tau = D / C[0]
        if tau * WINMULT < MAXLAG:
            return mean, sigma, tau
        Lh = L // 2
        Y = X[0:2 * Lh:2] + X[1:2 * Lh:2]
        _, s2, t2 = run(Y)
        if s2 is None:
            return mean, None, None
        D = 0.25 * s2 * s2 * L
        return mean, np.sqrt(D / L), D / C[0]

    mean, sigma, tau = run(np.asarray(x, dtype=np.float64))
    if tau is None:
        return mean, float("nan"), -1.0
    return mean, sigma, tau


class StretchSampler:
    """The reference's ensemble sampler (mcmc_init, mcmc_advance) with the
    forward models of an iteration evaluated in one batch.

    forward(params (n, ndim)) -> values (n, nvalue); a row of NaN marks a
        forward model that failed (an invalid atmosphere)
    log_prob(par (ndim,), val (nvalue,)) -> float; NaN marks an invalid point
    a           stretch scale (mcmc_opts::a)
    """

    def __init__(self, forward, log_prob, nwalker, ndim, nvalue, a=2.0, seed=0):
        if nwalker < 2:
            raise ValueError("nwalker must be at least 2")
        self.forward, self.log_prob = forward, log_prob
        self.a = float(a)
        self.rng = np.random.Generator(np.random.PCG64(seed))
        self.recs = ChainRecords(nwalker, ndim, nvalue)
        self.evaluations = 0

    def _lnp(self, par, val):
        return np.array([self.log_prob(par[k], val[k]) for k in range(len(par))])

    def _draws(self, n):
        r = self.rng.random(n)
        j = self.rng.integers(0, self.recs.nwalker - 1, n)
        return r, j

    def _best(self, par, val, lnp):
        rc = self.recs
        for k in range(len(lnp)):
            if lnp[k] > rc.opt_lnp:
                rc.opt_lnp = float(lnp[k])
                rc.opt_par = par[k].copy()
                rc.opt_val = val[k].copy()

    def init(self, pos):
        """mcmc_init (mcmc.cpp:699-736, mcmc_init.cpp): evaluate the start
        points; a walker whose point is invalid is moved by the stretch move
        (from the current positions, in place) up to 10 times."""
        rc = self.recs
        par = np.array(pos, dtype=np.float64).copy()
        val = self.forward(par)
        self.evaluations += len(par)
        lnp = self._lnp(par, val)
        for k in range(rc.nwalker):
            niter = 0
            while np.isnan(lnp[k]) and niter < 10:
                niter += 1
                r, j = self._draws(1)
                par[k], _ = stretch_proposal(par, k, r[0], j[0], self.a)
                val[k] = self.forward(par[k:k + 1])[0]
                self.evaluations += 1
                lnp[k] = self.log_prob(par[k], val[k])
            if np.isnan(lnp[k]):
                raise RuntimeError("starting point iteration > 10 times")
        self._best(par, val, lnp)
        rc.par.append(par)
        rc.val.append(val)
        rc.lnp.append(lnp)
        rc.newstate.append(np.ones(rc.nwalker, dtype=np.int32))
        rc.accept += rc.nwalker

    def advance(self):
        """mcmc_advance (mcmc.cpp:738-782): propose for every walker from the
        previous positions, evaluate all proposals as one batch, then accept
        or reject walker by walker."""
        rc = self.recs
        if rc.cur == 0:
            raise RuntimeError("the chain is not initialised (init)")
        old_par, old_val, old_lnp = rc.par[-1], rc.val[-1], rc.lnp[-1]
        r, j = self._draws(rc.nwalker)
        prop = np.empty_like(old_par)
        zz = np.empty(rc.nwalker)
        for k in range(rc.nwalker):
            prop[k], zz[k] = stretch_proposal(old_par, k, r[k], j[k], self.a)
        val = self.forward(prop)
        self.evaluations += rc.nwalker
        lnp1 = self._lnp(prop, val)
        u = self.rng.random(rc.nwalker)
        par, new_val, lnp = old_par.copy(), old_val.copy(), old_lnp.copy()
        newstate = np.zeros(rc.nwalker, dtype=np.int32)
        for k in range(rc.nwalker):
            pdiff = (rc.ndim - 1.) * np.log(zz[k]) + lnp1[k] - old_lnp[k]
            if pdiff > np.log(u[k]):  # NaN compares false: rejected
                par[k], new_val[k], lnp[k] = prop[k], val[k], lnp1[k]
                if lnp1[k] > rc.opt_lnp:
                    rc.opt_lnp = float(lnp1[k])
                    rc.opt_par, rc.opt_val = prop[k].copy(), val[k].copy()
                rc.accept += 1
                newstate[k] = 1
        rc.par.append(par)
        rc.val.append(new_val)
        rc.lnp.append(lnp)
        rc.newstate.append(newstate)

    def run(self, pos, nstep):
        """init, then nstep advances; returns the records."""
        self.init(pos)
        for _ in range(nstep):
            self.advance()
        return self.recs

    def statistics(self):
        """mcmc_statistics (mcmc.cpp:160-177): per dimension, the mean,
        error bar and autocorrelation time of the walker-averaged chain."""
        rc = self.recs
        x = np.array([p.mean(axis=0) for p in rc.par])  # (cur, ndim)
        out = [acor(x[:, d]) for d in range(rc.ndim)]
        return {"mean": np.array([o[0] for o in out]), "sigma": np.array([o[1] for o in out]),
                "tau": np.array([o[2] for o in out])}


# ------------------------------------------------------ forward models ----
class EnsembleForward:
    """Forward models of a batch of parameter vectors as members of one
    Ensemble: build(params) -> (config dict, primitive initial state),
    `steps` steps each, observe(config, final primitives) -> values.  A
    member whose state went invalid yields a row of NaN."""

    def __init__(self, build, observe, nvalue, steps, precision=nat.EXO_PREC_MIXED,
                 capacity=64, budget_bytes=150 * 10 ** 9, tile_cache=None):
        from .ensemble import Ensemble
        self.build, self.observe, self.nvalue, self.steps = build, observe, nvalue, steps
        self.precision = precision
        self.capacity = capacity
        self.ens = Ensemble(precision=precision, capacity=capacity, budget_bytes=budget_bytes)
        self.tile_cache = tile_cache
        self.cell_updates = 0

    def close(self):
        self.ens.close()

    def __call__(self, params):
        params = np.atleast_2d(params)
        out = np.full((len(params), self.nvalue), np.nan)
        for lo in range(0, len(params), self.capacity):
            chunk = params[lo:lo + self.capacity]
            slots, cfgs = [], []
            for p in chunk:
                cfg, w = self.build(p)
                cfg = dict(cfg, precision=self.precision)
                slots.append(self.ens.add(cfg, w))
                cfgs.append(cfg)
            if self.tile_cache is not None:
                self.ens.autotune(self.tile_cache)
            self.ens.step(self.steps)
            for n, (slot, cfg) in enumerate(zip(slots, cfgs)):
                if self.ens.invalid(slot) == 0:
                    out[lo + n] = self.observe(cfg, self.ens.primitive(slot))
                self.cell_updates += 6 * cfg["N"] ** 2 * cfg["L"] * self.steps
                self.ens.remove(slot)
        return out


class SequentialForward:
    """The same forward models one at a time, each on its own context (the
    reference's order of evaluation)."""

    def __init__(self, build, observe, nvalue, steps, precision=nat.EXO_PREC_FP64):
        self.build, self.observe, self.nvalue, self.steps = build, observe, nvalue, steps
        self.precision = precision
        self.cell_updates = 0

    def __call__(self, params):
        from .atmosphere import CubedSphereAtmosphere
        params = np.atleast_2d(params)
        out = np.full((len(params), self.nvalue), np.nan)
        for n, p in enumerate(params):
            cfg, w = self.build(p)
            cfg = dict(cfg, precision=self.precision)
            with CubedSphereAtmosphere(cfg) as a:
                a.set_primitive(w)
                a.step(self.steps)
                if a.invalid() == 0:
                    out[n] = self.observe(cfg, a.primitive())
            self.cell_updates += 6 * cfg["N"] ** 2 * cfg["L"] * self.steps
        return out


# ----------------------------------------- a temperature-profile problem --
def profile_problem(N=24, L=32, steps=20, Rd=287., gamma=1.4, g=9.81, ps=1e5, ptop=1e3,
                    seed=0):
    """A retrieval in the spirit of the reference's profile inversion
    (profile_inversion.cpp): the parameters are the surface and top
    temperatures (Ts, Ttop) of a dry adiabat capped by an isothermal layer
    (the profile of workloads.ensemble_member); the forward model runs the
    atmosphere `steps` steps from that profile (plus fixed seeded noise) and
    observes the horizontally averaged temperature of every level.
    Returns (build, observe, nvalue)."""
    from . import workloads as W
    from .atmosphere import cell_geometry, make_config
    import math

    def build(theta):
        Ts, Ttop = float(theta[0]), float(theta[1])
        cp = gamma / (gamma - 1.) * Rd
        lapse = g / cp
        Ttop = min(Ttop, Ts)
        zt = (Ts - Ttop) / lapse
        pt = ps * (Ttop / Ts) ** (cp / Rd)
        if pt <= ptop:
            ztop = (Ts - Ts * (ptop / ps) ** (Rd / cp)) / lapse
        else:
            ztop = zt + Rd * Ttop / g * math.log(pt / ptop)
        cfg = dict(N=N, L=L, eqn=nat.EXO_EQN_IDEAL, rsolver=nat.EXO_RS_LMARS, implicit_flag=9,
                   coriolis=nat.EXO_CORIOLIS_NONE, x1min=6.371e6, x1max=6.371e6 + ztop,
                   gamma=gamma, Rd=Rd, grav=-g, cfl=0.4, omega=0.)
        c = make_config(**cfg)
        _, _, m, x1v = cell_geometry(c)
        T0, p = W._adiabat_isothermal(x1v - c.x1min, Ts, Ttop, g, Rd, gamma, ps)
        rng = np.random.Generator(np.random.PCG64(seed))
        T = T0[None, None, None, :] + rng.standard_normal((6, N, N, L))
        U = 5. * rng.standard_normal((6, N, N, L))
        V = 5. * rng.standard_normal((6, N, N, L))
        w = np.zeros((6, 5, N + 6, N + 6, L + 6))
        sl = (slice(None), slice(3, 3 + N), slice(3, 3 + N), slice(3, 3 + L))
        w[:, 4][sl] = p[None, None, None, :]
        w[:, 0][sl] = p[None, None, None, :] / (Rd * T)
        w[:, 2][sl] = m[..., 0, None] * U + m[..., 1, None] * V
        w[:, 3][sl] = m[..., 2, None] * U + m[..., 3, None] * V
        return cfg, w

    def observe(cfg, w):
        wi = W.interior(w)
        return (wi[:, 4] / (wi[:, 0] * cfg["Rd"])).mean(axis=(0, 1, 2))

    return build, observe, L
