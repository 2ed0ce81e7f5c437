"""The oracle's FullCorrection and PartialCorrection against a second, plain
numpy statement of the same linear system.

The oracle solves the vertical block-tridiagonal system level by level
(ForwardSweep / BackwardSubstitution, forward_backward.hpp:15-126) with 5x5
Gauss-Jordan or 3x3 adjugate inverses.  Here the same blocks are written out
again from the reference formulas (partial_correction.cpp:26-173,
full_correction.cpp:32-165, flux_decomposition.hpp:14-120), assembled into
one dense matrix per column and solved by numpy's LU.  The two solutions
agree to rounding: relative difference below 1e-9 per variable."""
import numpy as np
import pytest

from _columns import column_problem

G = 3


def flux_jacobian(gm1, w):
    rho, v1, v2, v3, p = w
    s2 = v1 * v1 + v2 * v2 + v3 * v3
    c1 = ((gm1 - 1) * s2 / 2 - (gm1 + 1) / gm1 * p / rho) * v1
    c2 = (gm1 + 1) / gm1 * p / rho + s2 / 2 - gm1 * v1 * v1
    return np.array([[0., 1., 0., 0., 0.],
                     [gm1 * s2 / 2 - v1 * v1, (2. - gm1) * v1, -gm1 * v2, -gm1 * v3, gm1],
                     [-v1 * v2, v2, v1, 0., 0.],
                     [-v1 * v3, v3, 0., v1, 0.],
                     [c1, c2, -gm1 * v2 * v1, -gm1 * v3 * v1, (gm1 + 1) * v1]])


def abs_jacobian(gm1, gamma, wl, wr):
    """R |Lambda| R^-1 at the Roe average of the face between wl and wr."""
    sl, sr = np.sqrt(wl[0]), np.sqrt(wr[0])
    r = sl * sr
    u, v, w = [(sl * wl[n] + sr * wr[n]) / (sl + sr) for n in (1, 2, 3)]
    el = wl[4] / gm1 + 0.5 * wl[0] * (wl[1] ** 2 + wl[2] ** 2 + wl[3] ** 2)
    er = wr[4] / gm1 + 0.5 * wr[0] * (wr[1] ** 2 + wr[2] ** 2 + wr[3] ** 2)
    hbar = ((el + wl[4]) / sl + (er + wr[4]) / sr) / (sl + sr)
    p = (hbar - 0.5 * (u * u + v * v + w * w)) * gm1 / (gm1 + 1.) * r
    cs = np.sqrt(gamma * p / r)
    ke = 0.5 * (u * u + v * v + w * w)
    hp = (gm1 + 1.) / gm1 * p / r
    h = hp + ke
    R = np.array([[1., 1., 1., 0., 0.], [u - cs, u, u + cs, 0., 0.], [v, v, v, 1., 0.],
                  [w, w, w, 0., 1.], [h - u * cs, ke, h + u * cs, v, w]])
    lam = np.abs([u - cs, u, u + cs, u, u])
    return R @ np.diag(lam) @ np.linalg.inv(R)


def dense_correction(wcol, du, geo, x1f, x1v, dx1f, dt, gamma, grav, full):
    cos_t, sin_t, d2, d3 = geo
    L = du.shape[1]
    w = wcol.copy()
    w[2] += w[3] * cos_t
    w[3] *= sin_t
    gm1 = gamma - 1.
    sel = [0, 1, 2, 3, 4] if full else [0, 1, 4]
    m = len(sel)
    ix = np.ix_(sel, sel)
    phi = np.zeros((5, 5))
    phi[1, 0] = phi[4, 1] = grav
    bnd = np.diag([1., -1., 1., 1., 1.])[ix]
    J = [flux_jacobian(gm1, w[:, i]) for i in range(w.shape[1])]
    M = np.zeros((m * L, m * L))
    for lev in range(L):
        i = G + lev
        Am = abs_jacobian(gm1, gamma, w[:, i - 1], w[:, i])
        Ap = abs_jacobian(gm1, gamma, w[:, i], w[:, i + 1])
        al = d2 * d3 * x1f[i] ** 2 * sin_t
        ar = d2 * d3 * x1f[i + 1] ** 2 * sin_t
        vol = dx1f[i] * d2 * d3 * x1v[i] ** 2 * sin_t
        a = ((Am * al + Ap * ar + (ar - al) * J[i]) / (2 * vol) + np.eye(5) / dt - phi)[ix]
        b = (-(Am + J[i - 1]) * al / (2 * vol))[ix]
        c = (-(Ap - J[i + 1]) * ar / (2 * vol))[ix]
        if lev == 0:
            a = a + b @ bnd
        if lev == L - 1:
            a = a + c @ bnd
        s = slice(lev * m, lev * m + m)
        M[s, s] = a
        if lev > 0:
            M[s, slice((lev - 1) * m, lev * m)] = b
        if lev < L - 1:
            M[s, slice((lev + 1) * m, (lev + 2) * m)] = c
    rhs = (du[sel] / dt).T.reshape(-1)
    delta = np.linalg.solve(M, rhs).reshape(L, m).T
    out = du.copy()
    out[sel] = delta
    return out


@pytest.mark.parametrize("full", [False, True])
@pytest.mark.parametrize("L,dt", [(1, 20.0), (6, 60.0), (16, 400.0)])
def test_oracle_correction_solves_the_block_system(oracle_mod, full, L, dt):
    ncol = 5
    w, du, colgeo, x1f, x1v, dx1f, cfg = column_problem(oracle_mod, ncol, L, seed=L + 7 * full)
    got = oracle_mod.implicit_columns(w, du, colgeo, x1f, x1v, dx1f, dt, cfg["gamma"],
                                      cfg["grav"], full=full)
    for c in range(ncol):
        want = dense_correction(w[c], du[c], colgeo[c], x1f, x1v, dx1f, dt, cfg["gamma"],
                                cfg["grav"], full)
        for n in range(5):
            rel = np.linalg.norm(got[c, n] - want[n]) / np.linalg.norm(want[n])
            assert rel < 1e-9, (c, n, rel)
    if not full:
        # the tangential momenta keep their explicit update
        assert np.array_equal(got[:, 2:4], du[:, 2:4])
    # the correction is not the identity
    assert np.abs(got[:, [0, 1, 4]] - du[:, [0, 1, 4]]).max() > 0
