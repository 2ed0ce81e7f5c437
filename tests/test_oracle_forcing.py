"""The oracle's user sources against a plain numpy statement of the
reference's formulas, and two balance properties of the restated scheme.

* Held-Suarez forcing (examples/2023-Chen-exo3/hs94.cpp:59-155): Coriolis on
  the momenta in latitude-longitude, Rayleigh drag and Newtonian cooling.
  The numpy version goes through the latitude and the (U, V) -> (V2, V3) map
  of exo_cell_geometry (inverting the map instead of calling the transform
  the other way), so it agrees to rounding: 1e-12 relative.
* CalculateCoriolisForce3 (src/exo3/cubed_sphere.cpp:197-231) from the cell
  centres' tangents: 1e-13 relative.
* A shallow-water lake at rest and a uniform ideal gas at rest with HLLC
  stay at rest to rounding (the metric source terms balance the pressure
  fluxes, panel edges included)."""
import numpy as np
import pytest

from exocubed_b200 import _native as nat
from exocubed_b200 import workloads as W
from exocubed_b200.atmosphere import cell_geometry

G = 3


def _tangents(o, N):
    """tan(x2v[j]), tan(x3v[k]) of the interior cells, per panel."""
    X, Y = [], []
    for p in range(6):
        _, x2f, x3f = o.mesh(p)
        x2v = 0.5 * (x2f[1:] + x2f[:-1])
        x3v = 0.5 * (x3f[1:] + x3f[:-1])
        X.append(np.tan(x2v[G:G + N]))
        Y.append(np.tan(x3v[G:G + N]))
    return np.array(X), np.array(Y)   # [6][N] each: X over j, Y over k


def _state(cfg, seed):
    w = W.hs94_state(cfg, seed=seed)
    rng = np.random.default_rng(seed)
    W.interior(w)[:, 1] = 0.5 * rng.standard_normal(W.interior(w)[:, 1].shape)
    return w


def test_hs94_forcing_matches_numpy(oracle_mod):
    N, L = 8, 12
    cfg = W.hs94_config(N=N, L=L)
    o = oracle_mod.Oracle(cfg)
    w = _state(cfg, 3)
    wght = 123.0
    got = W.interior(o.user_sources(w, wght))
    lat, _, m, _ = cell_geometry(cfg)
    X, Y = _tangents(o, N)
    x = X[:, None, :, None]          # [6][k][j][i]
    y = Y[:, :, None, None]
    C, D = np.sqrt(x * x + 1), np.sqrt(y * y + 1)
    cth = -x * y / (C * D)
    wi = W.interior(w)
    rho, v1, v2, v3, p = (wi[:, n] for n in range(5))
    # Coriolis in latitude-longitude: (U, V) from (V2, V3) by the inverse map
    m4 = m.reshape(6, N, N, 2, 2)
    minv = np.linalg.inv(m4)
    U = minv[..., 0, 0, None] * v2 + minv[..., 0, 1, None] * v3
    V = minv[..., 1, 0, None] * v2 + minv[..., 1, 1, None] * v3
    f = 2 * cfg["omega"] * np.sin(lat)[..., None]
    llU, llV = f * rho * V, -f * rho * U
    acc2 = m4[..., 0, 0, None] * llU + m4[..., 0, 1, None] * llV
    acc3 = m4[..., 1, 0, None] * llU + m4[..., 1, 1, None] * llV
    want = np.zeros_like(got)
    want[:, 2] = wght * (acc2 + acc3 * cth)
    want[:, 3] = wght * (acc3 + acc2 * cth)
    # Rayleigh drag and Newtonian cooling
    Rd, gamma = cfg["Rd"], cfg["gamma"]
    cp = gamma / (gamma - 1.) * Rd
    day = 8.64e4
    Kf, Ka, Ks = cfg["hs_Kf"] / day, cfg["hs_Ka"] / day, cfg["hs_Ks"] / day
    sig = p / cfg["hs_p0"]
    sig_p = (sig - cfg["hs_sigmab"]) / (1 - cfg["hs_sigmab"])
    Kv = np.where(sig_p < 0, 0., sig_p * Kf)
    la = lat[..., None]
    Teq = (cfg["hs_Ts"] - cfg["hs_dT"] * np.sin(la) ** 2 -
           cfg["hs_dtheta"] * np.log(sig) * np.cos(la) ** 2) * sig ** (Rd / cp)
    Teq = np.maximum(Teq, 200.)
    Kt = Ka + (Ks - Ka) * np.where(sig_p < 0, 0., sig_p * np.cos(la) ** 4)
    T = p / rho / Rd
    m2, m3 = rho * v2, rho * v3
    want[:, 1] += -wght * Kv * rho * v1
    want[:, 2] += -wght * Kv * (m2 + m3 * cth)
    want[:, 3] += -wght * Kv * (m3 + m2 * cth)
    want[:, 4] += -wght * (cp - Rd) * rho * Kt * (T - Teq)
    assert np.array_equal(got[:, 0], want[:, 0])
    for n in range(1, 5):
        rel = np.linalg.norm(got[:, n] - want[:, n]) / np.linalg.norm(want[:, n])
        assert rel < 1e-12, (n, rel)
    # both parts are active: drag near the ground, cooling everywhere
    assert np.abs(want[:, 1]).max() > 0 and np.abs(want[:, 4]).max() > 0


def test_coriolis3_matches_numpy(oracle_mod):
    N, L = 8, 6
    cfg = W.dry_atmosphere_config(N=N, L=L, rsolver=nat.EXO_RS_HLLC,
                                  coriolis=nat.EXO_CORIOLIS_3D, omega=7.292e-5)
    o = oracle_mod.Oracle(cfg)
    w = W.dry_atmosphere_state(cfg, seed=4)
    rng = np.random.default_rng(4)
    W.interior(w)[:, 1] = rng.standard_normal(W.interior(w)[:, 1].shape)
    wght = 50.0
    got = W.interior(o.user_sources(w, wght))
    X, Y = _tangents(o, N)
    x = X[:, None, :, None]
    y = Y[:, :, None, None]
    C, D = np.sqrt(x * x + 1), np.sqrt(y * y + 1)
    delta = np.sqrt(x * x + y * y + 1)
    wi = W.interior(w)
    rho, v1, v2, v3 = (wi[:, n] for n in range(4))
    A = 2 * cfg["omega"] * C * D / delta ** 2 * rho
    polar = np.array([1, 0, 0, 0, 1, 0], bool)[:, None, None, None]  # blocks 1 and 5
    cF1 = np.where(polar, A * (y * C * v2 - x * D * v3), -A * D * v3)
    cF2 = np.where(polar, A * (-y * C * v1 - v3), A * x * v3)
    cF3 = np.where(polar, A * (x * D * v1 + v2), A * (D * v1 - x * v2))
    for n, cf in ((1, cF1), (2, cF2), (3, cF3)):
        rel = np.linalg.norm(got[:, n] - wght * cf) / np.linalg.norm(wght * cf)
        assert rel < 1e-13, (n, rel)
    assert not got[:, 0].any() and not got[:, 4].any()


def test_shallow_water_lake_at_rest(oracle_mod):
    cfg = dict(W.shallow_water_config(N=16), coriolis=nat.EXO_CORIOLIS_NONE)
    w = W.shallow_water_state(cfg, seed=0)
    w[:, 0] = 2.94e4
    w[:, 2:] = 0.
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(w)
    o.step(5)
    wi = W.interior(o.primitive())
    assert np.abs(wi[:, 2:4]).max() < 1e-10
    assert np.ptp(wi[:, 0]) < 1e-9 * 2.94e4


@pytest.mark.parametrize("implicit_flag", [0, 1, 9])
def test_uniform_gas_at_rest_with_hllc(oracle_mod, implicit_flag):
    cfg = W.dry_atmosphere_config(N=8, L=6, rsolver=nat.EXO_RS_HLLC, grav=0.0,
                                  implicit_flag=implicit_flag)
    w = W.dry_atmosphere_state(cfg, seed=0, wind_sigma=0., temp_sigma=0.)
    w[:, 0] = 1.0
    w[:, 1:4] = 0.
    w[:, 4] = 1e5
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(w)
    o.step(3)
    wi = W.interior(o.primitive())
    assert np.abs(wi[:, 1:4]).max() < 1e-10
    assert np.ptp(wi[:, 4]) < 1e-12 * 1e5
