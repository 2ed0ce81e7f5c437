"""Seeded synthetic initial states for the benchmark configurations.

The reference has no published benchmark inputs for this path; these stand
in for its problem generators (examples/2023-Chen-exo3/W92.cpp:72-113 for
the shallow-water sphere, hs94.cpp:251-291 for the dry atmosphere) with the
shapes, sizes and value distributions of the configurations:

  shallow_water   exo2, 6 x N x N x 3 layers: geopotential 2.94e4 m^2/s^2
                  plus a random real spherical-harmonic field of degree <= 8
                  with RMS 1 % of the base; solid-body rotation of 20-40 m/s
                  about a random axis.
  dry_atmosphere  exo3, 6 x N x N x L: isothermal 250 K hydrostatic column,
                  1e5 Pa at the surface, 1e3 Pa at the top; per-cell
                  temperature noise sigma 1 K at fixed pressure; horizontal
                  winds sigma 5 m/s per lat-lon component.

Every generator takes a numpy PCG64 seed and returns the primitive array
(6, nvar, N+6, N+6, L+6) with the interior filled (ghosts are zero).  The
cell geometry comes from the product library (`cell_geometry`) unless a
`geometry` callable with the same result is given: the CPU reference leg of
the benchmark passes the oracle's, so that it never loads the product.
"""
import math
import types

import numpy as np
from scipy.special import lpmv

from . import _native as nat
from .atmosphere import cell_geometry, make_config

G = nat.NGHOST


def _resolve(cfg, geometry):
    """(attribute view of cfg, geometry function).  Without a geometry
    function the configuration is completed with the library's defaults
    (make_config) and the library's geometry is used; with one, a dict is
    read as given."""
    if geometry is None:
        return (make_config(**cfg) if isinstance(cfg, dict) else cfg), cell_geometry
    return (types.SimpleNamespace(**cfg) if isinstance(cfg, dict) else cfg), geometry


def shallow_water_config(N=48, **kw):
    cfg = dict(N=N, L=3, eqn=nat.EXO_EQN_SHALLOW_YZ, rsolver=nat.EXO_RS_ROE_SHALLOW,
               implicit_flag=0, coriolis=nat.EXO_CORIOLIS_W92, x1min=6371000.,
               x1max=6371001., gamma=1.4, Rd=287., grav=0., cfl=0.4, omega=7.292e-5)
    cfg.update(kw)
    return cfg


def dry_atmosphere_config(N=96, L=64, rsolver=nat.EXO_RS_LMARS, T0=250., g=9.81,
                          Rd=287., gamma=1.4, ps=1e5, ptop=1e3, **kw):
    ztop = Rd * T0 / g * math.log(ps / ptop)
    cfg = dict(N=N, L=L, eqn=nat.EXO_EQN_IDEAL, rsolver=rsolver, implicit_flag=9,
               coriolis=nat.EXO_CORIOLIS_NONE, x1min=6.371e6, x1max=6.371e6 + ztop,
               gamma=gamma, Rd=Rd, grav=-g, cfl=0.4, omega=0.)
    cfg.update(kw)
    return cfg


def _real_sph_harm_field(lat, lon, lmax, rng):
    """sum_{l<=lmax, m} a_lm Y_lm(lat, lon) with a_lm ~ N(0, 1), real basis."""
    x = np.sin(lat)
    out = np.zeros_like(lat)
    for l in range(lmax + 1):
        for m in range(0, l + 1):
            norm = math.sqrt((2 * l + 1) / (4 * math.pi) *
                             math.factorial(l - m) / math.factorial(l + m))
            P = lpmv(m, l, x) * norm
            if m == 0:
                out += rng.standard_normal() * P
            else:
                out += rng.standard_normal() * math.sqrt(2) * P * np.cos(m * lon)
                out += rng.standard_normal() * math.sqrt(2) * P * np.sin(m * lon)
    return out


def _solid_body_uv(lat, lon, u0, axis):
    """East/north components of u0 * (axis x r_hat)."""
    cl, sl = np.cos(lat), np.sin(lat)
    co, so = np.cos(lon), np.sin(lon)
    r = np.stack([cl * co, cl * so, sl])
    v = u0 * np.cross(axis, r, axis=0)
    east = np.stack([-so, co, np.zeros_like(lon)])
    north = np.stack([-sl * co, -sl * so, cl])
    return (v * east).sum(0), (v * north).sum(0)


def shallow_water_state(cfg, seed=0, geometry=None):
    c, geo = _resolve(cfg, geometry)
    N, L = c.N, c.L
    lat, lon, m, _ = geo(cfg)
    rng = np.random.Generator(np.random.PCG64(seed))
    base = 2.94e4
    d = _real_sph_harm_field(lat, lon, 8, rng)
    d *= 0.01 * base / math.sqrt(np.mean(d * d))
    u0 = rng.uniform(20., 40.)
    axis = rng.standard_normal(3)
    axis /= np.linalg.norm(axis)
    U, V = _solid_body_uv(lat, lon, u0, axis)
    v2 = m[..., 0] * U + m[..., 1] * V
    v3 = m[..., 2] * U + m[..., 3] * V
    w = np.zeros((6, 4, N + 2 * G, N + 2 * G, L + 2 * G))
    sl = (slice(G, G + N), slice(G, G + N), slice(G, G + L))
    w[:, 0][(slice(None),) + sl] = (base + d)[..., None]
    w[:, 2][(slice(None),) + sl] = v2[..., None]
    w[:, 3][(slice(None),) + sl] = v3[..., None]
    return w


def dry_atmosphere_state(cfg, seed=0, T0=250., ps=1e5, temp_sigma=1.0, wind_sigma=5.0,
                         geometry=None):
    c, geo = _resolve(cfg, geometry)
    N, L = c.N, c.L
    Rd, g = c.Rd, -c.grav
    lat, lon, m, x1v = geo(cfg)
    rng = np.random.Generator(np.random.PCG64(seed))
    z = x1v - c.x1min
    p = ps * np.exp(-g * z / (Rd * T0))
    T = T0 + temp_sigma * rng.standard_normal((6, N, N, L))
    U = wind_sigma * rng.standard_normal((6, N, N, L))
    V = wind_sigma * rng.standard_normal((6, N, N, L))
    v2 = m[..., 0, None] * U + m[..., 1, None] * V
    v3 = m[..., 2, None] * U + m[..., 3, None] * V
    w = np.zeros((6, 5, N + 2 * G, N + 2 * G, L + 2 * G))
    sl = (slice(None), slice(G, G + N), slice(G, G + N), slice(G, G + L))
    w[:, 4][sl] = p[None, None, None, :]
    w[:, 0][sl] = p[None, None, None, :] / (Rd * T)
    w[:, 2][sl] = v2
    w[:, 3][sl] = v3
    return w


def interior(a):
    """View of the interior cells of a (6, nvar, nc3, nc2, nc1) array."""
    return a[:, :, G:-G, G:-G, G:-G]


ENSEMBLE_N = (24, 32, 48, 64, 96)
ENSEMBLE_L = (32, 48, 64, 96)


def _adiabat_isothermal(z, Ts, Ttop, g, Rd, gamma, ps):
    """Dry adiabat from (Ts, ps) up to T = Ttop, isothermal above: the
    analytic form of the column examples/2023-Chen-exo3/hs94.cpp:263-289
    integrates level by level.  Returns (T, p) at heights z."""
    cp = gamma / (gamma - 1.) * Rd
    lapse = g / cp
    zt = (Ts - Ttop) / lapse
    T = np.where(z < zt, Ts - lapse * z, Ttop)
    pt = ps * (Ttop / Ts) ** (cp / Rd)
    p = np.where(z < zt, ps * (np.maximum(T, Ttop) / Ts) ** (cp / Rd),
                 pt * np.exp(-g * (z - zt) / (Rd * Ttop)))
    return T, p


def member_config(N, L, Ts, Ttop, g, gamma, precision=nat.EXO_PREC_MIXED,
                  rsolver=nat.EXO_RS_LMARS, ps=1e5, ptop=1e3, Rd=287.):
    """Configuration of one forward-model atmosphere with the given profile
    parameters: dry adiabat from (Ts, ps) up to T = Ttop, isothermal above;
    the model top sits where the profile reaches ptop.  Returns (config
    dict, profile parameters)."""
    Ttop = min(Ttop, Ts)
    cp = gamma / (gamma - 1.) * Rd
    zt = (Ts - Ttop) / (g / cp)
    pt = ps * (Ttop / Ts) ** (cp / Rd)
    if pt <= ptop:
        ztop = (Ts - Ts * (ptop / ps) ** (Rd / cp)) / (g / cp)
    else:
        ztop = zt + Rd * Ttop / g * math.log(pt / ptop)
    cfg = dict(N=N, L=L, eqn=nat.EXO_EQN_IDEAL, rsolver=rsolver, implicit_flag=9,
               precision=precision, coriolis=nat.EXO_CORIOLIS_NONE, x1min=6.371e6,
               x1max=6.371e6 + ztop, gamma=gamma, Rd=Rd, grav=-g, cfl=0.4, omega=0.)
    return cfg, dict(Ts=Ts, Ttop=Ttop, ps=ps)


def ensemble_member_config(seed, precision=nat.EXO_PREC_MIXED, rsolver=nat.EXO_RS_LMARS,
                           ps=1e5, ptop=1e3, Rd=287.):
    """Configuration of one forward-model run of the batched ensemble.
    N ~ U{24,32,48,64,96}, L ~ U{32,48,64,96}, surface temperature
    U[150,400] K, top temperature U[100,250] K (at most the surface's),
    gravity U[3,25] m/s^2, gamma U[1.3,1.67]; member_config places the
    model top.  Returns (config dict, profile parameters)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    N = int(rng.choice(ENSEMBLE_N))
    L = int(rng.choice(ENSEMBLE_L))
    Ts = rng.uniform(150., 400.)
    Ttop = min(rng.uniform(100., 250.), Ts)
    g = rng.uniform(3., 25.)
    gamma = rng.uniform(1.3, 1.67)
    return member_config(N, L, Ts, Ttop, g, gamma, precision, rsolver, ps, ptop, Rd)


def member_state(cfg, prof, seed, temp_sigma=1.0, wind_sigma=5.0, geometry=None):
    """Primitive initial state of a member_config atmosphere: the profile
    plus temperature and wind noise as in dry_atmosphere_state, drawn from a
    generator seeded by (seed, 1)."""
    c, geo = _resolve(cfg, geometry)
    N, L, Rd, g = c.N, c.L, c.Rd, -c.grav
    rng = np.random.Generator(np.random.PCG64([seed, 1]))
    lat, lon, m, x1v = geo(cfg)
    T0, p = _adiabat_isothermal(x1v - c.x1min, prof["Ts"], prof["Ttop"], g, Rd, c.gamma,
                                prof["ps"])
    T = T0[None, None, None, :] + temp_sigma * rng.standard_normal((6, N, N, L))
    U = wind_sigma * rng.standard_normal((6, N, N, L))
    V = wind_sigma * rng.standard_normal((6, N, N, L))
    w = np.zeros((6, 5, N + 2 * G, N + 2 * G, L + 2 * G))
    sl = (slice(None), slice(G, G + N), slice(G, G + N), slice(G, G + L))
    w[:, 4][sl] = p[None, None, None, :]
    w[:, 0][sl] = p[None, None, None, :] / (Rd * T)
    w[:, 2][sl] = m[..., 0, None] * U + m[..., 1, None] * V
    w[:, 3][sl] = m[..., 2, None] * U + m[..., 3, None] * V
    return w


def ensemble_member(seed, precision=nat.EXO_PREC_MIXED, rsolver=nat.EXO_RS_LMARS,
                    temp_sigma=1.0, wind_sigma=5.0, geometry=None, **kw):
    """One forward-model run of the batched ensemble: (config dict, primitive
    array) for ensemble_member_config(seed)."""
    cfg, prof = ensemble_member_config(seed, precision, rsolver, **kw)
    return cfg, member_state(cfg, prof, seed, temp_sigma, wind_sigma, geometry)


def hs94_config(N=40, L=40, precision=nat.EXO_PREC_FP64, **kw):
    """The Held-Suarez benchmark of examples/2023-Chen-exo3/hs94.inp: six
    40x40 panels, 40 levels from 6371 to 6396 km, implicit_flag 1 (the
    partial vertical correction), CFL 0.9, gamma 1.4, g = 9.81, Rd = 287,
    Omega = 7.292e-5 and the HS94 forcing parameters of its <problem> and
    <thermodynamics> blocks.  The Riemann solver is HLLC, the one an exo3
    build compiles in (cmake/exo3.cmake: RSOLVER hllc_transform); the
    "--flux=lmars" of the input file's configure comment names an older
    build.  (LMARS has no cubed-sphere projection, lmars.cpp:24-110, so a
    resting atmosphere does not stay at rest with it on this grid.)"""
    cfg = dict(N=N, L=L, eqn=nat.EXO_EQN_IDEAL, rsolver=nat.EXO_RS_HLLC, implicit_flag=1,
               precision=precision, coriolis=nat.EXO_CORIOLIS_NONE,
               forcing=nat.EXO_FORCING_HS94, x1min=6.371e6, x1max=6.396e6, gamma=1.4,
               Rd=287., grav=-9.81, cfl=0.9, omega=7.292e-5,
               hs_p0=1.e5, hs_Ts=315., hs_dT=60., hs_dtheta=10., hs_Kf=1., hs_Ka=0.025,
               hs_Ks=0.25, hs_sigmab=0.7)
    cfg.update(kw)
    return cfg


def hs94_state(cfg, seed=0, z_iso=2.e4, wind_sigma=10., geometry=None):
    """MeshBlock::ProblemGenerator of hs94.cpp:246-291 restated: a dry adiabat
    from (Ts, p0) up to z_iso, isothermal above (Ttop = Ts + grav z_iso / cp),
    and wind noise of wind_sigma m/s in v2 and v3 of the adiabatic cells; the
    isothermal cells of a column keep the noise of its top adiabatic cell, as
    the reference's level loop leaves them.  Noise from a PCG64 generator."""
    c, geo = _resolve(cfg, geometry)
    N, L, Rd, g = c.N, c.L, c.Rd, -c.grav
    cp = c.gamma / (c.gamma - 1.) * Rd
    Ts, p0 = c.hs_Ts, c.hs_p0
    Ttop = Ts - g * z_iso / cp
    _, _, _, x1v = geo(cfg)
    z = x1v - c.x1min
    T, p = _adiabat_isothermal(z, Ts, Ttop, g, Rd, c.gamma, p0)
    rng = np.random.Generator(np.random.PCG64(seed))
    v2 = wind_sigma * rng.standard_normal((6, N, N, L))
    v3 = wind_sigma * rng.standard_normal((6, N, N, L))
    top = int(np.searchsorted(z, z_iso, side="right"))  # first isothermal level
    if 0 < top < L:
        v2[..., top:] = v2[..., top - 1:top]
        v3[..., top:] = v3[..., top - 1:top]
    w = np.zeros((6, 5, N + 2 * G, N + 2 * G, L + 2 * G))
    sl = (slice(None), slice(G, G + N), slice(G, G + N), slice(G, G + L))
    w[:, 4][sl] = p[None, None, None, :]
    w[:, 0][sl] = (p / (Rd * T))[None, None, None, :]
    w[:, 2][sl] = v2
    w[:, 3][sl] = v3
    return w
