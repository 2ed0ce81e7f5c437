"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker of the GPU path.  The oracle is a
C++ restatement of ExoCubed's cubed-sphere step (see exo_oracle.cpp's header
for the file:line of every piece it follows and the choices it makes where
the reference's Athena++ fork is not available).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

NGHOST = 3


class ExoConfig(ctypes.Structure):
    """Mirror of exo_config in include/exo_b200.h."""
    _fields_ = [
        ("N", ctypes.c_int), ("L", ctypes.c_int), ("eqn", ctypes.c_int),
        ("rsolver", ctypes.c_int), ("implicit_flag", ctypes.c_int),
        ("precision", ctypes.c_int), ("coriolis", ctypes.c_int),
        ("forcing", ctypes.c_int),
        ("x1min", ctypes.c_double), ("x1max", ctypes.c_double),
        ("gamma", ctypes.c_double), ("Rd", ctypes.c_double),
        ("grav", ctypes.c_double), ("cfl", ctypes.c_double),
        ("omega", ctypes.c_double), ("reserved1", ctypes.c_double),
        ("hs_p0", ctypes.c_double), ("hs_Ts", ctypes.c_double), ("hs_dT", ctypes.c_double),
        ("hs_dtheta", ctypes.c_double), ("hs_Kf", ctypes.c_double), ("hs_Ka", ctypes.c_double),
        ("hs_Ks", ctypes.c_double), ("hs_sigmab", ctypes.c_double),
    ]


def build():
    """Compile liboracle.so with its Makefile (gcc, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        d, p, i = ctypes.c_double, ctypes.c_void_p, ctypes.c_int
        dp = ctypes.POINTER(ctypes.c_double)
        L.ora_interp_weno5.restype = d
        L.ora_interp_weno5.argtypes = [d] * 5
        L.ora_interp_weno3.restype = d
        L.ora_interp_weno3.argtypes = [d] * 3
        L.ora_cov_to_contra.argtypes = [dp, d]
        L.ora_contra_to_cov.argtypes = [dp, d]
        L.ora_create.restype = p
        L.ora_create.argtypes = [ctypes.POINTER(ExoConfig)]
        L.ora_destroy.argtypes = [p]
        L.ora_set_primitive.argtypes = [p, dp]
        L.ora_set_conserved.argtypes = [p, dp]
        L.ora_get_conserved.argtypes = [p, dp]
        L.ora_get_primitive.argtypes = [p, dp]
        L.ora_get_flux.argtypes = [p, i, dp]
        L.ora_get_dt.restype = d
        L.ora_get_dt.argtypes = [p]
        L.ora_get_time.restype = d
        L.ora_get_time.argtypes = [p]
        L.ora_get_invalid.restype = i
        L.ora_get_invalid.argtypes = [p]
        L.ora_calculate_fluxes.argtypes = [p]
        L.ora_step.argtypes = [p, i, d]
        L.ora_get_mesh.argtypes = [p, i, dp, dp, dp]
        ip = ctypes.POINTER(ctypes.c_int)
        L.ora_vec_abp_from_rll.argtypes = [d, d, i, d, d, dp]
        L.ora_vec_rll_from_abp.argtypes = [d, d, i, d, d, dp]
        L.ora_rll_from_xyp.argtypes = [d, d, i, dp]
        L.ora_interp_loc.restype = d
        L.ora_interp_loc.argtypes = [i, i, i, i]
        L.ora_panel_tables.argtypes = [ip] * 5
        L.ora_get_dx1f.argtypes = [p, dp]
        L.ora_eos_range.restype = i
        L.ora_eos_range.argtypes = [p, i, dp, dp, i, i, i, i, i, i]
        L.ora_sound_speed.restype = d
        L.ora_sound_speed.argtypes = [p, dp]
        L.ora_pack_face.restype = i
        L.ora_pack_face.argtypes = [p, i, i, dp]
        L.ora_cell_geometry_at.argtypes = [p, i, i, i, i, dp]
        L.ora_face_geo.argtypes = [p, i, i, i, i, dp]
        L.ora_exchange_faces.argtypes = [p, dp, dp, dp, dp]
        L.ora_set_ghost_passes.restype = i
        L.ora_set_ghost_passes.argtypes = [p, i]
        L.ora_cell_geometry.restype = i
        L.ora_cell_geometry.argtypes = [ctypes.POINTER(ExoConfig), dp, dp, dp, dp]
        L.ora_riemann_face.argtypes = [i, i, i, d, dp, dp, dp, d, d, d, d]
        L.ora_correction_columns.argtypes = [i, i, i, dp, dp, dp, dp, dp, dp, d, d, d]
        L.ora_solve_implicit_3d.argtypes = [p, dp, dp, d]
        L.ora_user_sources.argtypes = [p, dp, dp, d]
        L.ora_change_to_perturbation.argtypes = [p, dp]
        L.ora_restore_from_perturbation.argtypes = [p, dp, dp, dp]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def to_struct(cfg):
    """dict (or ExoConfig) -> ExoConfig."""
    if isinstance(cfg, ExoConfig):
        return cfg
    s = ExoConfig()
    for k, v in cfg.items():
        setattr(s, k, v)
    return s


def cell_geometry(cfg):
    """(lat, lon, uv_to_v23, x1v) of the interior cells from the oracle's own
    mesh (GetLatLon / GetVyVz, cubed_sphere.cpp:78-162): the geometry that
    seeded initial states need, without the product library."""
    c = to_struct(cfg)
    N, L = c.N, c.L
    lat = np.empty((6, N, N))
    lon = np.empty((6, N, N))
    m = np.empty((6, N, N, 4))
    x1v = np.empty(L)
    if lib().ora_cell_geometry(ctypes.byref(c), _ptr(lat), _ptr(lon), _ptr(m), _ptr(x1v)):
        raise ValueError("oracle rejected the configuration")
    return lat, lon, m, x1v


class Oracle:
    """Six-panel cubed-sphere state advanced on the CPU."""

    def __init__(self, cfg):
        self.cfg = to_struct(cfg)
        self._h = lib().ora_create(ctypes.byref(self.cfg))
        if not self._h:
            raise ValueError("oracle rejected the configuration")
        c = self.cfg
        self.nvar = 4 if c.eqn == 0 else 5
        self.shape = (6, self.nvar, c.N + 2 * NGHOST, c.N + 2 * NGHOST, c.L + 2 * NGHOST)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().ora_destroy(self._h)
            self._h = None

    def set_ghost_passes(self, passes):
        """1 panel ghost sync per boundary update, or 2 as the reference's
        cubed-sphere task list runs them."""
        if lib().ora_set_ghost_passes(self._h, int(passes)):
            raise ValueError("passes must be 1 or 2")

    def set_primitive(self, w):
        w = np.ascontiguousarray(w, dtype=np.float64)
        assert w.shape == self.shape
        lib().ora_set_primitive(self._h, _ptr(w))

    def set_conserved(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        assert u.shape == self.shape
        lib().ora_set_conserved(self._h, _ptr(u))

    def conserved(self):
        a = np.empty(self.shape)
        lib().ora_get_conserved(self._h, _ptr(a))
        return a

    def primitive(self):
        a = np.empty(self.shape)
        lib().ora_get_primitive(self._h, _ptr(a))
        return a

    def flux(self, d):
        a = np.empty(self.shape)
        lib().ora_get_flux(self._h, d, _ptr(a))
        return a

    def calculate_fluxes(self):
        lib().ora_calculate_fluxes(self._h)

    def step(self, nsteps, dt_fixed=0.0):
        lib().ora_step(self._h, int(nsteps), float(dt_fixed))

    @property
    def dt(self):
        return lib().ora_get_dt(self._h)

    @property
    def time(self):
        return lib().ora_get_time(self._h)

    def invalid(self):
        return lib().ora_get_invalid(self._h)

    def change_to_perturbation(self, w):
        """ChangeToPerturbation on w (whole-array layout, in place)."""
        assert w.flags.c_contiguous and w.dtype == np.float64 and w.shape == self.shape
        lib().ora_change_to_perturbation(self._h, _ptr(w))

    def restore_from_perturbation(self, w, wl, wr):
        """RestoreFromPerturbation: w and the x1 face states wl, wr in place."""
        for a in (w, wl, wr):
            assert a.flags.c_contiguous and a.dtype == np.float64 and a.shape == self.shape
        lib().ora_restore_from_perturbation(self._h, _ptr(w), _ptr(wl), _ptr(wr))

    def user_sources(self, w, wght, out=None):
        """The user explicit sources alone (Coriolis, HS94 forcing) of
        primitives w, times wght, added to out (zeros if None)."""
        w = np.ascontiguousarray(w, dtype=np.float64)
        out = np.zeros(self.shape) if out is None else np.ascontiguousarray(out, dtype=np.float64).copy()
        lib().ora_user_sources(self._h, _ptr(w), _ptr(out), float(wght))
        return out

    def solve_implicit_3d(self, du, w, dt):
        """SolveImplicit3D: du (whole-array layout) corrected in place."""
        w = np.ascontiguousarray(w, dtype=np.float64)
        assert du.flags.c_contiguous and du.dtype == np.float64
        lib().ora_solve_implicit_3d(self._h, _ptr(du), _ptr(w), float(dt))

    def eos(self, to_prim, a, ranges):
        """ConservedToPrimitive (to_prim) or PrimitiveToConserved of the whole
        array a over ranges (il, iu, jl, ju, kl, ku); returns (out, invalid)
        with out zero outside the ranges."""
        a = np.ascontiguousarray(a, dtype=np.float64)
        out = np.zeros(self.shape)
        inv = lib().ora_eos_range(self._h, int(bool(to_prim)), _ptr(a), _ptr(out), *ranges)
        return out, inv

    def sound_speed(self, prim):
        w = np.zeros(5)
        w[:len(prim)] = prim
        return lib().ora_sound_speed(self._h, _ptr(w))

    def dx1f(self):
        out = np.zeros(self.cfg.L + 2 * NGHOST)
        lib().ora_get_dx1f(self._h, _ptr(out))
        return out

    def pack_face(self, p, s):
        """What panel p sends across side s (0 Up, 1 Down, 2 Left, 3 Right)
        from the current conserved state."""
        buf = np.zeros(self.nvar * 3 * (self.cfg.N + 6) * (self.cfg.L + 6))
        n = lib().ora_pack_face(self._h, p, s, _ptr(buf))
        return buf[:n]

    def cell_geometry_at(self, p, k, j, i):
        out = np.zeros(7)
        lib().ora_cell_geometry_at(self._h, p, k, j, i, _ptr(out))
        return out

    def face_geo(self, p, k, j, ivx):
        out = np.zeros(4)
        lib().ora_face_geo(self._h, p, k, j, ivx, _ptr(out))
        return out

    def exchange_faces(self, L2, R2, L3, R3):
        arrs = [np.ascontiguousarray(a, dtype=np.float64).copy() for a in (L2, R2, L3, R3)]
        for a in arrs:
            assert a.shape == self.shape
        lib().ora_exchange_faces(self._h, *[_ptr(a) for a in arrs])
        return arrs

    def mesh(self, panel):
        c = self.cfg
        x1f = np.empty(c.L + 2 * NGHOST + 1)
        x2f = np.empty(c.N + 2 * NGHOST + 1)
        x3f = np.empty(c.N + 2 * NGHOST + 1)
        lib().ora_get_mesh(self._h, panel, _ptr(x1f), _ptr(x2f), _ptr(x3f))
        return x1f, x2f, x3f


def interp_weno5(a, b, c, d, e):
    return lib().ora_interp_weno5(a, b, c, d, e)


def interp_weno3(a, b, c):
    return lib().ora_interp_weno3(a, b, c)


def cov_to_contra(w, cth):
    w = np.ascontiguousarray(w, dtype=np.float64).copy()
    lib().ora_cov_to_contra(_ptr(w), cth)
    return w


def contra_to_cov(w, cth):
    w = np.ascontiguousarray(w, dtype=np.float64).copy()
    lib().ora_contra_to_cov(_ptr(w), cth)
    return w


def riemann_face(rsolver, eqn, ivx, gamma, wl, wr, cosf=0.0, sinf=1.0, cthp=0.0, cthc=0.0):
    wl = np.ascontiguousarray(wl, dtype=np.float64).copy()
    wr = np.ascontiguousarray(wr, dtype=np.float64).copy()
    f = np.zeros(5)
    lib().ora_riemann_face(rsolver, eqn, ivx, gamma, _ptr(wl), _ptr(wr), _ptr(f),
                           cosf, sinf, cthp, cthc)
    return f


def implicit_columns(w, du, colgeo, x1f, x1v, dx1f, dt, gamma, grav, full=True):
    """FullCorrection (full=True) or PartialCorrection over a batch of
    columns; returns the corrected du."""
    w = np.ascontiguousarray(w, dtype=np.float64)
    out = np.ascontiguousarray(du, dtype=np.float64).copy()
    colgeo = np.ascontiguousarray(colgeo, dtype=np.float64)
    ncol, _, L = out.shape
    lib().ora_correction_columns(int(bool(full)), ncol, L, _ptr(w), _ptr(out), _ptr(colgeo),
                                 _ptr(np.ascontiguousarray(x1f)), _ptr(np.ascontiguousarray(x1v)),
                                 _ptr(np.ascontiguousarray(dx1f)), dt, gamma, grav)
    return out


def panel_tables():
    """(neighbour panel, arrival side, direction inversion, target side,
    pack order), each 6 x 4 (sides Up, Down, Left, Right)."""
    out = [np.zeros(24, dtype=np.int32) for _ in range(5)]
    lib().ora_panel_tables(*[a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) for a in out])
    return [a.reshape(6, 4) for a in out]


def vec_abp_from_rll(X, Y, blockID, U, V):
    out = np.zeros(2)
    lib().ora_vec_abp_from_rll(X, Y, blockID, U, V, _ptr(out))
    return out


def vec_rll_from_abp(X, Y, blockID, V2, V3):
    out = np.zeros(2)
    lib().ora_vec_rll_from_abp(X, Y, blockID, V2, V3, _ptr(out))
    return out


def rll_from_xyp(dX, dY, nP):
    out = np.zeros(2)
    lib().ora_rll_from_xyp(dX, dY, nP, _ptr(out))
    return out


def interp_loc(loc_n, N_blk, k, ghost):
    return lib().ora_interp_loc(loc_n, N_blk, k, int(bool(ghost)))
