"""Host-side mirror of the reference's per-MeshBlock operator interface.

`CubedSphereAtmosphere` owns one exo_ctx: the six panels of one atmosphere,
resident in HBM.  Its methods are the reference's hooks on that path:

  calculate_fluxes()  Hydro::CalculateFluxes (patches/19.calculate_fluxes.patch)
  step(n, dt)         DoTaskListOneStage x 3 per step (main.cpp.in:139-141)
  new_dt()            Mesh::NewTimeStep (patches/21.new_blockdt.patch)
  riemann_solver(...) Hydro::RiemannSolver on device rows (src/snap/riemann/*)

Arrays follow AthenaArray(n,k,j,i) per panel, six panels stacked:
shape (6, nvar, N+6, N+6, L+6).
"""
import ctypes
import os

import numpy as np

from . import _native as nat


def make_config(**kw):
    """exo_config with the defaults of kw['eqn'] (shallow water if absent)."""
    cfg = nat.ExoConfig()
    nat.check(nat.lib().exo_config_default(ctypes.byref(cfg), int(kw.get("eqn", 0))))
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg


def cell_geometry(cfg):
    """(lat, lon, uv_to_v23, x1v) of the interior cells; no GPU needed."""
    cfg = cfg if isinstance(cfg, nat.ExoConfig) else make_config(**cfg)
    N, L = cfg.N, cfg.L
    lat = np.empty((6, N, N))
    lon = np.empty((6, N, N))
    m = np.empty((6, N, N, 4))
    x1v = np.empty(L)
    nat.check(nat.lib().exo_cell_geometry(ctypes.byref(cfg), nat.dptr(lat), nat.dptr(lon),
                                          nat.dptr(m), nat.dptr(x1v)))
    return lat, lon, m, x1v


def mesh(cfg, panel):
    """(x1f, x2f, x3f) face coordinates of a panel, ghosts included; no GPU
    needed."""
    cfg = cfg if isinstance(cfg, nat.ExoConfig) else make_config(**cfg)
    x1f = np.empty(cfg.L + 7)
    x2f = np.empty(cfg.N + 7)
    x3f = np.empty(cfg.N + 7)
    nat.check(nat.lib().exo_mesh(ctypes.byref(cfg), int(panel), nat.dptr(x1f), nat.dptr(x2f),
                                 nat.dptr(x3f)))
    return x1f, x2f, x3f


class CubedSphereAtmosphere:
    """Six-panel cubed-sphere atmosphere advanced on the current CUDA device."""

    def __init__(self, cfg=None, **kw):
        if cfg is None:
            cfg = make_config(**kw)
        elif isinstance(cfg, dict):
            cfg = make_config(**cfg)
        self.cfg = cfg
        self._ctx = ctypes.c_void_p()
        nat.check(nat.lib().exo_create(ctypes.byref(cfg), ctypes.byref(self._ctx)))
        nv, n3, n2, n1 = (ctypes.c_int() for _ in range(4))
        nat.check(nat.lib().exo_shape(self._ctx, ctypes.byref(nv), ctypes.byref(n3),
                                      ctypes.byref(n2), ctypes.byref(n1)))
        self.nvar = nv.value
        self.shape = (6, nv.value, n3.value, n2.value, n1.value)

    def close(self):
        if getattr(self, "_ctx", None) and self._ctx.value:
            nat.lib().exo_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---------------------------------------------------------------- state
    def set_primitive(self, w):
        w = np.ascontiguousarray(w, dtype=np.float64)
        if w.shape != self.shape:
            raise ValueError(f"expected shape {self.shape}, got {w.shape}")
        nat.check(nat.lib().exo_set_primitive(self._ctx, nat.dptr(w)))

    def conserved(self, out=None):
        a = np.empty(self.shape) if out is None else out
        nat.check(nat.lib().exo_get_conserved(self._ctx, nat.dptr(a)))
        return a

    def primitive(self, out=None):
        a = np.empty(self.shape) if out is None else out
        nat.check(nat.lib().exo_get_primitive(self._ctx, nat.dptr(a)))
        return a

    def device_pointers(self):
        u, w = ctypes.c_void_p(), ctypes.c_void_p()
        nat.check(nat.lib().exo_device_state(self._ctx, ctypes.byref(u), ctypes.byref(w)))
        return u.value, w.value

    # ------------------------------------------------------------- stepping
    def step(self, nsteps=1, dt_fixed=0.0):
        nat.check(nat.lib().exo_step(self._ctx, int(nsteps), float(dt_fixed)))

    def stage(self, s):
        """One SSPRK(3,3) stage (0, 1, 2) on the CFL step; see exo_stage."""
        nat.check(nat.lib().exo_stage(self._ctx, int(s)))

    def boundary(self):
        """Ghost syncs and ConservedToPrimitive of the current state."""
        nat.check(nat.lib().exo_boundary(self._ctx))

    def solve_implicit_3d(self, du, w, dt):
        """ImplicitSolver::SolveImplicit3D: du corrected in place from w.  It
        uses the context's device arrays; load a state before stepping on."""
        assert du.shape == self.shape and du.flags.c_contiguous and du.dtype == np.float64
        w = np.ascontiguousarray(w, dtype=np.float64)
        nat.check(nat.lib().exo_solve_implicit_3d(self._ctx, nat.dptr(du), nat.dptr(w), float(dt)))

    def change_to_perturbation(self, w):
        """Decomposition::ChangeToPerturbation on w (whole-array layout, in place)."""
        assert w.shape == self.shape and w.flags.c_contiguous and w.dtype == np.float64
        nat.check(nat.lib().exo_change_to_perturbation(self._ctx, nat.dptr(w)))

    def restore_from_perturbation(self, w, wl, wr):
        """Decomposition::RestoreFromPerturbation: w, and the x1 face states wl,
        wr (same layout as w), restored in place."""
        for a in (w, wl, wr):
            assert a.shape == self.shape and a.flags.c_contiguous and a.dtype == np.float64
        nat.check(nat.lib().exo_restore_from_perturbation(self._ctx, nat.dptr(w), nat.dptr(wl),
                                                          nat.dptr(wr)))

    def set_max_redo(self, max_redo):
        """Redo of failed steps with half the time step (the reference's
        max_redo; 0 turns it off)."""
        nat.check(nat.lib().exo_set_max_redo(self._ctx, int(max_redo)))

    @property
    def redo_count(self):
        n = ctypes.c_int64()
        nat.check(nat.lib().exo_redo_count(self._ctx, ctypes.byref(n)))
        return n.value

    def write_netcdf(self, basename, file_id="out2", number=0, directory=".", blocks=1,
                     combine=False):
        """Primitive output in the reference's per-meshblock NetCDF layout
        (exocubed_b200.netcdf): blocks x blocks files per panel; with
        combine, joined into the one file the reference's CombineBlocks
        leaves.  Returns the paths written."""
        from . import netcdf
        paths = netcdf.write_prim_output(self.primitive(), lambda p: mesh(self.cfg, p), basename,
                                         file_id, number, self.time, directory, blocks)
        if combine:
            return [netcdf.combine_blocks(basename, file_id, number, directory)]
        return paths

    def checkpoint(self):
        """The run's checkpoint image (numpy uint8 array): configuration,
        clock, conserved and primitive arrays.  restore() or
        Ensemble.add_checkpoint() continue it bit for bit."""
        n = ctypes.c_size_t()
        nat.check(nat.lib().exo_checkpoint_bytes(self._ctx, ctypes.byref(n)))
        img = np.empty(n.value, dtype=np.uint8)
        nat.check(nat.lib().exo_checkpoint_save(self._ctx, img.ctypes.data, n.value))
        return img

    def restore(self, image):
        """Continue from a checkpoint image of this configuration (the
        precision may differ)."""
        img = np.ascontiguousarray(np.frombuffer(image, dtype=np.uint8))
        nat.check(nat.lib().exo_checkpoint_load(self._ctx, img.ctypes.data, img.size))

    def save_checkpoint(self, path):
        """Write the checkpoint image to a file."""
        img = self.checkpoint()
        with open(path, "wb") as f:
            f.write(img.tobytes())

    @classmethod
    def from_checkpoint(cls, path_or_image, precision=None):
        """A context built from a checkpoint's configuration and resumed from
        it; precision overrides the one it was written with."""
        if isinstance(path_or_image, (str, os.PathLike)):
            with open(path_or_image, "rb") as f:
                image = f.read()
        else:
            image = path_or_image
        cfg = dict(nat.checkpoint_header(image)["cfg"])
        if precision is not None:
            cfg["precision"] = precision
        a = cls(make_config(**cfg))
        a.restore(image)
        return a

    def synchronize(self):
        nat.check(nat.lib().exo_synchronize(self._ctx))

    @property
    def dt(self):
        d = ctypes.c_double()
        nat.check(nat.lib().exo_get_dt(self._ctx, ctypes.byref(d)))
        return d.value

    def new_dt(self):
        return self.dt

    @property
    def time(self):
        t, n = ctypes.c_double(), ctypes.c_int64()
        nat.check(nat.lib().exo_get_time(self._ctx, ctypes.byref(t), ctypes.byref(n)))
        return t.value

    @property
    def ncycle(self):
        """Steps taken."""
        t, n = ctypes.c_double(), ctypes.c_int64()
        nat.check(nat.lib().exo_get_time(self._ctx, ctypes.byref(t), ctypes.byref(n)))
        return n.value

    @property
    def tiles(self):
        """Threads per block of each kernel, indexed by EXO_K_* (exo_get_tiles)."""
        t = (ctypes.c_int * nat.EXO_TILE_COUNT)()
        nat.check(nat.lib().exo_get_tiles(self._ctx, t))
        return list(t)

    def set_tiles(self, threads):
        """Set launch tiles (entries 0 keep the current value); see exo_set_tiles."""
        t = (ctypes.c_int * nat.EXO_TILE_COUNT)(*[int(x) for x in threads])
        nat.check(nat.lib().exo_set_tiles(self._ctx, t))

    def autotune(self, cache=None):
        """Set the fastest measured tile of every kernel for this configuration
        (autotune.best_tiles: timed once on a throw-away context, then cached)
        and return the tiles.  The arithmetic per cell does not change."""
        from . import autotune
        tiles = autotune.best_tiles(self.cfg, cache)
        self.set_tiles(tiles)
        return self.tiles

    def invalid(self):
        f = ctypes.c_int()
        nat.check(nat.lib().exo_check_state(self._ctx, ctypes.byref(f)))
        return f.value

    @property
    def stream(self):
        s = ctypes.c_void_p()
        nat.check(nat.lib().exo_get_stream(self._ctx, ctypes.byref(s)))
        return s.value or 0

    def profile(self, enable=True):
        nat.check(nat.lib().exo_profile(self._ctx, 1 if enable else 0))

    def profile_read(self):
        out = {}
        for kid, name in enumerate(nat.KERNELS):
            n, ms = ctypes.c_int64(), ctypes.c_double()
            nat.check(nat.lib().exo_profile_read(self._ctx, kid, ctypes.byref(n), ctypes.byref(ms)))
            out[name] = (n.value, ms.value)
        return out

    def launch_count(self):
        n = ctypes.c_int64()
        nat.check(nat.lib().exo_launch_count(self._ctx, ctypes.byref(n)))
        return n.value

    def set_primitive_ptr(self, host_ptr):
        """exo_set_primitive from a raw host pointer (e.g. pinned memory)."""
        nat.check(nat.lib().exo_set_primitive(self._ctx, ctypes.cast(host_ptr, ctypes.POINTER(ctypes.c_double))))

    def conserved_ptr(self, host_ptr):
        nat.check(nat.lib().exo_get_conserved(self._ctx, ctypes.cast(host_ptr, ctypes.POINTER(ctypes.c_double))))

    # ---------------------------------------------------------- operators
    def calculate_fluxes(self):
        nat.check(nat.lib().exo_calculate_fluxes(self._ctx))

    def flux(self, d):
        a = np.empty(self.shape)
        nat.check(nat.lib().exo_get_flux(self._ctx, int(d), nat.dptr(a)))
        return a


def riemann_rows(rsolver, eqn, ivx, gamma, wl_ptr, wr_ptr, flx_ptr, n, cos_ptr=0, sin_ptr=0,
                 cthp_ptr=0, cthc_ptr=0, stream=0):
    """Raw-pointer form of exo_riemann (device pointers, (nvar, n) rows)."""
    nat.check(nat.lib().exo_riemann(int(rsolver), int(eqn), int(ivx), int(n), float(gamma),
                                    wl_ptr, wr_ptr, flx_ptr, cos_ptr or None, sin_ptr or None,
                                    cthp_ptr or None, cthc_ptr or None, stream or None))
