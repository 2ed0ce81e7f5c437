"""Host mirror of the exo_ensemble C ABI: many independent atmospheres of
uneven size advanced by one batched, graph-captured step.

The reference runs each forward model of its MCMC inversion as a separate
atmosphere (src/inversion/profile_inversion.cpp:112-120); here they share
the GPU: every kernel of a step is launched once for all members."""
import ctypes

import numpy as np

from . import _native as nat
from .atmosphere import make_config

G = nat.NGHOST


def _cfg(cfg):
    return cfg if isinstance(cfg, nat.ExoConfig) else make_config(**cfg)


def footprint(cfg):
    """Device bytes one member of this configuration holds."""
    b = ctypes.c_size_t()
    nat.check(nat.lib().exo_ensemble_footprint(ctypes.byref(_cfg(cfg)), ctypes.byref(b)))
    return b.value


class Ensemble:
    def __init__(self, precision=nat.EXO_PREC_MIXED, capacity=64, budget_bytes=150 * 10 ** 9):
        self.precision = precision
        self._h = ctypes.c_void_p()
        nat.check(nat.lib().exo_ensemble_create(int(precision), int(capacity),
                                                int(budget_bytes), ctypes.byref(self._h)))
        self.shapes = {}
        self.cfgs = {}

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            nat.lib().exo_ensemble_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, cfg, w):
        """Admit a member; returns its slot or raises ExoError (code 7 when
        it does not fit the slots or the memory budget)."""
        if isinstance(cfg, dict) and "precision" not in cfg:
            cfg = dict(cfg, precision=self.precision)
        c = _cfg(cfg)
        w = np.ascontiguousarray(w, dtype=np.float64)
        slot = ctypes.c_int()
        nat.check(nat.lib().exo_ensemble_add(self._h, ctypes.byref(c), nat.dptr(w),
                                             ctypes.byref(slot)))
        self.shapes[slot.value] = w.shape
        self.cfgs[slot.value] = {f: getattr(c, f) for f, _ in nat.ExoConfig._fields_}
        return slot.value

    def add_checkpoint(self, image):
        """Admit a member from a checkpoint image (CubedSphereAtmosphere.
        checkpoint or Ensemble.checkpoint); it continues the run that wrote
        it, in this ensemble's precision.  Returns its slot."""
        img = np.ascontiguousarray(np.frombuffer(image, dtype=np.uint8))
        slot = ctypes.c_int()
        nat.check(nat.lib().exo_ensemble_add_checkpoint(self._h, img.ctypes.data, img.size,
                                                        ctypes.byref(slot)))
        h = nat.checkpoint_header(img)
        c = dict(h["cfg"], precision=self.precision)
        nv = 4 if c["eqn"] == nat.EXO_EQN_SHALLOW_YZ else 5
        n2 = c["N"] + 6
        self.shapes[slot.value] = (6, nv, n2, n2, c["L"] + 6)
        self.cfgs[slot.value] = c
        return slot.value

    def checkpoint(self, slot):
        """Checkpoint image of one member (numpy uint8 array)."""
        n = ctypes.c_size_t()
        nat.check(nat.lib().exo_ensemble_checkpoint_bytes(self._h, slot, ctypes.byref(n)))
        img = np.empty(n.value, dtype=np.uint8)
        nat.check(nat.lib().exo_ensemble_checkpoint_save(self._h, slot, img.ctypes.data,
                                                         n.value))
        return img

    def try_add(self, cfg, w):
        try:
            return self.add(cfg, w)
        except nat.ExoError as e:
            if e.code == 7:
                return None
            raise

    def remove(self, slot):
        nat.check(nat.lib().exo_ensemble_remove(self._h, int(slot)))
        self.shapes.pop(slot, None)
        self.cfgs.pop(slot, None)

    def step(self, nsteps=1):
        nat.check(nat.lib().exo_ensemble_step(self._h, int(nsteps)))

    def synchronize(self):
        nat.check(nat.lib().exo_ensemble_synchronize(self._h))

    def conserved(self, slot):
        a = np.empty(self.shapes[slot])
        nat.check(nat.lib().exo_ensemble_get_conserved(self._h, int(slot), nat.dptr(a)))
        return a

    def primitive(self, slot):
        a = np.empty(self.shapes[slot])
        nat.check(nat.lib().exo_ensemble_get_primitive(self._h, int(slot), nat.dptr(a)))
        return a

    def member_time(self, slot):
        t, dt, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64()
        nat.check(nat.lib().exo_ensemble_member_time(self._h, int(slot), ctypes.byref(t),
                                                     ctypes.byref(dt), ctypes.byref(n)))
        return t.value, dt.value, n.value

    @property
    def tiles(self):
        t = (ctypes.c_int * nat.EXO_TILE_COUNT)()
        nat.check(nat.lib().exo_ensemble_get_tiles(self._h, t))
        return list(t)

    def set_tiles(self, threads):
        """Launch tiles of the batched step (exo_ensemble_set_tiles)."""
        t = (ctypes.c_int * nat.EXO_TILE_COUNT)(*[int(x) for x in threads])
        nat.check(nat.lib().exo_ensemble_set_tiles(self._h, t))

    def autotune(self, cache=None):
        """Tiles minimising the summed per-member kernel times (autotune.py)."""
        from . import autotune
        tiles = autotune.batch_tiles(list(self.cfgs.values()), cache)
        self.set_tiles(tiles)
        return tiles

    def invalid(self, slot):
        """Non-zero if the member's state turned invalid since the last call."""
        f = ctypes.c_int()
        nat.check(nat.lib().exo_ensemble_check_state(self._h, int(slot), ctypes.byref(f)))
        return f.value

    def stats(self):
        m, b, l = ctypes.c_int(), ctypes.c_size_t(), ctypes.c_int64()
        nat.check(nat.lib().exo_ensemble_stats(self._h, ctypes.byref(m), ctypes.byref(b),
                                               ctypes.byref(l)))
        return {"members": m.value, "bytes": b.value, "launches": l.value}

    @property
    def stream(self):
        s = ctypes.c_void_p()
        nat.check(nat.lib().exo_ensemble_get_stream(self._h, ctypes.byref(s)))
        return s.value or 0
