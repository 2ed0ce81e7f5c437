"""ctypes wrapper of the reference's own exo3 and Riemann sources, compiled
unchanged against the stand-in Athena++ headers of oracle/ref/stubs into
oracle/_ref/libref_<solver>.so (oracle/ref/Makefile; needs the reference
checkout, REF=/root/reference by default).

TEST INFRASTRUCTURE ONLY: tests/test_ref_pinned.py uses it to hold the
oracle to the reference's code bit for bit.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(_HERE, "_ref")
SOLVERS = {1: "lmars", 2: "hllc_transform", 0: "roe_shallow_yz", 3: "lmars_shallow_yz"}
REF = os.environ.get("EXO_REFERENCE_DIR", "/root/reference")
_libs = {}


def available():
    """True when the libraries exist or can be built here."""
    return all(os.path.exists(_path(s)) for s in SOLVERS.values()) or \
        os.path.isdir(os.path.join(REF, "src", "exo3"))


def _path(solver):
    return os.path.join(OUT, f"libref_{solver}.so")


def build():
    subprocess.run(["make", "-s", "-C", os.path.join(_HERE, "ref"), f"REF={REF}"], check=True)


def lib(rsolver=1):
    name = SOLVERS[rsolver]
    if name not in _libs:
        if not os.path.exists(_path(name)) and os.path.isdir(os.path.join(REF, "src")):
            build()
        L = ctypes.CDLL(_path(name), mode=ctypes.RTLD_LOCAL)
        d, i, p = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.ref_vec_abp_from_rll.argtypes = [d, d, i, d, d, dp]
        L.ref_vec_rll_from_abp.argtypes = [d, d, i, d, d, dp]
        L.ref_rll_from_xyp.argtypes = [d, d, i, dp]
        L.ref_interp_loc.restype = d
        L.ref_interp_loc.argtypes = [i, i, i, i]
        L.ref_find_block_id.restype = i
        L.ref_find_block_id.argtypes = [i, i, i]
        L.ref_transform_ox.restype = i
        L.ref_transform_ox.argtypes = [i, i, i, i, i, ip]
        L.ref_pack_data.restype = i
        L.ref_pack_data.argtypes = [dp] + [i] * 18 + [dp]
        L.ref_sphere_create.restype = p
        L.ref_sphere_create.argtypes = [i, i, i, d, dp, dp, dp, dp]
        L.ref_sphere_destroy.argtypes = [p]
        L.ref_sphere_set_neighbor.argtypes = [p, i, i, i]
        L.ref_sphere_gid.restype = i
        L.ref_sphere_gid.argtypes = [p, i]
        L.ref_cell_geometry.argtypes = [p, i, i, i, i, dp]
        L.ref_riemann.argtypes = [p, i, i, i, i, i, i, dp, dp, dp]
        L.ref_sphere_face_sync.restype = i
        L.ref_sphere_face_sync.argtypes = [p, dp, dp]
        _libs[name] = L
    return _libs[name]


def ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


_decomp = None


def decomposition_lib():
    """The reference's hydrostatic decomposition (change_to_perturbation.cpp,
    decomposition.cpp) on one panel: oracle/_ref/libref_decomposition.so."""
    global _decomp
    if _decomp is None:
        path = os.path.join(OUT, "libref_decomposition.so")
        if not os.path.exists(path) and os.path.isdir(os.path.join(REF, "src")):
            build()
        L = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
        d, i, p = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
        dp = ctypes.POINTER(ctypes.c_double)
        L.ref_decomp_create.restype = p
        L.ref_decomp_create.argtypes = [i, i, d, d, d, dp, dp, dp, dp]
        L.ref_decomp_destroy.argtypes = [p]
        L.ref_change_to_perturbation.argtypes = [p, dp]
        L.ref_restore_from_perturbation.argtypes = [p, dp, dp, dp, i, i, i, i]
        _decomp = L
    return _decomp


class DecomposedPanel:
    """One panel (MeshBlock) with the reference's Decomposition object."""

    def __init__(self, N, L, gamma, Rd, grav, x1f, dx1f, x2f, x3f):
        self.L_ = decomposition_lib()
        self._keep = [np.ascontiguousarray(a, dtype=np.float64) for a in (x1f, dx1f, x2f, x3f)]
        self.h = self.L_.ref_decomp_create(N, L, gamma, Rd, grav, *[ptr(a) for a in self._keep])

    def close(self):
        if self.h:
            self.L_.ref_decomp_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def change_to_perturbation(self, w):
        """w: one panel's primitives (5, N+6, N+6, L+6), changed in place."""
        assert w.flags.c_contiguous and w.dtype == np.float64
        self.L_.ref_change_to_perturbation(self.h, ptr(w))

    def restore_from_perturbation(self, w, wl, wr, k, j, il, iu):
        """w in place; wl, wr: face states of row (k, j), (5, L+6), in place."""
        for a in (w, wl, wr):
            assert a.flags.c_contiguous and a.dtype == np.float64
        self.L_.ref_restore_from_perturbation(self.h, ptr(w), ptr(wl), ptr(wr), k, j, il, iu)


class Sphere:
    """Six panels of one block each (MeshBlocks with the reference's
    GnomonicEquiangle, CubedSphere and Hydro objects) on a given mesh."""

    def __init__(self, rsolver, N, L, gamma, x1f, dx1f, x2f_panels, x3f_panels, nbr_panel):
        self.L_ = lib(rsolver)
        self.N, self.L = N, L
        self._keep = [np.ascontiguousarray(a, dtype=np.float64)
                      for a in (x1f, dx1f, x2f_panels, x3f_panels)]
        self.h = self.L_.ref_sphere_create(N, L, 1, gamma, *[ptr(a) for a in self._keep])
        if not self.h:
            raise ValueError("reference harness rejected the mesh")
        # one block per panel: the neighbour across side s of panel p is
        # panel nbr_panel[p][s] (1-based), whose gid is its index
        for p in range(6):
            for s in range(4):
                self.L_.ref_sphere_set_neighbor(self.h, p, s, int(nbr_panel[p][s]) - 1)

    def close(self):
        if self.h:
            self.L_.ref_sphere_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def cell_geometry(self, p, k, j, i):
        """Face1/2/3 areas, volume, centre widths 1/2/3 (the row forms), then
        the point forms of the areas and the volume."""
        out = np.zeros(11)
        self.L_.ref_cell_geometry(self.h, p, k, j, i, ptr(out))
        return out

    def riemann(self, p, k, j, ivx, il, iu, wl, wr):
        """Fluxes of faces il..iu of row (k, j) of panel p; wl, wr are
        (5, nc1) and are modified in place as the reference does."""
        nc1 = self.L + 6
        flx = np.zeros((5, nc1))
        self.L_.ref_riemann(self.h, p, k, j, ivx, il, iu, ptr(wl), ptr(wr), ptr(flx))
        return flx

    def face_sync(self, L, R):
        """L, R: (6, 2, 5, nc3, nc2, nc1) x2 and x3 face states, exchanged in place."""
        rc = self.L_.ref_sphere_face_sync(self.h, ptr(L), ptr(R))
        if rc:
            raise RuntimeError(f"reference face exchange failed ({rc})")
