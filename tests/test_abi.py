"""The C ABI library: it loads, exports every symbol include/exo_b200.h
declares, and its host-only entry points agree with the oracle bit for bit.
No compute call needs a GPU here."""
import ctypes
import os
import re

import numpy as np

from exocubed_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    text = open(os.path.join(ROOT, "include", "exo_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(exo_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(native):
    L = native.lib()
    declared = _declared_functions()
    assert len(declared) >= 15
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing
    assert sorted(native.EXPORTED) == declared


def test_config_defaults(native):
    from exocubed_b200.atmosphere import make_config
    c1 = make_config(eqn=0)
    assert (c1.N, c1.L, c1.rsolver) == (48, 3, native.EXO_RS_ROE_SHALLOW)
    c2 = make_config(eqn=1)
    assert (c2.N, c2.L, c2.implicit_flag, c2.rsolver) == (96, 64, 9, native.EXO_RS_LMARS)


def test_rejects_bad_configs(native):
    from exocubed_b200.atmosphere import make_config
    L = native.lib()
    ctx = ctypes.c_void_p()
    bad = make_config(eqn=0, N=7)  # odd edge count
    rc = L.exo_create(ctypes.byref(bad), ctypes.byref(ctx))
    assert rc != 0 and not ctx.value
    bad2 = make_config(eqn=1, rsolver=native.EXO_RS_ROE_SHALLOW)
    assert L.exo_create(ctypes.byref(bad2), ctypes.byref(ctx)) == native.EXO_OK + 1
    assert b"LMARS or HLLC" in L.exo_last_error()


def test_mesh_matches_oracle_bitwise(native, oracle_mod):
    from exocubed_b200.atmosphere import make_config
    for cfgd in (W.shallow_water_config(N=16), W.dry_atmosphere_config(N=12, L=10)):
        cfg = make_config(**cfgd)
        o = oracle_mod.Oracle(cfgd)
        for p in range(6):
            a = [np.empty(cfg.L + 7), np.empty(cfg.N + 7), np.empty(cfg.N + 7)]
            assert native.lib().exo_mesh(ctypes.byref(cfg), p, *[native.dptr(x) for x in a]) == 0
            b = o.mesh(p)
            for x, y in zip(a, b):
                assert np.array_equal(x, y)


def test_cell_geometry_is_a_sphere(native):
    from exocubed_b200.atmosphere import cell_geometry
    lat, lon, m, x1v = cell_geometry(W.shallow_water_config(N=16))
    assert np.all(np.abs(lat) <= np.pi / 2) and np.all((lon >= 0) & (lon <= 2 * np.pi))
    # equal-area-ish coverage: the six panels tile the sphere, the polar
    # panels (1 and 5) hold the poles
    assert lat[0].max() > 1.3 and lat[4].min() < -1.3
    assert np.isfinite(m).all() and x1v.shape == (3,)
