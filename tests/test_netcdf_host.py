"""NetCDF output in the reference's layout (src/outputs/netcdf.cpp), read
back with scipy's independent NetCDF classic reader; meshblock files and
their combination (src/outputs/combine_blocks.cpp, mppnccombine.cpp)."""
import os

import numpy as np
import pytest
from scipy.io import netcdf_file

from exocubed_b200 import netcdf as nc
from exocubed_b200 import workloads as W


def test_classic_file_round_trip(tmp_path):
    p = str(tmp_path / "t.nc")
    a = np.arange(12, dtype=np.float32).reshape(2, 3, 2)
    nc.write_classic(p, [("time", None), ("x", 3), ("y", 2)],
                     {"NumFilesInSet": np.array([6], np.int32), "title": "t"},
                     [("time", ["time"], {"units": "s"}, np.array([1.5, 2.5], np.float32)),
                      ("x", ["x"], {"axis": "X"}, np.array([1, 2, 3], np.float32)),
                      ("a", ["time", "x", "y"], {"units": "kg"}, a)], numrecs=2)
    f = netcdf_file(p, "r", mmap=False)
    assert f.dimensions == {"time": None, "x": 3, "y": 2}
    assert f.NumFilesInSet == 6 and f.title == b"t"
    assert np.array_equal(f.variables["time"][:], [1.5, 2.5])
    assert np.array_equal(f.variables["a"][:], a)
    assert f.variables["a"].units == b"kg"
    f.close()


def test_prim_output_layout(tmp_path, oracle_mod):
    cfg = W.dry_atmosphere_config(N=6, L=4)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(W.dry_atmosphere_state(cfg, seed=0))
    w = o.primitive()
    paths = nc.write_prim_output(w, o.mesh, "hs94", "out2", 3, time=120.0,
                                 directory=str(tmp_path))
    assert [p.split("/")[-1] for p in paths] == [f"hs94.block{b}.out2.00003.nc" for b in range(6)]
    f = netcdf_file(paths[5], "r", mmap=False)
    assert list(f.variables) == ["time", "x1", "x1f", "x2", "x2f", "x3", "x3f",
                                 "rho", "press", "vel1", "vel2", "vel3"]
    rho = f.variables["rho"]
    assert rho.dimensions == ("time", "x1", "x2", "x3") and rho.shape == (1, 4, 6, 6)
    assert rho.units == b"kg/m^3" and rho.long_name == b"density"
    # (time, x1, x2, x3) with x3 fastest: rho[0, i, j, k] = w(IDN, k, j, i) of panel 5
    want = W.interior(w)[5, 0].transpose(2, 1, 0).astype(np.float32)
    assert np.array_equal(rho[0], want)
    assert np.array_equal(f.variables["vel2"][0],
                          W.interior(w)[5, 2].transpose(2, 1, 0).astype(np.float32))
    assert list(f.variables["x2"].domain_decomposition) == [1, 12, 7, 12]
    assert list(f.variables["x3"].domain_decomposition) == [1, 18, 13, 18]
    assert f.variables["time"][0] == 120.0 and f.NumFilesInSet == 6
    f.close()


def test_coordinate_attributes(tmp_path, oracle_mod):
    cfg = W.dry_atmosphere_config(N=6, L=3)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(W.dry_atmosphere_state(cfg, seed=0))
    paths = nc.write_prim_output(o.primitive(), o.mesh, "t", directory=str(tmp_path))
    f = netcdf_file(paths[0], "r", mmap=False)
    # the long_names netcdf.cpp:147-205 writes for the coordinates
    for name, axis, long_name in (("x1", b"Z", b"Z-coordinate at cell center"),
                                  ("x1f", None, b"Z-coordinate at cell face"),
                                  ("x2", b"Y", b"Y-coordinate at cell center"),
                                  ("x2f", None, b"Y-coordinate at cell face"),
                                  ("x3", b"X", b"X-coordinate at cell center"),
                                  ("x3f", None, b"X-coordinate at cell face")):
        v = f.variables[name]
        assert v.long_name == long_name and v.units == b"m"
        assert getattr(v, "axis", None) == axis
    assert list(f.variables["x1f"].domain_decomposition) == [0, 3, 0, 3]
    f.close()


def test_meshblock_order():
    # one block per panel: gid = panel = lx2 + 2 lx3
    assert [l2 + 2 * l3 for l2, l3 in nc.meshblock_order(1)] == list(range(6))
    for nb in (2, 4):
        order = nc.meshblock_order(nb)
        assert len(order) == 6 * nb * nb
        panels = [l2 // nb + 2 * (l3 // nb) for l2, l3 in order]
        # the walk takes the panels in order, each panel's blocks together
        assert panels == sorted(panels)
        # within a panel, the Z-order of (lx2, lx3), x2 first
        assert order[:4] == [(0, 0), (1, 0), (0, 1), (1, 1)]
    with pytest.raises(ValueError):
        nc.meshblock_order(3)


def _panel_layout(w, names=("rho", "press", "vel1", "vel2", "vel3")):
    """Interior fields of the 2 x 3 panel layout as the combined file holds
    them: (1, L, 2N, 3N), x3 fastest."""
    index = {"rho": 0, "press": 4, "vel1": 1, "vel2": 2, "vel3": 3}
    wi = W.interior(w)
    N, L = wi.shape[2], wi.shape[4]
    out = {}
    for name in names:
        a = np.zeros((1, L, 2 * N, 3 * N), np.float32)
        for p in range(6):
            l2, l3 = p % 2, p // 2
            a[0, :, l2 * N:(l2 + 1) * N, l3 * N:(l3 + 1) * N] = \
                wi[p, index[name]].transpose(2, 1, 0).astype(np.float32)
        out[name] = a
    return out


def test_meshblock_files(tmp_path, oracle_mod):
    cfg = W.dry_atmosphere_config(N=8, L=3)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(W.dry_atmosphere_state(cfg, seed=1))
    w = o.primitive()
    paths = nc.write_prim_output(w, o.mesh, "hs", "out2", 7, time=3.0,
                                 directory=str(tmp_path), blocks=2)
    assert [os.path.basename(p) for p in paths] == [f"hs.block{g}.out2.00007.nc"
                                                     for g in range(24)]
    wi = W.interior(w)
    for gid, (l2, l3) in enumerate(nc.meshblock_order(2)):
        f = netcdf_file(paths[gid], "r", mmap=False)
        p, b2, b3 = l2 // 2 + 2 * (l3 // 2), l2 % 2, l3 % 2
        assert f.NumFilesInSet == 24
        assert f.variables["rho"].shape == (1, 3, 4, 4)
        want = wi[p, 4, b3 * 4:(b3 + 1) * 4, b2 * 4:(b2 + 1) * 4].transpose(2, 1, 0)
        assert np.array_equal(f.variables["press"][0], want.astype(np.float32))
        assert list(f.variables["x2"].domain_decomposition) == [1, 16, 4 * l2 + 1, 4 * l2 + 4]
        assert list(f.variables["x3f"].domain_decomposition) == [0, 24, 4 * l3, 4 * l3 + 4]
        f.close()
    with pytest.raises(ValueError):   # 16 blocks do not divide N = 8
        nc.write_prim_output(w, o.mesh, "hs", blocks=16, directory=str(tmp_path))


def test_read_classic_against_scipy_writer(tmp_path):
    p = str(tmp_path / "s.nc")
    f = netcdf_file(p, "w")
    f.createDimension("time", None)
    f.createDimension("x", 3)
    f.title = b"scipy"
    t = f.createVariable("time", "f4", ("time",))
    t[:] = [0.5, 1.5]
    x = f.createVariable("x", "f8", ("x",))
    x[:] = [1., 2., 3.]
    x.domain_decomposition = np.array([1, 6, 4, 6], np.int32)
    a = f.createVariable("a", "f4", ("time", "x"))
    a[:] = np.arange(6, dtype=np.float32).reshape(2, 3)
    f.close()
    dims, gatts, variables, numrecs = nc.read_classic(p)
    assert dims == [("time", None), ("x", 3)] and numrecs == 2
    assert gatts["title"] == "scipy"
    v = {name: (vd, atts, arr) for name, vd, atts, arr in variables}
    assert np.array_equal(v["time"][2], [0.5, 1.5])
    assert v["x"][2].dtype == np.float64 and np.array_equal(v["x"][2], [1., 2., 3.])
    assert list(v["x"][1]["domain_decomposition"]) == [1, 6, 4, 6]
    assert np.array_equal(v["a"][2], np.arange(6).reshape(2, 3))


@pytest.mark.parametrize("blocks", [1, 2])
def test_combine_blocks(tmp_path, oracle_mod, blocks):
    cfg = W.dry_atmosphere_config(N=8, L=3)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(W.dry_atmosphere_state(cfg, seed=2))
    w = o.primitive()
    d = str(tmp_path)
    paths = nc.write_prim_output(w, o.mesh, "hs", "out2", 1, time=9.0, directory=d,
                                 blocks=blocks)
    out = nc.combine_blocks("hs", "out2", 1, directory=d)
    assert os.path.basename(out) == "hs.out2.00001.nc"
    assert not any(os.path.exists(p) for p in paths)   # removed, as mppnccombine -r
    f = netcdf_file(out, "r", mmap=False)
    assert f.dimensions == {"time": None, "x1": 3, "x1f": 4, "x2": 16, "x2f": 17,
                            "x3": 24, "x3f": 25}
    assert not hasattr(f, "NumFilesInSet")
    assert not hasattr(f.variables["x2"], "domain_decomposition")
    assert f.variables["x2"].long_name == b"Y-coordinate at cell center"
    for name, want in _panel_layout(w).items():
        assert np.array_equal(f.variables[name][:], want), name
    assert f.variables["time"][0] == 9.0
    # cell centres along x2: the panel columns' own coordinates side by side
    x2 = np.concatenate([0.5 * (o.mesh(p)[1][3:12][1:] + o.mesh(p)[1][3:12][:-1])
                         for p in (4, 5)]).astype(np.float32)
    assert np.array_equal(f.variables["x2"][:], x2)
    f.close()
    with pytest.raises(RuntimeError):
        nc.combine_blocks("hs", "out2", 1, directory=d)


def test_single_level_has_no_x1_faces(tmp_path, oracle_mod):
    # the writer defines x1f only where a block has more than one level
    cfg = W.dry_atmosphere_config(N=6, L=1)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(W.dry_atmosphere_state(cfg, seed=0))
    paths = nc.write_prim_output(o.primitive(), o.mesh, "t", directory=str(tmp_path))
    f = netcdf_file(paths[0], "r", mmap=False)
    assert "x1f" not in f.dimensions and "x1f" not in f.variables
    assert f.variables["rho"].shape == (1, 1, 6, 6) and "x2f" in f.variables
    f.close()
    out = nc.combine_blocks("t", directory=str(tmp_path))
    f = netcdf_file(out, "r", mmap=False)
    assert f.variables["rho"].shape == (1, 1, 12, 18)
    f.close()
