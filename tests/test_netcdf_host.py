"""NetCDF output in the reference's layout (src/outputs/netcdf.cpp), read
back with scipy's independent NetCDF classic reader."""
import numpy as np
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
