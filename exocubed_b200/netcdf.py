"""NetCDF output of primitive fields in the reference's layout.

The reference writes one file per meshblock (src/outputs/netcdf.cpp:40-460),
named `<problem_id>.block<gid>.<file_id>.<5-digit number>.nc`, with the
dimensions time (unlimited), x1, x1f, x2, x2f, x3, x3f, the coordinate
variables of the same names (axis, units, long_name and a
domain_decomposition attribute), a global NumFilesInSet, and per output
variable a float array (time, x1, x2, x3) -- x3 varying fastest -- with the
units and long_name of its MetadataTable (src/outputs/output_utils.cpp:
25-50): rho [kg/m^3], press [pa], and the velocity vector as vel1, vel2,
vel3 [m/s].  Here a meshblock is a panel (gid = panel, at (lx2, lx3) =
(panel % 2, panel // 2) of the 2 x 3 panel layout).

The reference calls libnetcdf with NC_NETCDF4 (HDF5 storage); that library
is not linked here, so the files are written in the NetCDF classic
format (the published CDF-1 layout: big-endian header of dimension,
attribute and variable lists, then the fixed-size variables, then the
records), which every NetCDF reader opens with the same dimensions,
variables and attributes.
"""
import os
import struct

import numpy as np

NC_DIMENSION, NC_VARIABLE, NC_ATTRIBUTE = 0x0A, 0x0B, 0x0C
NC_CHAR, NC_INT, NC_FLOAT, NC_DOUBLE = 2, 4, 5, 6
_NPTYPE = {NC_CHAR: ">S1", NC_INT: ">i4", NC_FLOAT: ">f4", NC_DOUBLE: ">f8"}


def _pad4(b):
    return b + b"\0" * (-len(b) % 4)


def _name(s):
    b = s.encode()
    return struct.pack(">i", len(b)) + _pad4(b)


def _attrs(atts):
    if not atts:
        return struct.pack(">ii", 0, 0)
    out = struct.pack(">ii", NC_ATTRIBUTE, len(atts))
    for k, v in atts.items():
        out += _name(k)
        if isinstance(v, str):
            b = v.encode()
            out += struct.pack(">ii", NC_CHAR, len(b)) + _pad4(b)
        else:
            a = np.atleast_1d(v)
            t = NC_INT if a.dtype.kind in "iu" else (NC_FLOAT if a.dtype == np.float32 else NC_DOUBLE)
            a = a.astype(_NPTYPE[t])
            out += struct.pack(">ii", t, a.size) + _pad4(a.tobytes())
    return out


def write_classic(path, dims, gatts, variables, numrecs=1):
    """Write a NetCDF classic (CDF-1) file.
    dims       [(name, length)], length None for the unlimited dimension
    gatts      {name: str | number | array}
    variables  [(name, [dim names], atts dict, numpy array)]; a variable
               whose first dimension is the unlimited one holds numrecs
               records (array shape (numrecs, ...))."""
    dim_index = {d: n for n, (d, _) in enumerate(dims)}
    unlimited = [d for d, L in dims if L is None]
    rec_dim = unlimited[0] if unlimited else None
    dlist = struct.pack(">ii", NC_DIMENSION, len(dims))
    for d, L in dims:
        dlist += _name(d) + struct.pack(">i", 0 if L is None else L)
    head = b"CDF\x01" + struct.pack(">i", numrecs) + dlist + _attrs(gatts)
    specs = []
    for name, vd, atts, arr in variables:
        t = NC_FLOAT if arr.dtype == np.float32 else (NC_INT if arr.dtype.kind in "iu" else NC_DOUBLE)
        data = np.ascontiguousarray(arr, dtype=_NPTYPE[t])
        is_rec = bool(vd) and vd[0] == rec_dim
        slab = data[0:1] if is_rec else data  # slices keep the big-endian dtype
        vsize = len(_pad4(slab.tobytes()))
        specs.append((name, vd, atts, t, data, is_rec, vsize))

    def var_list(offsets):
        out = struct.pack(">ii", NC_VARIABLE, len(specs))
        for (name, vd, atts, t, data, is_rec, vsize), off in zip(specs, offsets):
            out += _name(name) + struct.pack(">i", len(vd))
            out += b"".join(struct.pack(">i", dim_index[d]) for d in vd)
            out += _attrs(atts) + struct.pack(">iii", t, vsize, off)
        return out

    # fixed-size variables follow the header in order; each record holds
    # the record variables' slabs in order
    hsize = len(head) + len(var_list([0] * len(specs)))
    offsets, pos = [0] * len(specs), hsize
    for n, s in enumerate(specs):
        if not s[5]:
            offsets[n] = pos
            pos += s[6]
    for n, s in enumerate(specs):
        if s[5]:
            offsets[n] = pos
            pos += s[6]
    with open(path, "wb") as f:
        f.write(head + var_list(offsets))
        for s in specs:
            if not s[5]:
                f.write(_pad4(s[4].tobytes()))
        for r in range(numrecs):
            for s in specs:
                if s[5]:
                    f.write(_pad4(s[4][r:r + 1].tobytes()))


# the reference's MetadataTable entries used by primitive output
_META = {"x1": ("height at cell center", "m"), "x1f": ("height at cell boundary", "m"),
         "x2": ("distance at cell center", "m"), "x2f": ("distance at cell boundary", "m"),
         "x3": ("distance at cell center", "m"), "x3f": ("distance at cell boundary", "m"),
         "rho": ("density", "kg/m^3"), "press": ("pressure", "pa"),
         "vel": ("velocity", "m/s")}


def write_prim_output(w, mesh, basename, file_id="out2", number=0, time=0.0, directory="."):
    """Write the primitives w (6, nvar, nc3, nc2, nc1) of one atmosphere as
    six per-panel files in the reference's layout; mesh(panel) -> (x1f,
    x2f, x3f) face coordinates including ghosts (CubedSphereAtmosphere /
    oracle mesh).  Returns the file paths."""
    G = 3
    nv = w.shape[1]
    N, L = w.shape[3] - 2 * G, w.shape[4] - 2 * G
    names = ["rho", "press", "vel1", "vel2", "vel3"] if nv == 5 else ["rho", "vel1", "vel2",
                                                                      "vel3"]
    index = {"rho": 0, "press": 4, "vel1": 1, "vel2": 2, "vel3": 3}
    paths = []
    for p in range(6):
        x1f, x2f, x3f = mesh(p)
        x1f, x2f, x3f = x1f[G:G + L + 1], x2f[G:G + N + 1], x3f[G:G + N + 1]
        x1v = 0.5 * (x1f[1:] + x1f[:-1])
        x2v = 0.5 * (x2f[1:] + x2f[:-1])
        x3v = 0.5 * (x3f[1:] + x3f[:-1])
        lx2, lx3 = p % 2, p // 2
        dims = [("time", None), ("x1", L), ("x1f", L + 1), ("x2", N), ("x2f", N + 1),
                ("x3", N), ("x3f", N + 1)]

        def coord(name, axis, vals, pos):
            atts = {}
            if axis:
                atts["axis"] = axis
            long_name, units = _META[name]
            atts["units"] = units
            atts["long_name"] = long_name
            atts["domain_decomposition"] = np.array(pos, dtype=np.int32)
            return (name, [name], atts, np.asarray(vals, dtype=np.float32))

        variables = [("time", ["time"], {"axis": "T", "units": "s", "long_name": "time"},
                      np.array([time], dtype=np.float32))]
        variables += [coord("x1", "Z", x1v, [1, L, 1, L]), coord("x1f", None, x1f, [0, L, 0, L]),
                      coord("x2", "Y", x2v, [1, 2 * N, N * lx2 + 1, N * (lx2 + 1)]),
                      coord("x2f", None, x2f, [0, 2 * N, N * lx2, N * (lx2 + 1)]),
                      coord("x3", "X", x3v, [1, 3 * N, N * lx3 + 1, N * (lx3 + 1)]),
                      coord("x3f", None, x3f, [0, 3 * N, N * lx3, N * (lx3 + 1)])]
        for name in names:
            f = w[p, index[name], G:G + N, G:G + N, G:G + L]          # (k, j, i)
            data = np.transpose(f, (2, 1, 0))[None].astype(np.float32)  # (time, i, j, k)
            long_name, units = _META["vel" if name.startswith("vel") else name]
            variables.append((name, ["time", "x1", "x2", "x3"],
                              {"units": units, "long_name": long_name}, data))
        path = os.path.join(directory, f"{basename}.block{p}.{file_id}.{number:05d}.nc")
        write_classic(path, dims, {"NumFilesInSet": np.array([6], dtype=np.int32)}, variables)
        paths.append(path)
    return paths
