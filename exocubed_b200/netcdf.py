"""NetCDF output of primitive fields in the reference's layout.

The reference writes one file per meshblock (src/outputs/netcdf.cpp:40-460),
named `<problem_id>.block<gid>.<file_id>.<5-digit number>.nc`, with the
dimensions time (unlimited), x1, x1f, x2, x2f, x3, x3f, the coordinate
variables of the same names (axis, units, the long_names the writer spells
out, "Z-", "Y-" and "X-coordinate at cell center / face" (netcdf.cpp:
147-205), and a domain_decomposition attribute: first and last global index,
first and last index of this block), a global NumFilesInSet (the number of
meshblocks), and per output variable a float array (time, x1, x2, x3) -- x3
varying fastest -- with the units and long_name of its MetadataTable entry
(src/outputs/output_utils.cpp:25-50): rho [kg/m^3], press [pa], and the
velocity vector as vel1, vel2, vel3 [m/s].

Meshblocks.  The mesh lays the six panels out as 2 x 3 (panel = lx2 + 2 lx3
at the panel level, CubedSphere::FindBlockID, src/exo3/cubed_sphere.cpp:
82-84); a panel of nb x nb meshblocks (nb a power of two, the shift in
FindBlockID) puts block (b2, b3) of panel p at lx2 = nb (p % 2) + b2,
lx3 = nb (p // 2) + b3.  Athena++ numbers the meshblocks (gid) in the order
of a depth-first walk of its block tree, children with the x1 bit fastest,
then x2, then x3: the Z-order of (lx2, lx3).  That walk takes the panels in
order and each panel's blocks one after the other.

combine_blocks joins one output's block files into
`<problem_id>.<file_id>.<number>.nc` the way the reference's
NetcdfOutput::CombineBlocks (src/outputs/combine_blocks.cpp:19-83) does it
with its restatement of mppnccombine (src/outputs/mppnccombine.cpp): each
dimension takes the full size its coordinate's domain_decomposition names,
every decomposed variable is placed at its block's offset (files in the
sorted order of the glob, so a face shared by two blocks holds the later
file's value), the other variables come from the first file,
domain_decomposition and NumFilesInSet are dropped, and the block files are
removed afterwards.

The reference calls libnetcdf with NC_NETCDF4 (HDF5 storage); that library
is not linked here, so the files are written in the NetCDF classic
format (the published CDF-1 layout: big-endian header of dimension,
attribute and variable lists, then the fixed-size variables, then the
records), which every NetCDF reader opens with the same dimensions,
variables and attributes.
"""
import glob
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


# units and long_name of the output variables (MetadataTable,
# src/outputs/output_utils.cpp:25-50)
_META = {"rho": ("density", "kg/m^3"), "press": ("pressure", "pa"),
         "vel": ("velocity", "m/s")}
# the coordinates' long_names as the writer spells them (netcdf.cpp:147-205)
_COORD_LONG = {"x1": "Z-coordinate at cell center", "x1f": "Z-coordinate at cell face",
               "x2": "Y-coordinate at cell center", "x2f": "Y-coordinate at cell face",
               "x3": "X-coordinate at cell center", "x3f": "X-coordinate at cell face"}


def meshblock_order(nb):
    """(lx2, lx3) of the 6 nb^2 meshblocks of a cubed sphere with nb x nb
    blocks per panel, in gid order (the Z-order of (lx2, lx3), x2 bit
    first).  nb must be a power of two (FindBlockID's shift)."""
    if nb < 1 or nb & (nb - 1):
        raise ValueError(f"blocks per panel edge must be a power of two (got {nb})")

    def z(l2, l3):
        key = 0
        for b in range(12):
            key |= ((l2 >> b) & 1) << (2 * b) | ((l3 >> b) & 1) << (2 * b + 1)
        return key

    return sorted(((l2, l3) for l3 in range(3 * nb) for l2 in range(2 * nb)),
                  key=lambda c: z(*c))


def write_prim_output(w, mesh, basename, file_id="out2", number=0, time=0.0, directory=".",
                      blocks=1):
    """Write the primitives w (6, nvar, nc3, nc2, nc1) of one atmosphere as
    one file per meshblock in the reference's layout, each panel cut into
    blocks x blocks meshblocks of N / blocks cells a side; mesh(panel) ->
    (x1f, x2f, x3f) face coordinates including ghosts (CubedSphereAtmosphere
    / oracle mesh).  Returns the file paths in gid order."""
    G = 3
    nv = w.shape[1]
    N, L = w.shape[3] - 2 * G, w.shape[4] - 2 * G
    nb = int(blocks)
    order = meshblock_order(nb)
    if N % nb:
        raise ValueError(f"{nb} blocks per panel edge do not divide N = {N}")
    n = N // nb
    names = ["rho", "press", "vel1", "vel2", "vel3"] if nv == 5 else ["rho", "vel1", "vel2",
                                                                      "vel3"]
    index = {"rho": 0, "press": 4, "vel1": 1, "vel2": 2, "vel3": 3}
    # a face dimension and its coordinate exist only where the block has
    # more than one cell along the axis (netcdf.cpp:110-133)
    dims = [("time", None), ("x1", L)] + ([("x1f", L + 1)] if L > 1 else []) + \
        [("x2", n)] + ([("x2f", n + 1)] if n > 1 else []) + \
        [("x3", n)] + ([("x3f", n + 1)] if n > 1 else [])
    gatts = {"NumFilesInSet": np.array([6 * nb * nb], dtype=np.int32)}
    faces = [mesh(p) for p in range(6)]

    def coord(name, axis, vals, pos):
        atts = {"axis": axis} if axis else {}
        atts["units"] = "m"
        atts["long_name"] = _COORD_LONG[name]
        atts["domain_decomposition"] = np.array(pos, dtype=np.int32)
        return (name, [name], atts, np.asarray(vals, dtype=np.float32))

    paths = []
    for gid, (lx2, lx3) in enumerate(order):
        p = lx2 // nb + 2 * (lx3 // nb)
        j0, k0 = G + (lx2 % nb) * n, G + (lx3 % nb) * n
        x1f, x2f, x3f = faces[p]
        x1f, x2f, x3f = x1f[G:G + L + 1], x2f[j0:j0 + n + 1], x3f[k0:k0 + n + 1]
        x1v = 0.5 * (x1f[1:] + x1f[:-1])
        x2v = 0.5 * (x2f[1:] + x2f[:-1])
        x3v = 0.5 * (x3f[1:] + x3f[:-1])
        variables = [("time", ["time"], {"axis": "T", "units": "s", "long_name": "time"},
                      np.array([time], dtype=np.float32))]
        variables.append(coord("x1", "Z", x1v, [1, L, 1, L]))
        if L > 1:
            variables.append(coord("x1f", None, x1f, [0, L, 0, L]))
        variables.append(coord("x2", "Y", x2v, [1, 2 * N, n * lx2 + 1, n * (lx2 + 1)]))
        if n > 1:
            variables.append(coord("x2f", None, x2f, [0, 2 * N, n * lx2, n * (lx2 + 1)]))
        variables.append(coord("x3", "X", x3v, [1, 3 * N, n * lx3 + 1, n * (lx3 + 1)]))
        if n > 1:
            variables.append(coord("x3f", None, x3f, [0, 3 * N, n * lx3, n * (lx3 + 1)]))
        for name in names:
            f = w[p, index[name], k0:k0 + n, j0:j0 + n, G:G + L]       # (k, j, i)
            data = np.transpose(f, (2, 1, 0))[None].astype(np.float32)  # (time, i, j, k)
            long_name, units = _META["vel" if name.startswith("vel") else name]
            variables.append((name, ["time", "x1", "x2", "x3"],
                              {"units": units, "long_name": long_name}, data))
        path = os.path.join(directory, f"{basename}.block{gid}.{file_id}.{number:05d}.nc")
        write_classic(path, dims, gatts, variables)
        paths.append(path)
    return paths


_NC_TYPES = {1: ">i1", 2: ">S1", 3: ">i2", 4: ">i4", 5: ">f4", 6: ">f8"}


def read_classic(path):
    """(dims, gatts, variables, numrecs) of a NetCDF classic file (CDF-1 or
    CDF-2), in write_classic's argument form: dims [(name, length or None)],
    gatts {name: str | array}, variables [(name, [dims], atts, array)] with
    record variables shaped (numrecs, ...)."""
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:3] != b"CDF" or buf[3] not in (1, 2):
        raise ValueError(f"{path}: not a NetCDF classic file")
    off64 = buf[3] == 2
    pos = [4]

    def i32():
        v = struct.unpack_from(">i", buf, pos[0])[0]
        pos[0] += 4
        return v

    def name():
        ln = i32()
        s = buf[pos[0]:pos[0] + ln].decode()
        pos[0] += ln + (-ln % 4)
        return s

    def attrs():
        tag, cnt = i32(), i32()
        out = {}
        for _ in range(cnt if tag == NC_ATTRIBUTE else 0):
            k, t, ln = name(), i32(), i32()
            dt = np.dtype(_NC_TYPES[t])
            raw = buf[pos[0]:pos[0] + ln * dt.itemsize]
            pos[0] += len(_pad4(raw))
            out[k] = raw.decode() if t == NC_CHAR else np.frombuffer(raw, dt).copy()
        return out

    numrecs = i32()
    tag, cnt = i32(), i32()
    dims = []
    for _ in range(cnt if tag == NC_DIMENSION else 0):
        d, ln = name(), i32()
        dims.append((d, None if ln == 0 else ln))
    gatts = attrs()
    tag, cnt = i32(), i32()
    specs = []
    for _ in range(cnt if tag == NC_VARIABLE else 0):
        v, nd = name(), i32()
        vd = [dims[i32()][0] for _ in range(nd)]
        atts, t, vsize = attrs(), i32(), i32()
        begin = struct.unpack_from(">q" if off64 else ">i", buf, pos[0])[0]
        pos[0] += 8 if off64 else 4
        specs.append((v, vd, atts, t, vsize, begin))
    sizes = dict(dims)
    recs = [s for s in specs if s[1] and sizes[s[1][0]] is None]
    recsize = sum(s[4] for s in recs)
    if len(recs) == 1:  # a lone record variable's records are not padded
        s = recs[0]
        recsize = int(np.prod([sizes[d] for d in s[1][1:]], dtype=np.int64)) * \
            np.dtype(_NC_TYPES[s[3]]).itemsize
    variables = []
    for v, vd, atts, t, vsize, begin in specs:
        dt = np.dtype(_NC_TYPES[t])
        is_rec = bool(vd) and sizes[vd[0]] is None
        shape = [sizes[d] for d in (vd[1:] if is_rec else vd)]
        cnt = int(np.prod(shape, dtype=np.int64))
        if is_rec:
            arr = np.stack([np.frombuffer(buf, dt, cnt, begin + r * recsize).reshape(shape)
                            for r in range(numrecs)]) if numrecs else np.zeros([0] + shape, dt)
        else:
            arr = np.frombuffer(buf, dt, cnt, begin).reshape(shape)
        variables.append((v, vd, atts, arr.astype(dt.newbyteorder("="))))
    return dims, gatts, variables, numrecs


def combine_blocks(basename, file_id="out2", number=0, directory=".", remove=True):
    """Join the block files `<basename>.block*.<file_id>.<number>.nc` of one
    output into `<basename>.<file_id>.<number>.nc` (NetcdfOutput::
    CombineBlocks with mppnccombine -r; the module docstring gives the
    rules).  Returns the combined file's path; raises RuntimeError when no
    block file matches."""
    tag = f"{file_id}.{number:05d}.nc"
    files = sorted(glob.glob(os.path.join(glob.escape(directory),
                                          glob.escape(basename) + ".block*." + tag)))
    if not files:
        raise RuntimeError(f"no block files {basename}.block*.{tag} in {directory}")
    out = os.path.join(directory, f"{basename}.{tag}")
    if os.path.exists(out):
        os.remove(out)
    dims0, gatts0, vars0, nrec0 = read_classic(files[0])
    full = {}      # dimension -> full length
    for v, vd, atts, arr in vars0:
        if "domain_decomposition" in atts and v in dict(dims0):
            d = atts["domain_decomposition"]
            full[v] = int(d[1] - d[0] + 1)
    sizes0 = dict(dims0)
    out_dims = [(d, None if ln is None else full.get(d, ln)) for d, ln in dims0]
    out_vars = []
    for v, vd, atts, arr in vars0:
        decomposed = any(d in full for d in vd)
        rec = bool(vd) and sizes0[vd[0]] is None
        if decomposed:
            shape = ([arr.shape[0]] if rec else []) + [full.get(d, sizes0[d]) for d in
                                                       (vd[1:] if rec else vd)]
            data = np.zeros(shape, arr.dtype)
        else:
            data = arr
        out_vars.append([v, vd, {k: a for k, a in atts.items() if k != "domain_decomposition"},
                         data, decomposed, rec])
    for path in files:
        dims, gatts, variables, nrec = read_classic(path)
        if nrec != nrec0:
            raise RuntimeError(f"{path}: {nrec} records, the first file has {nrec0}")
        start = {}
        for v, vd, atts, arr in variables:
            if "domain_decomposition" in atts and v in full:
                d = atts["domain_decomposition"]
                start[v] = int(d[2] - d[0])
        for (v, vd, atts, arr), o in zip(variables, out_vars):
            if not o[4]:
                continue
            dd = vd[1:] if o[5] else vd
            sl = tuple(slice(start.get(d, 0), start.get(d, 0) + n) for d, n in
                       zip(dd, arr.shape[1:] if o[5] else arr.shape))
            o[3][(slice(None),) + sl if o[5] else sl] = arr
    gatts = {k: a for k, a in gatts0.items() if k != "NumFilesInSet"}
    if "filename" in gatts:
        gatts["filename"] = out
    write_classic(out, out_dims, gatts, [tuple(o[:4]) for o in out_vars], numrecs=nrec0)
    if remove:
        for path in files:
            os.remove(path)
    return out
