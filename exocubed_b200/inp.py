"""Athena++ input files (`.inp`) as exo_config dictionaries.

The reference drives a run with an Athena++ input file (examples/2023-Chen-
exo3/*.inp): <block> headers followed by `key = value  # comment` lines.  The
keys this path reads are the ones the reference's step reads:

  <mesh>          nx1 (levels), nx2 = 2 N and nx3 = 3 N (the cubed sphere laid
                  out as 2 x 3 panels of N x N), x1min, x1max
  <meshblock>     nx2, nx3 (one block per panel is N x N)
  <time>          cfl_number; xorder must be 5 and integrator rk3
  <hydro>         gamma, grav_acc1, implicit_flag
  <thermodynamics> Rd, dT, dtheta (Held-Suarez)
  <problem>       Omega, and p0, Ts, Kf, Ka, Ks, sigmab (Held-Suarez)
  <job>           problem_id, which names the problem generator

What the input file does not say is compiled into a reference build: the
equation set (shallow water for the exo2 problems W92 and zonal, the
problem_ids of W92.inp and steady_zonal.inp; the ideal gas otherwise), the
Riemann solver (roe_shallow_yz, cmake/parameters.cmake:39, and
hllc_transform, cmake/exo3.cmake:14) and the
user source the problem generator enrolls (W92.cpp:154 and
steady_zonal.cpp:134: the lat-lon Coriolis form; hs94.cpp:242: the
Held-Suarez forcing).  Those follow problem_id here and can be overridden.
"""
import re

from . import _native as nat

SHALLOW_PROBLEMS = ("W92", "zonal")   # W92.inp, steady_zonal.inp
W92_CORIOLIS = ("W92", "zonal")
HS94_PROBLEMS = ("hs94",)


def parse_inp(text):
    """{block: {key: value string}} of an Athena++ input file's text (the
    <comment> block and comments dropped)."""
    blocks, cur = {}, None
    for raw in text.splitlines():
        line = raw.split("#", 1)[0].strip()
        if not line:
            continue
        m = re.fullmatch(r"<\s*([^>]+?)\s*>", line)
        if m:
            cur = m.group(1)
            blocks.setdefault(cur, {})
            continue
        if cur is None or "=" not in line:
            continue
        k, v = line.split("=", 1)
        blocks[cur][k.strip()] = v.strip()
    blocks.pop("comment", None)
    return blocks


def _num(blocks, block, key, default=None):
    v = blocks.get(block, {}).get(key)
    if v is None:
        if default is None:
            raise ValueError(f"<{block}> {key} is missing")
        return default
    return float(v)


def meshblocks_per_edge(source):
    """Meshblocks along a panel edge (<mesh> nx2 / 2 over <meshblock> nx2)
    of an input file (a path or its text): the `blocks` of the NetCDF
    output.  <meshblock> nx3 must equal nx2, and the count must divide the
    panel and be a power of two (CubedSphere::FindBlockID,
    src/exo3/cs_find_block_id.cpp:11-13, shifts by it)."""
    text = source
    if "\n" not in source and "<" not in source:
        with open(source) as f:
            text = f.read()
    b = parse_inp(text)
    N = int(_num(b, "mesh", "nx2")) // 2
    bx2 = int(_num(b, "meshblock", "nx2", N))
    bx3 = int(_num(b, "meshblock", "nx3", bx2))
    nb = N // bx2 if bx2 else 0
    if bx3 != bx2 or bx2 < 1 or N % bx2 or nb & (nb - 1):
        raise ValueError(f"<meshblock> nx2 = {bx2}, nx3 = {bx3} do not cut a {N}^2 panel "
                         f"into a power-of-two square of blocks")
    return nb


def config_from_inp(source, precision=nat.EXO_PREC_FP64, eqn=None, rsolver=None,
                    problem=None):
    """(config dict, notes) of an input file (a path or its text).  notes
    lists what the file asks for that this path runs differently."""
    text = source
    if "\n" not in source and "<" not in source:
        with open(source) as f:
            text = f.read()
    b = parse_inp(text)
    notes = []
    problem = problem or b.get("job", {}).get("problem_id", "")
    xorder = int(_num(b, "time", "xorder", 5))
    integ = b.get("time", {}).get("integrator", "rk3")
    if xorder != 5 or integ != "rk3":
        raise ValueError(f"only xorder = 5 and integrator = rk3 are built "
                         f"(got {xorder}, {integ})")
    nx2, nx3 = int(_num(b, "mesh", "nx2")), int(_num(b, "mesh", "nx3"))
    if nx2 % 2 or nx3 != 3 * (nx2 // 2):
        raise ValueError(f"<mesh> nx2 = {nx2}, nx3 = {nx3} is not a 2 x 3 panel layout")
    N = nx2 // 2
    bx2 = int(_num(b, "meshblock", "nx2", N))
    if bx2 < N:
        notes.append(f"meshblocks of {bx2}^2 step as one {N}^2 block per panel "
                     f"(multi-block ghost interpolation is not built); output files "
                     f"follow the {N // bx2} x {N // bx2} blocks (meshblocks_per_edge)")
    if eqn is None:
        eqn = nat.EXO_EQN_SHALLOW_YZ if problem in SHALLOW_PROBLEMS else nat.EXO_EQN_IDEAL
    shallow = eqn == nat.EXO_EQN_SHALLOW_YZ
    if rsolver is None:
        rsolver = nat.EXO_RS_ROE_SHALLOW if shallow else nat.EXO_RS_HLLC
    cfg = dict(N=N, L=int(_num(b, "mesh", "nx1")), eqn=eqn, rsolver=rsolver,
               implicit_flag=0 if shallow else int(_num(b, "hydro", "implicit_flag", 0)),
               precision=precision, coriolis=nat.EXO_CORIOLIS_NONE,
               forcing=nat.EXO_FORCING_NONE,
               x1min=_num(b, "mesh", "x1min"), x1max=_num(b, "mesh", "x1max"),
               gamma=_num(b, "hydro", "gamma", 1.4),
               Rd=_num(b, "thermodynamics", "Rd", 287.),
               grav=0. if shallow else _num(b, "hydro", "grav_acc1", 0.),
               cfl=_num(b, "time", "cfl_number"),
               omega=_num(b, "problem", "Omega", 0.))
    if problem in W92_CORIOLIS:
        cfg["coriolis"] = nat.EXO_CORIOLIS_W92
        if cfg["omega"] == 0.:
            cfg["omega"] = 7.292e-5  # om_earth of W92.cpp / steady_zonal.cpp
    if problem in HS94_PROBLEMS:
        cfg["forcing"] = nat.EXO_FORCING_HS94
        cfg.update(hs_p0=_num(b, "problem", "p0"), hs_Ts=_num(b, "problem", "Ts"),
                   hs_dT=_num(b, "thermodynamics", "dT"),
                   hs_dtheta=_num(b, "thermodynamics", "dtheta"),
                   hs_Kf=_num(b, "problem", "Kf"), hs_Ka=_num(b, "problem", "Ka"),
                   hs_Ks=_num(b, "problem", "Ks"), hs_sigmab=_num(b, "problem", "sigmab"))
    for blk, key in (("mesh", "ix1_bc"), ("mesh", "ox1_bc")):
        v = b.get(blk, {}).get(key, "reflecting")
        if v != "reflecting":
            notes.append(f"<{blk}> {key} = {v}: radial boundaries are reflecting here")
    return cfg, notes
