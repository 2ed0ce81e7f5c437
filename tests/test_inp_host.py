"""Athena++ input files as configurations (exocubed_b200.inp): the keys of
the reference's examples/2023-Chen-exo3/hs94.inp and W92.inp, written out
here in the same form, give the configurations of the workloads module, and
the oracle steps them."""
import numpy as np
import pytest

from exocubed_b200 import _native as nat
from exocubed_b200 import workloads as W
from exocubed_b200.inp import config_from_inp, meshblocks_per_edge, parse_inp

HS94_LIKE = """
<comment>
problem   = Held-Suarez   # ignored
<job>
problem_id = hs94        # problem ID
<time>
cfl_number = 0.9
integrator = rk3
xorder     = 5
<mesh>
nx1        = 40
x1min      = 6.371E6
x1max      = 6.396E6
ix1_bc     = reflecting
ox1_bc     = reflecting
nx2        = 80
nx3        = 120
<meshblock>
nx1        = 40
nx2        = 40
nx3        = 40
<hydro>
gamma          = 1.4
grav_acc1      = -9.81
implicit_flag  = 1
<thermodynamics>
dT         = 60.
dtheta     = 10.
Rd         = 287.
cp         = 1004.
<problem>
Omega      = 7.292E-5
p0         = 1.E5
Ts         = 315.
Kf         = 1.
Ka         = 0.025
Ks         = 0.25
sigmab     = 0.7
z_iso      = 2.E4
"""

W92_LIKE = """
<job>
problem_id = W92
<time>
cfl_number = 0.7
xorder     = 5
integrator = rk3
<mesh>
nx1        = 3
x1min      = 6371000.
x1max      = 6371001.
nx2        = 96
nx3        = 144
<meshblock>
nx2        = 48
nx3        = 48
<hydro>
gamma       = 1.4
"""


def test_parse_blocks_and_comments():
    b = parse_inp(HS94_LIKE)
    assert "comment" not in b
    assert b["job"]["problem_id"] == "hs94"
    assert b["mesh"]["x1max"] == "6.396E6"


def test_hs94_input_gives_the_hs94_workload(oracle_mod):
    cfg, notes = config_from_inp(HS94_LIKE)
    want = W.hs94_config()
    for k, v in want.items():
        assert cfg[k] == v, k
    assert notes == []
    o = oracle_mod.Oracle(dict(cfg, N=8, L=20, cfl=0.4))
    o.set_primitive(W.hs94_state(dict(cfg, N=8, L=20), seed=0))
    o.step(2)
    assert np.isfinite(W.interior(o.conserved())).all()


def test_w92_input_gives_the_shallow_water_case(oracle_mod):
    cfg, notes = config_from_inp(W92_LIKE)
    assert cfg["eqn"] == nat.EXO_EQN_SHALLOW_YZ and cfg["N"] == 48 and cfg["L"] == 3
    assert cfg["rsolver"] == nat.EXO_RS_ROE_SHALLOW
    assert cfg["coriolis"] == nat.EXO_CORIOLIS_W92 and cfg["omega"] == 7.292e-5
    assert cfg["cfl"] == 0.7 and cfg["implicit_flag"] == 0
    small = dict(cfg, N=12)
    o = oracle_mod.Oracle(small)
    o.set_primitive(W.shallow_water_state(small, seed=0))
    o.step(2)
    assert np.isfinite(W.interior(o.conserved())).all()


def test_multi_block_and_unsupported_inputs():
    cfg, notes = config_from_inp(HS94_LIKE.replace("nx2        = 40\nnx3        = 40",
                                                   "nx2        = 20\nnx3        = 20"))
    assert cfg["N"] == 40 and len(notes) == 1 and "one 40^2 block" in notes[0]
    with pytest.raises(ValueError):
        config_from_inp(HS94_LIKE.replace("xorder     = 5", "xorder     = 3"))
    with pytest.raises(ValueError):
        config_from_inp(HS94_LIKE.replace("nx3        = 120", "nx3        = 100"))


def test_meshblocks_per_edge():
    blocks20 = HS94_LIKE.replace("nx2        = 40\nnx3        = 40",
                                 "nx2        = 20\nnx3        = 20")
    assert meshblocks_per_edge(HS94_LIKE) == 1
    assert meshblocks_per_edge(blocks20) == 2   # hs94-stable20.inp's 20 x 20 blocks
    assert "(meshblocks_per_edge)" in config_from_inp(blocks20)[1][0]
    for nx2, nx3 in ((20, 40), (8, 8), (30, 30)):   # not square / not a power of two
        with pytest.raises(ValueError):
            meshblocks_per_edge(HS94_LIKE.replace(
                "nx2        = 40\nnx3        = 40", f"nx2        = {nx2}\nnx3        = {nx3}"))
