"""Generates the golden fixtures of tests/golden/ (run from the repository
root on the CPU: python tests/golden/make_golden.py).

reference_kats.json  the known-answer tests of the reference project,
                     read as text from its tests/test_weno.cpp (interp_weno3,
                     interp_weno5) and tests/test_transform.cpp
                     (CovariantToContravariant, ContravariantToCovariant):
                     inputs, expected values and tolerances.  Needs the
                     reference checkout at /root/reference; without it the
                     committed file is kept.
oracle_small.npz     outputs of the oracle on small seeded cases, frozen so
                     that a later change of the oracle or of the CUDA path
                     shows up against a fixed record: the shallow-water case
                     (6x8x8, 5 CFL steps), the dry gas without gravity
                     (6x8x8x6, 2 steps of 50 s), the Held-Suarez case
                     (6x8x8x20, CFL 0.4, 2 steps; norms and one panel), and
                     the full and partial column corrections (4 columns of
                     8 levels).
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))
REF = "/root/reference/tests"


def _num(expr):
    """Value of a numeric literal expression of the test files: numbers,
    '/', '*', '+', '-', parentheses and sqrt(...)."""
    if not re.fullmatch(r"[0-9eE.+\-*/() sqrt]+", expr):
        raise ValueError(expr)
    return float(eval(expr, {"__builtins__": {}}, {"sqrt": np.sqrt}))


def reference_kats():
    weno = open(os.path.join(REF, "test_weno.cpp")).read()
    tran = open(os.path.join(REF, "test_transform.cpp")).read()
    out = {"source": "reference tests/test_weno.cpp, tests/test_transform.cpp"}

    def body(text, name):
        m = re.search(r"TEST\(" + name + r",\s*test1?_?\w*\)\s*\{(.*?)\n\}", text, re.S)
        return m.group(1)

    def assigns(b):
        return {k: v for k, v in re.findall(r"double\s+(\w+)\s*=\s*([^;]+);", b)}

    for fn in ("interp_weno3", "interp_weno5"):
        b = body(weno, fn)
        a = assigns(b)
        args = re.search(fn + r"\(([^)]*)\);", b).group(1).split(",")
        tol = _num(re.search(r"EXPECT_NEAR\([^,]+,[^,]+,\s*([^)]+)\)", b).group(1))
        out[fn] = {"args": [_num(a[x.strip()]) for x in args],
                   "expected": _num(a["expected_result"]), "tol": tol}
    for fn in ("CovariantToContravariant", "ContravariantToCovariant"):
        b = body(tran, fn)
        w = [_num(x) for x in re.search(r"Real w\[5\]\s*=\s*\{([^}]*)\}", b).group(1).split(",")]
        cth = _num(re.search(r"Real cth\s*=\s*([^;]+);", b).group(1))
        exp = [_num(e) for _, e in re.findall(r"EXPECT_DOUBLE_EQ\(w\[(\d)\],\s*([^)]*\)?)\);", b)]
        out[fn] = {"w": w, "cth": cth, "expected": exp, "ulps": 4}
    return out


def oracle_cases():
    from oracle import oracle as om
    from exocubed_b200 import workloads as W
    from _columns import column_problem
    res = {}
    cfg = W.shallow_water_config(N=8)
    o = om.Oracle(cfg)
    o.set_primitive(W.shallow_water_state(cfg, seed=0))
    o.step(5)
    res["c1_u"] = W.interior(o.conserved())
    res["c1_dt"] = np.array([o.dt])
    cfg = W.dry_atmosphere_config(N=8, L=6, rsolver=2, grav=0.0)
    o = om.Oracle(cfg)
    o.set_primitive(W.dry_atmosphere_state(cfg, seed=1))
    o.step(2, 50.0)
    res["dry_u"] = W.interior(o.conserved())
    cfg = W.hs94_config(N=8, L=20, cfl=0.4)
    o = om.Oracle(cfg)
    o.set_primitive(W.hs94_state(cfg, seed=2))
    o.step(2)
    u = W.interior(o.conserved())
    res["hs94_norms"] = np.array([np.linalg.norm(u[:, n]) for n in range(5)])
    res["hs94_panel0"] = u[0]
    res["hs94_dt"] = np.array([o.dt])
    for full in (True, False):
        w, du, colgeo, x1f, x1v, dx1f, c = column_problem(om, 4, 8, seed=3)
        out = om.implicit_columns(w, du, colgeo, x1f, x1v, dx1f, 300.0, c["gamma"], c["grav"],
                                  full=full)
        res["columns_full" if full else "columns_partial"] = out
    return res


if __name__ == "__main__":
    if os.path.isdir(REF):
        with open(os.path.join(HERE, "reference_kats.json"), "w") as f:
            json.dump(reference_kats(), f, indent=1)
        print("wrote reference_kats.json")
    else:
        print("no reference checkout: reference_kats.json kept")
    np.savez_compressed(os.path.join(HERE, "oracle_small.npz"), **oracle_cases())
    print("wrote oracle_small.npz")
