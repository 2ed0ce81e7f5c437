"""Host logic of bench.py without a GPU: the algorithmic bytes behind
roofline.achieved, the workload descriptions per precision, and the
ncu-measured traffic that roofline.traffic reads for every kernel a C3 line
can name as dominant."""
import json
import os

import pytest

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("precision,flag,want", [
    (0, 9, 640), (1, 9, 640), (2, 9, 400),   # w, du, u 120 + u 40 + factors 2 x 30 values
    (0, 1, 352), (1, 1, 352), (2, 1, 256),   # partial correction: 2 x 12 values
])
def test_implicit_bytes_per_cell(precision, flag, want):
    assert bench.alg_bytes_per_cell("implicit", precision, flag) == want


def test_other_kernels_bytes_per_cell():
    assert bench.alg_bytes_per_cell("flux_x1", 1) == 80
    assert bench.alg_bytes_per_cell("flux_x23", 1) == 80
    assert bench.alg_bytes_per_cell("flux_x23", 0) == 160
    assert bench.alg_bytes_per_cell("update", 1) == 280
    assert bench.alg_bytes_per_cell("update", 2) == 280
    assert bench.alg_bytes_per_cell("update", 0) == 320
    assert bench.alg_bytes_per_cell("prim_ghost", 0) == 80
    assert bench.alg_bytes_per_cell("prim_ghost", 1) == 100


def test_workload_descriptions_follow_the_precision():
    cfg0, d0 = bench.workload_config("c3", 0)
    cfg1, d1 = bench.workload_config("c3", 1)
    cfg2, d2 = bench.workload_config("c3", 2)
    assert cfg0.get("precision", 0) == 0 and "FP64" in d0 and "mixed" not in d0
    assert cfg1["precision"] == 1 and "mixed FP32/FP64" in d1 and "implicit blocks" not in d1
    assert cfg2["precision"] == 2 and "FP32 implicit blocks" in d2
    assert (cfg1["N"], cfg1["L"]) == (192, 96)


@pytest.mark.parametrize("precision", [0, 1, 2])
@pytest.mark.parametrize("flag", [1, 9])
def test_measured_traffic_for_every_dominant_kernel(precision, flag):
    table = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
    for kernel in ("flux_x1", "flux_x23", "update", "implicit", "prim_ghost"):
        entry = table.get(bench.traffic_key(kernel, precision, flag))
        assert entry is not None, (kernel, precision, flag)
        assert os.path.exists(os.path.join(ROOT, entry["source"])), entry["source"]
        # measured bytes stay near the algorithmic count (no hidden re-reads)
        alg = bench.alg_bytes_per_cell(kernel, precision, flag)
        assert 0.8 * alg < entry["bytes_per_cell"] < 1.6 * alg, (kernel, entry, alg)


def test_state_bytes_follow_the_step_rule():
    # the state arrays each kernel reads or writes once; no scratch or copies
    assert bench.state_bytes_per_cell("implicit", 1) == 160
    assert bench.state_bytes_per_cell("implicit", 0) == 160
    assert bench.state_bytes_per_cell("update", 1) == 160
    assert bench.state_bytes_per_cell("flux_x23", 1) == 20
    assert bench.state_bytes_per_cell("prim_ghost", 0) == 80
    for k in ("flux_x1", "flux_x23", "update", "implicit", "prim_ghost"):
        for p in (0, 1, 2):
            assert bench.state_bytes_per_cell(k, p) <= bench.alg_bytes_per_cell(k, p)


def test_reference_leg_never_loads_the_product_library():
    """The CPU leg (bench.py --impl reference, cpu_baseline) builds its state
    on the oracle's mesh and steps the oracle; the product library must not
    be mapped into that process."""
    import subprocess
    import sys
    code = (
        "import sys, types, json\n"
        f"sys.path.insert(0, {ROOT!r})\n"
        "import bench\n"
        "a = types.SimpleNamespace(workload='c1', cpu_warmup=0, cpu_steps=1)\n"
        "bench.cpu_worker(a)\n"
        "print(json.dumps({'mapped': 'libexo_b200' in open('/proc/self/maps').read()}))\n")
    env = dict(os.environ, OMP_NUM_THREADS="4")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env,
                       check=True, timeout=600)
    lines = [json.loads(x) for x in r.stdout.strip().splitlines()]
    assert lines[0]["steps"] == 1 and lines[0]["cells"] == 6 * 48 * 48 * 3
    assert lines[-1]["mapped"] is False


@pytest.mark.parametrize("N", [6, 8, 48])
def test_oracle_geometry_is_the_library_geometry(N, native):
    """Seeded states generated on the oracle's mesh equal those generated on
    the library's, bit for bit, so both arms start from the same state."""
    import numpy as np

    from exocubed_b200 import workloads as W
    from exocubed_b200.atmosphere import cell_geometry
    from oracle import oracle
    cfg = W.dry_atmosphere_config(N=N, L=7)
    for a, b in zip(oracle.cell_geometry(cfg), cell_geometry(cfg)):
        assert np.array_equal(a, b)
    for seed in (0, 3):
        c, w_ora = W.ensemble_member(seed, geometry=oracle.cell_geometry)
        _, w_lib = W.ensemble_member(seed)
        assert np.array_equal(w_ora, w_lib)
    sw = W.shallow_water_config(N=N)
    assert np.array_equal(W.shallow_water_state(sw, 1, geometry=oracle.cell_geometry),
                          W.shallow_water_state(sw, 1))


def test_launch_gaps_from_graph_and_kernel_times():
    """launch_gaps: the per-kernel event times of the profiled steps summed
    per step, against the timed graph steps."""
    import bench
    meas = {"ms": 300.0, "prof_steps": 5,
            "prof": {"implicit": (15, 60.0), "update": (15, 20.0), "other": (10, 0.5),
                     "flux_x1": (15, 60.0), "flux_x23": (15, 5.0), "prim_ghost": (15, 2.0)}}
    g = bench.launch_gaps(meas, 10)
    assert g["graph_ms_per_step"] == 30.0
    assert abs(g["kernel_ms_per_step"] - 147.5 / 5) < 1e-12
    assert abs(g["gap_frac"] - (1 - 29.5 / 30.0)) < 1e-12
