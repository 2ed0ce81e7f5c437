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
    assert bench.alg_bytes_per_cell("flux_x23", 0) == 120
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
