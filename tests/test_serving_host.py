"""Serving host logic without a GPU: arrival generation and summaries."""
import numpy as np

from exocubed_b200.serving import Record, poisson_arrivals, summarize


def test_poisson_arrivals_rate():
    t = poisson_arrivals(100.0, 20000, seed=3)
    assert np.all(np.diff(t) > 0)
    assert abs(len(t) / t[-1] - 100.0) < 3.0
    assert np.array_equal(t, poisson_arrivals(100.0, 20000, seed=3))


def test_summary_percentiles_and_throughput():
    recs = []
    for n in range(100):
        r = Record(n, arrival=0.01 * n, cells=1000, steps=10)
        r.admitted = r.arrival
        r.done = r.arrival + 1.0 + 0.01 * n
        recs.append(r)
    s = summarize(recs)
    assert abs(s["p50_s"] - 1.495) < 1e-9
    assert abs(s["p99_s"] - (1.0 + 0.01 * 98.01)) < 1e-9
    assert abs(s["span_s"] - (0.99 + 1.99)) < 1e-12
    assert abs(s["cell_updates_per_s"] - 100 * 1000 * 10 / s["span_s"]) < 1e-6
