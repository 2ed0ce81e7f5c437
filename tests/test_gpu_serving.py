"""Continuous-batching server: requests that arrive while others run are
admitted as slots and memory free up, advance in the same batched launches,
and every result equals the same request run alone, bit for bit."""
import numpy as np
import pytest

from exocubed_b200 import CubedSphereAtmosphere
from exocubed_b200 import _native as nat
from exocubed_b200 import workloads as W
from exocubed_b200.ensemble import footprint
from exocubed_b200.serving import Request, Server, summarize

pytestmark = pytest.mark.gpu


def _requests(precision, steps=5):
    shapes = [(8, 16), (6, 20), (10, 16), (8, 24), (12, 16), (6, 24), (10, 20)]
    arrivals = [0, 0, 1, 3, 3, 6, 9]
    out = []
    for n, ((N, L), a) in enumerate(zip(shapes, arrivals)):
        cfg, _ = W.ensemble_member_config(100 + n, precision=precision)
        cfg.update(N=N, L=L)
        out.append(Request(n, cfg, W.dry_atmosphere_state(cfg, seed=100 + n), a, steps))
    return out


def _alone(r, precision):
    with CubedSphereAtmosphere(dict(r.cfg, precision=precision)) as a:
        a.set_primitive(r.w)
        a.step(r.steps)
        return a.conserved()


@pytest.mark.parametrize("precision", [nat.EXO_PREC_MIXED, nat.EXO_PREC_FP64])
def test_results_equal_alone_and_in_the_mix(precision):
    reqs = _requests(precision)
    srv = Server(precision=precision, capacity=3, max_chunk=2, keep_results=True)
    recs = srv.run(reqs, clock="steps")
    srv.close()
    for r, rec in zip(reqs, recs):
        assert rec.done - rec.admitted >= r.steps
        assert rec.valid and np.isfinite(rec.result).all(), r.rid
        assert np.array_equal(rec.result, _alone(r, precision)), r.rid
    # three slots: at no step were more than three requests on the device
    for t in range(int(max(rec.done for rec in recs)) + 1):
        assert sum(rec.admitted <= t < rec.done for rec in recs) <= 3
    # requests overlapped: some request ran while another was admitted
    assert any(a.admitted < b.admitted < a.done for a in recs for b in recs)


def test_budget_limits_resident_members():
    prec = nat.EXO_PREC_MIXED
    reqs = _requests(prec)
    sizes = sorted(footprint(dict(r.cfg, precision=prec)) for r in reqs)
    budget = sizes[-1] + sizes[-2]           # room for two members at most
    srv = Server(precision=prec, capacity=8, budget_bytes=budget, max_chunk=3,
                 keep_results=True)
    recs = srv.run(reqs, clock="steps")
    srv.close()
    for t in range(int(max(rec.done for rec in recs)) + 1):
        res = [footprint(dict(r.cfg, precision=prec)) for r, rec in zip(reqs, recs)
               if rec.admitted <= t < rec.done]
        assert sum(res) <= budget
    for r, rec in zip(reqs, recs):
        assert np.array_equal(rec.result, _alone(r, prec))


def test_wall_clock_serving_reports_latency():
    prec = nat.EXO_PREC_MIXED
    reqs = _requests(prec)
    for r in reqs:
        r.arrival = 0.01 * r.arrival
    srv = Server(precision=prec, capacity=4)
    recs = srv.run(reqs)
    srv.close()
    s = summarize(recs)
    assert s["requests"] == len(reqs)
    assert 0 < s["p50_s"] <= s["p99_s"] <= s["max_s"]
    assert all(rec.admitted >= rec.arrival for rec in recs)


@pytest.mark.parametrize("precision", [nat.EXO_PREC_FP64, nat.EXO_PREC_MIXED])
def test_served_results_against_the_oracle(oracle_mod, precision):
    """Every served request's conserved state after its steps against the
    oracle's run of the same member: the FP64 path to 1e-9 relative L2 per
    variable (only the last bits of log/exp/pow differ), the mixed path to
    1e-5 in density and energy."""
    reqs = _requests(precision, steps=3)[:4]
    srv = Server(precision=precision, capacity=3, max_chunk=2, keep_results=True)
    recs = srv.run(reqs, clock="steps")
    srv.close()
    for r, rec in zip(reqs, recs):
        o = oracle_mod.Oracle(dict(r.cfg, precision=0))
        o.set_primitive(r.w)
        o.step(r.steps)
        assert o.invalid() == 0 and rec.valid
        got, want = W.interior(rec.result), W.interior(o.conserved())
        for n in range(5):
            rel = np.linalg.norm(got[:, n] - want[:, n]) / np.linalg.norm(want[:, n])
            if precision == nat.EXO_PREC_FP64:
                assert rel < 1e-9, (r.rid, n, rel)
            elif n in (0, 4):
                assert rel < 1e-5, (r.rid, n, rel)
