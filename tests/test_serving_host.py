"""Admission logic of the continuous-batching server, on the CPU with a fake
ensemble: a request the device refuses while nothing else runs on it is
rejected (it never fits) instead of being waited for."""
import numpy as np

from exocubed_b200 import serving
from exocubed_b200 import workloads as W


class _FakeEnsemble:
    """Admits members whose N is at most max_n; each step advances the clock."""

    def __init__(self, max_n):
        self.max_n = max_n
        self.slots = {}
        self.steps = 0

    def try_add(self, cfg, w):
        if cfg["N"] > self.max_n:
            return None
        slot = len(self.slots) + 100
        self.slots[slot] = cfg
        return slot

    def step(self, n):
        self.steps += n

    def conserved(self, slot):
        return np.zeros(1)

    def invalid(self, slot):
        return 0

    def remove(self, slot):
        self.slots.pop(slot)

    def autotune(self, cache):
        pass


def _server(max_n):
    srv = serving.Server.__new__(serving.Server)
    srv.tile_cache, srv.precision, srv.capacity = None, 1, 4
    srv.budget, srv.max_chunk, srv.keep = 10 ** 15, 8, False
    srv.ens = _FakeEnsemble(max_n)
    return srv


def _req(rid, N, arrival, steps=5):
    cfg = W.dry_atmosphere_config(N=N, L=4)
    return serving.Request(rid, cfg, None, arrival, steps)


def test_unadmittable_request_is_rejected_not_waited_for():
    srv = _server(max_n=8)
    reqs = [_req(0, 16, 0.0), _req(1, 8, 0.0), _req(2, 16, 3.0), _req(3, 8, 4.0)]
    recs = srv.run(reqs, clock="steps")
    by = {r.rid: r for r in recs}
    assert by[0].rejected and not by[0].valid
    assert by[2].rejected
    assert not by[1].rejected and by[1].valid and by[1].done >= 5
    assert not by[3].rejected and by[3].valid
    s = serving.summarize(recs)
    assert s["rejected"] == 2 and s["requests"] == 2


def test_everything_rejected_ends():
    srv = _server(max_n=4)
    recs = srv.run([_req(0, 8, 0.0), _req(1, 8, 2.0)], clock="steps")
    assert all(r.rejected for r in recs)
    assert serving.summarize(recs) == {"requests": 0, "rejected": 2}
