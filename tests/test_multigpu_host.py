"""Members and serving requests spread over ranks (exocubed_b200/multigpu.py)
without a GPU: placement by footprint, and two gloo ranks on 127.0.0.1 that
each advance their share with a stand-in ensemble and server, gathered on
rank 0 in input order.  Unmeasured on more than one GPU (the GPU machines
at hand give one device); the placement and gather logic is what runs on
the host here."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from exocubed_b200 import multigpu


def test_place_largest_first_to_the_emptiest_device():
    sizes = [5, 9, 3, 7, 2, 8]
    where = multigpu.place(sizes, [20, 20])
    load = multigpu.balance(where, sizes, 2)
    assert load.sum() == sum(sizes) and abs(load[0] - load[1]) <= max(sizes)
    assert all(w in (0, 1) for w in where)
    # every member fits its device's budget
    assert (multigpu.balance(multigpu.place(sizes, [30, 6]), sizes, 2) <= [30, 6]).all()
    with pytest.raises(ValueError):
        multigpu.place([10, 10], [9, 9])


class _FakeEnsemble:
    """Steps a member by scaling its state: enough to see who ran what."""

    def __init__(self, rank):
        self.rank = rank
        self.slots = {}

    def add(self, cfg, w):
        self.slots[len(self.slots)] = (cfg, np.array(w, dtype=np.float64))
        return len(self.slots) - 1

    def step(self, n):
        for s, (c, w) in self.slots.items():
            self.slots[s] = (c, w * (1.0 + 0.5 * n) + self.rank * 0.0)

    def conserved(self, s):
        return self.slots[s][1]

    def invalid(self, s):
        return 0

    def close(self):
        pass


def _members():
    rng = np.random.default_rng(5)
    return [(dict(N=8 + 2 * (m % 3), L=4 + m), rng.standard_normal(3 + m)) for m in range(7)]


def _footprint(cfg):
    return 1000 * cfg["N"] * cfg["N"] * cfg["L"]


class _FakeServer:
    def __init__(self, rank):
        self.rank = rank

    def run(self, reqs, clock="wall"):
        from exocubed_b200.serving import Record
        out = []
        for r in reqs:
            rec = Record(r.rid, r.arrival, cells=6 * r.cfg["N"] ** 2 * r.cfg["L"], steps=r.steps)
            rec.admitted, rec.done = r.arrival, r.arrival + 1.0 + self.rank
            out.append(rec)
        return out

    def close(self):
        pass


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    res = multigpu.run_members(_members(), 3, pg=dist, budget_bytes=10 ** 9,
                               footprint=_footprint,
                               ensemble_factory=lambda: _FakeEnsemble(rank))
    from exocubed_b200.serving import Request
    reqs = [Request(q, dict(N=8, L=4 + q), None, 0.1 * q, 10) for q in range(6)]
    recs = multigpu.serve(reqs, pg=dist, server_factory=lambda: _FakeServer(rank),
                          footprint=_footprint)
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        states, where = res
        q.put(("members", [s.tolist() for s, _ in states], where,
               [r.rid for r in recs], [r.done - r.arrival for r in recs]))
    else:
        q.put(("other", res, recs))


@pytest.mark.timeout(120)
def test_two_gloo_ranks_share_and_gather():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=90) for _ in range(world)]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    r0 = [o for o in out if o[0] == "members"][0]
    other = [o for o in out if o[0] == "other"][0]
    assert other[1] is None and other[2] is None
    _, states, where, rids, latencies = r0
    want = [(w * (1.0 + 0.5 * 3)).tolist() for _, w in _members()]
    assert states == want                      # every member, in input order
    assert set(where) == {0, 1}                # both ranks took members
    assert rids == list(range(6))              # every request, in order
    assert {round(x, 9) for x in latencies} == {1.0, 2.0}   # served on both ranks
