"""Multi-rank host logic of bench.py without a GPU: two gloo ranks on
127.0.0.1 exercise the barrier, the max-over-ranks timing reduction and the
per-rank member seeds (every rank advances its own members: weak scaling
with no data-path collective)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    w, r, local, pg = bench.dist_setup(world)
    bench.barrier(pg)
    m = bench.max_over_ranks(pg, 10.0 + r)      # each rank's own time
    seeds = bench.member_seeds(r, 4)
    bench.barrier(pg)
    pg.destroy_process_group()
    q.put((r, w, m, seeds))


@pytest.mark.timeout(120)
def test_two_gloo_ranks_max_and_disjoint_members():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=90) for _ in range(world))
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1] and all(o[1] == 2 for o in out)
    assert all(o[2] == 11.0 for o in out)       # the max over ranks, seen by both
    assert not set(out[0][3]) & set(out[1][3])


def test_single_rank_needs_no_process_group():
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    w, r, local, pg = bench.dist_setup(1)
    assert (w, r, pg) == (1, 0, None)
    assert bench.max_over_ranks(pg, 3.5) == 3.5
