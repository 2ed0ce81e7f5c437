"""Ensemble members and serving requests spread over several GPUs.

Members are independent, so they shard with no data-path collective: one
process per GPU (torch.distributed, NCCL on GPUs or gloo on the host), each
holding one exo_ensemble on its own device; no kernel reads another GPU's
memory.  The host places members by device-memory footprint and gathers the
results on rank 0 -- the arrangement the reference's MCMC inversion would
get by farming its forward models out to ranks
(src/inversion/profile_inversion.cpp:112-120, one model at a time per rank
there).

place(footprints, budgets)      greedy assignment, largest member first, to
                                the device with the most memory left
run_members(members, steps, ..) every rank advances its share in one
                                batched ensemble; rank 0 receives every
                                member's conserved state in input order
serve(requests, ..)             every rank serves its share of a request
                                stream with its own continuous-batching
                                server; rank 0 receives every record
"""
import numpy as np


def place(footprints, budgets):
    """Device index for each member: members are taken largest first and go
    to the device with the most memory left that can hold them.  Raises
    ValueError when a member fits no device."""
    left = [int(b) for b in budgets]
    out = [None] * len(footprints)
    for m in sorted(range(len(footprints)), key=lambda q: (-footprints[q], q)):
        d = max(range(len(left)), key=lambda q: (left[q], -q))
        if footprints[m] > left[d]:
            raise ValueError(f"member {m} ({footprints[m]} bytes) fits no device")
        out[m] = d
        left[d] -= footprints[m]
    return out


def _world(pg):
    if pg is None:
        return 1, 0
    return pg.get_world_size(), pg.get_rank()


def _gather(pg, obj):
    """obj of every rank, on rank 0 (None elsewhere)."""
    world, rank = _world(pg)
    if world == 1:
        return [obj]
    out = [None] * world if rank == 0 else None
    pg.gather_object(obj, out, dst=0)
    return out


def run_members(members, steps, pg=None, precision=1, budget_bytes=150 * 10 ** 9,
                footprint=None, ensemble_factory=None):
    """members: [(cfg dict, primitive array)] (the same list on every rank).
    Every rank admits the members place() gives it into one ensemble on its
    device, advances them `steps` batched steps and sends their conserved
    states to rank 0, which returns them in input order (other ranks return
    None).  footprint / ensemble_factory default to the library's."""
    world, rank = _world(pg)
    if footprint is None:
        from .ensemble import footprint
    if ensemble_factory is None:
        from .ensemble import Ensemble

        def ensemble_factory():
            return Ensemble(precision=precision, capacity=max(1, len(members)),
                            budget_bytes=budget_bytes)
    sizes = [footprint(dict(c, precision=precision)) for c, _ in members]
    where = place(sizes, [budget_bytes] * world)
    mine = [m for m in range(len(members)) if where[m] == rank]
    results = {}
    if mine:
        ens = ensemble_factory()
        try:
            slots = {m: ens.add(dict(members[m][0], precision=precision), members[m][1])
                     for m in mine}
            ens.step(steps)
            results = {m: (ens.conserved(s), ens.invalid(s) == 0) for m, s in slots.items()}
        finally:
            ens.close()
    parts = _gather(pg, results)
    if parts is None:
        return None
    merged = {}
    for p in parts:
        merged.update(p)
    return [merged[m] for m in range(len(members))], where


def serve(requests, pg=None, server_factory=None, clock="wall", footprint=None,
          precision=1, budget_bytes=150 * 10 ** 9):
    """requests: serving.Request list (the same on every rank).  Requests are
    placed on ranks by footprint (place()), every rank serves its share with
    its own server (server_factory()), and rank 0 returns all records in
    request order (other ranks return None)."""
    world, rank = _world(pg)
    if footprint is None:
        from .ensemble import footprint
    if server_factory is None:
        from .serving import Server

        def server_factory():
            return Server(precision=precision, budget_bytes=budget_bytes)
    sizes = [footprint(dict(r.cfg, precision=precision)) for r in requests]
    where = place(sizes, [budget_bytes * max(1, len(requests))] * world)
    mine = [r for q, r in enumerate(requests) if where[q] == rank]
    recs = []
    if mine:
        srv = server_factory()
        try:
            recs = srv.run(mine, clock=clock)
        finally:
            srv.close()
    parts = _gather(pg, recs)
    if parts is None:
        return None
    byid = {r.rid: r for p in parts for r in p}
    return [byid[r.rid] for r in requests]


def balance(where, sizes, ndev):
    """Bytes placed on each device (for reports and tests)."""
    out = np.zeros(ndev, dtype=np.int64)
    for m, d in enumerate(where):
        out[d] += sizes[m]
    return out
