"""Serving forward-model runs with continuous batching.

Requests (an exo3 atmosphere and a number of steps) arrive over time.  The
server keeps one batched ensemble resident on the GPU: a request is admitted
as soon as a member slot and enough of the device-memory budget are free
(its footprint: state, fluxes, scratch and tables), it joins the batch at
the next step boundary, advances in the same batched launches as every other
member, and leaves with its conserved state read back once it has taken its
steps.  Requests that arrive while others run therefore overlap with them on
the device; a member's result does not depend on who else is in the batch
(the batched kernels treat every member independently), which
tests/test_gpu_serving.py checks bit for bit.

The reference runs these forward models one at a time inside its MCMC
inversion (src/inversion/profile_inversion.cpp:112-120); the one-at-a-time
FP64 path is served_one_at_a_time() below, for comparison.
"""
import collections
import dataclasses
import time

import numpy as np

from . import _native as nat
from .atmosphere import CubedSphereAtmosphere
from .ensemble import Ensemble, footprint


@dataclasses.dataclass
class Request:
    rid: int
    cfg: dict
    w: np.ndarray          # primitive initial state (6, nvar, nc3, nc2, nc1)
    arrival: float         # seconds (wall clock) or steps (step clock) after start
    steps: int = 200


@dataclasses.dataclass
class Record:
    rid: int
    arrival: float
    admitted: float = float("nan")
    done: float = float("nan")
    cells: int = 0
    steps: int = 0
    valid: bool = True
    rejected: bool = False  # could not be admitted even with the device empty
    result: np.ndarray = None

    @property
    def latency(self):
        return self.done - self.arrival


def poisson_arrivals(rate, n, seed=0):
    """n arrival times (seconds) of a Poisson process of the given rate."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.cumsum(rng.exponential(1.0 / rate, n))


class Server:
    """Continuous-batching server over one Ensemble.

    precision      EXO_PREC_MIXED, EXO_PREC_MIXED_F32_SOLVE or EXO_PREC_FP64 (every
                   member the same)
    capacity       member slots
    budget_bytes   device memory the members may hold together
    max_chunk      steps launched between two admission checks (a chunk never
                   runs a member past its last step)
    keep_results   keep each request's final conserved state in its record
    tile_cache     an autotune.TileCache: when given, the batch's launch tiles
                   follow its members (autotune.batch_tiles) after every
                   membership change
    """

    def __init__(self, precision=nat.EXO_PREC_MIXED, capacity=64, budget_bytes=150 * 10 ** 9,
                 max_chunk=8, keep_results=False, tile_cache=None):
        self.tile_cache = tile_cache
        self.precision = precision
        self.capacity = capacity
        self.budget = budget_bytes
        self.max_chunk = max_chunk
        self.keep = keep_results
        self.ens = Ensemble(precision=precision, capacity=capacity, budget_bytes=budget_bytes)

    def close(self):
        self.ens.close()

    def run(self, requests, clock="wall"):
        """Serve the requests (sorted by arrival) to completion; returns one
        Record per request.  clock="wall": arrivals are seconds after the
        call and times are wall-clock seconds; clock="steps": arrivals and
        times count batched steps (a deterministic schedule for tests)."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        for r in reqs:
            need = footprint(dict(r.cfg, precision=self.precision))
            if need > self.budget:
                raise ValueError(f"request {r.rid} needs {need} bytes, above the whole budget")
        recs = {r.rid: Record(r.rid, r.arrival, cells=6 * r.cfg["N"] ** 2 * r.cfg["L"],
                              steps=r.steps) for r in reqs}
        pending = collections.deque(reqs)
        queue = collections.deque()
        active = {}                      # slot -> [request, steps left]
        t0 = time.perf_counter()
        nstep = 0

        def now():
            return time.perf_counter() - t0 if clock == "wall" else float(nstep)

        changed = False
        while pending or queue or active:
            t = now()
            while pending and pending[0].arrival <= t:
                queue.append(pending.popleft())
            # admission, first come first served: the head waits for room
            while queue:
                r = queue[0]
                cfg = dict(r.cfg, precision=self.precision)
                slot = self.ens.try_add(cfg, r.w)
                if slot is None and not active:
                    # refused with nothing else on the device (its memory
                    # could not be had): it never fits, so it is rejected
                    # rather than waited for
                    queue.popleft()
                    rec = recs[r.rid]
                    rec.rejected, rec.valid = True, False
                    rec.admitted = rec.done = now()
                    continue
                if slot is None:
                    break
                queue.popleft()
                active[slot] = [r, r.steps]
                recs[r.rid].admitted = now()
                changed = True
            if not active:
                if pending:
                    if clock == "wall":
                        time.sleep(max(0.0, min(pending[0].arrival - now(), 0.05)))
                    else:
                        nstep = int(np.ceil(pending[0].arrival))
                continue
            if changed and self.tile_cache is not None:
                self.ens.autotune(self.tile_cache)
            changed = False
            chunk = min(self.max_chunk, min(left for _, left in active.values()))
            if clock == "steps" and pending:
                chunk = max(1, min(chunk, int(np.ceil(pending[0].arrival)) - nstep))
            self.ens.step(chunk)
            nstep += chunk
            finished = []
            for slot, entry in active.items():
                entry[1] -= chunk
                if entry[1] == 0:
                    finished.append(slot)
            for slot in finished:
                r = active.pop(slot)[0]
                u = self.ens.conserved(slot)   # waits for the member's last step
                rec = recs[r.rid]
                rec.valid = self.ens.invalid(slot) == 0
                self.ens.remove(slot)
                changed = True
                rec.done = now()
                if self.keep:
                    rec.result = u
        return [recs[r.rid] for r in reqs]


def served_one_at_a_time(requests, precision=nat.EXO_PREC_FP64, keep_results=False):
    """The plain path: each request on its own context, one after another,
    first come first served; wall-clock records like Server.run."""
    reqs = sorted(requests, key=lambda r: r.arrival)
    out = []
    t0 = time.perf_counter()
    for r in reqs:
        wait = r.arrival - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        rec = Record(r.rid, r.arrival, cells=6 * r.cfg["N"] ** 2 * r.cfg["L"], steps=r.steps)
        rec.admitted = time.perf_counter() - t0
        with CubedSphereAtmosphere(dict(r.cfg, precision=precision)) as a:
            a.set_primitive(r.w)
            a.step(r.steps)
            u = a.conserved()
            rec.valid = a.invalid() == 0
        rec.done = time.perf_counter() - t0
        if keep_results:
            rec.result = u
        out.append(rec)
    return out


def summarize(records):
    """p50/p99 latency (seconds), throughput (requests/s and cell-updates/s)
    over a finished run; rejected requests are counted apart and take no
    part in the latency and throughput figures."""
    rejected = sum(1 for r in records if r.rejected)
    records = [r for r in records if not r.rejected]
    if not records:
        return {"requests": 0, "rejected": rejected}
    lat = np.array([r.latency for r in records])
    span = max(r.done for r in records) - min(r.arrival for r in records)
    cu = sum(r.cells * r.steps for r in records)
    return {"requests": len(records), "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()),
            "max_s": float(lat.max()), "span_s": float(span),
            "requests_per_s": len(records) / span, "cell_updates_per_s": cu / span,
            "all_valid": all(r.valid for r in records), "rejected": rejected}
