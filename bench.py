"""Benchmark: cell-updates/s of the cubed-sphere finite-volume step on B200.

Default workload (c3): the exo3 dry ideal-gas atmosphere, 6 panels x 192 x
192 x 96 levels, WENO5 + LMARS + the 5x5 implicit vertical solver
(implicit_flag 9), SSPRK(3,3), CFL time step, on a seeded synthetic state
(isothermal 250 K hydrostatic column, 1 K temperature noise, 5 m/s winds).
A "step" is one SSPRK(3,3) step of the whole atmosphere; one cell-update is
one interior cell advanced one step (6*N*N*L per step).

The line's value is the mixed-precision path (FP32 reconstruction, x2/x3
Riemann fluxes and their divergence; FP64 decomposition, x1 fluxes,
implicit solve, state and RK accumulation; --precision 2 also runs the
implicit solve's blocks in FP32);
"fp64" is the plain FP64 path on the same workload in the same run;
"accuracy" compares the two after --accuracy-steps steps; "serving" is a
short continuous-batching sample (ensemble-member requests, p50/p99 latency)
with the FP64 one-at-a-time path beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload c1|c2|c2s|c3|c4] [--precision 0|1|2]
  python bench.py --accuracy 1000            (mixed vs FP64 after 1000 steps)
  python bench.py --serve 10,100,2000        (serving sweep, one line per rate)

Multi-GPU: one process per GPU; every rank advances its own atmosphere (an
independent ensemble member), so there is no data-path collective and the
scaling is weak.  Timing: CUDA events on the library's stream, barrier +
synchronize on both sides, max over ranks.

--impl reference times the reference's CPU algorithm on this host's cores.
The reference itself cannot be built here (its Athena++ fork, MPI, NetCDF
and Eigen are not available), so the C++ restatement in oracle/ stands in
for it ("kind": "port"); it computes in FP64 and runs a bounded sample of
full steps of the same workload (--ref-steps).
"""
import argparse
import dataclasses
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_CELL_UPDATE = 320  # 8 registers x 5 vars x 8 B per SSPRK(3,3) step


RSOLVER = {1: "LMARS", 2: "HLLC"}
_RS = [None]  # the --rsolver choice for exo3 workloads (None: LMARS)
_IMP = [None]  # the --implicit-flag choice for exo3 workloads (None: 9)


def workload_config(name, precision=0):
    cfg, desc = _workload(name)
    if _RS[0] is not None and cfg["eqn"] == 1:
        cfg = dict(cfg, rsolver=_RS[0])
        desc = desc.replace("LMARS", RSOLVER[_RS[0]])
    if _IMP[0] is not None and cfg["eqn"] == 1:
        cfg = dict(cfg, implicit_flag=_IMP[0])
        desc = desc.replace("implicit(9)", f"implicit({_IMP[0]})")
    if precision in (1, 2):
        cfg = dict(cfg, precision=precision)
        desc = desc.replace("FP64", "mixed FP32/FP64" + (" (FP32 implicit blocks)"
                                                         if precision == 2 else ""))
    return cfg, desc


def _workload(name):
    from exocubed_b200 import workloads as W
    if name == "c2":
        return (W.dry_atmosphere_config(N=96, L=64, rsolver=1),
                "exo3 dry ideal gas 6x96x96x64 FP64 WENO5+LMARS+implicit(9), SSPRK3, CFL 0.4")
    if name == "c2s":  # profiling size: 6x64x64x64, state arrays 63 MB each
        return (W.dry_atmosphere_config(N=64, L=64, rsolver=1),
                "exo3 dry ideal gas 6x64x64x64 FP64 WENO5+LMARS+implicit(9), SSPRK3, CFL 0.4")
    if name == "c1":
        return (W.shallow_water_config(N=48),
                "exo2 shallow water 6x48x48x3 FP64 WENO5+Roe, SSPRK3, CFL 0.4")
    if name == "c3":
        return (W.dry_atmosphere_config(N=192, L=96, rsolver=1),
                "exo3 dry ideal gas 6x192x192x96 FP64 WENO5+LMARS+implicit(9), SSPRK3, CFL 0.4")
    if name == "hs94":  # examples/2023-Chen-exo3/hs94.inp
        return (W.hs94_config(),
                "exo3 Held-Suarez 6x40x40x40 FP64 WENO5+HLLC+implicit(1)+HS94 forcing, "
                "SSPRK3, CFL 0.9")
    raise ValueError(name)


def make_state(cfg, seed, geometry=None):
    """Seeded initial primitives of a workload; geometry: None (the product
    library's cell geometry) or the oracle's (CPU legs, which must not load
    the product library)."""
    from exocubed_b200 import workloads as W
    if cfg["eqn"] == 0:
        return W.shallow_water_state(cfg, seed=seed, geometry=geometry)
    if cfg.get("forcing", 0) == 1:
        return W.hs94_state(cfg, seed=seed, geometry=geometry)
    return W.dry_atmosphere_state(cfg, seed=seed, geometry=geometry)


def cells_of(cfg):
    return 6 * cfg["N"] * cfg["N"] * cfg["L"]


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ distributed --
def dist_setup(gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, x):
    if pg is None:
        return x
    import torch
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def member_seeds(rank, n):
    """Seeds of the ensemble members rank `rank` advances: disjoint across
    ranks, so N ranks hold N different ensembles (weak scaling)."""
    return [10_000 * rank + i for i in range(n)]


# ---------------------------------------------------------- CPU baseline --
def cpu_worker(args):
    """Runs in a fresh process: times the oracle on all host cores.  The
    state is generated on the oracle's own mesh, so this process never loads
    the product library."""
    import numpy as np  # noqa: F401
    from oracle import oracle
    cfg, _ = workload_config(args.workload)
    o = oracle.Oracle(cfg)
    o.set_primitive(make_state(cfg, 0, geometry=oracle.cell_geometry))
    o.step(args.cpu_warmup)
    t0 = time.perf_counter()
    o.step(args.cpu_steps)
    el = time.perf_counter() - t0
    print(json.dumps({"seconds": el, "steps": args.cpu_steps,
                      "cells": cells_of(cfg), "threads": os.cpu_count()}))


def run_cpu(workload, steps, warmup):
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = str(os.cpu_count())
    env.pop("CUDA_VISIBLE_DEVICES", None)
    cmd = [sys.executable, os.path.abspath(__file__), "--cpu-worker", "--workload", workload,
           "--cpu-steps", str(steps), "--cpu-warmup", str(warmup)]
    if _RS[0] is not None:
        cmd += ["--rsolver", str(_RS[0])]
    if _IMP[0] is not None:
        cmd += ["--implicit-flag", str(_IMP[0])]
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, check=True)
    return json.loads(r.stdout.strip().splitlines()[-1])


# -------------------------------------------------------------- our arm --
# algorithmic DRAM bytes per interior cell and launch, by kernel and flux type
# (each array element read or written once; the implicit solve's factors
# (A c)_i and delta_i, 30 values per level with the full correction and 12
# with the partial one, FP32 at precision 2 and FP64 otherwise, are written
# and read back)
def alg_bytes_per_cell(kernel, precision, implicit_flag=9):
    mixed = precision in (1, 2)
    t = 4 if mixed else 8
    # flux_x23: a block per line of faces reads every cell once per direction
    x23 = 10 * t + 10 * t
    factors = (30 if implicit_flag & 8 else 12) * (4 if precision == 2 else 8) * 2
    # the x1 fluxes are FP64 in both builds (5 values of 8 bytes per cell)
    return {"flux_x1": 40 + 40, "flux_x23": x23, "update": 120 + 40 + 10 * t + 80,
            "implicit": 160 + factors, "prim_ghost": 80 + (20 if mixed else 0),
            "other": 0}[kernel]


def state_bytes_per_cell(kernel, precision):
    """Compulsory bytes per interior cell and launch: the state arrays the
    kernel must read or write, each once (u, u1, du, w in FP64; the FP32
    primitive copy where the mixed x2/x3 sweep reads nothing else).  Face
    fluxes, the implicit solve's factor scratch, FP32 flux copies, halos and
    tables are implementation traffic and are not counted (the 320 B per
    cell-update rule of the step applied to one kernel)."""
    mixed = precision in (1, 2)
    return {"flux_x1": 40,                        # w
            "flux_x23": 20 if mixed else 40,      # w32 / w
            "update": 160,                        # u, u1, w read; du (or u) written
            "implicit": 160,                      # w, du, u read; u written
            "prim_ghost": 80,                     # u read; w written
            "other": 0}[kernel]


def traffic_key(kernel, precision, implicit_flag=9):
    """Key of a kernel's ncu-measured DRAM bytes per cell in profiles/traffic.json."""
    key = f"{kernel}:{'mixed' if precision in (1, 2) else 'fp64'}"
    if kernel == "implicit" and precision == 2:
        key += "_f32_solve"
    if kernel == "implicit" and not implicit_flag & 8:
        key += ":partial"
    return key


def alu_peaks():
    """FP64 and FP32 FMA rates of this GPU (exo_measure_fma_peak), measured
    in the same run, before any timed region."""
    from exocubed_b200 import _native as nat
    f64, f32 = nat.fma_peak(True), nat.fma_peak(False)
    return {"fp64_flops_per_s": f64, "fp32_flops_per_s": f32,
            "how": "independent FMA chains on every SM, best of 3 event-timed launches"}


def measure_path(cfg, state, steps, warmup, pg, local, sample_clocks, tune=True):
    """Device-timed steps of one atmosphere with the state resident (launch
    tiles autotuned before the clock starts unless tune is False)."""
    import torch

    from exocubed_b200.atmosphere import CubedSphereAtmosphere
    g = CubedSphereAtmosphere(cfg)
    tiles = g.autotune() if tune else g.tiles
    g.set_primitive(state)
    stream = torch.cuda.ExternalStream(g.stream)
    g.step(warmup)
    g.synchronize()
    clocks = ClockSampler(local)
    if sample_clocks:
        clocks.start()
    launches0 = g.launch_count()
    barrier(pg)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    g.step(steps)  # CFL steps replay the library's captured step graph
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier(pg)
    ms = e0.elapsed_time(e1)
    launches = g.launch_count() - launches0
    clk = clocks.stop() if sample_clocks else None
    # per-kernel times from a few more steps launched one by one between events
    g.profile(True)
    g.step(min(steps, 5))
    g.synchronize()
    prof = g.profile_read()
    g.profile(False)
    out = {"ms": max_over_ranks(pg, ms), "prof": prof, "prof_steps": min(steps, 5),
           "launches": launches, "clocks": clk, "invalid": g.invalid(), "tiles": tiles}
    g.close()
    return out


def launch_gaps(meas, steps):
    """The captured step graph (the timed steps) against the same kernels
    launched one by one between CUDA events (the profiled steps): the share
    of the step outside the kernels, i.e. launch gaps a persistent kernel
    could remove."""
    graph = meas["ms"] / steps
    kern = sum(v[1] for v in meas["prof"].values()) / max(meas["prof_steps"], 1)
    return {"graph_ms_per_step": graph, "kernel_ms_per_step": kern,
            "gap_frac": 1.0 - kern / graph,
            "note": "per-kernel CUDA-event times of the same step summed, against the graph "
                    "replay; a negative value means the events' own overhead exceeds the gaps"}


def measure_e2e(cfg, state, steps, pg, tune=True):
    """The same steps through the public API with the state in pinned host
    memory: upload, steps, download inside the timed region."""
    import torch

    from exocubed_b200.atmosphere import CubedSphereAtmosphere
    h_in = torch.from_numpy(state).pin_memory()
    h_out = torch.empty(state.shape, dtype=torch.float64).pin_memory()
    g = CubedSphereAtmosphere(cfg)
    if tune:
        g.autotune()
    s2 = torch.cuda.ExternalStream(g.stream)
    g.set_primitive_ptr(h_in.data_ptr())
    g.step(1)
    g.synchronize()
    barrier(pg)
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(s2)
    g.set_primitive_ptr(h_in.data_ptr())
    g.step(steps)
    g.conserved_ptr(h_out.data_ptr())
    f1.record(s2)
    f1.synchronize()
    barrier(pg)
    ms = max_over_ranks(pg, f0.elapsed_time(f1))
    g.close()
    return ms, state.nbytes


def fp64_reference(cfg, state, steps):
    """(dt, interior primitives) of the FP64 path after steps steps of its
    first CFL step."""
    from exocubed_b200 import workloads as W
    from exocubed_b200.atmosphere import CubedSphereAtmosphere
    ref = CubedSphereAtmosphere(dict(cfg, precision=0))
    ref.set_primitive(state)
    dt = ref.dt
    ref.step(steps, dt)
    wr = W.interior(ref.primitive())
    ref.close()
    return dt, wr


def accuracy(cfg, state, steps, precision=1, ref=None):
    """A mixed precision (1 or 2) against the FP64 path on the same state,
    the FP64 path's first CFL step held fixed: relative L2 / Linf per field.
    ref: fp64_reference(cfg, state, steps), computed here when None."""
    import numpy as np

    from exocubed_b200 import workloads as W
    from exocubed_b200.atmosphere import CubedSphereAtmosphere
    dt, wr = ref if ref is not None else fp64_reference(cfg, state, steps)
    mix = CubedSphereAtmosphere(dict(cfg, precision=precision))
    mix.set_primitive(state)
    mix.step(steps, dt)
    wm = W.interior(mix.primitive())
    invalid = mix.invalid()
    mix.close()
    names = ["rho", "v1", "v2", "v3", "p"] if cfg["eqn"] == 1 else ["phi", "v1", "v2", "v3"]
    err = {}
    for n, name in enumerate(names):
        if name == "v1" and cfg["eqn"] == 0:
            continue
        d = wm[:, n] - wr[:, n]
        scale = np.linalg.norm(wr[:, n])
        err[name] = {"rel_l2": float(np.linalg.norm(d) / scale) if scale > 0
                     else float(np.linalg.norm(d)),
                     "linf": float(np.abs(d).max()),
                     "rel_linf": float(np.abs(d).max() / max(np.abs(wr[:, n]).max(), 1e-300))}
    return {"steps": steps, "precision": precision, "dt": dt, "simulated_seconds": dt * steps,
            "fields": err,
            "state_valid": invalid == 0}


ORACLE_RUN = os.path.join(ROOT, "tests", "golden", "oracle_c2_lmars.npz")


def accuracy_vs_oracle(precisions=(0, 1, 2), path=ORACLE_RUN):
    """The GPU paths against the oracle's own long run of the C2 workload
    (6x96x96x64, LMARS, implicit_flag 9, seeded state 0; the oracle's first
    CFL step held fixed; tests/golden/make_oracle_runs.py): relative L2 and
    L-inf of each primitive variable on the run's 8192 sampled interior
    cells after each of its checkpoints (10, 100, 1000 steps)."""
    import numpy as np

    from exocubed_b200 import workloads as W
    from exocubed_b200.atmosphere import CubedSphereAtmosphere
    if not os.path.exists(path):
        return None
    fx = np.load(path)
    N, L, rs, seed = int(fx["N"]), int(fx["L"]), int(fx["rsolver"]), int(fx["seed"])
    dt = float(fx["dt"])
    idx = fx["cells"]
    cfg = W.dry_atmosphere_config(N=N, L=L, rsolver=rs)
    state = W.dry_atmosphere_state(cfg, seed=seed)
    names = ["rho", "v1", "v2", "v3", "p"]
    out = {"workload": f"exo3 dry ideal gas 6x{N}x{N}x{L} LMARS implicit(9), seeded state {seed}, "
                       f"dt = {dt:.6g} s fixed (the oracle's first CFL step)",
           "vs": "oracle (FP64 C++ restatement, its own run on the same seeded state)",
           "cells_sampled": int(idx.shape[1]), "paths": {}}
    for prec in precisions:
        a = CubedSphereAtmosphere(dict(cfg, precision=prec))
        a.set_primitive(state)
        done, rows = 0, {}
        for n in [int(x) for x in fx["checkpoints"]]:
            a.step(n - done, dt)
            done = n
            w = a.primitive()
            g = w[idx[0], :, idx[1], idx[2], idx[3]].T
            o = fx[f"sample_{n}"]
            rows[str(n)] = {
                name: {"rel_l2": float(np.linalg.norm(g[q] - o[q]) / np.linalg.norm(o[q])),
                       "linf": float(np.abs(g[q] - o[q]).max()),
                       "rel_linf": float(np.abs(g[q] - o[q]).max() / np.abs(o[q]).max())}
                for q, name in enumerate(names)}
            rows[str(n)]["state_valid"] = a.invalid() == 0
        a.close()
        out["paths"][{0: "fp64", 1: "mixed", 2: "mixed_f32_solve"}[prec]] = rows
    return out


def measure_ensemble(members, prec, steps, warmup, pg=None, cache=None, tune=True):
    """Device-timed batched steps of an ensemble (state resident): ms, launches, validity."""
    import torch

    from exocubed_b200.ensemble import Ensemble
    ens = Ensemble(precision=prec, capacity=len(members))
    slots = [ens.add(dict(c, precision=prec), w) for c, w in members]
    tiles = ens.autotune(cache) if tune else ens.tiles
    stream = torch.cuda.ExternalStream(ens.stream)
    ens.step(warmup)
    ens.synchronize()
    l0 = ens.stats()["launches"]
    barrier(pg)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ens.step(steps)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier(pg)
    ms = max_over_ranks(pg, e0.elapsed_time(e1))
    out = {"ms": ms, "launches": ens.stats()["launches"] - l0, "tiles": tiles,
           "valid": all(ens.invalid(s) == 0 for s in slots)}
    ens.close()
    return out


def ensemble_sample(nmembers, steps, warmup, cache=None):
    """The C4 batched ensemble in the default line: nmembers atmospheres of
    the member distribution, mixed precision and the plain FP64 path on the
    same members, one graph-captured batched step per step."""
    from exocubed_b200 import workloads as W
    members = [W.ensemble_member(sd, precision=1) for sd in member_seeds(0, nmembers)]
    cells = sum(cells_of(c) for c, _ in members)
    mixed = measure_ensemble(members, 1, steps, warmup, cache=cache)
    fp64 = measure_ensemble(members, 0, steps, warmup, cache=cache)
    return {"members": nmembers, "cells_per_step": cells, "steps": steps, "warmup": warmup,
            "workload": "batched ensemble of exo3 dry atmospheres, N in {24..96}, L in {32..96}, "
                        "Ts 150-400 K, gravity 3-25, gamma 1.3-1.67, one graph launch per step",
            "mixed": {"value": cells * steps / (mixed["ms"] / 1e3),
                      "ms_per_step": mixed["ms"] / steps, "gpu_launches": mixed["launches"],
                      "state_valid": mixed["valid"]},
            "fp64": {"value": cells * steps / (fp64["ms"] / 1e3),
                     "ms_per_step": fp64["ms"] / steps, "state_valid": fp64["valid"]},
            "mixed_over_fp64": fp64["ms"] / mixed["ms"],
            "tiles": "autotuned per kernel over the members (autotune.batch_tiles)"}


def serving_sample(rate, nreq, steps, fp64_baseline=True, cache=None):
    """A short continuous-batching run (mixed) and, for the same requests,
    the plain FP64 path one request at a time."""
    from exocubed_b200 import autotune
    from exocubed_b200 import workloads as W
    from exocubed_b200.serving import (Request, Server, poisson_arrivals,
                                       served_one_at_a_time, summarize)
    t_arr = poisson_arrivals(rate, nreq, seed=int(rate))
    reqs = []
    for n, a in enumerate(t_arr):
        cfg, w = W.ensemble_member(50_000 + n, precision=1)
        reqs.append(Request(n, cfg, w, float(a), steps))
    cache = cache if cache is not None else autotune.TileCache()
    autotune.batch_tiles([r.cfg for r in reqs], cache)  # measured before the clock starts
    srv = Server(precision=1, capacity=64, budget_bytes=150 * 10 ** 9, max_chunk=8,
                 tile_cache=cache)
    srv.run(reqs[:2], clock="steps")  # warm-up: graph capture, pools
    mixed = summarize(srv.run(reqs))
    srv.close()
    base = None
    if fp64_baseline:
        base = summarize(served_one_at_a_time(
            [dataclasses.replace(r, cfg=dict(r.cfg, precision=0)) for r in reqs]))
    return {"rate_per_s": rate, "requests": nreq, "steps_per_request": steps,
            "members": "ensemble distribution (N in 24..96, L in 32..96, varied gas and gravity)",
            "continuous_batching_mixed": mixed, "one_at_a_time_fp64": base}


def run_ours(args):
    import torch

    world, rank, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    prec = args.precision
    cfg, desc = workload_config(args.workload, prec)
    state = make_state(cfg, seed=rank)
    cells = cells_of(cfg)

    tune = not args.no_autotune
    alu = alu_peaks()
    main = measure_path(cfg, state, args.steps, args.warmup, pg, local, rank == 0, tune)
    ms_e2e, nbytes = measure_e2e(cfg, state, args.steps, pg, tune)
    plain = None
    if prec == 1 and not args.no_fp64:
        plain = measure_path(dict(cfg, precision=0), state, args.steps, args.warmup, pg, local,
                             False, tune)
    # the same workload with the implicit solve's blocks in FP32 as well
    f32s = None
    if prec == 1 and not args.no_f32_solve and cfg["eqn"] == 1 and cfg["implicit_flag"] & 1:
        f32s = measure_path(dict(cfg, precision=2), state, args.steps, args.warmup, pg, local,
                            False, tune)
    value = world * cells * args.steps / (main["ms"] / 1e3)
    e2e_value = world * cells * args.steps / (ms_e2e / 1e3)

    # dominant kernel and its roofline (algorithmic bytes per launch)
    prof = main["prof"]
    dom = max((k for k in prof if k != "other"), key=lambda k: prof[k][1])
    n_l, t_l = prof[dom]
    iflag = cfg.get("implicit_flag", 9)
    if dom == "implicit" and prec == 2 and iflag & 8:
        n_l //= 2  # the FP32-block full solve is a forward and a backward launch
    avg_ms = t_l / max(n_l, 1)
    alg_bytes = state_bytes_per_cell(dom, prec) * cells
    all_bytes = alg_bytes_per_cell(dom, prec, iflag) * cells
    peak, peak_kind = load_peaks()
    achieved = alg_bytes / (avg_ms / 1e3) / 1e9
    achieved_all = all_bytes / (avg_ms / 1e3) / 1e9
    traffic = None
    fp64_flops = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        tr = json.load(open(tp)).get(traffic_key(dom, prec, iflag))
        if tr:  # DRAM bytes per cell measured by ncu, scaled to this launch
            traffic = tr["bytes_per_cell"] * cells
            if tr.get("fp64_flops_per_cell"):  # ncu: dadd + dmul + 2 dfma per cell
                fp64_flops = tr["fp64_flops_per_cell"] * cells
    shares = {k: round(v[1] / sum(x[1] for x in prof.values()), 4) for k, v in prof.items()}

    extra = {}
    if rank == 0 and world == 1:
        if args.accuracy_steps > 0 and prec in (1, 2):
            c0 = workload_config(args.workload, 0)[0]
            ref = fp64_reference(c0, state, args.accuracy_steps)
            extra["accuracy"] = accuracy(c0, state, args.accuracy_steps, prec, ref)
            if f32s is not None:
                extra["accuracy_f32_solve"] = accuracy(c0, state, args.accuracy_steps, 2, ref)
        if args.oracle_accuracy:
            extra["accuracy_vs_oracle"] = accuracy_vs_oracle()
        from exocubed_b200 import autotune
        cache = autotune.TileCache()
        if args.ensemble_members > 0:
            extra["ensemble"] = ensemble_sample(args.ensemble_members, args.ensemble_steps,
                                                3, cache)
        if args.serve_requests > 0:
            extra["serving"] = serving_sample(args.serve_rate, args.serve_requests,
                                              args.serve_steps, not args.no_fp64_baseline,
                                              cache)
        if not args.no_cpu_baseline:
            r = run_cpu(args.workload, args.cpu_steps, args.cpu_warmup)
            extra["cpu_baseline"] = {
                "value": r["cells"] * r["steps"] / r["seconds"], "unit": "cell-updates/s",
                "cores": r["threads"], "kind": "port",
                "sample": f"oracle/ C++ restatement, OpenMP on {r['threads']} threads, "
                          f"{r['steps']} full step(s) of the same workload after "
                          f"{args.cpu_warmup} warm-up step(s)"}
    if rank != 0:
        if pg is not None:
            pg.destroy_process_group()
        return
    line = {
        "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": main["ms"] / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if prec == 0 else "f32+f64",
        "data": "synthetic",
        "config": {"workload": desc, "cells_per_step": cells, "replicas": world,
                   "l2": "every state array is larger than the 126 MB L2",
                   "parallelism": f"replicas x{world}",
                   "tiles": dict(zip(["x1", "x23", "update", "implicit", "prim_ghost",
                                      "roundtrip"], main["tiles"])),
                   "tiles_from": "autotuner (before the timed region)" if tune
                                 else "defaults"},
        "fp64": None if plain is None else {
            "value": world * cells * args.steps / (plain["ms"] / 1e3),
            "ms_per_step": plain["ms"] / args.steps,
            "note": "the plain FP64 path on the same workload, same run"},
        "mixed_f32_solve": None if f32s is None else {
            "value": world * cells * args.steps / (f32s["ms"] / 1e3),
            "ms_per_step": f32s["ms"] / args.steps,
            "accuracy_rel_l2": {k: v["rel_l2"] for k, v in
                                extra.get("accuracy_f32_solve", {}).get("fields", {}).items()},
            "note": "--precision 2 on the same workload, same run: the implicit solve's blocks "
                    "in FP32 as well (state and corrected update FP64)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "kernel": dom,
                     "peak_kind": peak_kind,
                     "bytes_per_cell": state_bytes_per_cell(dom, prec),
                     "ms_per_launch": avg_ms,
                     "with_intermediates": {
                         "bytes_per_cell": alg_bytes_per_cell(dom, prec, iflag),
                         "achieved": achieved_all, "frac": achieved_all / peak,
                         "note": "adds the kernel's face fluxes, factor scratch and FP32 "
                                 "copies to its state bytes"},
                     "step_frac": value / world * BYTES_PER_CELL_UPDATE / 1e9 / peak,
                     "alu_peaks": alu,
                     "fp64_pipe_frac": (fp64_flops / (avg_ms / 1e3) / alu["fp64_flops_per_s"]
                                        if fp64_flops and alu else None)},
        "kernel_share": shares,
        "launch_gaps": launch_gaps(main, args.steps),
        "cpu_baseline": extra.get("cpu_baseline"),
        "e2e": {"value": e2e_value, "unit": "cell-updates/s",
                "h2d_bytes_per_step": nbytes / args.steps, "d2h_bytes_per_step": nbytes / args.steps,
                "steps_per_request": args.steps},
        "gpu_launches": main["launches"],
        "clocks": main["clocks"],
        "state_valid": main["invalid"] == 0,
    }
    if "accuracy" in extra:
        line["accuracy"] = dict(extra["accuracy"], vs="the plain FP64 GPU path on the same state")
    if extra.get("accuracy_vs_oracle"):
        line["accuracy_vs_oracle"] = extra["accuracy_vs_oracle"]
    if "ensemble" in extra:
        line["ensemble"] = extra["ensemble"]
    if "serving" in extra:
        line["serving"] = extra["serving"]
    print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()


def run_ensemble(args):
    """Batched ensemble: args.members independent atmospheres drawn from the
    member distribution (uneven N, L, gas and gravity), advanced together by
    one graph-captured batched step per step; every rank runs its own
    ensemble (seeds differ by rank)."""
    import numpy as np
    import torch

    from exocubed_b200 import workloads as W
    from exocubed_b200.ensemble import Ensemble

    world, rank, local, pg = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    prec = args.precision
    members = [W.ensemble_member(sd, precision=prec) for sd in member_seeds(rank, args.members)]
    cells = sum(cells_of(c) for c, _ in members)
    ens = Ensemble(precision=prec, capacity=args.members)
    slots = [ens.add(c, w) for c, w in members]
    t_tune = time.perf_counter()
    tiles = ens.autotune() if not args.no_autotune else ens.tiles
    t_tune = time.perf_counter() - t_tune
    stream = torch.cuda.ExternalStream(ens.stream)
    ens.step(args.warmup)
    ens.synchronize()
    clocks = ClockSampler(local)
    if rank == 0:
        clocks.start()
    l0 = ens.stats()["launches"]
    barrier(pg)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ens.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier(pg)
    ms_max = max_over_ranks(pg, e0.elapsed_time(e1))
    launches = ens.stats()["launches"] - l0
    clk = clocks.stop() if rank == 0 else None
    valid = all(ens.invalid(s) == 0 for s in slots)
    nbytes_state = sum(w.nbytes for _, w in members)
    ens.close()

    # end to end: every member admitted from pinned host memory, K steps,
    # every member's conserved state read back
    pinned = [(c, torch.from_numpy(w).pin_memory().numpy()) for c, w in members]
    outs = [np.empty_like(w) for _, w in pinned]
    ens = Ensemble(precision=prec, capacity=args.members)
    ens.set_tiles(tiles)
    s2 = torch.cuda.ExternalStream(ens.stream)
    barrier(pg)
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(s2)
    slots = [ens.add(c, w) for c, w in pinned]
    ens.step(args.steps)
    for s, o in zip(slots, outs):
        o[...] = ens.conserved(s)
    f1.record(s2)
    f1.synchronize()
    barrier(pg)
    ms_e2e = max_over_ranks(pg, f0.elapsed_time(f1))
    ens.close()

    value = world * cells * args.steps / (ms_max / 1e3)
    peak, peak_kind = load_peaks()
    achieved = value / world * BYTES_PER_CELL_UPDATE / 1e9
    if rank == 0:
        Ns = [c["N"] for c, _ in members]
        Ls = [c["L"] for c, _ in members]
        print(json.dumps({
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if prec == 0 else "f32+f64", "data": "synthetic",
            "config": {"workload": f"batched ensemble of {args.members} exo3 dry atmospheres, "
                                   f"N in {sorted(set(Ns))}, L in {sorted(set(Ls))}, "
                                   f"{'FP64' if prec == 0 else 'mixed FP32/FP64'}, "
                                   "one graph-captured batched SSPRK3 step per step",
                       "members": args.members, "cells_per_step": cells,
                       "tiles": dict(zip(["x1", "x23", "update", "implicit", "prim_ghost",
                                          "roundtrip"], tiles)),
                       "autotune_s": round(t_tune, 2),
                       "l2": f"{nbytes_state / 1e9:.1f} GB of member state exceeds the 126 MB L2"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": "whole batched step (320 B per cell-update)",
                         "peak_kind": peak_kind},
            "e2e": {"value": world * cells * args.steps / (ms_e2e / 1e3), "unit": "cell-updates/s",
                    "h2d_bytes_per_step": nbytes_state / args.steps,
                    "d2h_bytes_per_step": nbytes_state / args.steps,
                    "steps_per_request": args.steps},
            "gpu_launches": launches, "clocks": clk, "state_valid": bool(valid)}))
    if pg is not None:
        pg.destroy_process_group()


def run_serving(args):
    """Serving sweep: for each arrival rate, a Poisson stream of args.requests
    forward-model requests (ensemble members, 200 steps each) served by the
    continuous-batching server in mixed precision, and the same requests on
    the plain FP64 path one at a time; one JSON line per rate."""
    import torch

    from exocubed_b200 import workloads as W
    from exocubed_b200.serving import (Request, Server, poisson_arrivals,
                                       served_one_at_a_time, summarize)
    torch.cuda.init()
    for rate in [float(x) for x in args.serve.split(",")]:
        t_arr = poisson_arrivals(rate, args.requests, seed=int(rate))
        reqs = []
        for n, a in enumerate(t_arr):
            cfg, w = W.ensemble_member(50_000 + n, precision=1)
            reqs.append(Request(n, cfg, w, float(a), args.serve_steps))
        cache = None
        if not args.no_autotune:
            from exocubed_b200 import autotune
            cache = autotune.TileCache()
            autotune.batch_tiles([r.cfg for r in reqs], cache)  # measured before the clock starts
        srv = Server(precision=1, capacity=64, budget_bytes=150 * 10 ** 9, max_chunk=8,
                     tile_cache=cache)
        srv.run(reqs[:2], clock="steps")  # warm-up: graph capture, pools
        mixed = summarize(srv.run(reqs))
        srv.close()
        base = None
        if not args.no_fp64_baseline:
            base = summarize(served_one_at_a_time(
                [dataclasses.replace(r, cfg=dict(r.cfg, precision=0)) for r in reqs]))
        print(json.dumps({"serving": {
            "rate_per_s": rate, "requests": args.requests, "steps_per_request": args.serve_steps,
            "members": "ensemble distribution (N in 24..96, L in 32..96, varied gas and gravity)",
            "continuous_batching_mixed": mixed, "one_at_a_time_fp64": base}}), flush=True)


def run_mcmc(args):
    """MCMC driver: the stretch-move sampler with args.mcmc walkers over the
    temperature-profile problem (each forward model a 6 x 32^2 x 48
    atmosphere run args.mcmc_steps steps), its forward models batched in one
    mixed-precision ensemble, against the same sampler evaluating them one
    at a time on FP64 contexts (the reference's order).  Reports walker
    evaluations per second and cell-updates per second of both."""
    import time

    import numpy as np
    import torch

    from exocubed_b200.inversion import (EnsembleForward, SequentialForward, StretchSampler,
                                         profile_problem)
    torch.cuda.init()
    nw, steps, iters = args.mcmc, args.mcmc_steps, args.mcmc_iters
    build, observe, nvalue = profile_problem(N=32, L=48, steps=steps)
    obs = SequentialForward(build, observe, nvalue, steps, precision=0)(
        np.array([[285., 205.]]))[0]

    def log_prob(theta, val):
        Ts, Ttop = theta
        if not (200. < Ts < 350. and 150. < Ttop < Ts) or np.isnan(val).any():
            return -np.inf
        return float(-0.5 * (((val - obs) / 2.0) ** 2).sum())

    rng = np.random.default_rng(0)
    pos = np.stack([280. + 5 * rng.standard_normal(nw), 200. + 5 * rng.standard_normal(nw)], 1)
    out = {}
    for name, fwd in (("batched_mixed", EnsembleForward(build, observe, nvalue, steps,
                                                        precision=1, capacity=nw)),
                      ("one_at_a_time_fp64", SequentialForward(build, observe, nvalue, steps,
                                                               precision=0))):
        fwd(pos[:2])  # warm-up: contexts, pools, graph capture
        fwd.cell_updates = 0
        sampler = StretchSampler(fwd, log_prob, nw, 2, nvalue, seed=1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rec = sampler.run(pos, iters)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        out[name] = {"seconds": el, "evaluations": sampler.evaluations,
                     "evaluations_per_s": sampler.evaluations / el,
                     "cell_updates_per_s": fwd.cell_updates / el,
                     "acceptance": rec.acceptance_fraction(),
                     "best_theta": [float(x) for x in rec.opt_par]}
        if hasattr(fwd, "close"):
            fwd.close()
    print(json.dumps({"mcmc": {
        "walkers": nw, "iterations": iters, "forward": f"6x32x32x48 dry atmosphere, {steps} steps",
        "speedup": out["batched_mixed"]["evaluations_per_s"] /
        out["one_at_a_time_fp64"]["evaluations_per_s"], **out}}), flush=True)


def run_accuracy(args):
    """Mixed precision against the FP64 path after args.accuracy steps."""
    import torch  # noqa: F401  (CUDA context)
    cfg, desc = workload_config(args.workload, 0)
    res = accuracy(cfg, make_state(cfg, seed=0), args.accuracy,
                   args.precision if args.precision in (1, 2) else 1)
    res["workload"] = desc.replace("FP64", "mixed vs FP64")
    print(json.dumps({"accuracy": res}))


def run_reference(args):
    """The reference arm: the oracle (the reference's algorithm restated in
    C++, FP64, OpenMP on all host threads) on the same workload.  It times
    the --steps steps after the --warmup warm-up steps it reports (or, with
    --ref-steps, that many) in a process that never loads the product
    library; under torchrun only rank 0 runs."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg, desc = workload_config(args.workload, 0)
    steps = args.steps if args.ref_steps <= 0 else min(args.steps, args.ref_steps)
    warm = args.warmup
    r = run_cpu(args.workload, steps, warm)
    v = r["cells"] * r["steps"] / r["seconds"]
    line = {
        "impl": "reference", "metric": "cell-updates/s", "value": v, "unit": "cell-updates/s",
        "n_gpus": world, "steps": r["steps"], "warmup": warm,
        "ms_per_step": r["seconds"] / r["steps"] * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc, "cells_per_step": r["cells"]},
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": r["threads"],
                         "kind": "port",
                         "sample": f"{r['steps']} full FP64 step(s) of the workload after "
                                   f"{warm} warm-up step(s); the reference cannot be built "
                                   "here, its C++ restatement (oracle/) runs with OpenMP on "
                                   "all host threads, on a state generated on its own mesh"},
        "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=["c1", "c2", "c2s", "c3", "c4", "hs94"])
    ap.add_argument("--members", type=int, default=64, help="ensemble members (c4)")
    ap.add_argument("--serve", default="", help="comma-separated arrival rates (req/s): serving sweep")
    ap.add_argument("--requests", type=int, default=24, help="requests per rate (serving)")
    ap.add_argument("--serve-steps", type=int, default=200)
    ap.add_argument("--no-fp64-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch tiles")
    ap.add_argument("--precision", type=int, default=1, choices=[0, 1, 2],
                    help="0: FP64; 1: mixed (FP32 reconstruction, x2/x3 Riemann and "
                         "divergence); 2: mixed with FP32 implicit blocks")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison leg")
    ap.add_argument("--no-f32-solve", action="store_true",
                    help="skip the leg with FP32 implicit blocks (--precision 2)")
    ap.add_argument("--accuracy-steps", type=int, default=100,
                    help="steps of the mixed-vs-FP64 error check in the bench line (0: none)")
    ap.add_argument("--serve-requests", type=int, default=32,
                    help="requests of the serving sample in the bench line (0: none)")
    ap.add_argument("--no-oracle-accuracy", dest="oracle_accuracy", action="store_false",
                    help="skip the 1000-step C2 comparison with the oracle's run")
    ap.add_argument("--ensemble-members", type=int, default=64,
                    help="members of the C4 ensemble sample in the bench line (0: none)")
    ap.add_argument("--ensemble-steps", type=int, default=10)
    ap.add_argument("--serve-rate", type=float, default=2.0,
                    help="arrival rate (req/s) of the serving sample: at 2 req/s the batching "
                         "server keeps up with the stream and the one-at-a-time FP64 path does not")
    ap.add_argument("--ref-steps", type=int, default=0,
                    help="full steps the reference arm times at most (0: all of --steps)")
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--cpu-warmup", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-worker", action="store_true")
    ap.add_argument("--accuracy", type=int, default=0,
                    help="run N steps mixed vs FP64 and report the field errors")
    ap.add_argument("--rsolver", type=int, default=None, choices=[1, 2],
                    help="Riemann solver of exo3 workloads: 1 LMARS (default), 2 HLLC")
    ap.add_argument("--mcmc", type=int, default=0,
                    help="walkers: run the MCMC driver comparison instead of a step benchmark")
    ap.add_argument("--mcmc-steps", type=int, default=50, help="steps per forward model (mcmc)")
    ap.add_argument("--mcmc-iters", type=int, default=3, help="sampler iterations (mcmc)")
    ap.add_argument("--implicit-flag", type=int, default=None, choices=[1, 9],
                    help="implicit_flag of exo3 workloads: 9 full 5x5 (default), 1 partial 3x3")
    args = ap.parse_args()
    _RS[0] = args.rsolver
    _IMP[0] = args.implicit_flag
    if args.cpu_worker:
        cpu_worker(args)
    elif args.accuracy > 0:
        run_accuracy(args)
    elif args.serve:
        run_serving(args)
    elif args.mcmc:
        run_mcmc(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == "c4":
        run_ensemble(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
