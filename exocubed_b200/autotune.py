"""Autotuner of the launch tiles (threads per block) of the step's kernels.

For one atmosphere configuration it times every kernel of a few real steps
at each candidate tile (one candidate per kernel per trial, the kernels
timed separately by the library's event profiler) on a throw-away context
with a synthetic state of that configuration, and caches the per-launch
times under the key (N, L, equation set, solver, implicit flag, precision).

A single atmosphere takes, per kernel, the fastest candidate.  A batch of
uneven members runs each kernel as one launch, so it takes, per kernel, the
candidate with the least total time over its members' cached tables.

Tiles change only the launch shape: every cell's arithmetic is the same, so
results do not depend on them (tests/test_gpu_tiles.py checks it bit for
bit).  The cache is a JSON file ($EXO_TILE_CACHE, default
~/.cache/exocubed_b200/tiles.json).
"""
import json
import os
import threading

from . import _native as nat

# candidate tiles per kernel id; EXO_K_OTHER (the round trip of atmospheres
# without the implicit solver) is timed inside EXO_K_UPDATE and follows it
CANDIDATES = {
    nat.EXO_K_FLUX_X1: (1, 2, 3, 4),     # radial columns per block
    nat.EXO_K_FLUX_X23: (128,),          # both x2/x3 forms run 128 threads a block
    nat.EXO_K_UPDATE: (32, 64, 128, 256),
    nat.EXO_K_IMPLICIT: (32, 64, 128),
    nat.EXO_K_PRIM_GHOST: (64, 128, 256, 512),
}
NTRIAL = max(len(c) for c in CANDIDATES.values())  # trials measure every kernel at once

_lock = threading.Lock()


def cache_path():
    return os.environ.get("EXO_TILE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "exocubed_b200",
                                       "tiles.json"))


def config_key(cfg):
    c = cfg if isinstance(cfg, dict) else cfg.as_dict()
    return (f"N{c['N']}_L{c['L']}_eqn{c['eqn']}_rs{c['rsolver']}_imp{c['implicit_flag']}"
            f"_prec{c['precision']}")


class TileCache:
    """Per-configuration tables {kernel id: {threads: ms per launch}}."""

    def __init__(self, path=None):
        self.path = path or cache_path()
        self.tables = {}
        if os.path.exists(self.path):
            try:
                with open(self.path) as f:
                    raw = json.load(f)
                self.tables = {k: {int(kid): {int(t): float(ms) for t, ms in v.items()}
                                   for kid, v in tab.items()} for k, tab in raw.items()}
            except (OSError, ValueError):
                self.tables = {}

    def save(self):
        d = os.path.dirname(self.path)
        if d:
            os.makedirs(d, exist_ok=True)
        tmp = f"{self.path}.{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump({k: {str(kid): {str(t): ms for t, ms in v.items()} for kid, v in tab.items()}
                       for k, tab in self.tables.items()}, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)


def _synthetic_state(cfg):
    from . import workloads as W
    if cfg["eqn"] == nat.EXO_EQN_SHALLOW_YZ:
        return W.shallow_water_state(cfg, seed=0)
    return W.dry_atmosphere_state(cfg, seed=0)


def measure(cfg, steps=2):
    """Per-launch milliseconds of each tuned kernel at each candidate tile,
    on a throw-away context of this configuration."""
    from .atmosphere import CubedSphereAtmosphere
    cfg = cfg if isinstance(cfg, dict) else cfg.as_dict()
    table = {k: {} for k in CANDIDATES}
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(_synthetic_state(cfg))
        for trial in range(NTRIAL):
            tiles = [0] * nat.EXO_TILE_COUNT
            for k, cand in CANDIDATES.items():
                tiles[k] = cand[min(trial, len(cand) - 1)]
            tiles[nat.EXO_K_OTHER] = tiles[nat.EXO_K_UPDATE]
            a.set_tiles(tiles)
            a.step(1)  # warm-up at this shape
            a.profile(True)
            a.step(steps)
            prof = a.profile_read()
            a.profile(False)
            for k in CANDIDATES:
                n, ms = prof[nat.KERNELS[k]]
                if n > 0:
                    table[k][tiles[k]] = ms / n
    return {k: v for k, v in table.items() if v}


def table_for(cfg, cache=None):
    """The configuration's table, measured once and cached."""
    cache = cache if cache is not None else TileCache()
    key = config_key(cfg)
    with _lock:
        if key not in cache.tables:
            cache.tables[key] = measure(cfg)
            cache.save()
        return cache.tables[key]


def _pick(tables, weights=None):
    tiles = [0] * nat.EXO_TILE_COUNT
    for k, cand in CANDIDATES.items():
        best, best_t = None, None
        for c in cand:
            tot, seen = 0.0, False
            for n, tab in enumerate(tables):
                if k in tab and c in tab[k]:
                    tot += tab[k][c] * (weights[n] if weights else 1.0)
                    seen = True
            if seen and (best_t is None or tot < best_t):
                best, best_t = c, tot
        tiles[k] = best or 0
    tiles[nat.EXO_K_OTHER] = tiles[nat.EXO_K_UPDATE]
    return tiles


def best_tiles(cfg, cache=None):
    """Fastest tile per kernel for one atmosphere (0 = keep the default)."""
    return _pick([table_for(cfg, cache)])


def batch_tiles(cfgs, cache=None):
    """Tiles of one batched launch per kernel over members of these
    configurations: per kernel, the least summed member time."""
    cache = cache if cache is not None else TileCache()
    return _pick([table_for(c, cache) for c in cfgs])
