"""exo_implicit_columns_noalloc: the vertical implicit solve for callers that
cannot allocate device memory while they step (a host application whose
memory pool owns the GPU, a loop that must not stall on the synchronization
cudaMalloc/cudaFree can cause, a fixed memory budget).  Its scratch is a
fixed 8 MiB device array inside the library instead of caller memory.

Checked against the allocating entry point exo_implicit_columns, which runs
the same kernel on caller-provided scratch: the results must be identical,
on two calls in a row (the second one sees the first call's leftovers in the
shared array), and the second call must not change the device's free memory.
This file is named so that pytest collects it last.
"""
import numpy as np
import pytest

from exocubed_b200 import workloads as W

pytestmark = pytest.mark.gpu
G = 3


def _columns(oracle_mod, ncol, L, seed):
    N = 8
    cfg = W.dry_atmosphere_config(N=N, L=L, rsolver=2)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(W.dry_atmosphere_state(cfg, seed=seed))
    wfull = o.primitive()
    x1f, _, _ = o.mesh(0)
    rng = np.random.default_rng(seed)
    w = np.stack([wfull[rng.integers(6), :, G + rng.integers(N), G + rng.integers(N), :]
                  for _ in range(ncol)])
    scale = np.abs(w[:, :, G:G + L]).mean(axis=(0, 2))
    du = 1e-4 * scale[None, :, None] * rng.standard_normal((ncol, 5, L))
    cth = 0.5 * rng.uniform(-1, 1, ncol)
    colgeo = np.stack([cth, np.sqrt(1 - cth ** 2), np.full(ncol, np.pi / 2 / N),
                       np.full(ncol, np.pi / 2 / N)], axis=1)
    return dict(w=w, du=du, g=colgeo, x1f=x1f, x1v=0.5 * (x1f[1:] + x1f[:-1]),
                dx1f=np.diff(x1f)), cfg


def _solve(native, torch, arrays, cfg, dt, noalloc):
    ncol, _, L = arrays["du"].shape
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in arrays.items()}
    torch.cuda.synchronize()
    args = [ncol, L, t["w"].data_ptr(), t["du"].data_ptr(), t["g"].data_ptr(),
            t["x1f"].data_ptr(), t["x1v"].data_ptr(), t["dx1f"].data_ptr(), dt,
            cfg["gamma"], cfg["grav"]]
    if noalloc:
        free0 = torch.cuda.mem_get_info()[0]
        rc = native.lib().exo_implicit_columns_noalloc(*args, None)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
    else:
        scratch = torch.empty(ncol * L * 30, dtype=torch.float64, device="cuda")
        rc = native.lib().exo_implicit_columns(*args, scratch.data_ptr(), None)
        torch.cuda.synchronize()
        free0 = free1 = 0
    assert rc == 0, native.lib().exo_last_error()
    return t["du"].cpu().numpy(), free0 - free1


def test_noalloc_matches_allocating_entry_point_twice(oracle_mod, native):
    torch = pytest.importorskip("torch")
    # the last case fills the fixed array to its last whole column level:
    # 4369 columns x 8 levels = NOALLOC_SCRATCH_DOUBLES // 30 column levels
    assert 4369 * 8 == native.NOALLOC_SCRATCH_DOUBLES // 30
    cases = [(_columns(oracle_mod, 300, 40, seed=21), 900.0),
             (_columns(oracle_mod, 120, 64, seed=22), 300.0),
             (_columns(oracle_mod, 4369, 8, seed=23), 600.0)]
    for n, ((arrays, cfg), dt) in enumerate(cases):
        want, _ = _solve(native, torch, arrays, cfg, dt, noalloc=False)
        got, freed = _solve(native, torch, arrays, cfg, dt, noalloc=True)
        assert np.isfinite(got).all()
        assert np.array_equal(got, want), np.abs(got - want).max()
        if n >= 1:  # after the first call's one-time set-up: nothing is allocated
            assert freed == 0


def test_noalloc_rejects_batches_beyond_its_scratch(native):
    torch = pytest.importorskip("torch")
    limit = native.NOALLOC_SCRATCH_DOUBLES // 30
    L = 64
    ncol = limit // L + 1
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda").data_ptr()
    rc = native.lib().exo_implicit_columns_noalloc(ncol, L, dummy, dummy, dummy, dummy, dummy,
                                                   dummy, 1.0, 1.4, -9.81, None)
    assert rc == 7  # EXO_ERR_CAPACITY
    assert b"exceeds the fixed scratch" in native.lib().exo_last_error()
