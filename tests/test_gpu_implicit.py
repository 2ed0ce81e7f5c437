"""exo_implicit_columns (the FullCorrection hook over a batch of columns)
against the oracle's restatement of ImplicitSolver::FullCorrection.

No transcendental function enters the block-tridiagonal solve (only +, -, *,
/ and sqrt), so the comparison is bit-exact."""
import numpy as np
import pytest

from exocubed_b200 import workloads as W

pytestmark = pytest.mark.gpu
G = 3


def column_problem(oracle_mod, ncol, L, seed):
    """Realistic columns: primitives of a perturbed isothermal atmosphere with
    reflected ghosts, an explicit update of the right scale, metric values of
    real cells."""
    N = 8
    cfg = W.dry_atmosphere_config(N=N, L=L, rsolver=2)
    o = oracle_mod.Oracle(cfg)
    o.set_primitive(W.dry_atmosphere_state(cfg, seed=seed))
    wfull = o.primitive()
    x1f, _, _ = o.mesh(0)
    x1v = 0.5 * (x1f[1:] + x1f[:-1])
    dx1f = np.diff(x1f)
    rng = np.random.default_rng(seed)
    cols = []
    for c in range(ncol):
        p, k, j = rng.integers(6), G + rng.integers(N), G + rng.integers(N)
        cols.append(wfull[p, :, k, j, :])
    w = np.stack(cols)                                   # [ncol][5][L+6]
    scale = np.abs(w[:, :, G:G + L]).mean(axis=(0, 2))
    du = 1e-4 * scale[None, :, None] * rng.standard_normal((ncol, 5, L))
    du[:, 1:4] = 1e-3 * rng.standard_normal((ncol, 3, L))
    cth = 0.5 * rng.uniform(-1, 1, ncol)
    colgeo = np.stack([cth, np.sqrt(1 - cth ** 2),
                       np.pi / 2 / N * rng.uniform(0.8, 1.0, ncol),
                       np.pi / 2 / N * rng.uniform(0.8, 1.0, ncol)], axis=1)
    return w, du, colgeo, x1f, x1v, dx1f, cfg


@pytest.mark.parametrize("ncol,L,dt", [(1, 12, 30.0), (257, 16, 400.0), (1000, 40, 1500.0)])
def test_implicit_columns_bitwise(oracle_mod, native, ncol, L, dt):
    torch = pytest.importorskip("torch")
    w, du, colgeo, x1f, x1v, dx1f, cfg = column_problem(oracle_mod, ncol, L, seed=ncol)
    ref = oracle_mod.implicit_columns(w, du, colgeo, x1f, x1v, dx1f, dt, cfg["gamma"], cfg["grav"])
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda()
         for k, v in dict(w=w, du=du, g=colgeo, x1f=x1f, x1v=x1v, dx1f=dx1f).items()}
    scratch = torch.empty(ncol * L * 30, dtype=torch.float64, device="cuda")
    rc = native.lib().exo_implicit_columns(
        ncol, L, t["w"].data_ptr(), t["du"].data_ptr(), t["g"].data_ptr(), t["x1f"].data_ptr(),
        t["x1v"].data_ptr(), t["dx1f"].data_ptr(), dt, cfg["gamma"], cfg["grav"],
        scratch.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    got = t["du"].cpu().numpy()
    assert np.isfinite(got).all()
    assert np.array_equal(got, ref), np.abs(got - ref).max()
    # the correction is not the identity: the implicit solve changed du
    assert np.abs(got - du).max() > 0


def test_implicit_columns_rejects_bad_args(native):
    L = native.lib()
    assert L.exo_implicit_columns(-1, 4, None, None, None, None, None, None, 1., 1.4, -9.8,
                                  None, None) == 1
    assert L.exo_implicit_columns(0, 4, None, None, None, None, None, None, 1., 1.4, -9.8,
                                  None, None) == 0
