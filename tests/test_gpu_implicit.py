"""exo_implicit_columns (the FullCorrection hook over a batch of columns)
against the oracle's restatement of ImplicitSolver::FullCorrection.

No transcendental function enters the block-tridiagonal solve (only +, -, *,
/ and sqrt), so the comparison is bit-exact."""
import numpy as np
import pytest

from _columns import column_problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ncol,L,dt", [(1, 12, 30.0), (257, 16, 400.0), (1000, 40, 1500.0),
                                       (70, 250, 200.0)])
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
