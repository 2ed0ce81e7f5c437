"""Host side of the batched ensemble, no GPU: the member generator follows
its stated distributions and profile, and the footprint the admission
ledger charges is the sum of the member's device arrays."""
import numpy as np
import pytest

from exocubed_b200 import _native as nat
from exocubed_b200 import workloads as W
from exocubed_b200.ensemble import footprint


def test_member_distribution_and_profile():
    cfgs = [W.ensemble_member_config(seed)[0] for seed in range(200)]
    assert {c["N"] for c in cfgs} == set(W.ENSEMBLE_N)
    assert {c["L"] for c in cfgs} == set(W.ENSEMBLE_L)
    for c in cfgs:
        assert 1.3 <= c["gamma"] <= 1.67 and 3 <= -c["grav"] <= 25
        assert c["precision"] == nat.EXO_PREC_MIXED and c["implicit_flag"] == 9
    cells = np.mean([6 * c["N"] ** 2 * c["L"] for c in cfgs])
    assert 0.8e6 < cells < 1.7e6  # about 1.24 M cells per member on average
    # the analytic column: adiabat below the tropopause, isothermal above,
    # continuous at the joint and hydrostatic (dp/dz = -g rho) everywhere
    Ts, Tt, g, Rd, gam = 300., 180., 9.0, 287., 1.4
    z = np.linspace(0., 40e3, 40001)
    T, p = W._adiabat_isothermal(z, Ts, Tt, g, Rd, gam, 1e5)
    assert T[0] == Ts and T[-1] == Tt and T.min() == Tt
    dpdz = np.gradient(p, z)
    rho = p / (Rd * T)
    assert np.max(np.abs(dpdz + g * rho) / (g * rho))[()] < 2e-3


def test_member_state_top_pressure():
    cfg, w = W.ensemble_member(3)
    ptop = w[:, 4, 3:-3, 3:-3, 3:-3][..., -1].mean()
    assert 1e3 < ptop < 1.3e3  # the top cell centre sits just below p = 1e3 Pa
    assert (w[:, 0, 3:-3, 3:-3, 3:-3] > 0).all()


def test_footprint_counts_member_arrays():
    cfg = W.dry_atmosphere_config(N=16, L=20)
    cells = 6 * 5 * (16 + 6) ** 2 * (20 + 6)
    f64 = footprint(dict(cfg, precision=nat.EXO_PREC_FP64))
    mix = footprint(dict(cfg, precision=nat.EXO_PREC_MIXED))
    assert f64 >= 7 * cells * 8      # u, w, u1, du, three flux arrays
    assert mix > f64                 # plus the FP32 primitive and flux copies
    # FP32 implicit blocks take the same arrays (the solve's scratch is sized for FP64)
    assert footprint(dict(cfg, precision=nat.EXO_PREC_MIXED_F32_SOLVE)) == mix
    with pytest.raises(nat.ExoError):
        footprint(dict(cfg, precision=3))
    big = footprint(dict(cfg, N=96, L=96))
    assert big > 50 * f64
