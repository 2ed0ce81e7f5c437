"""Autotuner host logic, no GPU: keys, cache round trip, and the choice of
one tile per kernel for a batch (least summed member time)."""
from exocubed_b200 import _native as nat
from exocubed_b200 import autotune
from exocubed_b200 import workloads as W


def test_config_key_distinguishes_what_changes_the_kernels():
    a = W.dry_atmosphere_config(N=24, L=32, precision=1)
    assert autotune.config_key(a) == "N24_L32_eqn1_rs1_imp9_prec1"
    assert autotune.config_key(dict(a, precision=0)) != autotune.config_key(a)
    assert autotune.config_key(dict(a, grav=-3.0)) == autotune.config_key(a)


def test_cache_round_trip(tmp_path):
    c = autotune.TileCache(str(tmp_path / "t.json"))
    c.tables["k"] = {nat.EXO_K_UPDATE: {64: 0.5, 128: 0.25}}
    c.save()
    d = autotune.TileCache(str(tmp_path / "t.json"))
    assert d.tables == c.tables


def test_batch_choice_minimises_summed_time():
    K = nat.EXO_K_IMPLICIT
    small = {K: {32: 1.0, 64: 2.0, 128: 3.0}}
    big = {K: {32: 10.0, 64: 6.0, 128: 9.0}}
    assert autotune._pick([small])[K] == 32
    assert autotune._pick([big])[K] == 64
    assert autotune._pick([small, big])[K] == 64      # 8.0 < 11.0 < 12.0
    assert autotune._pick([small, small, small, small, small, big])[K] == 32
    t = autotune._pick([{nat.EXO_K_UPDATE: {256: 1.0, 64: 2.0}}])
    assert t[nat.EXO_K_UPDATE] == 256 and t[nat.EXO_K_OTHER] == 256
    assert t[nat.EXO_K_FLUX_X1] == 0 and t[nat.EXO_K_PRIM_GHOST] == 0  # not measured: keep
