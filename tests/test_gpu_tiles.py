"""Launch tiles and their autotuner: any tile gives the same result to the
bit (only the launch shape changes), invalid tiles are refused, and the
autotuner measures each configuration once and caches it."""
import numpy as np
import pytest

from exocubed_b200 import CubedSphereAtmosphere
from exocubed_b200 import _native as nat
from exocubed_b200 import autotune
from exocubed_b200 import workloads as W
from exocubed_b200.ensemble import Ensemble

pytestmark = pytest.mark.gpu


def _run(cfg, w, tiles, steps=3):
    with CubedSphereAtmosphere(cfg) as a:
        if tiles:
            a.set_tiles(tiles)
        a.set_primitive(w)
        a.step(steps)
        return a.conserved(), a.tiles


@pytest.mark.parametrize("precision", [nat.EXO_PREC_FP64, nat.EXO_PREC_MIXED])
@pytest.mark.parametrize("implicit", [9, 0])
def test_tiles_do_not_change_results(precision, implicit):
    cfg = W.dry_atmosphere_config(N=10, L=20, implicit_flag=implicit, precision=precision)
    w = W.dry_atmosphere_state(cfg, seed=5)
    ref, t0 = _run(cfg, w, None)
    assert t0[1:] == [128, 128, 64, 256, 128]
    assert t0[0] == 4
    for tiles in ([1, 64, 256, 32, 512, 64], [2, 256, 64, 128, 128, 256], [8, 32, 32, 32, 32, 32]):
        got, t = _run(cfg, w, tiles)
        assert t == tiles
        assert np.array_equal(got, ref), tiles


def test_ensemble_tiles_keep_members_exact():
    prec = nat.EXO_PREC_MIXED
    members = []
    for n, (N, L) in enumerate([(8, 16), (10, 12), (6, 20)]):
        cfg = W.dry_atmosphere_config(N=N, L=L, precision=prec, g=6. + 3 * n)
        members.append((cfg, W.dry_atmosphere_state(cfg, seed=60 + n)))
    alone = [_run(c, w, None)[0] for c, w in members]
    ens = Ensemble(precision=prec, capacity=4)
    slots = [ens.add(c, w) for c, w in members]
    ens.step(1)
    ens.set_tiles([2, 256, 64, 128, 512, 64])   # changes shape mid-run
    ens.step(2)
    ens.synchronize()
    assert ens.tiles == [2, 256, 64, 128, 512, 64]
    for s, a in zip(slots, alone):
        assert np.array_equal(ens.conserved(s), a)
    ens.close()


def test_invalid_tiles_are_refused():
    cfg = W.dry_atmosphere_config(N=6, L=8)
    with CubedSphereAtmosphere(cfg) as a:
        for bad in ([0, 100, 0, 0, 0, 0], [0, 0, 0, 96, 0, 0], [0, 0, 1024, 0, 0, 0],
                    [9, 0, 0, 0, 0, 0]):
            with pytest.raises(nat.ExoError) as e:
                a.set_tiles(bad)
            assert e.value.code == 1
        assert a.tiles[1:] == [128, 128, 64, 256, 128]


def test_autotune_measures_once_and_caches(tmp_path, monkeypatch):
    cache = autotune.TileCache(str(tmp_path / "tiles.json"))
    cfg = W.dry_atmosphere_config(N=12, L=16, precision=nat.EXO_PREC_MIXED)
    tiles = autotune.best_tiles(cfg, cache)
    for k, cand in autotune.CANDIDATES.items():
        assert tiles[k] in cand
    assert (tmp_path / "tiles.json").exists()
    monkeypatch.setattr(autotune, "measure", lambda *a, **k: pytest.fail("measured twice"))
    assert autotune.best_tiles(cfg, autotune.TileCache(str(tmp_path / "tiles.json"))) == tiles


def test_atmosphere_autotune_sets_the_tuned_tiles(tmp_path):
    cache = autotune.TileCache(str(tmp_path / "tiles.json"))
    cfg = W.dry_atmosphere_config(N=12, L=16, precision=nat.EXO_PREC_MIXED)
    state = W.dry_atmosphere_state(cfg, seed=3)
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(state)
        a.step(2)
        want = a.conserved()
    with CubedSphereAtmosphere(cfg) as a:
        tiles = a.autotune(cache)
        assert tiles == a.tiles
        for k, cand in autotune.CANDIDATES.items():
            assert tiles[k] in cand
        a.set_primitive(state)
        a.step(2)
        assert np.array_equal(a.conserved(), want)
