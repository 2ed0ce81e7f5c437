"""Checkpoints: a run resumed from its image takes the same bits as the run
that never stopped (MeshBlock::Impl::SaveAllStates / LoadAllStates,
src/impl.cpp:306-332, and Athena++ restart files, src/mesh_setup.cpp:25-97,
for the hydro state), in a context, in an ensemble and across the two."""
import numpy as np
import pytest

from exocubed_b200 import _native as nat
from exocubed_b200 import workloads as W
from exocubed_b200.atmosphere import CubedSphereAtmosphere
from exocubed_b200.ensemble import Ensemble

pytestmark = pytest.mark.gpu

CASES = {
    "shallow": (lambda: W.shallow_water_config(N=12), W.shallow_water_state),
    "dry": (lambda: W.dry_atmosphere_config(N=8, L=12, rsolver=nat.EXO_RS_HLLC),
            W.dry_atmosphere_state),
    "hs94": (lambda: W.hs94_config(N=8, L=20, cfl=0.4), W.hs94_state),
}


def _clock(a):
    return a.time, a.ncycle, a.dt


@pytest.mark.parametrize("precision", [nat.EXO_PREC_FP64, nat.EXO_PREC_MIXED])
@pytest.mark.parametrize("case", sorted(CASES))
def test_resume_is_bitwise(case, precision, tmp_path):
    mk_cfg, mk_state = CASES[case]
    cfg = dict(mk_cfg(), precision=precision)
    state = mk_state(cfg, seed=3)
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(state)
        a.step(6)
        want_u, want_w, want_clock = a.conserved(), a.primitive(), _clock(a)
        assert np.isfinite(W.interior(want_u)).all() and a.invalid() == 0
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(state)
        a.step(3)
        a.save_checkpoint(tmp_path / "run.ckpt")
        img = a.checkpoint()
    with CubedSphereAtmosphere.from_checkpoint(tmp_path / "run.ckpt") as b:
        b.step(3)
        assert np.array_equal(b.conserved(), want_u)
        assert np.array_equal(b.primitive(), want_w)
        assert _clock(b) == want_clock
    h = nat.checkpoint_header(img)
    assert h["magic"] == b"EXOCKPT1" and h["ncycle"] == 3 and h["cfg"]["N"] == cfg["N"]


@pytest.mark.parametrize("precision", [nat.EXO_PREC_FP64, nat.EXO_PREC_MIXED])
def test_checkpoint_moves_between_context_and_ensemble(precision):
    cfgs = [dict(W.hs94_config(N=8, L=20, cfl=0.4), precision=precision),
            dict(W.dry_atmosphere_config(N=10, L=8), precision=precision)]
    states = [W.hs94_state(cfgs[0], seed=1), W.dry_atmosphere_state(cfgs[1], seed=2)]
    # context -> ensemble: the member continues the context's run
    with CubedSphereAtmosphere(cfgs[0]) as a:
        a.set_primitive(states[0])
        a.step(2)
        img = a.checkpoint()
        a.step(3)
        want0 = a.conserved()
    with Ensemble(precision=precision, capacity=4) as e:
        other = e.add(cfgs[1], states[1])
        s0 = e.add_checkpoint(img)
        e.step(3)
        assert np.array_equal(e.conserved(s0), want0)
        # ensemble -> ensemble and ensemble -> context
        img1 = e.checkpoint(other)
        e.step(2)
        want1 = e.conserved(other)
    with Ensemble(precision=precision, capacity=2) as f:
        s1 = f.add_checkpoint(img1)
        f.step(2)
        assert np.array_equal(f.conserved(s1), want1)
    with CubedSphereAtmosphere.from_checkpoint(img1) as b:
        b.step(2)
        assert np.array_equal(b.conserved(), want1)


def test_resume_in_the_other_precision():
    cfg = W.dry_atmosphere_config(N=8, L=12)
    state = W.dry_atmosphere_state(cfg, seed=6)
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(state)
        a.step(2)
        img = a.checkpoint()
        a.step(2)
        want = W.interior(a.conserved())
    with CubedSphereAtmosphere.from_checkpoint(img, precision=nat.EXO_PREC_MIXED) as b:
        b.step(2)
        got = W.interior(b.conserved())
        assert b.invalid() == 0
    for n in (0, 4):
        rel = np.linalg.norm(got[:, n] - want[:, n]) / np.linalg.norm(want[:, n])
        assert 0 < rel < 1e-6, (n, rel)


def test_load_rejects_foreign_images():
    cfg = W.dry_atmosphere_config(N=8, L=12)
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(W.dry_atmosphere_state(cfg, seed=0))
        img = a.checkpoint()
        with CubedSphereAtmosphere(dict(cfg, N=10)) as other:
            with pytest.raises(nat.ExoError) as ei:
                other.restore(img)
            assert ei.value.code == nat.EXO_ERR_ARG
        bad = img.copy()
        bad[0] = ord("X")
        with pytest.raises(nat.ExoError):
            a.restore(bad)
        with pytest.raises(nat.ExoError):
            a.restore(img[:-8])
        with pytest.raises(nat.ExoError):
            a.restore(img[:100])
        # the context still runs after the refused loads
        a.step(1)
        assert a.invalid() == 0


def test_netcdf_output_of_a_run(tmp_path):
    from scipy.io import netcdf_file
    cfg = W.dry_atmosphere_config(N=8, L=12)
    with CubedSphereAtmosphere(cfg) as a:
        a.set_primitive(W.dry_atmosphere_state(cfg, seed=0))
        a.step(2)
        paths = a.write_netcdf("exo3", "out2", 1, directory=str(tmp_path))
        combined = a.write_netcdf("exo3", "out2", 2, directory=str(tmp_path), blocks=2,
                                  combine=True)
        w = a.primitive()
        t = a.time
    f = netcdf_file(paths[2], "r", mmap=False)
    assert np.array_equal(f.variables["press"][0],
                          W.interior(w)[2, 4].transpose(2, 1, 0).astype(np.float32))
    assert f.variables["time"][0] == np.float32(t)
    f.close()
    # 2 x 2 meshblocks per panel joined into one file of the 2 x 3 panel layout
    assert len(combined) == 1 and combined[0].endswith("exo3.out2.00002.nc")
    f = netcdf_file(combined[0], "r", mmap=False)
    press = f.variables["press"][0]
    assert press.shape == (12, 16, 24)
    wi = W.interior(w)
    for p in range(6):
        l2, l3 = p % 2, p // 2
        assert np.array_equal(press[:, 8 * l2:8 * l2 + 8, 8 * l3:8 * l3 + 8],
                              wi[p, 4].transpose(2, 1, 0).astype(np.float32))
    f.close()
