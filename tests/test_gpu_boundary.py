"""The boundary's panel-exchange, equation-of-state and array-view hooks
through the C ABI, against the oracle (which tests/test_ref_pinned.py holds
to the reference's own PackData, face-state exchange and solver code):

  exo_panel_pack              CubedSphereUtility::PackData         bitwise
  exo_save_lr3d / exo_synchronize_faces / exo_load_lr3d
                              CubedSphere::Save/LoadLR3DValues,
                              SynchronizeFluxes*                   bitwise
  exo_conserved_to_primitive / exo_primitive_to_conserved / exo_sound_speed
                              EquationOfState hooks               bitwise
  exo_*_views                 the whole-array entry points on strided
                              per-panel views (host and device)    bitwise
"""
import ctypes

import numpy as np
import pytest

from exocubed_b200 import _native as nat
from exocubed_b200 import workloads as W
from exocubed_b200.atmosphere import CubedSphereAtmosphere

pytestmark = pytest.mark.gpu
G = 3
SIDE_OX = {0: (-1, 0), 1: (1, 0), 2: (0, -1), 3: (0, 1)}


def _cfg(eqn, N=8, L=4):
    return W.dry_atmosphere_config(N=N, L=L) if eqn else dict(W.shallow_water_config(N=N))


def _random_conserved(shape, eqn, rng):
    nv, N, L = shape[1], shape[2] - 2 * G, shape[4] - 2 * G
    u = np.zeros(shape)
    sl = (slice(None), slice(G, G + N), slice(G, G + N), slice(G, G + L))
    for n in range(nv):
        u[:, n][sl] = rng.standard_normal((6, N, N, L)) * (10.0 ** n) + (5.0 if n == 0 else 0)
    if eqn:
        u[:, 4][sl] = 2.5e5 + 1e3 * rng.random((6, N, N, L))
    return u


@pytest.mark.parametrize("eqn,N", [(1, 8), (0, 8), (1, 12)])
def test_panel_pack_matches_the_oracle(oracle_mod, eqn, N):
    torch = pytest.importorskip("torch")
    cfg = _cfg(eqn, N)
    o = oracle_mod.Oracle(cfg)
    o.set_conserved(_random_conserved(o.shape, eqn, np.random.default_rng(N + eqn)))
    u = o.conserved()
    nv, nc3, nc2, nc1 = u.shape[1:]
    L = nc1 - 2 * G
    with CubedSphereAtmosphere(cfg) as a:
        h = a._ctx
        for p in range(6):
            src = torch.from_numpy(np.ascontiguousarray(u[p])).cuda()
            for s in range(4):
                ox2, ox3 = SIDE_OX[s]
                sj = G + N - G if ox2 > 0 else G
                ej = G + G - 1 if ox2 < 0 else G + N - 1
                sk = G + N - G if ox3 > 0 else G
                ek = G + G - 1 if ox3 < 0 else G + N - 1
                buf = torch.zeros(nv * nc3 * nc2 * nc1, dtype=torch.float64, device="cuda")
                off = ctypes.c_int(5)
                nat.check(nat.lib().exo_panel_pack(h, src.data_ptr(), buf.data_ptr(), 0, nv - 1,
                                                   G, G + L - 1, sj, ej, sk, ek,
                                                   ctypes.byref(off), 0, ox2, ox3, p, None))
                a.synchronize()
                want = o.pack_face(p, s)
                assert off.value == 5 + want.size
                got = buf.cpu().numpy()[5:5 + want.size]
                assert np.array_equal(got, want), (p, s)
            # a corner: PackDataR0, a plain copy of the range
            buf = torch.zeros(nv * nc3 * nc2 * nc1, dtype=torch.float64, device="cuda")
            off = ctypes.c_int(0)
            nat.check(nat.lib().exo_panel_pack(h, src.data_ptr(), buf.data_ptr(), 0, nv - 1, G,
                                               G + L - 1, G + N - G, G + N - 1, G + N - G,
                                               G + N - 1, ctypes.byref(off), 0, 1, 1, p, None))
            a.synchronize()
            ref = u[p][:, G + N - G:G + N, G + N - G:G + N, G:G + L].ravel()
            assert off.value == ref.size
            assert np.array_equal(buf.cpu().numpy()[:ref.size], ref)
        # a range that is not the edge band is refused
        with pytest.raises(nat.ExoError) as ei:
            nat.check(nat.lib().exo_panel_pack(h, src.data_ptr(), buf.data_ptr(), 0, nv - 1, G,
                                               G + L - 1, G, G + 1, G, G + N - 1,
                                               ctypes.byref(off), 0, -1, 0, 0, None))
        assert ei.value.code == nat.EXO_ERR_SHAPE


def test_face_state_exchange_matches_the_oracle(oracle_mod):
    N, L = 8, 4
    cfg = _cfg(1, N, L)
    o = oracle_mod.Oracle(cfg)
    rng = np.random.default_rng(11)
    arrs = [rng.standard_normal(o.shape) * 30 for _ in range(4)]
    want = o.exchange_faces(*arrs)
    nv, nc3, nc2, nc1 = o.shape[1:]
    got = [np.zeros(o.shape) for _ in range(4)]
    with CubedSphereAtmosphere(cfg) as a:
        h, lib = a._ctx, nat.lib()
        for d, (Lq, Rq) in ((2, (0, 1)), (3, (2, 3))):
            for p in range(6):
                for k in range(nc3):
                    for j in range(nc2):
                        lrow = np.ascontiguousarray(arrs[Lq][p, :, k, j, :])
                        rrow = np.ascontiguousarray(arrs[Rq][p, :, k, j, :])
                        nat.check(lib.exo_save_lr3d(h, lrow.ctypes.data, rrow.ctypes.data, d, p,
                                                    k, j, 0, nc1 - 1, None))
                        a.synchronize()
        nat.check(lib.exo_synchronize_faces(h, None))
        for d, (Lq, Rq) in ((2, (0, 1)), (3, (2, 3))):
            for p in range(6):
                for k in range(nc3):
                    for j in range(nc2):
                        lrow = np.zeros((nv, nc1))
                        rrow = np.zeros((nv, nc1))
                        nat.check(lib.exo_load_lr3d(h, lrow.ctypes.data, rrow.ctypes.data, d, p,
                                                    k, j, 0, nc1 - 1, None))
                        a.synchronize()
                        got[Lq][p, :, k, j, :] = lrow
                        got[Rq][p, :, k, j, :] = rrow
    for q in range(4):
        assert np.array_equal(got[q], want[q]), q
    assert not np.array_equal(want[0], arrs[0])


@pytest.mark.parametrize("eqn", [1, 0])
def test_equation_of_state_hooks_match_the_oracle(oracle_mod, eqn):
    torch = pytest.importorskip("torch")
    cfg = _cfg(eqn, 8, 4)
    o = oracle_mod.Oracle(cfg)
    state = (W.dry_atmosphere_state(cfg, seed=5) if eqn else W.shallow_water_state(cfg, seed=5))
    # fill the ghost bands and corners too: the hooks convert any range
    w = state.copy()
    rng = np.random.default_rng(3)
    ghost = w[:, 0] == 0
    w[:, 0][ghost] = (1.0 if eqn else 2.9e4) * (1 + 0.01 * rng.random(np.count_nonzero(ghost)))
    if eqn:
        w[:, 4][ghost] = 1e4 * (1 + rng.random(np.count_nonzero(ghost)))
    nc3, nc2, nc1 = w.shape[2:]
    full = (0, nc1 - 1, 0, nc2 - 1, 0, nc3 - 1)
    inner = (G, nc1 - G - 1, G, nc2 - G - 1, 1, nc3 - 2)
    with CubedSphereAtmosphere(cfg) as a:
        h, lib = a._ctx, nat.lib()
        for ranges in (full, inner):
            wd = torch.from_numpy(w).cuda()
            ud = torch.zeros_like(wd)
            nat.check(lib.exo_primitive_to_conserved(h, wd.data_ptr(), ud.data_ptr(), *ranges,
                                                     None))
            a.synchronize()
            u_ref, _ = o.eos(False, w, ranges)
            assert np.array_equal(ud.cpu().numpy(), u_ref)
            back = torch.zeros_like(wd)
            nat.check(lib.exo_conserved_to_primitive(h, ud.data_ptr(), back.data_ptr(), *ranges,
                                                     None))
            a.synchronize()
            w_ref, inv = o.eos(True, u_ref, ranges)
            assert np.array_equal(back.cpu().numpy(), w_ref) and inv == 0
            assert a.invalid() == 0
        # a negative density sets the sticky flag, as in the oracle
        u_bad = u_ref.copy()
        u_bad[2, 0, G + 1, G + 2, G + 1] = -1.0
        ub = torch.from_numpy(u_bad).cuda()
        back = torch.zeros_like(ub)
        nat.check(lib.exo_conserved_to_primitive(h, ub.data_ptr(), back.data_ptr(), *full, None))
        a.synchronize()
        _, inv = o.eos(True, u_bad, full)
        if eqn:
            assert inv == 1 and a.invalid() == 1
        # SoundSpeed of a row of cells
        n = 257
        prim = np.zeros((5, n))
        prim[0] = 1.0 + rng.random(n) if eqn else 2.9e4 * (1 + 0.05 * rng.random(n))
        prim[4] = 1e5 * (1 + rng.random(n))
        pd = torch.from_numpy(prim).cuda()
        cs = torch.zeros(n, dtype=torch.float64, device="cuda")
        nat.check(lib.exo_sound_speed(h, n, pd.data_ptr(), cs.data_ptr(), None))
        a.synchronize()
        want = np.array([o.sound_speed(prim[:, m]) for m in range(n)])
        assert np.array_equal(cs.cpu().numpy(), want)


def _strided_panels(w):
    """Six panel arrays of w (6, nv, nc3, nc2, nc1) as non-contiguous views:
    stored (nc1, nc2, nc3, nv) with padding, viewed back in (n, k, j, i) order."""
    out = []
    for p in range(6):
        store = np.full((w.shape[4] + 1, w.shape[3], w.shape[2], w.shape[1] + 2), np.nan)
        v = store[:-1, :, :, 1:-1].transpose(3, 2, 1, 0)
        v[...] = w[p]
        out.append(v)
    return out


def test_array_views_host_and_device(oracle_mod):
    torch = pytest.importorskip("torch")
    cfg = W.dry_atmosphere_config(N=8, L=6)
    state = W.dry_atmosphere_state(cfg, seed=2)
    lib = nat.lib()
    with CubedSphereAtmosphere(cfg) as ref:
        ref.set_primitive(state)
        u_ref, w_ref = ref.conserved(), ref.primitive()
        du = np.zeros_like(state)
        W.interior(du)[...] = 1e-5 * np.random.default_rng(1).standard_normal(
            W.interior(du).shape) * np.abs(W.interior(state)).mean(axis=(0, 2, 3, 4))[
                None, :, None, None, None]
        du_ref = du.copy()
        ref.solve_implicit_3d(du_ref, w_ref, 200.0)
    # host views, strided and permuted
    with CubedSphereAtmosphere(cfg) as a:
        h = a._ctx
        views = _strided_panels(state)
        nat.check(lib.exo_set_primitive_views(h, nat.views_of(views)))
        out = _strided_panels(np.zeros_like(state))
        nat.check(lib.exo_get_conserved_views(h, nat.views_of(out)))
        assert np.array_equal(np.stack([np.array(x) for x in out]), u_ref)
        out = _strided_panels(np.zeros_like(state))
        nat.check(lib.exo_get_primitive_views(h, nat.views_of(out)))
        assert np.array_equal(np.stack([np.array(x) for x in out]), w_ref)
        dv = _strided_panels(du)
        nat.check(lib.exo_solve_implicit_3d_views(h, nat.views_of(dv), nat.views_of(
            _strided_panels(w_ref)), 200.0))
        assert np.array_equal(np.stack([np.array(x) for x in dv]), du_ref)
    # device views: torch tensors stored (nc1, nc2, nc3, nv), permuted
    with CubedSphereAtmosphere(cfg) as a:
        h = a._ctx
        dev = [torch.from_numpy(np.ascontiguousarray(state[p].transpose(3, 2, 1, 0))).cuda()
               .permute(3, 2, 1, 0) for p in range(6)]
        trip = [(t.data_ptr(), tuple(t.shape), t.stride()) for t in dev]
        nat.check(lib.exo_set_primitive_views(h, nat.views_of(trip, device=0)))
        outs = [torch.zeros(state.shape[1:][::-1], dtype=torch.float64, device="cuda")
                .permute(3, 2, 1, 0) for _ in range(6)]
        trip = [(t.data_ptr(), tuple(t.shape), t.stride()) for t in outs]
        nat.check(lib.exo_get_conserved_views(h, nat.views_of(trip, device=0)))
        got = np.stack([t.cpu().numpy() for t in outs])
        assert np.array_equal(got, u_ref)
        # views of the wrong shape are refused
        bad = nat.views_of(_strided_panels(state))
        bad[3].nx1 = 5
        with pytest.raises(nat.ExoError) as ei:
            nat.check(lib.exo_set_primitive_views(h, bad))
        assert ei.value.code == nat.EXO_ERR_SHAPE
