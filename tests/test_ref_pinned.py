"""The oracle held to the reference's own code, bit for bit.

The reference cannot be built as a whole here (its Athena++ fork, MPI,
Eigen and NetCDF are missing), but its cubed-sphere and Riemann sources
compile unchanged against a few stand-in Athena++ headers
(oracle/ref/stubs, oracle/ref/Makefile -> oracle/_ref/libref_<solver>.so,
MPI replaced by an in-process message board).  These tests run the
reference's functions and the oracle's restatements on the same seeded
inputs and require identical bits:

  src/exo3/cubed_sphere_transform.cpp   VecTransABPFromRLL, VecTransRLLFromABP,
                                        RLLFromXYP
  src/exo3/cubed_sphere_utility.cpp     CalculateInterpLocations, PackData
                                        (InteprolateX2/X3, PackDataR0..R3)
  src/exo3/cs_find_block_id.cpp,        FindBlockID, TransformOX (the panel
  src/exo3/cs_transform_ox.cpp          connectivity tables)
  src/exo3/gnomonic_equiangle.cpp       areas, volumes, widths in the row
                                        forms the flux divergence and the
                                        time step call (with the
                                        constructor's metric tables) and,
                                        through the solvers, PrimToLocal2/3
                                        and FluxToGlobal2/3
  src/exo3/cubed_sphere.cpp             SaveLR3DValues, SynchronizeFluxes*,
                                        LoadLR3DValues (face-state exchange)
  src/snap/riemann/lmars.cpp, hllc_transform.cpp, roe_shallow_yz.cpp,
  lmars_shallow_yz.cpp                  Hydro::RiemannSolver rows
  src/snap/decomposition/change_to_perturbation.cpp, decomposition.cpp
                                        ChangeToPerturbation (hydrostatic face
                                        pressure, log-mean and isentropic
                                        reference state, bottom entropy) and
                                        RestoreFromPerturbation on one panel

The stand-ins supply no arithmetic of their own except the equation of
state's sound speed (ideal_moist_hydro.cpp with no vapour), which HLLC
calls, and the dry polytropic index 1 + (gamma - 1) feps / fsig of canoe's
Thermodynamics, which the decomposition reads.  Through these pins and the GPU parity tests, the CUDA path is held
to the same reference code.
"""
import numpy as np
import pytest

from exocubed_b200 import workloads as W
from oracle import oracle, reference

pytestmark = pytest.mark.skipif(not reference.available(),
                                reason="needs the reference checkout or oracle/_ref")
G = 3
UP, DOWN, LEFT, RIGHT = range(4)
SIDE_OX = {UP: (-1, 0), DOWN: (1, 0), LEFT: (0, -1), RIGHT: (0, 1)}


@pytest.fixture(scope="module")
def ref():
    oracle.lib()
    return reference.lib(1)


def test_vector_transforms_bitwise(ref):
    rng = np.random.default_rng(1)
    for _ in range(400):
        X, Y = np.tan(rng.uniform(-np.pi / 4, np.pi / 4, 2))
        U, V = 40 * rng.standard_normal(2)
        for b in range(1, 7):
            out = np.zeros(2)
            ref.ref_vec_abp_from_rll(X, Y, b, U, V, reference.ptr(out))
            assert np.array_equal(out, oracle.vec_abp_from_rll(X, Y, b, U, V))
            ref.ref_vec_rll_from_abp(X, Y, b, U, V, reference.ptr(out))
            assert np.array_equal(out, oracle.vec_rll_from_abp(X, Y, b, U, V))
        for nP in range(6):
            ref.ref_rll_from_xyp(X, Y, nP, reference.ptr(out))
            assert np.array_equal(out, oracle.rll_from_xyp(X, Y, nP))
    # the polar panels' special cases at the panel centre
    for nP in (0, 4):
        for dY in (-0.5, 0.0, 0.5):
            out = np.zeros(2)
            ref.ref_rll_from_xyp(0.0, dY, nP, reference.ptr(out))
            assert np.array_equal(out, oracle.rll_from_xyp(0.0, dY, nP))


@pytest.mark.parametrize("N_blk", [6, 8, 12, 48, 96])
def test_interp_locations_bitwise(ref, N_blk):
    for k in range(3):
        for loc_n in range(-N_blk // 2, N_blk // 2 + 1):
            for ghost in (0, 1):
                assert ref.ref_interp_loc(loc_n, N_blk, k, ghost) == \
                    oracle.interp_loc(loc_n, N_blk, k, ghost)


def test_panel_connectivity_matches_the_reference(ref):
    """FindBlockID and TransformOX against the oracle's tables (one block per
    panel: level 2, the 2 x 3 layout of panels)."""
    import ctypes
    nbr_panel, nbr_side, _, _, _ = oracle.panel_tables()
    for p in range(6):
        lx2, lx3 = p % 2, p // 2
        assert ref.ref_find_block_id(lx2, lx3, 2) == p + 1
        for s in range(4):
            ox2, ox3 = SIDE_OX[s]
            out = (ctypes.c_int * 4)()
            assert ref.ref_transform_ox(ox2, ox3, lx2, lx3, 2, out) == 0
            tox = (out[2], out[3])
            assert tox == SIDE_OX[int(nbr_side[p][s])], (p, s, tuple(out))
    # blocks of a panel split 2 x 2 (level 3) and 4 x 4 (level 4) keep its id
    for level, nb in ((3, 2), (4, 4)):
        for lx3 in range(3 * nb):
            for lx2 in range(2 * nb):
                assert ref.ref_find_block_id(lx2, lx3, level) == (lx3 // nb) * 2 + lx2 // nb + 1


def _random_conserved(o, rng):
    u = np.zeros(o.shape)
    c = o.cfg
    sl = (slice(None), slice(G, G + c.N), slice(G, G + c.N), slice(G, G + c.L))
    for n in range(o.nvar):
        u[:, n][sl] = rng.standard_normal((6, c.N, c.N, c.L)) * (10.0 ** n) + (5.0 if n == 0 else 0)
    if o.nvar == 5:
        u[:, 4][sl] = 2.5e5 + 1e3 * rng.random((6, c.N, c.N, c.L))
    return u


@pytest.mark.parametrize("eqn,N", [(1, 6), (1, 8), (0, 8), (1, 12)])
def test_pack_data_bitwise(ref, eqn, N):
    """CubedSphereUtility::PackData (interpolation along the panel edge, the
    vector rotation and the per-(panel, side) traversal order) against the
    oracle's ghost-exchange sender, for every panel and side."""
    cfg = (W.dry_atmosphere_config(N=N, L=4) if eqn else W.shallow_water_config(N=N))
    o = oracle.Oracle(cfg)
    rng = np.random.default_rng(N + eqn)
    o.set_conserved(_random_conserved(o, rng))
    u = o.conserved()
    nv, nc3, nc2, nc1 = u.shape[1:]
    L = cfg["L"]
    for p in range(6):
        lx2, lx3 = p % 2, p // 2
        src = np.ascontiguousarray(u[p])
        for s in range(4):
            ox2, ox3 = SIDE_OX[s]
            si, ei = G, G + L - 1
            sj = G + N - G if ox2 > 0 else G
            ej = G + G - 1 if ox2 < 0 else G + N - 1
            sk = G + N - G if ox3 > 0 else G
            ek = G + G - 1 if ox3 < 0 else G + N - 1
            buf = np.zeros(nv * nc3 * nc2 * nc1)
            n = ref.ref_pack_data(reference.ptr(src), nv, nc3, nc2, nc1, 0, nv - 1, si, ei, sj,
                                  ej, sk, ek, 0, ox2, ox3, lx2, lx3, 2, reference.ptr(buf))
            want = o.pack_face(p, s)
            assert n == want.size, (p, s, n, want.size)
            assert np.array_equal(buf[:n], want), (p, s, np.abs(buf[:n] - want).max())


def _sphere(o, rsolver, nbr_panel):
    c = o.cfg
    x1f = o.mesh(0)[0]
    x2 = np.stack([o.mesh(p)[1] for p in range(6)])
    x3 = np.stack([o.mesh(p)[2] for p in range(6)])
    return reference.Sphere(rsolver, c.N, c.L, c.gamma, x1f, o.dx1f(), x2, x3, nbr_panel)


def test_geometry_bitwise(ref):
    """GnomonicEquiangle's constructor tables, areas, volume and widths on the
    oracle's mesh, ghosts included."""
    cfg = W.dry_atmosphere_config(N=8, L=5)
    o = oracle.Oracle(cfg)
    sph = _sphere(o, 1, oracle.panel_tables()[0])
    for p in range(6):
        for k in range(0, 14, 3):
            for j in range(0, 14, 2):
                for i in (0, 2, 3, 5, 7, 10):
                    got = sph.cell_geometry(p, k, j, i)
                    assert np.array_equal(got[:7], o.cell_geometry_at(p, k, j, i)), (p, k, j, i)
                    # the point forms agree to rounding (another product order)
                    np.testing.assert_allclose(got[7:], got[:4], rtol=4e-16)
    sph.close()


def _rows(rng, eqn, nc1):
    wl = np.zeros((5, nc1))
    wr = np.zeros((5, nc1))
    for w in (wl, wr):
        if eqn == 0:
            w[0] = 2.9e4 * (1 + 0.05 * rng.standard_normal(nc1))
        else:
            w[0] = 1.0 + 0.1 * rng.random(nc1)
            w[4] = 1e5 * (1 + 0.1 * rng.random(nc1))
            w[1] = 20 * rng.standard_normal(nc1)
        w[2] = 30 * rng.standard_normal(nc1)
        w[3] = 30 * rng.standard_normal(nc1)
    return wl, wr


@pytest.mark.parametrize("rsolver,eqn", [(1, 1), (2, 1), (0, 0), (3, 0)])
def test_riemann_rows_bitwise(ref, rsolver, eqn):
    """Hydro::RiemannSolver of each solver file on rows of faces, with the
    real gnomonic projections (PrimToLocal2/3, FluxToGlobal2/3) and the
    covariant flux projection, against the oracle's solver on the face
    geometry of the same rows."""
    N, L = 8, 6
    cfg = (W.dry_atmosphere_config(N=N, L=L, rsolver=rsolver) if eqn
           else W.shallow_water_config(N=N, rsolver=rsolver))
    cfg["L"] = L
    o = oracle.Oracle(cfg)
    sph = _sphere(o, rsolver, oracle.panel_tables()[0])
    nv = 5 if eqn else 4
    nc1 = L + 2 * G
    rng = np.random.default_rng(7 + rsolver)
    # x1 faces of the shallow-water solvers project with an angle the
    # reference never sets (roe_shallow_yz.cpp:96-121); the flux there is dead
    dirs = (1, 2, 3) if eqn else (2, 3)
    for p in (0, 2, 4, 5):
        for (k, j) in ((G, G), (G + 2, G + 5), (G + N - 1, G + N), (G + N, G + 1)):
            for ivx in dirs:
                wl, wr = _rows(rng, eqn, nc1)
                got = sph.riemann(p, k, j, ivx, G, G + L - 1, wl.copy(), wr.copy())
                fg = o.face_geo(p, k, j, ivx)
                for i in range(G, G + L):
                    want = oracle.riemann_face(rsolver, eqn, ivx, cfg["gamma"], wl[:, i],
                                               wr[:, i], *fg)
                    assert np.array_equal(got[:nv, i], want[:nv]), (p, k, j, ivx, i)
    sph.close()


def test_face_state_exchange_bitwise(ref):
    """CubedSphere::SaveLR3DValues -> SynchronizeFluxesSend/Recv/Wait ->
    LoadLR3DValues over the six panels (MPI replaced by the in-process board)
    against the oracle's exchange of panel-edge face states."""
    N, L = 8, 4
    cfg = W.dry_atmosphere_config(N=N, L=L)
    o = oracle.Oracle(cfg)
    sph = _sphere(o, 1, oracle.panel_tables()[0])
    rng = np.random.default_rng(3)
    arrs = [rng.standard_normal(o.shape) * 30 for _ in range(4)]
    want = o.exchange_faces(*arrs)   # L2, R2, L3, R3 after the exchange
    Lr = np.ascontiguousarray(np.stack([arrs[0], arrs[2]], axis=1))  # (6, 2, 5, ...)
    Rr = np.ascontiguousarray(np.stack([arrs[1], arrs[3]], axis=1))
    sph.face_sync(Lr, Rr)
    assert np.array_equal(Lr[:, 0], want[0])
    assert np.array_equal(Rr[:, 0], want[1])
    assert np.array_equal(Lr[:, 1], want[2])
    assert np.array_equal(Rr[:, 1], want[3])
    # the exchange changed something (the edges were overwritten)
    assert not np.array_equal(want[0], arrs[0])
    sph.close()


@pytest.mark.parametrize("rsolver,seed", [(1, 4), (2, 9)])
def test_decomposition_bitwise(ref, rsolver, seed):
    """ChangeToPerturbation and RestoreFromPerturbation of the reference
    (one panel, reflecting radial boundaries, no vertical neighbours) against
    the oracle's, panel by panel, on a seeded dry state."""
    N, L = 8, 10
    cfg = W.dry_atmosphere_config(N=N, L=L, rsolver=rsolver)
    o = oracle.Oracle(cfg)
    o.set_primitive(W.dry_atmosphere_state(cfg, seed=seed, geometry=oracle.cell_geometry))
    w0 = o.primitive()
    w_ora = w0.copy()
    o.change_to_perturbation(w_ora)
    rng = np.random.default_rng(seed)
    wl = w_ora.copy() + rng.standard_normal(w_ora.shape) * 1e-3
    wr = w_ora.copy() + rng.standard_normal(w_ora.shape) * 1e-3
    wl_ora, wr_ora, w_back = wl.copy(), wr.copy(), w_ora.copy()
    o.restore_from_perturbation(w_back, wl_ora, wr_ora)
    x1f = o.mesh(0)[0]
    for p in range(6):
        _, x2f, x3f = o.mesh(p)
        pan = reference.DecomposedPanel(N, L, cfg["gamma"], cfg["Rd"], cfg["grav"],
                                        x1f, o.dx1f(), x2f, x3f)
        wp = np.ascontiguousarray(w0[p])
        pan.change_to_perturbation(wp)
        inner = (slice(None), slice(G, G + N), slice(G, G + N), slice(None))
        assert np.array_equal(wp[inner], w_ora[p][inner]), p
        for k in range(G, G + N):
            for j in range(G, G + N):
                lrow = np.ascontiguousarray(wl[p, :, k, j, :])
                rrow = np.ascontiguousarray(wr[p, :, k, j, :])
                pan.restore_from_perturbation(wp, lrow, rrow, k, j, G, G + L)
                assert np.array_equal(lrow[:, G:G + L + 1], wl_ora[p, :, k, j, G:G + L + 1])
                assert np.array_equal(rrow[:, G:G + L + 1], wr_ora[p, :, k, j, G:G + L + 1])
        assert np.array_equal(wp[inner], w_back[p][inner]), p
        pan.close()


def _unpack(buf, order, nv, K, J, I):
    """The inverse of PackDataR0..R3 (oracle pack_order): the (n, k, j, i)
    array a packed buffer was traversed from."""
    if order in (0, 2):
        a = buf.reshape(nv, K, J, I)
        return a if order == 0 else a[:, ::-1, ::-1, :]
    b = buf.reshape(nv, J, K, I).transpose(0, 2, 1, 3)
    return b[:, :, ::-1, :] if order == 1 else b[:, ::-1, :, :]


def _pack(a, order):
    if order == 0:
        return a.ravel()
    if order == 2:
        return a[:, ::-1, ::-1, :].ravel()
    if order == 1:
        return a[:, :, ::-1, :].transpose(0, 2, 1, 3).ravel()
    return a[:, ::-1, :, :].transpose(0, 2, 1, 3).ravel()


@pytest.mark.parametrize("N,nb", [(16, 2), (32, 4)])
def test_multiblock_pack_data_equals_one_block_per_panel(ref, N, nb):
    """Multi-block panels: with nb x nb blocks per panel, the
    reference's own PackData (cubed_sphere_utility.cpp:92-369: N_blk the whole
    panel edge, n_start the block's offset along it) sends, from every block
    on a panel edge, exactly the slice of what one block per panel sends,
    bit for bit, once the block's ghost cells along the edge hold the
    neighbouring blocks' current values (the reference's second ghost pass).
    So a run with blocks per panel gives the one-block-per-panel result, and
    the one-block layout stands in for it.  Blocks are 8 cells wide here: the
    reference tells a block's low-side band from its high-side band by
    comparing the band's start with the other direction's end less NGHOST
    (`sk < ej - NGHOST` in InteprolateX2), which for blocks of G + 1 = 4
    cells or fewer treats a low-side band as a high-side one and reverses
    its rows (a block-size limit of the reference, not of this layout)."""
    L = 4
    n = N // nb
    level = 2 + int(np.log2(nb))
    cfg = W.dry_atmosphere_config(N=N, L=L)
    o = oracle.Oracle(cfg)
    rng = np.random.default_rng(17 + nb)
    o.set_conserved(_random_conserved(o, rng))
    u = o.conserved()
    nv, nc1 = u.shape[1], u.shape[4]
    pack = oracle.panel_tables()[4]
    for p in range(6):
        for s in range(4):
            ox2, ox3 = SIDE_OX[s]
            order = int(pack[p][s])
            K1, J1 = (N, G) if ox2 else (G, N)
            whole = _unpack(o.pack_face(p, s), order, nv, K1, J1, L)
            for b in range(nb):
                bx = (0 if ox2 < 0 else nb - 1) if ox2 else b
                by = (0 if ox3 < 0 else nb - 1) if ox3 else b
                blk = np.ascontiguousarray(u[p][:, by * n:by * n + n + 2 * G,
                                                 bx * n:bx * n + n + 2 * G, :])
                sj = G + n - G if ox2 > 0 else G
                ej = G + G - 1 if ox2 < 0 else G + n - 1
                sk = G + n - G if ox3 > 0 else G
                ek = G + G - 1 if ox3 < 0 else G + n - 1
                buf = np.zeros(blk.size)
                cnt = ref.ref_pack_data(reference.ptr(blk), nv, n + 2 * G, n + 2 * G, nc1, 0,
                                        nv - 1, G, G + L - 1, sj, ej, sk, ek, 0, ox2, ox3,
                                        (p % 2) * nb + bx, (p // 2) * nb + by, level,
                                        reference.ptr(buf))
                part = whole[:, b * n:(b + 1) * n] if ox2 else whole[:, :, b * n:(b + 1) * n]
                want = _pack(np.ascontiguousarray(part), order)
                assert cnt == want.size, (p, s, b, cnt, want.size)
                assert np.array_equal(buf[:cnt], want), (p, s, b, np.abs(buf[:cnt] - want).max())
