// harness.cpp -- drives the reference's own exo3 and Riemann sources,
// compiled unchanged against the stand-in headers of oracle/ref/stubs, so
// that the oracle (oracle/exo_oracle.cpp) can be checked against code the
// reference itself ships.  Test infrastructure only: tests/ loads the
// resulting oracle/_ref/libref_<solver>.so; the product never does.
//
// Compiled into one library per Riemann solver (each of
// src/snap/riemann/{lmars,hllc_transform,roe_shallow_yz,lmars_shallow_yz}.cpp
// defines Hydro::RiemannSolver), together with src/exo3/
// {gnomonic_equiangle,cubed_sphere,cubed_sphere_utility,
// cubed_sphere_transform,cs_transform_ox,cs_find_block_id}.cpp.
#include <athena/athena.hpp>
#include <athena/bvals/bvals.hpp>
#include <athena/coordinates/coordinates.hpp>
#include <athena/eos/eos.hpp>
#include <athena/hydro/hydro.hpp>
#include <athena/mesh/mesh.hpp>
#include <exo3/cubed_sphere.hpp>
#include <exo3/cubed_sphere_utility.hpp>
#include <exo3/gnomonic_equiangle.hpp>

#include <memory>
#include <vector>

namespace CubedSphereUtility {
// defined in cubed_sphere_utility.cpp, not declared in its header
Real CalculateInterpLocations(int loc_n, int N_blk, int k, bool GhostZone);
}  // namespace CubedSphereUtility

// The Coordinates stand-in's constructor: index ranges and sizes from the
// MeshBlock, faces and radial widths from the mesh the harness was given.
Coordinates::Coordinates(MeshBlock* pmb, ParameterInput*, bool) : pmy_block(pmb) {
  il = pmb->is; iu = pmb->ie;
  jl = pmb->js; ju = pmb->je;
  kl = pmb->ks; ku = pmb->ke;
  ng = pmb->is;
  nc1 = pmb->ncells1; nc2 = pmb->ncells2; nc3 = pmb->ncells3;
  x1f.NewAthenaArray(nc1 + 1); x2f.NewAthenaArray(nc2 + 1); x3f.NewAthenaArray(nc3 + 1);
  dx1f.NewAthenaArray(nc1); dx2f.NewAthenaArray(nc2); dx3f.NewAthenaArray(nc3);
  x1v.NewAthenaArray(nc1); x2v.NewAthenaArray(nc2); x3v.NewAthenaArray(nc3);
  dx1v.NewAthenaArray(nc1); dx2v.NewAthenaArray(nc2); dx3v.NewAthenaArray(nc3);
  x1s2.NewAthenaArray(nc1); x1s3.NewAthenaArray(nc1);
  x2s1.NewAthenaArray(nc2); x2s3.NewAthenaArray(nc2);
  x3s1.NewAthenaArray(nc3); x3s2.NewAthenaArray(nc3);
  for (auto* a : {&h2f, &dh2fd1, &h31f, &dh31fd1, &h2v, &dh2vd1, &h31v, &dh31vd1})
    a->NewAthenaArray(nc1);
  for (auto* a : {&h32f, &dh32fd2, &h32v, &dh32vd2}) a->NewAthenaArray(nc2);
  for (int i = 0; i <= nc1; ++i) x1f(i) = pmb->mesh_x1f[i];
  for (int j = 0; j <= nc2; ++j) x2f(j) = pmb->mesh_x2f[j];
  for (int k = 0; k <= nc3; ++k) x3f(k) = pmb->mesh_x3f[k];
  for (int i = 0; i < nc1; ++i) dx1f(i) = pmb->mesh_dx1f[i];
  for (int j = 0; j < nc2; ++j) dx2f(j) = x2f(j + 1) - x2f(j);
  for (int k = 0; k < nc3; ++k) dx3f(k) = x3f(k + 1) - x3f(k);
}

namespace {

// Six panels of nb x nb blocks each, every block a MeshBlock with the
// reference's GnomonicEquiangle, CubedSphere and Hydro objects.
struct Sphere {
  int N, L, nb, level;
  Mesh mesh;
  EquationOfState eos;
  std::vector<std::unique_ptr<MeshBlock>> blocks;
  std::vector<std::unique_ptr<MeshBlock::Impl>> impls;
  std::vector<std::unique_ptr<BoundaryValues>> bvals;
  std::vector<std::unique_ptr<Hydro>> hydros;
  std::vector<std::vector<Real>> meshes;  // x1f, x2f, x3f, dx1f per block
};

int log2i(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return l;
}

// gid of the block at (lx2, lx3) of the 2 x 3 layout of panels, each split
// into nb x nb blocks: Athena++'s Z-order is not needed, any fixed numbering
// that both sides of an exchange agree on is
int gid_of(int lx2, int lx3, int nb) { return lx3 * 2 * nb + lx2; }

}  // namespace

extern "C" {

void ref_vec_abp_from_rll(double X, double Y, int blockID, double U, double V, double* out) {
  CubedSphereUtility::VecTransABPFromRLL(X, Y, blockID, U, V, &out[0], &out[1]);
}
void ref_vec_rll_from_abp(double X, double Y, int blockID, double V2, double V3, double* out) {
  CubedSphereUtility::VecTransRLLFromABP(X, Y, blockID, V2, V3, &out[0], &out[1]);
}
void ref_rll_from_xyp(double dX, double dY, int nP, double* out) {
  CubedSphereUtility::RLLFromXYP(dX, dY, nP, out[0], out[1]);
}
double ref_interp_loc(int loc_n, int N_blk, int k, int ghost) {
  return CubedSphereUtility::CalculateInterpLocations(loc_n, N_blk, k, ghost != 0);
}

// CubedSphere::FindBlockID; -1 where the reference raises its error
int ref_find_block_id(int lx2, int lx3, int level) {
  LogicalLocation loc;
  loc.lx2 = lx2; loc.lx3 = lx3; loc.level = level;
  try {
    return CubedSphere::FindBlockID(loc);
  } catch (...) {
    return -1;
  }
}

// CubedSphere::TransformOX: out = (ox2, ox3, tox2, tox3) after the call;
// returns -1 where the reference raises its error
int ref_transform_ox(int ox2, int ox3, int lx2, int lx3, int level, int* out) {
  LogicalLocation loc;
  loc.lx2 = lx2; loc.lx3 = lx3; loc.level = level;
  int tox2 = 0, tox3 = 0;
  try {
    CubedSphere::TransformOX(&ox2, &ox3, &tox2, &tox3, loc);
  } catch (...) {
    return -1;
  }
  out[0] = ox2; out[1] = ox3; out[2] = tox2; out[3] = tox3;
  return 0;
}

// CubedSphereUtility::PackData on src (nv, nc3, nc2, nc1); returns the
// number of values written to buf, -1 on an error raised by the reference
int ref_pack_data(const double* src, int nv, int nc3, int nc2, int nc1, int sn, int en, int si,
                  int ei, int sj, int ej, int sk, int ek, int ox1, int ox2, int ox3, int lx2,
                  int lx3, int level, double* buf) {
  AthenaArray<Real> a;
  a.Wrap(const_cast<double*>(src), nv, nc3, nc2, nc1);
  LogicalLocation loc;
  loc.lx2 = lx2; loc.lx3 = lx3; loc.level = level;
  int offset = 0;
  try {
    CubedSphereUtility::PackData(a, buf, sn, en, si, ei, sj, ej, sk, ek, offset, ox1, ox2, ox3,
                                 loc);
  } catch (...) {
    return -1;
  }
  return offset;
}

// Six panels of nb x nb blocks of (N/nb)^2 x L cells; per block (panel-major,
// then lx3, then lx2 inside the panel) its x2f and x3f (N/nb + 7 values each);
// x1f (L + 7) and dx1f (L + 6) are shared.
void* ref_sphere_create(int N, int L, int nb, double gamma, const double* x1f,
                        const double* dx1f, const double* x2f_blocks,
                        const double* x3f_blocks) {
  if (nb < 1 || N % nb) return nullptr;
  auto* s = new Sphere();
  s->N = N; s->L = L; s->nb = nb;
  s->level = 2 + log2i(nb);
  s->eos.gamma = gamma;
  const int n = N / nb, G = 3;
  int b = 0;
  for (int p = 0; p < 6; ++p)
    for (int by = 0; by < nb; ++by)
      for (int bx = 0; bx < nb; ++bx, ++b) {
        auto mb = std::make_unique<MeshBlock>();
        int lx2 = (p % 2) * nb + bx, lx3 = (p / 2) * nb + by;
        mb->loc.lx2 = lx2; mb->loc.lx3 = lx3; mb->loc.level = s->level;
        mb->gid = gid_of(lx2, lx3, nb);
        mb->pmy_mesh = &s->mesh;
        mb->block_size.nx1 = L; mb->block_size.nx2 = n; mb->block_size.nx3 = n;
        mb->is = G; mb->ie = G + L - 1;
        mb->js = G; mb->je = G + n - 1;
        mb->ks = G; mb->ke = G + n - 1;
        mb->ncells1 = L + 2 * G; mb->ncells2 = n + 2 * G; mb->ncells3 = n + 2 * G;
        std::vector<Real> m;
        m.insert(m.end(), x1f, x1f + L + 2 * G + 1);
        m.insert(m.end(), dx1f, dx1f + L + 2 * G);
        m.insert(m.end(), x2f_blocks + (size_t)b * (n + 2 * G + 1),
                 x2f_blocks + (size_t)(b + 1) * (n + 2 * G + 1));
        m.insert(m.end(), x3f_blocks + (size_t)b * (n + 2 * G + 1),
                 x3f_blocks + (size_t)(b + 1) * (n + 2 * G + 1));
        s->meshes.push_back(std::move(m));
        const std::vector<Real>& mm = s->meshes.back();
        mb->mesh_x1f = mm.data();
        mb->mesh_dx1f = mm.data() + (L + 2 * G + 1);
        mb->mesh_x2f = mm.data() + (L + 2 * G + 1) + (L + 2 * G);
        mb->mesh_x3f = mb->mesh_x2f + (n + 2 * G + 1);
        mb->peos = &s->eos;
        s->impls.push_back(std::make_unique<MeshBlock::Impl>());
        mb->pimpl = s->impls.back().get();
        s->bvals.push_back(std::make_unique<BoundaryValues>());
        mb->pbval = s->bvals.back().get();
        s->hydros.push_back(std::make_unique<Hydro>());
        mb->phydro = s->hydros.back().get();
        mb->phydro->pmy_block = mb.get();
        s->blocks.push_back(std::move(mb));
      }
  // geometry and cubed-sphere objects once every block exists
  for (auto& mb : s->blocks) {
    mb->pcoord = new GnomonicEquiangle(mb.get(), nullptr, false);
    mb->pimpl->pexo3 = new CubedSphere(mb.get());
  }
  // the four face neighbours of every block: the logical neighbour inside
  // the 2 x 3 layout or, across a panel edge, the block TransformOX's
  // target side names (found by matching the return exchange)
  for (auto& mb : s->blocks) {
    BoundaryValues& bv = *mb->pbval;
    bv.nneighbor = 0;
    const int dirs[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};  // (ox2, ox3)
    for (auto& d : dirs) {
      NeighborBlock& nbk = bv.neighbor[bv.nneighbor++];
      nbk.ni.ox1 = 0; nbk.ni.ox2 = d[0]; nbk.ni.ox3 = d[1];
      nbk.snb.rank = 0; nbk.snb.level = s->level;
      nbk.snb.gid = -1;
    }
  }
  return s;
}

void ref_sphere_destroy(void* h) {
  auto* s = static_cast<Sphere*>(h);
  if (!s) return;
  for (auto& mb : s->blocks) {
    delete mb->pimpl->pexo3;
    delete mb->pcoord;
  }
  delete s;
}

// set the gid of neighbour slot `slot` (0: ox2 = -1, 1: ox2 = +1, 2: ox3 = -1,
// 3: ox3 = +1) of block b
void ref_sphere_set_neighbor(void* h, int b, int slot, int gid) {
  static_cast<Sphere*>(h)->blocks[b]->pbval->neighbor[slot].snb.gid = gid;
}
int ref_sphere_gid(void* h, int b) { return static_cast<Sphere*>(h)->blocks[b]->gid; }

// The row forms the flux divergence and the time step call (Face1Area,
// Face2Area, Face3Area, CellVolume, CenterWidth1/2/3) at cell (k, j, i) of
// block b; out[7..10] = the point forms GetFace1Area, GetFace2Area,
// GetFace3Area, GetCellVolume (which multiply in another order)
void ref_cell_geometry(void* h, int b, int k, int j, int i, double* out) {
  MeshBlock* mb = static_cast<Sphere*>(h)->blocks[b].get();
  Coordinates* c = mb->pcoord;
  AthenaArray<Real> w;
  w.NewAthenaArray(mb->ncells1 + 1);
  c->Face1Area(k, j, i, i, w);
  out[0] = w(i);
  c->Face2Area(k, j, i, i, w);
  out[1] = w(i);
  c->Face3Area(k, j, i, i, w);
  out[2] = w(i);
  c->CellVolume(k, j, i, i, w);
  out[3] = w(i);
  out[7] = c->GetFace1Area(k, j, i);
  out[8] = c->GetFace2Area(k, j, i);
  out[9] = c->GetFace3Area(k, j, i);
  out[10] = c->GetCellVolume(k, j, i);
  c->CenterWidth1(k, j, i, i, w);
  out[4] = w(i);
  c->CenterWidth2(k, j, i, i, w);
  out[5] = w(i);
  c->CenterWidth3(k, j, i, i, w);
  out[6] = w(i);
}

// Hydro::RiemannSolver of this library's solver on faces il..iu of row
// (k, j) of block b in direction ivx: wl, wr (NWAVE x ncells1, modified in
// place as the reference does), flx (NHYDRO x ncells1) receives the row
void ref_riemann(void* h, int b, int k, int j, int ivx, int il, int iu, double* wl, double* wr,
                 double* flx) {
  MeshBlock* mb = static_cast<Sphere*>(h)->blocks[b].get();
  const int nc1 = mb->ncells1, nc2 = mb->ncells2, nc3 = mb->ncells3;
  AthenaArray<Real> awl, awr, af, dxw;
  awl.Wrap(wl, 1, 1, NWAVE, nc1);
  awr.Wrap(wr, 1, 1, NWAVE, nc1);
  af.NewAthenaArray(NHYDRO, nc3, nc2, nc1);
  dxw.NewAthenaArray(nc1);
  mb->phydro->RiemannSolver(k, j, il, iu, ivx, awl, awr, af, dxw);
  for (int n = 0; n < NHYDRO; ++n)
    for (int i = 0; i < nc1; ++i) flx[(size_t)n * nc1 + i] = af(n, k, j, i);
}

// The panel-edge face-state exchange (SaveLR3DValues on every row,
// SynchronizeFluxesSend/Recv/Wait on every block, LoadLR3DValues): L and R
// hold, per block, dir (0: x2, 1: x3), NWAVE x nc3 x nc2 x nc1 face states
// in and out.
int ref_sphere_face_sync(void* h, double* L, double* R) {
  auto* s = static_cast<Sphere*>(h);
  const int nblk = (int)s->blocks.size();
  auto slab = [&](double* a, int b, int d) -> double* {
    MeshBlock* mb = s->blocks[b].get();
    size_t n = (size_t)NWAVE * mb->ncells3 * mb->ncells2 * mb->ncells1;
    return a + ((size_t)b * 2 + d) * n;
  };
  try {
    for (int b = 0; b < nblk; ++b) {
      MeshBlock* mb = s->blocks[b].get();
      const int nc1 = mb->ncells1, nc2 = mb->ncells2, nc3 = mb->ncells3;
      for (int d = 0; d < 2; ++d) {
        AthenaArray<Real> l4, r4;
        l4.Wrap(slab(L, b, d), NWAVE, nc3, nc2, nc1);
        r4.Wrap(slab(R, b, d), NWAVE, nc3, nc2, nc1);
        AthenaArray<Real> lrow, rrow;
        lrow.NewAthenaArray(NWAVE, nc1);
        rrow.NewAthenaArray(NWAVE, nc1);
        for (int k = 0; k < nc3; ++k)
          for (int j = 0; j < nc2; ++j) {
            for (int n = 0; n < NWAVE; ++n)
              for (int i = 0; i < nc1; ++i) {
                lrow(n, i) = l4(n, k, j, i);
                rrow(n, i) = r4(n, k, j, i);
              }
            mb->pimpl->pexo3->SaveLR3DValues(lrow, rrow, d + 1, k, j, 0, nc1 - 1);
          }
      }
    }
    for (int b = 0; b < nblk; ++b) s->blocks[b]->pimpl->pexo3->SynchronizeFluxesSend();
    for (int b = 0; b < nblk; ++b) s->blocks[b]->pimpl->pexo3->SynchronizeFluxesRecv();
    for (int b = 0; b < nblk; ++b) s->blocks[b]->pimpl->pexo3->SynchronizeFluxesWait();
    if (!mpi_inproc_board().empty()) return -2;  // a message nobody received
    for (int b = 0; b < nblk; ++b) {
      MeshBlock* mb = s->blocks[b].get();
      const int nc1 = mb->ncells1, nc2 = mb->ncells2, nc3 = mb->ncells3;
      for (int d = 0; d < 2; ++d) {
        AthenaArray<Real> l4, r4;
        l4.Wrap(slab(L, b, d), NWAVE, nc3, nc2, nc1);
        r4.Wrap(slab(R, b, d), NWAVE, nc3, nc2, nc1);
        AthenaArray<Real> lrow, rrow;
        lrow.NewAthenaArray(NWAVE, nc1);
        rrow.NewAthenaArray(NWAVE, nc1);
        for (int k = 0; k < nc3; ++k)
          for (int j = 0; j < nc2; ++j) {
            mb->pimpl->pexo3->LoadLR3DValues(lrow, rrow, d + 1, k, j, 0, nc1 - 1);
            for (int n = 0; n < NWAVE; ++n)
              for (int i = 0; i < nc1; ++i) {
                l4(n, k, j, i) = lrow(n, i);
                r4(n, k, j, i) = rrow(n, i);
              }
          }
      }
    }
  } catch (...) {
    mpi_inproc_board().clear();
    return -1;
  }
  return 0;
}

}  // extern "C"
