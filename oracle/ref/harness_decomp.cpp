// harness_decomp.cpp -- drives the reference's own hydrostatic decomposition
// (src/snap/decomposition/change_to_perturbation.cpp and decomposition.cpp),
// compiled unchanged against the stand-in headers of oracle/ref/stubs, on
// one panel at a time (one MeshBlock, no vertical neighbours, reflecting
// radial boundaries).  Test infrastructure only: tests/test_ref_pinned.py
// holds the oracle's decomposition to it.
#include <athena/athena.hpp>
#include <athena/coordinates/coordinates.hpp>
#include <athena/hydro/hydro.hpp>
#include <athena/mesh/mesh.hpp>
#include <exo3/gnomonic_equiangle.hpp>
#include <snap/decomposition/decomposition.hpp>
#include <snap/thermodynamics/thermodynamics.hpp>

#include <memory>
#include <vector>

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

struct Panel {
  Mesh mesh;
  MeshBlock mb;
  MeshBlock::Impl impl;
  BoundaryValues bval;
  Hydro hydro;
  std::vector<Real> x1f, dx1f, x2f, x3f;
  std::unique_ptr<GnomonicEquiangle> coord;
};

}  // namespace

extern "C" {

// One panel of N x N x L cells with the given mesh, gamma and x1 gravity
void* ref_decomp_create(int N, int L, double gamma, double Rd, double grav, const double* x1f,
                        const double* dx1f, const double* x2f, const double* x3f) {
  const int G = 3;
  auto* s = new Panel();
  Thermodynamics::GetInstance()->gammad = gamma;
  Thermodynamics::GetInstance()->Rd = Rd;
  MeshBlock& mb = s->mb;
  mb.loc.lx2 = 0; mb.loc.lx3 = 0; mb.loc.level = 2;
  mb.pmy_mesh = &s->mesh;
  mb.block_size.nx1 = L; mb.block_size.nx2 = N; mb.block_size.nx3 = N;
  mb.is = G; mb.ie = G + L - 1;
  mb.js = G; mb.je = G + N - 1;
  mb.ks = G; mb.ke = G + N - 1;
  mb.ncells1 = L + 2 * G; mb.ncells2 = N + 2 * G; mb.ncells3 = N + 2 * G;
  s->x1f.assign(x1f, x1f + L + 2 * G + 1);
  s->dx1f.assign(dx1f, dx1f + L + 2 * G);
  s->x2f.assign(x2f, x2f + N + 2 * G + 1);
  s->x3f.assign(x3f, x3f + N + 2 * G + 1);
  mb.mesh_x1f = s->x1f.data();
  mb.mesh_dx1f = s->dx1f.data();
  mb.mesh_x2f = s->x2f.data();
  mb.mesh_x3f = s->x3f.data();
  mb.pimpl = &s->impl;
  mb.pbval = &s->bval;
  s->hydro.pmy_block = &mb;
  s->hydro.hsrc.g1 = grav;
  mb.phydro = &s->hydro;
  s->coord.reset(new GnomonicEquiangle(&mb, nullptr, false));
  mb.pcoord = s->coord.get();
  s->impl.pdec = std::make_shared<Decomposition>(&mb);
  return s;
}

void ref_decomp_destroy(void* h) { delete static_cast<Panel*>(h); }

// Decomposition::ChangeToPerturbation on the interior columns of one
// panel's primitives w (NHYDRO, N+6, N+6, L+6), in place
void ref_change_to_perturbation(void* h, double* w) {
  auto* s = static_cast<Panel*>(h);
  MeshBlock& mb = s->mb;
  AthenaArray<Real> a;
  a.Wrap(w, NHYDRO, mb.ncells3, mb.ncells2, mb.ncells1);
  s->impl.pdec->ChangeToPerturbation(a, mb.ks, mb.ke, mb.js, mb.je);
}

// Decomposition::RestoreFromPerturbation of row (k, j): w (whole panel) and
// the x1 face states wl, wr (NHYDRO, L+6) of that row, faces il..iu
void ref_restore_from_perturbation(void* h, double* w, double* wl, double* wr, int k, int j,
                                   int il, int iu) {
  auto* s = static_cast<Panel*>(h);
  MeshBlock& mb = s->mb;
  AthenaArray<Real> a, l, r;
  a.Wrap(w, NHYDRO, mb.ncells3, mb.ncells2, mb.ncells1);
  l.Wrap(wl, 1, 1, NHYDRO, mb.ncells1);
  r.Wrap(wr, 1, 1, NHYDRO, mb.ncells1);
  s->impl.pdec->RestoreFromPerturbation(a, l, r, k, j, il, iu);
}

}  // extern "C"
