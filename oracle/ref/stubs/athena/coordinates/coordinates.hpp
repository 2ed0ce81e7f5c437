// Harness stand-in for Athena++'s Coordinates base class: the members and
// virtual interface the reference's GnomonicEquiangle (src/exo3/
// gnomonic_equiangle.hpp) overrides, and a constructor that takes the mesh
// (face positions of the three directions and the radial widths) from the
// MeshBlock instead of Athena++'s mesh generator.  Test infrastructure only.
#ifndef REF_STUB_COORDINATES_HPP_
#define REF_STUB_COORDINATES_HPP_

#include "../athena.hpp"
#include "../mesh/mesh.hpp"

class Coordinates {
 public:
  Coordinates(MeshBlock* pmb, ParameterInput* pin, bool flag = false);
  virtual ~Coordinates() = default;

  MeshBlock* pmy_block;
  AthenaArray<Real> dx1f, dx2f, dx3f, x1f, x2f, x3f;
  AthenaArray<Real> dx1v, dx2v, dx3v, x1v, x2v, x3v;
  AthenaArray<Real> x1s2, x1s3, x2s1, x2s3, x3s1, x3s2;
  AthenaArray<Real> h2f, dh2fd1, h31f, h32f, dh31fd1, dh32fd2;
  AthenaArray<Real> h2v, dh2vd1, h31v, h32v, dh31vd1, dh32vd2;

  virtual void Face1Area(const int k, const int j, const int il, const int iu,
                         AthenaArray<Real>& area) {}
  virtual void Face2Area(const int k, const int j, const int il, const int iu,
                         AthenaArray<Real>& area) {}
  virtual void Face3Area(const int k, const int j, const int il, const int iu,
                         AthenaArray<Real>& area) {}
  virtual Real GetFace1Area(const int k, const int j, const int i) { return 0; }
  virtual Real GetFace2Area(const int k, const int j, const int i) { return 0; }
  virtual Real GetFace3Area(const int k, const int j, const int i) { return 0; }
  virtual void VolCenterFace1Area(const int k, const int j, const int il, const int iu,
                                  AthenaArray<Real>& area) {}
  virtual void VolCenterFace2Area(const int k, const int j, const int il, const int iu,
                                  AthenaArray<Real>& area) {}
  virtual void VolCenterFace3Area(const int k, const int j, const int il, const int iu,
                                  AthenaArray<Real>& area) {}
  virtual void CellVolume(const int k, const int j, const int il, const int iu,
                          AthenaArray<Real>& vol) {}
  virtual Real GetCellVolume(const int k, const int j, const int i) { return 0; }
  virtual void CenterWidth1(const int k, const int j, const int il, const int iu,
                            AthenaArray<Real>& dx1) {}
  virtual void CenterWidth2(const int k, const int j, const int il, const int iu,
                            AthenaArray<Real>& dx2) {}
  virtual void CenterWidth3(const int k, const int j, const int il, const int iu,
                            AthenaArray<Real>& dx3) {}
  virtual void CellMetric(const int k, const int j, const int il, const int iu,
                          AthenaArray<Real>& g, AthenaArray<Real>& g_inv) {}
  virtual void Face1Metric(const int k, const int j, const int il, const int iu,
                           AthenaArray<Real>& g, AthenaArray<Real>& g_inv) {}
  virtual void Face2Metric(const int k, const int j, const int il, const int iu,
                           AthenaArray<Real>& g, AthenaArray<Real>& g_inv) {}
  virtual void Face3Metric(const int k, const int j, const int il, const int iu,
                           AthenaArray<Real>& g, AthenaArray<Real>& g_inv) {}
  virtual void PrimToLocal1(const int k, const int j, const int il, const int iu,
                            const AthenaArray<Real>& b1_vals, AthenaArray<Real>& prim_left,
                            AthenaArray<Real>& prim_right, AthenaArray<Real>& bx) {}
  virtual void PrimToLocal2(const int k, const int j, const int il, const int iu,
                            const AthenaArray<Real>& b2_vals, AthenaArray<Real>& prim_left,
                            AthenaArray<Real>& prim_right, AthenaArray<Real>& bx) {}
  virtual void PrimToLocal3(const int k, const int j, const int il, const int iu,
                            const AthenaArray<Real>& b3_vals, AthenaArray<Real>& prim_left,
                            AthenaArray<Real>& prim_right, AthenaArray<Real>& bx) {}
  virtual void FluxToGlobal1(const int k, const int j, const int il, const int iu,
                             const AthenaArray<Real>& cons, const AthenaArray<Real>& bbx,
                             AthenaArray<Real>& flux, AthenaArray<Real>& ey,
                             AthenaArray<Real>& ez) {}
  virtual void FluxToGlobal2(const int k, const int j, const int il, const int iu,
                             const AthenaArray<Real>& cons, const AthenaArray<Real>& bbx,
                             AthenaArray<Real>& flux, AthenaArray<Real>& ey,
                             AthenaArray<Real>& ez) {}
  virtual void FluxToGlobal3(const int k, const int j, const int il, const int iu,
                             const AthenaArray<Real>& cons, const AthenaArray<Real>& bbx,
                             AthenaArray<Real>& flux, AthenaArray<Real>& ey,
                             AthenaArray<Real>& ez) {}
  virtual void AddCoordTermsDivergence(const Real dt, const AthenaArray<Real>* flux,
                                       const AthenaArray<Real>& prim,
                                       const AthenaArray<Real>& bcc, AthenaArray<Real>& u) {}

 protected:
  int il, iu, jl, ju, kl, ku, ng;
  int nc1, nc2, nc3;
  AthenaArray<Real> g_, gi_;
  AthenaArray<Real> coord_vol_i_, coord_area2_i_, coord_area2_i1_, coord_area3_i_,
      coord_area3_i1_;
};

#endif
