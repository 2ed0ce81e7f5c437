// harness stand-in for Athena++'s Hydro: the Riemann solver hook the
// reference's src/snap/riemann/*.cpp define, and the constant-gravity source
// whose x1 acceleration the decomposition reads
#ifndef REF_STUB_HYDRO_HPP_
#define REF_STUB_HYDRO_HPP_
#include "../athena.hpp"
class HydroSourceTerms {
 public:
  Real g1 = 0.;
  Real GetG1() const { return g1; }
};
class Hydro {
 public:
  MeshBlock* pmy_block = nullptr;
  HydroSourceTerms hsrc;
  void RiemannSolver(const int k, const int j, const int il, const int iu, const int ivx,
                     AthenaArray<Real>& wl, AthenaArray<Real>& wr, AthenaArray<Real>& flx,
                     const AthenaArray<Real>& dxw);
};
#endif
