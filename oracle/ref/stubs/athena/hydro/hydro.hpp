// harness stand-in for Athena++'s Hydro: the Riemann solver hook the
// reference's src/snap/riemann/*.cpp define
#ifndef REF_STUB_HYDRO_HPP_
#define REF_STUB_HYDRO_HPP_
#include "../athena.hpp"
class Hydro {
 public:
  MeshBlock* pmy_block = nullptr;
  void RiemannSolver(const int k, const int j, const int il, const int iu, const int ivx,
                     AthenaArray<Real>& wl, AthenaArray<Real>& wr, AthenaArray<Real>& flx,
                     const AthenaArray<Real>& dxw);
};
#endif
