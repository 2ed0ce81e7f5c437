// harness stand-in: with no clouds (NCLOUD = 0) the LMARS sedimentation loop
// never runs, but it must compile
#ifndef REF_STUB_MICRO_HPP_
#define REF_STUB_MICRO_HPP_
#include <athena/athena.hpp>
class Microphysics {
 public:
  AthenaArray<Real>& GetSedimentationVelocityFace(int dir) { return vsed_; }
  void SetFluidMassFlux(int dir, int n, int k, int j, int i, Real v) {}

 private:
  AthenaArray<Real> vsed_;
};
#endif
