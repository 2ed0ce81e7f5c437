// harness stand-in for canoe's Thermodynamics with no vapour: the dry gas
// constant and the polytropic index the decomposition reads
// (thermodynamics.hpp GetGamma with fsig = feps = 1)
#ifndef REF_STUB_THERMO_HPP_
#define REF_STUB_THERMO_HPP_
#include <athena/athena.hpp>
class Thermodynamics {
 public:
  Real Rd = 287., gammad = 1.4;
  static Thermodynamics* GetInstance() { static Thermodynamics t; return &t; }
  Real GetCvRatioMass(int) const { return 1.; }
  Real GetMuRatio(int) const { return 1.; }
  Real GetRd() const { return Rd; }
  Real GetGamma(MeshBlock*, int, int, int) const {
    Real fsig = 1., feps = 1.;
    return 1. + (gammad - 1.) * feps / fsig;
  }
};
#endif
