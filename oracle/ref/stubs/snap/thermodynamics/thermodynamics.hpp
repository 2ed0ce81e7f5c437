// harness stand-in: with no vapour the Riemann solvers never call it
#ifndef REF_STUB_THERMO_HPP_
#define REF_STUB_THERMO_HPP_
#include <athena/athena.hpp>
class Thermodynamics {
 public:
  static Thermodynamics* GetInstance() { static Thermodynamics t; return &t; }
  Real GetCvRatioMass(int) const { return 1.; }
  Real GetMuRatio(int) const { return 1.; }
};
#endif
