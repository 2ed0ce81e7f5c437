// Harness stand-in for the equation of state the reference's Riemann
// solvers call: canoe's ideal_moist_hydro.cpp with no vapour (the sound
// speed of src/snap/eos/ideal_moist_hydro.cpp:226-238 with fsig = feps = 1).
#ifndef REF_STUB_EOS_HPP_
#define REF_STUB_EOS_HPP_
#include <cmath>
#include "../athena.hpp"
class EquationOfState {
 public:
  Real gamma = 1.4;
  Real GetGamma() const { return gamma; }
  Real SoundSpeed(const Real prim[]) {
    Real fsig = 1., feps = 1.;
    return std::sqrt((1. + (gamma - 1) * feps / fsig) * prim[IPR] / prim[IDN]);
  }
  Real EgasFromRhoP(Real rho, Real p) { return p / (gamma - 1.); }
  Real AsqFromRhoP(Real rho, Real p) { return gamma * p / rho; }
};
#endif
