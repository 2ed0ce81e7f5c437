// harness stand-in for Athena++'s bvals.hpp: the neighbour list the
// reference's face-state exchange walks (CubedSphere::SynchronizeFluxes*)
#ifndef REF_STUB_BVALS_HPP_
#define REF_STUB_BVALS_HPP_
#include "../athena.hpp"
struct NeighborIndexes { int ox1 = 0, ox2 = 0, ox3 = 0; };
struct SimpleNeighborBlock { int rank = 0, level = 0, gid = 0; };
struct NeighborBlock {
  SimpleNeighborBlock snb;
  NeighborIndexes ni;
};
class BoundaryValues {
 public:
  int nneighbor = 0;
  NeighborBlock neighbor[4];
};
#endif
