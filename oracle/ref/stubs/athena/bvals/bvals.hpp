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
enum class BoundaryFlag { block = -1, undef, reflect, outflow, user, periodic, polar };
enum BoundaryFace { undef = -1, inner_x1, outer_x1, inner_x2, outer_x2, inner_x3, outer_x3 };
class BoundaryValues {
 public:
  int nneighbor = 0;
  NeighborBlock neighbor[4];
  BoundaryFlag block_bcs[6] = {BoundaryFlag::reflect, BoundaryFlag::reflect,
                               BoundaryFlag::block,   BoundaryFlag::block,
                               BoundaryFlag::block,   BoundaryFlag::block};
};
#endif
