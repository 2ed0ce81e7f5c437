// Harness stand-in for Athena++'s Mesh and MeshBlock: index ranges, the
// logical location, the mesh the Coordinates stand-in reads, and the
// pointers the reference's sources follow.  Test infrastructure only.
#ifndef REF_STUB_MESH_HPP_
#define REF_STUB_MESH_HPP_

#include <memory>

#include "../athena.hpp"
#include "../bvals/bvals.hpp"

struct RegionSize {
  int nx1 = 1, nx2 = 1, nx3 = 1;
  Real x1rat = 1.0, x2rat = 1.0, x3rat = 1.0;
};

class MeshBlock;
class Mesh {
 public:
  bool multilevel = false;
  // blocks of this process by gid (the harness has no local neighbours)
  MeshBlock* FindMeshBlock(int) { return nullptr; }
};

class CubedSphere;
class Microphysics;
class Decomposition;

class MeshBlock {
 public:
  // what MeshBlock::Impl holds for the reference's sources
  struct Impl {
    CubedSphere* pexo3 = nullptr;
    Microphysics* pmicro = nullptr;
    std::shared_ptr<Decomposition> pdec;
  };

  Mesh* pmy_mesh = nullptr;
  Coordinates* pcoord = nullptr;
  EquationOfState* peos = nullptr;
  Hydro* phydro = nullptr;
  BoundaryValues* pbval = nullptr;
  Impl* pimpl = nullptr;
  LogicalLocation loc;
  RegionSize block_size;
  int is = 0, ie = 0, js = 0, je = 0, ks = 0, ke = 0;
  int ncells1 = 1, ncells2 = 1, ncells3 = 1;
  int gid = 0;
  // the mesh for the Coordinates stand-in: faces (ncells + 1 each) and the
  // radial face widths (ncells1)
  const Real* mesh_x1f = nullptr;
  const Real* mesh_x2f = nullptr;
  const Real* mesh_x3f = nullptr;
  const Real* mesh_dx1f = nullptr;
};

#endif
