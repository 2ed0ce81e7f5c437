// harness stand-in for canoe's impl.hpp: MeshBlock::Impl lives in the
// MeshBlock stand-in; its cubed-sphere object is the reference's CubedSphere
#ifndef REF_STUB_IMPL_HPP_
#define REF_STUB_IMPL_HPP_
#include <athena/coordinates/coordinates.hpp>
#include <athena/mesh/mesh.hpp>
#include <exo3/cubed_sphere.hpp>
#endif
