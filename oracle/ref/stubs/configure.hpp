// harness stand-in for canoe's generated configure.hpp: the cubed-sphere dry
// build (no vapour, no clouds)
#ifndef REF_STUB_CONFIGURE_HPP_
#define REF_STUB_CONFIGURE_HPP_
#define CUBED_SPHERE
#define NVAPOR 0
#define NCLOUD 0
#endif
