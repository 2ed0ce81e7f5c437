// harness stand-in for Athena++'s globals.hpp
#ifndef REF_STUB_GLOBALS_HPP_
#define REF_STUB_GLOBALS_HPP_
namespace Globals {
static const int my_rank = 0, nranks = 1, mpi_tag_ub = 32767;
}
#endif
