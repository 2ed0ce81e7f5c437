// harness stand-in for Athena++'s generated defs.hpp
#ifndef REF_STUB_DEFS_HPP_
#define REF_STUB_DEFS_HPP_
#ifndef EQUATION_OF_STATE
#define EQUATION_OF_STATE "ideal_moist"
#endif
#endif
