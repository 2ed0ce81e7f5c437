// harness stand-in for Athena++'s parameter_input.hpp
#ifndef REF_STUB_PARAMETER_INPUT_HPP_
#define REF_STUB_PARAMETER_INPUT_HPP_
class ParameterInput {};
#endif
