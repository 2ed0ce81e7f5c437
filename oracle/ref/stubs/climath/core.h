// harness stand-in for climath/core.h
#ifndef REF_STUB_CLIMATH_CORE_H_
#define REF_STUB_CLIMATH_CORE_H_
inline double sqr(double x) { return x * x; }
inline double cub(double x) { return x * x * x; }
#endif
