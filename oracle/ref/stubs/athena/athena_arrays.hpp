// harness stand-in: AthenaArray lives in athena.hpp
#include "athena.hpp"
