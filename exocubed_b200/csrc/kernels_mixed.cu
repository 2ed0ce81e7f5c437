// kernels_mixed.cu -- the mixed-precision build of the step: WENO5, the
// Riemann solvers and the flux divergence in FP32; the hydrostatic
// decomposition, the implicit vertical solve, the equation of state and the
// conserved-state accumulation across RK stages in FP64.
#define EXO_KNS mixed
#define EXO_MIXED 1
#define EXO_FLUX_T float
#include "exo_kernels.cuh"
