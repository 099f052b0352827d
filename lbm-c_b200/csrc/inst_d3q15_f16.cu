// Kernel instantiations for D3Q15 with __half population storage.
#include "instances.cuh"

LBMC_DEFINE_OPS(ops_d3q15_f16, D3Q15, __half)
