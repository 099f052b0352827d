// Kernel instantiations for D3Q15 with float population storage.
#include "instances.cuh"

LBMC_DEFINE_OPS(ops_d3q15_f32, D3Q15, float)
