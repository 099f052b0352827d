// Kernel instantiations for D3Q15 with double population storage.
#include "instances.cuh"

LBMC_DEFINE_OPS(ops_d3q15_f64, D3Q15, double)
