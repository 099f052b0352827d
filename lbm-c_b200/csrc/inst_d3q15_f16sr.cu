// Kernel instantiations for D3Q15 with FP16 storage written by stochastic rounding.
#include "instances.cuh"

LBMC_DEFINE_OPS(ops_d3q15_f16sr, D3Q15, half_sr)
