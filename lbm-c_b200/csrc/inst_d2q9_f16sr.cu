// Kernel instantiations for D2Q9 with FP16 storage written by stochastic rounding.
#include "instances.cuh"

LBMC_DEFINE_OPS(ops_d2q9_f16sr, D2Q9, half_sr)
