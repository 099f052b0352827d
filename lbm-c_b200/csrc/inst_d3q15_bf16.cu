// Kernel instantiations for D3Q15 with __nv_bfloat16 population storage.
#include "instances.cuh"

LBMC_DEFINE_OPS(ops_d3q15_bf16, D3Q15, __nv_bfloat16)
