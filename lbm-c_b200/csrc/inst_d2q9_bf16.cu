// Kernel instantiations for D2Q9 with __nv_bfloat16 population storage.
#include "instances.cuh"

LBMC_DEFINE_OPS(ops_d2q9_bf16, D2Q9, __nv_bfloat16)
