// Kernel instantiations for D2Q9 with __half population storage.
#include "instances.cuh"

LBMC_DEFINE_OPS(ops_d2q9_f16, D2Q9, __half)
