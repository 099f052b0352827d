// Kernel instantiations for D2Q9 with float population storage.
#include "instances.cuh"

LBMC_DEFINE_OPS(ops_d2q9_f32, D2Q9, float)
