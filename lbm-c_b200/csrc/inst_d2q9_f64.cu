// Kernel instantiations for D2Q9 with double population storage.
#include "instances.cuh"

LBMC_DEFINE_OPS(ops_d2q9_f64, D2Q9, double)
