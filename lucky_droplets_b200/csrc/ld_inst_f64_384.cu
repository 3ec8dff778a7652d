// Kernel instance: precision double, N = 384.
#include "ld_ops.cuh"
LD_DEFINE_TABLE(f64, double, 384)
