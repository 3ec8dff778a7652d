// Kernel instance: precision float, N = 96.
#include "ld_ops.cuh"
LD_DEFINE_TABLE(f32, float, 96)
