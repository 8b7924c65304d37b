// Fused stage, order N = 1.
#define BBW_FUSED_N 1
#include "fused_inst.cuh"
