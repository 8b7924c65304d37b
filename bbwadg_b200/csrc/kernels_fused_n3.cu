// Fused stage, order N = 3.
#define BBW_FUSED_N 3
#include "fused_inst.cuh"
