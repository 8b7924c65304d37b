// Fused stage, order N = 6.
#define BBW_FUSED_N 6
#include "fused_inst.cuh"
