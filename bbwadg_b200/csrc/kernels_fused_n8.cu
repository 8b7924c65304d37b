// Fused stage, order N = 8.
#define BBW_FUSED_N 8
#include "fused_inst.cuh"
