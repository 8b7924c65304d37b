// Fused stage, order N = 7.
#define BBW_FUSED_N 7
#include "fused_inst.cuh"
