// Fused stage, order N = 2.
#define BBW_FUSED_N 2
#include "fused_inst.cuh"
