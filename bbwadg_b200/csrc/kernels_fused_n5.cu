// Fused stage, order N = 5.
#define BBW_FUSED_N 5
#include "fused_inst.cuh"
