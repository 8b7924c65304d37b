// Fused stage, order N = 4.
#define BBW_FUSED_N 4
#include "fused_inst.cuh"
