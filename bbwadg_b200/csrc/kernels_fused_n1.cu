// Fused stage, order N = 1, 32-element tiles.
#define BBW_FUSED_N 1
#define BBW_FUSED_E 32
#include "fused_inst.cuh"
