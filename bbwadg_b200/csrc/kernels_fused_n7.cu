// Fused stage, order N = 7, 32-element tiles.
#define BBW_FUSED_N 7
#define BBW_FUSED_E 32
#include "fused_inst.cuh"
