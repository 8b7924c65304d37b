// Fused stage, order N = 8, 32-element tiles.
#define BBW_FUSED_N 8
#define BBW_FUSED_E 32
#include "fused_inst.cuh"
