// Fused stage, order N = 6, 32-element tiles.
#define BBW_FUSED_N 6
#define BBW_FUSED_E 32
#include "fused_inst.cuh"
