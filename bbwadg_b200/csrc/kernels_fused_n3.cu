// Fused stage, order N = 3, 32-element tiles.
#define BBW_FUSED_N 3
#define BBW_FUSED_E 32
#include "fused_inst.cuh"
