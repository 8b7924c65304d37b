// Fused stage, order N = 4, 32-element tiles.
#define BBW_FUSED_N 4
#define BBW_FUSED_E 32
#include "fused_inst.cuh"
