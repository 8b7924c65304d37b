// Fused stage, order N = 5, 32-element tiles.
#define BBW_FUSED_N 5
#define BBW_FUSED_E 32
#include "fused_inst.cuh"
