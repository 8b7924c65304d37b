// Fused stage, order N = 2, 32-element tiles.
#define BBW_FUSED_N 2
#define BBW_FUSED_E 32
#include "fused_inst.cuh"
