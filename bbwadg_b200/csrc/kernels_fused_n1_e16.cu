// Fused stage, order N = 1, 16-element tiles.
#define BBW_FUSED_N 1
#define BBW_FUSED_E 16
#include "fused_inst.cuh"
