// Fused stage, order N = 7, 16-element tiles.
#define BBW_FUSED_N 7
#define BBW_FUSED_E 16
#include "fused_inst.cuh"
