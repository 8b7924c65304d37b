// Fused stage, order N = 8, 16-element tiles.
#define BBW_FUSED_N 8
#define BBW_FUSED_E 16
#include "fused_inst.cuh"
