// Fused stage, order N = 4, 16-element tiles.
#define BBW_FUSED_N 4
#define BBW_FUSED_E 16
#include "fused_inst.cuh"
