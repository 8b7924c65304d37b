// Fused stage, order N = 3, 16-element tiles.
#define BBW_FUSED_N 3
#define BBW_FUSED_E 16
#include "fused_inst.cuh"
