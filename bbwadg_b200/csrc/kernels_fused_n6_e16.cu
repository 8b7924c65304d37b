// Fused stage, order N = 6, 16-element tiles.
#define BBW_FUSED_N 6
#define BBW_FUSED_E 16
#include "fused_inst.cuh"
