// Fused stage, order N = 5, 16-element tiles.
#define BBW_FUSED_N 5
#define BBW_FUSED_E 16
#include "fused_inst.cuh"
