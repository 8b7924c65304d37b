// Fused stage, order N = 2, 16-element tiles.
#define BBW_FUSED_N 2
#define BBW_FUSED_E 16
#include "fused_inst.cuh"
