// ccz4_tma_cfg16.cu -- the TMA stage kernel in configuration 16 of TMA_CFGS
// (ccz4_kernels.h).
#include "ccz4_stage_tma.cuh"

GRANITE_TMA_CFG_UNIT(16, false)
