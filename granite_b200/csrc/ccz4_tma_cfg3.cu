// ccz4_tma_cfg3.cu -- the TMA stage kernel in configuration 3 of TMA_CFGS
// (ccz4_kernels.h).
#include "ccz4_stage_tma.cuh"

GRANITE_TMA_CFG_UNIT(3, false)
