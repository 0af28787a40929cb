// ccz4_tma_cfg15.cu -- the TMA stage kernel in configuration 15 of TMA_CFGS
// (ccz4_kernels.h).
#include "ccz4_stage_tma.cuh"

GRANITE_TMA_CFG_UNIT(15, false)
