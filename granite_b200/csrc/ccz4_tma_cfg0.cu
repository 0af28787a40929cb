// ccz4_tma_cfg0.cu -- the TMA stage kernel in configuration 0 of TMA_CFGS
// (ccz4_kernels.h); with the store epilogue of the drop-in RHS.
#include "ccz4_stage_tma.cuh"

GRANITE_TMA_CFG_UNIT(0, true)
