// ccz4_tma_cfg5.cu -- configuration 5 of TMA_CFGS (ccz4_kernels.h): the
// warp-specialized mixed RK kernels (ccz4_stage_ws.cuh; 3 TMA slots, 6
// derivative slots) and, for FP64, the fused kernel of configuration 4's shape.
#include "ccz4_stage_ws.cuh"

namespace granite_b200 {
static_assert(TMA_CFGS[5].ws == 1 && TMA_CFGS[5].tz == 2 && TMA_CFGS[5].nbuf == 3, "configuration 5");
using WsCfg5 = WsCfgT<3, 6>;
using WsFused5 = TmaCfgT<2, 3, true, false, 2>;
cudaError_t configure_tma_cfg5(int nsm, int grids[3][2][2]) { return WsConfigOps<WsCfg5, WsFused5>::configure(nsm, grids); }
cudaError_t launch_tma_cfg5(int pm, int epi, bool sel, const DevBlock* blocks, const Tile* tiles, int ntiles,
                            const StageArgs& args, cudaStream_t stream, int grid) {
    return WsConfigOps<WsCfg5, WsFused5>::launch(pm, epi, sel, blocks, tiles, ntiles, args, stream, grid);
}
}  // namespace granite_b200
