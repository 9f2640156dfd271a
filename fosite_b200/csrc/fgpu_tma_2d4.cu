// fgpu_tma_2d4.cu -- the TMA-staged stage kernels of 2D meshes, 32 x 4 tiles (layout 7;
// fgpu_tma.cuh).
#include "fgpu_tma_nd.cuh"

namespace fgpu {
cudaError_t tma_stage_launch_2d4(bool euler, bool prim, int limiter, bool constant_recon, const Grid& g,
                                 cudaStream_t s, const StageArgs& A, const CUtensorMap& map) {
  return launch_nd<2, 4>(euler, prim, limiter, constant_recon, g, 1, s, A, map);
}
void tma_stage_configure_2d4(bool euler, bool prim) { configure_nd<2, 4>(euler, prim); }
}  // namespace fgpu
