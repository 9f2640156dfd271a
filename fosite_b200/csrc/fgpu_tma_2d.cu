// fgpu_tma_2d.cu -- the TMA-staged stage kernels of 2D meshes, 32 x 8 tiles (single grids and
// batches; fgpu_tma.cuh).  The 32 x 4 tiles are in fgpu_tma_2d4.cu.
#include "fgpu_tma_nd.cuh"

namespace fgpu {
cudaError_t tma_stage_launch_2d(bool euler, bool prim, int limiter, bool constant_recon, int ty, const Grid& g,
                                cudaStream_t s, const StageArgs& A, const CUtensorMap& map) {
  if (ty == 4) return tma_stage_launch_2d4(euler, prim, limiter, constant_recon, g, s, A, map);
  return launch_nd<2, kTmaTY>(euler, prim, limiter, constant_recon, g, 1, s, A, map);
}
cudaError_t tma_batched_launch_2d(bool euler, bool prim, int lim, bool red, const StageArgs* args,
                                  const CUtensorMap* maps, const int4* tiles, int ntiles, cudaStream_t s) {
  if (euler) {
    if (prim) launch_batched_lim<2, true, true>(lim, red, args, maps, tiles, ntiles, s);
    else launch_batched_lim<2, true, false>(lim, red, args, maps, tiles, ntiles, s);
  } else {
    if (prim) launch_batched_lim<2, false, true>(lim, red, args, maps, tiles, ntiles, s);
    else launch_batched_lim<2, false, false>(lim, red, args, maps, tiles, ntiles, s);
  }
  return cudaGetLastError();
}
void tma_stage_configure_2d(bool euler, bool prim) {
  configure_nd<2, kTmaTY>(euler, prim);
  tma_stage_configure_2d4(euler, prim);
}
}  // namespace fgpu
