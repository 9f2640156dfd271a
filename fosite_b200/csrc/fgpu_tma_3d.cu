// fgpu_tma_3d.cu -- the TMA-staged stage kernels of 3D meshes (fgpu_tma.cuh).
#include "fgpu_tma_nd.cuh"

namespace fgpu {
cudaError_t tma_stage_launch_3d(bool euler, bool prim, int limiter, bool constant_recon, const Grid& g, int kchunk,
                                cudaStream_t s, const StageArgs& A, const CUtensorMap& map) {
  return launch_nd<3, kTmaTY>(euler, prim, limiter, constant_recon, g, kchunk, s, A, map);
}
void tma_stage_configure_3d(bool euler, bool prim) { configure_nd<3, kTmaTY>(euler, prim); }
}  // namespace fgpu
