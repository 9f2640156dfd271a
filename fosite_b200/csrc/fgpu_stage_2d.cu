// fgpu_stage_2d.cu -- the shared-memory stage kernels of 2D meshes (fgpu_stage_nd.cuh).
#include "fgpu_stage_nd.cuh"

namespace fgpu {
cudaError_t legacy_stage_launch_2d(bool euler, bool prim, int variant, const Grid& g, cudaStream_t s,
                                   const StageArgs& A) {
  return launch_nd<2>(euler, prim, variant, g, 1, s, A);
}
cudaError_t legacy_batched_launch_2d(bool euler, bool prim, int variant, const StageArgs* args, const int4* tiles,
                                     int ntiles, int sms, cudaStream_t s) {
  return batched_nd<2>(euler, prim, variant, args, tiles, ntiles, sms, s);
}
void legacy_stage_configure_2d(bool euler, bool prim) { configure_nd<2>(euler, prim); }
}  // namespace fgpu
