// fgpu_stage_3d.cu -- the shared-memory stage kernels of 3D meshes (fgpu_stage_nd.cuh).
#include "fgpu_stage_nd.cuh"

namespace fgpu {
cudaError_t legacy_stage_launch_3d(bool euler, bool prim, int variant, const Grid& g, int kchunk, cudaStream_t s,
                                   const StageArgs& A) {
  return launch_nd<3>(euler, prim, variant, g, kchunk, s, A);
}
cudaError_t legacy_batched_launch_3d(bool euler, bool prim, int variant, const StageArgs* args, const int4* tiles,
                                     int ntiles, int sms, cudaStream_t s) {
  return batched_nd<3>(euler, prim, variant, args, tiles, ntiles, sms, s);
}
void legacy_stage_configure_3d(bool euler, bool prim) { configure_nd<3>(euler, prim); }
}  // namespace fgpu
