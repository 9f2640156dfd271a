// fgpu_stage_launch.h -- host entry of the shared-memory stage kernels (stage_kernel and
// batched_stage_kernel of fgpu_kernels.cuh, stage2_kernel of fgpu_stage2.cuh).
//
// The kernel instantiations live in their own translation units (fgpu_stage_2d.cu,
// fgpu_stage_3d.cu) so that they compile in parallel with the rest of the library.
#pragma once
#include <cuda_runtime.h>
#include "fgpu_kernels.cuh"

namespace fgpu {

// height of the base tile (the batches' tile queues are built for it): 2D 32 x 8, 3D 32 x 4
constexpr int kBaseTY2 = 8, kBaseTY3 = 4;

// Launch one stage on a shared-memory layout: 0 the base tile (2D 32x8, 3D 32x4 marching in
// z), 2/3 the base tile with a register cap for more resident blocks (2D 2/3, 3D 4/6 per SM),
// 4/5 a taller tile (2D 32x16, 3D 32x8 with 2/3 blocks per SM) that halves the y halo, 1 the
// warp-shuffle window; any other id launches layout 0.
cudaError_t legacy_stage_launch_2d(bool euler, bool prim, int variant, const Grid& g, cudaStream_t s,
                                   const StageArgs& A);
cudaError_t legacy_stage_launch_3d(bool euler, bool prim, int variant, const Grid& g, int kchunk, cudaStream_t s,
                                   const StageArgs& A);
// Batches: layouts 0, 2, 3 (any other id: 0) over the tile queue (grid, bx, by, bz) of base
// tiles, one persistent launch sized by the occupancy calculator for `sms` SMs.
cudaError_t legacy_batched_launch_2d(bool euler, bool prim, int variant, const StageArgs* args, const int4* tiles,
                                     int ntiles, int sms, cudaStream_t s);
cudaError_t legacy_batched_launch_3d(bool euler, bool prim, int variant, const StageArgs* args, const int4* tiles,
                                     int ntiles, int sms, cudaStream_t s);
// opt the kernels into their dynamic shared memory (once per device)
void legacy_stage_configure_2d(bool euler, bool prim);
void legacy_stage_configure_3d(bool euler, bool prim);

}  // namespace fgpu
