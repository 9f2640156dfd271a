// fgpu_tma_launch.h -- host entry of the TMA-staged stage kernel (fgpu_tma.cuh).
//
// The kernel instantiations live in their own translation units (fgpu_tma_2d.cu,
// fgpu_tma_3d.cu) so that they compile in parallel with the rest of the library.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdlib>
#include "fgpu_kernels.cuh"

namespace fgpu {

// tile shapes of the TMA layouts: 32 x 8 cells (layout 6; 3D: a three-plane ring, two blocks
// per SM; 2D: one plane, three blocks per SM) and, for 2D meshes, 32 x 4 cells (layout 7, six
// blocks per SM: twice the blocks on small grids)
constexpr int kTmaTX = 32, kTmaTY = 8;

// Launch one stage on the TMA layout.  limiter / constant_recon are the config's: the
// minmod, MC (theta = 1) and van Leer limiters of linear reconstruction have kernels with the
// limiter compiled in, every other case the kernel that reads it from the arguments.
cudaError_t tma_stage_launch_2d(bool euler, bool prim, int limiter, bool constant_recon, int ty, const Grid& g,
                                cudaStream_t s, const StageArgs& A, const CUtensorMap& map);
cudaError_t tma_stage_launch_3d(bool euler, bool prim, int limiter, bool constant_recon, const Grid& g, int kchunk,
                                cudaStream_t s, const StageArgs& A, const CUtensorMap& map);
// Batched ensembles of 2D grids on the 32 x 8 TMA layout: one block per entry (grid, bx, byb, 0)
// of the block queue, the block computing tiles byb * kchunk .. of column bx of the grid, kchunk
// taken from the grid's stage arguments; args[grid] and maps[grid] (device arrays) the stage
// arguments and the tensor map of the stage input of each grid; lim the compiled-in limiter
// shared by every grid (compiled_limiter), 0 when the grids differ or read it from their
// arguments.
// red: some grid's stage reduces CFL / CheckData / error-norm maxima (else the kernel form without
// the reductions runs).
cudaError_t tma_batched_launch_2d(bool euler, bool prim, int lim, bool red, const StageArgs* args,
                                  const CUtensorMap* maps, const int4* tiles, int ntiles, cudaStream_t s);
// the 32 x 4 tiles (own translation unit)
cudaError_t tma_stage_launch_2d4(bool euler, bool prim, int limiter, bool constant_recon, const Grid& g,
                                 cudaStream_t s, const StageArgs& A, const CUtensorMap& map);
void tma_stage_configure_2d4(bool euler, bool prim);
// 2D TMA tiles computed by one block (a column of tiles whose boxes are double-buffered): as
// many as keep about three waves of resident blocks on the device, at most 8; FGPU_TMA_TPB
// fixes the count
inline int tma_tiles_per_block(long long tiles, int blocks_per_sm) {
  if (const char* e = std::getenv("FGPU_TMA_TPB")) {
    const int v = std::atoi(e);
    if (v > 0) return v;
  }
  static int sms = [] {
    int d = 0, n = 148;
    if (cudaGetDevice(&d) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, d);
    return n > 0 ? n : 148;
  }();
  const long long per = tiles / (3LL * sms * blocks_per_sm);
  return (int)(per < 1 ? 1 : (per > 8 ? 8 : per));
}
// the limiter code a stage's TMA kernel is compiled for: minmod, MC with theta = 1 (LIM_MC1),
// van Leer; 0 when the kernel reads limiter, theta and reconstruction order from the arguments
inline int compiled_limiter(int limiter, bool constant_recon, double theta) {
  if (constant_recon) return 0;
  if (limiter == LIM_MC) return theta == 1.0 ? LIM_MC1 : 0;
  return (limiter == LIM_MINMOD || limiter == LIM_VANLEER) ? limiter : 0;
}
// opt the kernels into their dynamic shared memory (once per device)
void tma_stage_configure_2d(bool euler, bool prim);
void tma_stage_configure_3d(bool euler, bool prim);

}  // namespace fgpu
