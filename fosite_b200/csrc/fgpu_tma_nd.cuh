// fgpu_tma_nd.cuh -- instantiations of the TMA-staged stage kernel for one dimensionality and
// tile height (included by fgpu_tma_2d.cu, fgpu_tma_2d4.cu and fgpu_tma_3d.cu).
#pragma once
#include "fgpu_tma.cuh"
#include "fgpu_tma_launch.h"

namespace fgpu {
namespace {

// resident blocks per SM requested from the register allocator: the 32 x 8 tile two (3D) or
// three (2D), the 32 x 4 tile (2D) six
template <int ND, int TY> struct TmaMinBlocks { static constexpr int N = ND == 3 ? 2 : (TY == 4 ? 6 : 3); };

// a stage that reduces CFL / CheckData / error-norm maxima; the others run the kernel form whose
// maxima are compiled out (their registers go to the stencil: 10% on the 3D Butcher stages)
inline bool stage_reduces(const StageArgs& A) { return A.cfl_mode || A.last_stage || A.err_low; }

template <int ND, bool EU, bool PRIM, int TY, int LIM>
struct TmaKernel {
  static constexpr int MINB = TmaMinBlocks<ND, TY>::N;
  static constexpr int NTH = kTmaTX * TY;   // one thread per cell
  static constexpr size_t SMEM = TmaLayout<Phys<ND, EU>::V, kTmaTX, TY, TmaSlots<ND>::N>::SMEM;
  template <bool RED>
  static void configure_red() {
    cudaFuncSetAttribute(tma_stage_kernel<ND, EU, PRIM, kTmaTX, TY, MINB, LIM, NTH, RED>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
    if constexpr (ND == 2 && TY == kTmaTY)
      cudaFuncSetAttribute(batched_tma_stage_kernel<ND, EU, PRIM, kTmaTX, TY, MINB, LIM, NTH, RED>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
  }
  static void configure() {
    configure_red<true>();
    configure_red<false>();
  }
  static void launch_batched(bool red, const StageArgs* args, const CUtensorMap* maps, const int4* tiles, int ntiles,
                             cudaStream_t s) {
    if constexpr (ND == 2 && TY == kTmaTY) {
      if (red)
        batched_tma_stage_kernel<ND, EU, PRIM, kTmaTX, TY, MINB, LIM, NTH, true><<<ntiles, NTH, SMEM, s>>>(args, maps, tiles);
      else
        batched_tma_stage_kernel<ND, EU, PRIM, kTmaTX, TY, MINB, LIM, NTH, false><<<ntiles, NTH, SMEM, s>>>(args, maps, tiles);
    }
  }
  static void launch(const Grid& g, int kchunk, cudaStream_t s, const StageArgs& A, const CUtensorMap& map) {
    const int tx = (g.nx + kTmaTX - 1) / kTmaTX, ty = (g.ny + TY - 1) / TY;
    const bool red = stage_reduces(A);
    if constexpr (ND == 3) {
      dim3 grid(tx, ty, (g.nz + kchunk - 1) / kchunk);
      if (red) tma_stage_kernel<ND, EU, PRIM, kTmaTX, TY, MINB, LIM, NTH, true><<<grid, NTH, SMEM, s>>>(A, map);
      else tma_stage_kernel<ND, EU, PRIM, kTmaTX, TY, MINB, LIM, NTH, false><<<grid, NTH, SMEM, s>>>(A, map);
    } else {
      // 2D: each block computes a column of tma_tiles_per_block tiles, the next tile's box
      // arriving while the current one is computed
      StageArgs B = A;
      B.kchunk = tma_tiles_per_block((long long)tx * ty, MINB);
      dim3 grid(tx, (ty + B.kchunk - 1) / B.kchunk, 1);
      if (red) tma_stage_kernel<ND, EU, PRIM, kTmaTX, TY, MINB, LIM, NTH, true><<<grid, NTH, SMEM, s>>>(B, map);
      else tma_stage_kernel<ND, EU, PRIM, kTmaTX, TY, MINB, LIM, NTH, false><<<grid, NTH, SMEM, s>>>(B, map);
    }
  }
};

template <int ND, bool EU, bool PRIM, int TY>
void configure_all() {
  TmaKernel<ND, EU, PRIM, TY, 0>::configure();
  TmaKernel<ND, EU, PRIM, TY, LIM_MINMOD>::configure();
  TmaKernel<ND, EU, PRIM, TY, LIM_MC1>::configure();
  TmaKernel<ND, EU, PRIM, TY, LIM_VANLEER>::configure();
}

template <int ND, bool EU, bool PRIM, int TY>
void launch_lim(int limiter, bool constant_recon, const Grid& g, int kchunk, cudaStream_t s, const StageArgs& A,
                const CUtensorMap& map) {
  // MC with theta = 1 has its own kernel; MC with another theta reads it from the arguments
  const int lim = compiled_limiter(limiter, constant_recon, A.theta);
  switch (lim) {
    case LIM_MINMOD: TmaKernel<ND, EU, PRIM, TY, LIM_MINMOD>::launch(g, kchunk, s, A, map); break;
    case LIM_MC1: TmaKernel<ND, EU, PRIM, TY, LIM_MC1>::launch(g, kchunk, s, A, map); break;
    case LIM_VANLEER: TmaKernel<ND, EU, PRIM, TY, LIM_VANLEER>::launch(g, kchunk, s, A, map); break;
    default: TmaKernel<ND, EU, PRIM, TY, 0>::launch(g, kchunk, s, A, map); break;
  }
}

template <int ND, int TY>
cudaError_t launch_nd(bool euler, bool prim, int limiter, bool constant_recon, const Grid& g, int kchunk,
                      cudaStream_t s, const StageArgs& A, const CUtensorMap& map) {
  if (euler) {
    if (prim) launch_lim<ND, true, true, TY>(limiter, constant_recon, g, kchunk, s, A, map);
    else launch_lim<ND, true, false, TY>(limiter, constant_recon, g, kchunk, s, A, map);
  } else {
    if (prim) launch_lim<ND, false, true, TY>(limiter, constant_recon, g, kchunk, s, A, map);
    else launch_lim<ND, false, false, TY>(limiter, constant_recon, g, kchunk, s, A, map);
  }
  return cudaGetLastError();
}

template <int ND, bool EU, bool PRIM>
void launch_batched_lim(int lim, bool red, const StageArgs* args, const CUtensorMap* maps, const int4* tiles,
                        int ntiles, cudaStream_t s) {
  switch (lim) {
    case LIM_MINMOD: TmaKernel<ND, EU, PRIM, kTmaTY, LIM_MINMOD>::launch_batched(red, args, maps, tiles, ntiles, s); break;
    case LIM_MC1: TmaKernel<ND, EU, PRIM, kTmaTY, LIM_MC1>::launch_batched(red, args, maps, tiles, ntiles, s); break;
    case LIM_VANLEER: TmaKernel<ND, EU, PRIM, kTmaTY, LIM_VANLEER>::launch_batched(red, args, maps, tiles, ntiles, s); break;
    default: TmaKernel<ND, EU, PRIM, kTmaTY, 0>::launch_batched(red, args, maps, tiles, ntiles, s); break;
  }
}

template <int ND, int TY>
void configure_nd(bool euler, bool prim) {
  if (euler) prim ? configure_all<ND, true, true, TY>() : configure_all<ND, true, false, TY>();
  else prim ? configure_all<ND, false, true, TY>() : configure_all<ND, false, false, TY>();
}

}  // namespace
}  // namespace fgpu
