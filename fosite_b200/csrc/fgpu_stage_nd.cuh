// fgpu_stage_nd.cuh -- instantiations of the shared-memory stage kernels for one dimensionality
// (included by fgpu_stage_2d.cu and fgpu_stage_3d.cu).
#pragma once
#include <algorithm>
#include "fgpu_kernels.cuh"
#include "fgpu_stage2.cuh"
#include "fgpu_stage_launch.h"

namespace fgpu {
namespace {

// A shared-memory tile layout of the stage kernel: TX x TY cells per block,
// MINB resident blocks per SM requested from the register allocator.
template <int ND, bool EU, bool PRIM, int TX, int TY, int MINB>
struct TileLayout {
  static constexpr size_t SMEM = stage_smem_bytes<Phys<ND, EU>::V, TX, TY>();
  // the tiles use more than the default 48 KB of dynamic shared memory: opt in (per device)
  static void configure(bool batched) {
    cudaFuncSetAttribute(stage_kernel<ND, EU, PRIM, TX, TY, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)SMEM);
    if (batched)
      cudaFuncSetAttribute(batched_stage_kernel<ND, EU, PRIM, TX, TY, MINB>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
  }
  static void launch(const Grid& g, int kchunk, cudaStream_t s, const StageArgs& A) {
    const int kz = ND == 3 ? (g.nz + kchunk - 1) / kchunk : 1;
    dim3 grid((g.nx + TX - 1) / TX, (g.ny + TY - 1) / TY, kz);
    stage_kernel<ND, EU, PRIM, TX, TY, MINB><<<grid, TX * TY, SMEM, s>>>(A);
  }
  // one persistent launch over a batch's tile queue
  static void launch_batched(const StageArgs* args, const int4* tiles, int ntiles, int sms, cudaStream_t s) {
    auto k = batched_stage_kernel<ND, EU, PRIM, TX, TY, MINB>;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, TX * TY, SMEM) != cudaSuccess || per_sm < 1)
      per_sm = 1;
    const int blocks = std::max(1, std::min(ntiles, per_sm * sms));
    k<<<blocks, TX * TY, SMEM, s>>>(args, tiles, ntiles);
  }
};
template <int ND> struct TileShapes;
template <> struct TileShapes<2> { static constexpr int TY = kBaseTY2, M2 = 2, M3 = 3, TY4 = 16, M4 = 1, M5 = 1; };
template <> struct TileShapes<3> { static constexpr int TY = kBaseTY3, M2 = 4, M3 = 6, TY4 = 8, M4 = 2, M5 = 3; };

template <int ND, bool EU, bool PRIM>
void configure_t() {
  using S = TileShapes<ND>;
  TileLayout<ND, EU, PRIM, 32, S::TY, 1>::configure(true);
  TileLayout<ND, EU, PRIM, 32, S::TY, S::M2>::configure(true);
  TileLayout<ND, EU, PRIM, 32, S::TY, S::M3>::configure(true);
  TileLayout<ND, EU, PRIM, 32, S::TY4, S::M4>::configure(false);
  TileLayout<ND, EU, PRIM, 32, S::TY4, S::M5>::configure(false);
}

template <int ND, bool EU, bool PRIM>
void launch_t(int variant, const Grid& g, int kchunk, cudaStream_t s, const StageArgs& A) {
  using S = TileShapes<ND>;
  switch (variant) {
    case 1: {
      // warp-shuffle layout: 32 x 8 points per block, 30 x 6 output cells
      constexpr int NW = 8;
      const int kz = ND == 3 ? (g.nz + kchunk - 1) / kchunk : 1;
      dim3 grid((g.nx + 29) / 30, (g.ny + NW - 3) / (NW - 2), kz);
      stage2_kernel<ND, EU, PRIM, NW><<<grid, 32 * NW, 0, s>>>(A);
      break;
    }
    case 2: TileLayout<ND, EU, PRIM, 32, S::TY, S::M2>::launch(g, kchunk, s, A); break;
    case 3: TileLayout<ND, EU, PRIM, 32, S::TY, S::M3>::launch(g, kchunk, s, A); break;
    case 4: TileLayout<ND, EU, PRIM, 32, S::TY4, S::M4>::launch(g, kchunk, s, A); break;
    case 5: TileLayout<ND, EU, PRIM, 32, S::TY4, S::M5>::launch(g, kchunk, s, A); break;
    default: TileLayout<ND, EU, PRIM, 32, S::TY, 1>::launch(g, kchunk, s, A); break;
  }
}

template <int ND, bool EU, bool PRIM>
void batched_t(int variant, const StageArgs* args, const int4* tiles, int ntiles, int sms, cudaStream_t s) {
  using S = TileShapes<ND>;
  if (variant == 2) TileLayout<ND, EU, PRIM, 32, S::TY, S::M2>::launch_batched(args, tiles, ntiles, sms, s);
  else if (variant == 3) TileLayout<ND, EU, PRIM, 32, S::TY, S::M3>::launch_batched(args, tiles, ntiles, sms, s);
  else TileLayout<ND, EU, PRIM, 32, S::TY, 1>::launch_batched(args, tiles, ntiles, sms, s);
}

template <int ND>
cudaError_t launch_nd(bool euler, bool prim, int variant, const Grid& g, int kchunk, cudaStream_t s,
                      const StageArgs& A) {
  if (euler) prim ? launch_t<ND, true, true>(variant, g, kchunk, s, A) : launch_t<ND, true, false>(variant, g, kchunk, s, A);
  else prim ? launch_t<ND, false, true>(variant, g, kchunk, s, A) : launch_t<ND, false, false>(variant, g, kchunk, s, A);
  return cudaGetLastError();
}

template <int ND>
cudaError_t batched_nd(bool euler, bool prim, int variant, const StageArgs* args, const int4* tiles, int ntiles,
                       int sms, cudaStream_t s) {
  if (euler) {
    if (prim) batched_t<ND, true, true>(variant, args, tiles, ntiles, sms, s);
    else batched_t<ND, true, false>(variant, args, tiles, ntiles, sms, s);
  } else {
    if (prim) batched_t<ND, false, true>(variant, args, tiles, ntiles, sms, s);
    else batched_t<ND, false, false>(variant, args, tiles, ntiles, sms, s);
  }
  return cudaGetLastError();
}

template <int ND>
void configure_nd(bool euler, bool prim) {
  if (euler) prim ? configure_t<ND, true, true>() : configure_t<ND, true, false>();
  else prim ? configure_t<ND, false, true>() : configure_t<ND, false, false>();
}

}  // namespace
}  // namespace fgpu
