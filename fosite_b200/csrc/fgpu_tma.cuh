// fgpu_tma.cuh -- stage kernel with TMA-staged halo planes (sm_100a).
//
// Same right-hand side and epilogues as stage_tile (fgpu_kernels.cuh: fosite's ComputeRHS,
// timedisc_base.f90:1073-1271, fused with its consumer), laid out for the Blackwell memory
// system:
//   * every x-y plane of a tile, halo included, arrives in shared memory by one bulk tensor
//     copy (cp.async.bulk.tensor, 4-D map x, y, z, variable) completing on an mbarrier;
//     a 3D tile marches along z with a ring of three plane slots, the copy of plane k+3
//     issued while plane k is computed, so the stencil reads each cell from HBM once per
//     stage and never waits on a load in its inner phases; a 2D block computes a column of
//     tiles with two box slots, the copy of the next tile in flight while one is computed,
//     and reduces its CFL / error maxima once for the column;
//   * interior tiles need no boundary logic at all; tiles touching an x or y face fill
//     their ghost cells once per plane in shared memory (CenterBoundary rules,
//     boundary_generic.f90:287-418), the z ghosts of the own column come from the same
//     rules;
//   * the own column's z neighbours come from the ring (planes k, k+1) and a register
//     lookahead (plane k+2, loaded one plane early); its z slope and flux are computed after
//     the plane's x-y fluxes, right before the epilogue that consumes them;
//   * stages that reduce nothing (no CFL, CheckData or error norm) run a form of the kernel
//     whose maxima are compiled out: registers decide the speed of this kernel;
//   * the epilogue's streams (base and earlier k of a Butcher stage, the Shu-Osher start
//     state) are brought into L2 one plane ahead by bulk prefetches, one tile row per thread;
//   * the x and y interface fluxes run in warp-sized chunks of one direction each, so that
//     the flux code is specialised for its direction; the common limiters (minmod, MC with
//     theta = 1, van Leer) are compiled in.
// Requirements (checked on the host): even nx (16-byte strides of the tensor map), no
// viscous source, no accretion rows, a plain or formed stage input (no k-sums in the
// stencil).  FARGO frame changes (2D) are applied where the staged points are converted.
#pragma once
#include <cuda.h>
#include <type_traits>
#include "fgpu_kernels.cuh"

namespace fgpu {

// ------------------------------------------------------------------ PTX wrappers
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count) : "memory");
}
// orders this thread's generic-proxy shared-memory accesses with later async-proxy ones
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned long long* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for phase `parity` of an mbarrier, for at most about two seconds of SM clock;
// false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, unsigned parity) {
  if (mbar_test(b, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_test(b, parity))
    if (clock64() - t0 > 4000000000LL) return false;
  return true;
}
// bulk tensor copy of one box (coordinates x, y, z; the variable coordinate 0) into shared
// memory, completing on the mbarrier; RANK 4 (x, y, z, var) or 3 (x, y, var)
template <int RANK>
__device__ __forceinline__ void tma_load_box(void* dst, const CUtensorMap* map, unsigned long long* bar, int x, int y,
                                             int z) {
  if (RANK == 4)
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(smem_addr(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(0), "r"(smem_addr(bar))
        : "memory");
  else
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_addr(dst)),
        "l"(map), "r"(x), "r"(y), "r"(0), "r"(smem_addr(bar))
        : "memory");
}
// L2 prefetch of `bytes` contiguous bytes (16-byte aligned address, multiple of 16 bytes)
__device__ __forceinline__ void bulk_prefetch_l2(const void* p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// ------------------------------------------------------------------ layout
// Shared memory of one TMA tile: NSLOT staged planes [V][TY+4][TX+4] (the box of one tensor
// copy, 128-byte aligned), the x and y slopes and interface fluxes, NSLOT mbarriers.
template <int V, int TX, int TY, int NSLOT>
struct TmaLayout {
  static constexpr int RW = TX + 4, RH = TY + 4;
  static constexpr int PLANE = V * RH * RW;
  static constexpr unsigned PLANE_BYTES = 8u * PLANE;
  static constexpr int NSX = V * TY * (TX + 2), NSY = V * (TY + 2) * TX;
  static constexpr int NFX = V * TY * (TX + 1), NFY = V * (TY + 1) * TX;
  static constexpr size_t SMEM = 8 * ((size_t)NSLOT * PLANE + NSX + NSY + NFX + NFY + NSLOT);
  static_assert(PLANE_BYTES % 128 == 0, "plane slots must stay 128-byte aligned");
};
// plane slots: a 3D tile's ring of three z planes; a 2D block's two boxes (the tile being
// computed and the next tile of its column, whose copy is in flight)
template <int ND> struct TmaSlots { static constexpr int N = ND == 3 ? 3 : 2; };

// ------------------------------------------------------------------ the tile
// LIM > 0: the limiter is compiled in (linear reconstruction with that limiter); LIM = 0: the
// limiter and the reconstruction order are read from the arguments.  NT threads (at least
// TX * TY; thread t owns cell (t % TX, t / TX) of the tile when t < TX * TY, the others share
// the halo, slope and flux items).  RED = false: a stage without CFL, CheckData or error-norm
// reduction (cfl_mode 0, not the last stage, no err_low), whose maxima are then dead code and
// hold no registers across the planes.
template <int ND, bool EU, bool PRIM, int TX, int TY, int LIM, int NT = TX * TY, bool RED = true>
__device__ __forceinline__ void tma_stage_tile(const StageArgs& A, const CUtensorMap* tmap, const int bx, const int by,
                                               const int bz) {
  using PH = Phys<ND, EU>;
  using CE = Cells<ND, EU>;
  constexpr int V = PH::V;
  static_assert(NT >= TX * TY && NT % 32 == 0, "every cell of the tile needs a thread");
  constexpr int NSLOT = TmaSlots<ND>::N;
  using L = TmaLayout<V, TX, TY, NSLOT>;
  constexpr int RW = L::RW, RHW = L::RH * L::RW;
  // dynamic shared memory, 128-byte aligned (the plane slots are tensor-copy destinations);
  // every pointer below is an offset from the shared array, so accesses stay shared-space
  extern __shared__ __align__(128) double tma_smem_raw[];
  double* const ring = tma_smem_raw;
  double* const Sx = ring + NSLOT * L::PLANE;   // [V][TY][TX+2]
  double* const Sy = Sx + L::NSX;               // [V][TY+2][TX]
  double* const Fx = Sy + L::NSY;               // [V][TY][TX+1]
  double* const Fy = Fx + L::NFX;               // [V][TY+1][TX]
  unsigned long long* const mbar = reinterpret_cast<unsigned long long*>(Fy + L::NFY);
  __shared__ double sred[RED_STRIDE * ((NT + 31) / 32)];
  __shared__ int abort_flag;

  if (A.ctl && (A.ctl->stop | A.ctl->brk)) return;
  if (gated_out(A.ctl, A.gate)) return;
  const Grid& g = A.g;
  const PhysP& P = A.ph;
  const MetricP& M = A.mt;
  const double dt = A.dt_dev ? *A.dt_dev : A.dt;
  const bool roundtrip = EU && A.in.roundtrip;
  const StateRef& SR = A.rin.base ? A.rin : A.in;
  const int lim = LIM > 0 ? LIM : A.limiter;
  const bool crec = LIM > 0 ? false : A.constant_recon != 0;   // constant reconstruction (no slopes)
  // FARGO (2D): the stage input's frame changes (the chain of the stored state) and the
  // subtraction of the background velocity apply to every staged point
  constexpr bool FG = ND == 2;
  const bool frames = FG && (A.w_sub != nullptr || A.in.pre.n != 0);
  // the staged values are the reconstruction variables as they stand (a formed primitive
  // stage state, or a conservative state without the CHECK_PMIN round trip or frame
  // changes), else every staged point is converted once
  const bool raw_ok = PRIM ? (SR.ready != 0) : (!roundtrip && !frames);
  const int tid = threadIdx.x;
  const int tx = tid % TX, ty = tid / TX;
  const int i0 = bx * TX;
  const int ex = min(TX, g.nx - i0);
  const int i = i0 + tx;
  const int ip = i + 2;
  // 3D: planes k0 .. k1-1 of the tile (bx, by); 2D: the block computes tiles jb0 .. jb0+k1-1 of
  // column bx (by counts blocks of A.kchunk tiles), "plane" kp being tile jb0 + kp
  int k0 = 0, k1 = 1, jb0 = by;
  if (ND == 3) {
    k0 = bz * A.kchunk;
    k1 = min(g.nz, k0 + A.kchunk);
  } else {
    jb0 = by * A.kchunk;
    k1 = min(A.kchunk, (g.ny + TY - 1) / TY - jb0);
  }
  auto tile_j0 = [&](int kp) { return ND == 3 ? by * TY : (jb0 + kp) * TY; };
  int j0 = tile_j0(k0), ey = min(TY, g.ny - j0);
  bool own = tx < ex && ty < ey;
  int j = j0 + ty;
  // the tile's staged box reaches ghost cells of an x or y face
  bool xy_ghosts = i0 == 0 || i0 + ex + 2 > g.nx || j0 == 0 || j0 + ey + 2 > g.ny;
  bool prep_sync = !raw_ok || xy_ghosts;
  auto set_tile = [&](int kp) {   // 2D: the block's current tile becomes tile jb0 + kp
    j0 = tile_j0(kp);
    ey = min(TY, g.ny - j0);
    own = tx < ex && ty < ey;
    j = j0 + ty;
    xy_ghosts = i0 == 0 || i0 + ex + 2 > g.nx || j0 == 0 || j0 + ey + 2 > g.ny;
    prep_sync = !raw_ok || xy_ghosts;
  };

  // reconstruction variables of a raw staged value of cell (gi, gj) (in place), and of a face
  // ghost; with FARGO the stored state's frame chain first, the co-moving frame last (the
  // order of ComputeRHS: AddBackgroundVelocity, CenterBoundary, SubtractBackgroundVelocity)
  auto conv = [&](double* u, int gi, int gj) {
    if (FG && A.in.pre.n) apply_chain<V>(A.in.pre, u, g, gi, gj);
    if (PRIM) {
      double p[V];
      PH::c2p(u, p, P);
      if (roundtrip) p[V - 1] = dmax(p[V - 1], P.pmin);
      if (FG && A.w_sub) sub_velocity(p, A.w_sub[fargo_ix(g, gi, gj)], g.fdir);
#pragma unroll
      for (int v = 0; v < V; ++v) u[v] = p[v];
    } else {
      if (roundtrip) {
        double p[V];
        PH::c2p(u, p, P);
        p[V - 1] = dmax(p[V - 1], P.pmin);
        PH::p2c(p, u, P);
      }
      if (FG && A.w_sub) frame_change<V>(u, -1.0, A.w_sub[fargo_ix(g, gi, gj)], g.fdir);
    }
  };
  auto ghost = [&](int d, int gi, int gj, int gk, double* R) {
    double p[V];
    CE::face_ghost_p(SR, g, P, M, d, gi, gj, gk, p);
    if (roundtrip) p[V - 1] = dmax(p[V - 1], P.pmin);
    if (PRIM) {
      if (FG && A.w_sub) sub_velocity(p, A.w_sub[fargo_ix(g, gi, gj)], g.fdir);
#pragma unroll
      for (int v = 0; v < V; ++v) R[v] = p[v];
    } else {
      PH::p2c(p, R, P);
      if (FG && A.w_sub) frame_change<V>(R, -1.0, A.w_sub[fargo_ix(g, gi, gj)], g.fdir);
    }
  };
  // A face ghost of a staged plane from its mirror cell in the same box, for the boundaries
  // whose ghosts copy an interior cell (reflecting, axis, no gradients; boundary_reflecting.f90:
  // 89-204, boundary_axis.f90, boundary_nogradients.f90:75-125) while the staged values are the
  // reconstruction variables: the arithmetic of face_ghost_p on the same values, no global
  // load.  False when the face has another rule or the mirror cell lies outside the box.
  auto box_ghost = [&](const double* S, int d, int lx, int ly, int gi, int gj, double* R) -> bool {
    if (!raw_ok) return false;
    const int x = d == 0 ? gi : gj, nd = d == 0 ? g.nx : g.ny;
    const bool lo = x < 0;
    const int type = g.bc[2 * d + (lo ? 0 : 1)];
    if (type != BC_REFLECTING && type != BC_AXIS && type != BC_NOGRAD) return false;
    const int sdep = lo ? -x : x - (nd - 1);
    const int mirror = type == BC_NOGRAD ? (lo ? 0 : nd - 1) : (lo ? sdep - 1 : nd - sdep);
    const int lm = mirror - (d == 0 ? i0 : j0) + 2;   // the mirror's box coordinate along d
    if (lm < 2 || lm > (d == 0 ? ex : ey) + 1) return false;
    const double* src = S + (d == 0 ? ly * RW + lm : lm * RW + lx);
    double p[V];
    if (PRIM) {
#pragma unroll
      for (int v = 0; v < V; ++v) p[v] = src[v * RHW];
    } else {
      double u[V];
#pragma unroll
      for (int v = 0; v < V; ++v) u[v] = src[v * RHW];
      PH::c2p(u, p, P);
    }
    if (type != BC_NOGRAD) {
      if (d == 0) p[1] = -p[1];
      else p[2] = -p[2];
      if (type == BC_AXIS && d == 0 && M.curv) p[2] = -p[2];
    }
    if (roundtrip) p[V - 1] = dmax(p[V - 1], P.pmin);
    if (PRIM) {
#pragma unroll
      for (int v = 0; v < V; ++v) R[v] = p[v];
    } else {
      PH::p2c(p, R, P);
    }
    return true;
  };
  // own column at plane gk: raw loads (interior planes), then the reconstruction variables
  auto col_load = [&](int gk, double* u) {
    if (gk >= 0 && gk < g.nz) {
      const double* b = SR.base + CE::lin(g, i, j, gk);
#pragma unroll
      for (int v = 0; v < V; ++v) u[v] = __ldg(b + (long long)v * g.n);
    }
  };
  auto col_finish = [&](int gk, double* u) {
    if (gk < 0 || gk >= g.nz) ghost(2, i, j, gk, u);
    else if (!raw_ok) conv(u, i, j);
  };

  auto slot = [&](int kp) { return ring + ((kp - k0) % NSLOT) * L::PLANE; };
  auto issue = [&](int kp) {   // one thread: the tensor copy of plane kp's box into its slot
    unsigned long long* b = &mbar[(kp - k0) % NSLOT];
    mbar_expect_tx(b, L::PLANE_BYTES);
    tma_load_box<ND + 1>(slot(kp), tmap, b, i0 - 2, tile_j0(kp) - 2, ND == 3 ? kp : 0);
  };
  // planes k0 .. k1-1 are staged by tensor copies (the first NSLOT now, then plane
  // k+NSLOT-1 once every thread is past plane k-1); 3D: the own column of planes k1, k1+1
  // comes from the lookahead
  if (tid == 0) {
    abort_flag = 0;
    for (int s = 0; s < NSLOT; ++s) mbar_init(&mbar[s], 1);
    fence_proxy_async();
    for (int kp = k0; kp < min(k1, k0 + NSLOT); ++kp) issue(kp);
  }
  __syncthreads();

  // wait for plane kp's copy, then fill its ghost cells / convert its raw values in place
  int waited = 0;   // thread 0: planes k0 .. k0+waited-1 seen complete (or given up on)
  auto prepare = [&](int kp) {
    if (kp >= k1) {   // own column only (the next chunk's plane or a z ghost)
      if (own) {
        double u[V];
        col_load(kp, u);
        col_finish(kp, u);
        double* S = slot(kp);
#pragma unroll
        for (int v = 0; v < V; ++v) S[v * RHW + (ty + 2) * RW + tx + 2] = u[v];
      }
      return;
    }
    if (!mbar_wait(&mbar[(kp - k0) % NSLOT], (unsigned)(((kp - k0) / NSLOT) & 1))) abort_flag = 1;
    if (tid == 0) waited = kp + 1 - k0;
    if (prep_sync) {
      double* S = slot(kp);

      constexpr int NXB = (TX + 4) * TY, NYB = TX * 4;
      for (int t = tid; t < NXB + NYB; t += NT) {
        int lx, ly;
        if (t < NXB) {
          lx = t % (TX + 4);
          ly = 2 + t / (TX + 4);
          if (lx >= ex + 4 || ly >= ey + 2) continue;
        } else {
          const int u = t - NXB, q = u / TX;
          lx = 2 + u % TX;
          ly = q < 2 ? q : ey + q;
          if (lx >= ex + 2) continue;
        }
        const int gi = i0 + lx - 2, gj = j0 + ly - 2;
        const bool gx = gi < 0 || gi >= g.nx, gy = gj < 0 || gj >= g.ny;
        if (gx || gy || !raw_ok) {
          double R[V];
          if (gx || gy) {
            if (!box_ghost(S, gx ? 0 : 1, lx, ly, gi, gj, R)) ghost(gx ? 0 : 1, gi, gj, ND == 3 ? kp : 0, R);
          } else {
#pragma unroll
            for (int v = 0; v < V; ++v) R[v] = S[v * RHW + ly * RW + lx];
            conv(R, gi, gj);
          }
#pragma unroll
          for (int v = 0; v < V; ++v) S[v * RHW + ly * RW + lx] = R[v];
        }
      }
      fence_proxy_async();
      __syncthreads();
    }
  };

  // epilogue streams of plane kp brought into L2 (one bulk prefetch per tile row, spread over
  // the block): stream q < nf: the next Butcher stage's base and earlier k; then the stage
  // input's base and k (the last stage's high/low-order sums, or cvar read by the sources);
  // y0; err_low
  const int nf = A.fnext_out ? A.fnext.nk : 0;
  const bool in_needed = A.last_stage || (PRIM && !roundtrip && (M.curv || A.has_accel || A.out_base ||
                                                                 A.out_mode == OUT_SSPRK)) ||
                         (!PRIM && roundtrip);
  const int nin = !in_needed ? 0 : (A.last_stage ? A.nstage : A.in.nk + 1);
  const int nstreams = nf + nin + (A.out_mode == OUT_SSPRK ? 1 : 0) + (A.err_low ? 1 : 0);
  auto stream = [&](int q) -> const double* {
    if (q < nf) return q == 0 ? A.fnext.base : A.fnext.K[q - 1];
    q -= nf;
    if (q < nin) return q == 0 ? A.in.base : A.in.K[q - 1];
    q -= nin;
    if (A.out_mode == OUT_SSPRK) {
      if (q == 0) return A.y0;
      q -= 1;
    }
    return A.err_low;
  };
  auto prefetch_epilogue = [&](int kp) {
    if (kp >= k1) return;
    const int rows = TY * V * nstreams;
    const int pj0 = tile_j0(kp), pey = min(TY, g.ny - pj0), pk = ND == 3 ? kp : 0;
    for (int r = tid; r < rows; r += NT) {
      const int jr = r % TY, vq = r / TY, v = vq % V, q = vq / V;
      if (jr < pey) bulk_prefetch_l2(stream(q) + (long long)v * g.n + CE::lin(g, i0, pj0 + jr, pk), 8u * ex);
    }
  };

  double cflv[4] = {0.0, 0.0, 0.0, 0.0};
  double errv = 0.0;
  int flags = 0;
  int issued = min(k1, k0 + NSLOT) - k0;   // thread 0: planes k0 .. k0+issued-1 copied

  // z state of the own column (3D): lookahead raw values of plane k+2, z slope at k, z flux at k-1/2
  double la[V], sz0[V], Fzm[V];
  if (ND == 3) {
    prepare(k0);
    if (own) {
      double Ra[V], Rb[V], Rc[V], Rd[V];
      col_load(k0 - 2, Ra);
      col_load(k0 - 1, Rb);
      col_load(k0 + 1, Rd);
      col_finish(k0 - 2, Ra);
      col_finish(k0 - 1, Rb);
      col_finish(k0 + 1, Rd);
      const double* S0 = slot(k0);
#pragma unroll
      for (int v = 0; v < V; ++v) Rc[v] = S0[v * RHW + (ty + 2) * RW + tx + 2];
      double szm[V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        szm[v] = crec ? 0.0 : slope(lim, A.theta, A.invd[2], Ra[v], Rb[v], Rc[v]);
        sz0[v] = crec ? 0.0 : slope(lim, A.theta, A.invd[2], Rb[v], Rc[v], Rd[v]);
      }
      double RL[V], RR[V];
      const double oT = M.offzT[k0 - 1 + 2], oB = M.offzB[k0 + 2];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        RL[v] = crec ? Rb[v] : Rb[v] + szm[v] * oT;
        RR[v] = crec ? Rc[v] : Rc[v] + sz0[v] * oB;
      }
      kt_flux<ND, EU, PRIM, 2>(2, RL, RR, EU ? 0.0 : M.cs[6 * M.nxp + ip], EU ? 0.0 : M.cs[5 * M.nxp + ip],
                               M.dAzB[ip], P, Fzm);
      col_load(k0 + 2, la);
    }
  }
  prefetch_epilogue(k0);

  bool aborted = false;
  constexpr int NSXI = TY * (TX + 2), NSYI = (TY + 2) * TX;   // slope items (x, y)
  constexpr int NFXI = TY * (TX + 1), NFYI = (TY + 1) * TX;   // interface-flux items (x, y)
  for (int k = k0; k < k1; ++k) {
    const double* S = slot(k);
    const int oc = (ty + 2) * RW + tx + 2;   // the own cell in a staged plane
    if (ND == 3) {
      prepare(k + 1);
    } else {
      set_tile(k);
      prepare(k);
    }
    // ---- x and y slopes of plane k: items over the full tile shape (ey rows x ex+2 cells for x,
    // ey+2 rows x ex cells for y), one code path for both directions, the ones outside a
    // partial edge tile skipped
    if (!crec) {
      for (int t = tid; t < NSXI + NSYI; t += NT) {
        int cidx, step, sidx, sstride;
        double* Sout;
        double invd;
        if (t < NSXI) {
          const int r = t / (TX + 2), c = t % (TX + 2) - 1;
          if (r >= ey || c > ex) continue;
          cidx = (r + 2) * RW + (c + 2); step = 1;
          Sout = Sx; sidx = r * (TX + 2) + (c + 1); sstride = TY * (TX + 2);
          invd = A.invd[0];
        } else {
          const int u = t - NSXI;
          const int c = u % TX, r = u / TX - 1;
          if (c >= ex || r > ey) continue;
          cidx = (r + 2) * RW + (c + 2); step = RW;
          Sout = Sy; sidx = (r + 1) * TX + c; sstride = (TY + 2) * TX;
          invd = A.invd[1];
        }
#pragma unroll
        for (int v = 0; v < V; ++v) {
          const double* R = S + v * RHW + cidx;
          Sout[v * sstride + sidx] = slope(lim, A.theta, invd, R[-step], R[0], R[step]);
        }
      }
    }
    __syncthreads();
    // every thread is past plane k-1's epilogue: its slot takes plane k+NSLOT-1
    if (tid == 0 && k >= k0 + 1 && k + NSLOT - 1 < k1) { issue(k + NSLOT - 1); ++issued; }
    // ---- x and y interface fluxes of plane k: warp-sized chunks of items, each chunk of one
    // direction, so that the direction is a compile-time constant of the flux code
    auto xy_flux = [&](auto dir, int t) {
      constexpr int D = decltype(dir)::value;
      double RL[V], RR[V], F[V];
      int lidx, ridx, sL, sR, sstride, fstride;
      const double* Sl;
      double* Fout;
      double oL, oR, csL, csR, dA;
      if (D == 0) {
        const int r = t / (TX + 1), f = t % (TX + 1);
        if (r >= ey || f > ex) return;
        const int gl = i0 + f - 1 + 2;   // padded i of the left cell
        oL = M.offxE[gl]; oR = M.offxW[gl + 1];
        lidx = (r + 2) * RW + (f + 1); ridx = lidx + 1;
        Sl = Sx; sL = r * (TX + 2) + f; sR = sL + 1; sstride = TY * (TX + 2);
        csL = EU ? 0.0 : M.cs[2 * M.nxp + gl]; csR = EU ? 0.0 : M.cs[1 * M.nxp + gl + 1];
        dA = M.dAxW[gl + 1];
        Fout = Fx + r * (TX + 1) + f; fstride = TY * (TX + 1);
      } else {
        const int c = t % TX, f = t / TX;
        if (c >= ex || f > ey) return;
        const int gjl = j0 + f - 1 + 2, gi = i0 + c + 2;
        oL = M.offyN[gjl]; oR = M.offyS[gjl + 1];
        lidx = (f + 1) * RW + (c + 2); ridx = lidx + RW;
        Sl = Sy; sL = f * TX + c; sR = sL + TX; sstride = (TY + 2) * TX;
        csL = EU ? 0.0 : M.cs[4 * M.nxp + gi]; csR = EU ? 0.0 : M.cs[3 * M.nxp + gi];
        dA = M.dAyS[gi];
        Fout = Fy + f * TX + c; fstride = (TY + 1) * TX;
      }
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const double rl = S[v * RHW + lidx], rr = S[v * RHW + ridx];
        RL[v] = crec ? rl : rl + Sl[v * sstride + sL] * oL;
        RR[v] = crec ? rr : rr + Sl[v * sstride + sR] * oR;
      }
      kt_flux<ND, EU, PRIM, D>(D, RL, RR, csL, csR, dA, P, F);
#pragma unroll
      for (int v = 0; v < V; ++v) Fout[v * fstride] = F[v];
    };
    {
      constexpr int CX = (NFXI + 31) / 32, CY = (NFYI + 31) / 32;
      const int warp = tid >> 5, lane = tid & 31;
      for (int c = warp; c < CX + CY; c += NT / 32) {
        if (c < CX) {
          const int t = c * 32 + lane;
          if (t < NFXI) xy_flux(std::integral_constant<int, 0>(), t);
        } else {
          const int t = (c - CX) * 32 + lane;
          if (t < NFYI) xy_flux(std::integral_constant<int, 1>(), t);
        }
      }
    }
    __syncthreads();
    if (abort_flag) { aborted = true; break; }   // block-uniform: read after the barrier
    prefetch_epilogue(k + 1);
    double divZ[V];
    // ---- z: slope at k+1 and the flux at k+1/2 of the own column (planes k, k+1 staged, k+2
    // from the lookahead, whose registers then take plane k+3's raw values), computed after
    // the x-y fluxes so that divZ is live only into the epilogue (5% on the 3D stage)
    if (ND == 3 && own) {
      const double* S1 = slot(k + 1);
      col_finish(k + 2, la);
      double sz1[V], RL[V], RR[V], Fzp[V];
      const double oT = M.offzT[k + 2], oB = M.offzB[k + 1 + 2];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const double r0 = S[v * RHW + oc], r1 = S1[v * RHW + oc];
        sz1[v] = crec ? 0.0 : slope(lim, A.theta, A.invd[2], r0, r1, la[v]);
        RL[v] = crec ? r0 : r0 + sz0[v] * oT;
        RR[v] = crec ? r1 : r1 + sz1[v] * oB;
      }
      col_load(k + 3, la);
      kt_flux<ND, EU, PRIM, 2>(2, RL, RR, EU ? 0.0 : M.cs[6 * M.nxp + ip], EU ? 0.0 : M.cs[5 * M.nxp + ip],
                               M.dAzB[ip], P, Fzp);
      const double dVz = M.dxdydV[ip];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        divZ[v] = dVz * (Fzp[v] - Fzm[v]);
        Fzm[v] = Fzp[v];
        sz0[v] = sz1[v];
      }
    }
    // ---- divergence, sources and the stage's consumer (no barrier after it: the slot of
    // plane k is next written after the following plane's slope barrier)
    if (own) {
      double rhs[V], R0[V];
      const double dVx = M.dydzdV[ip], dVy = M.dzdxdV[ip];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const double divX = dVx * (Fx[(v * TY + ty) * (TX + 1) + tx + 1] - Fx[(v * TY + ty) * (TX + 1) + tx]);
        const double divY = dVy * (Fy[(v * (TY + 1) + ty + 1) * TX + tx] - Fy[(v * (TY + 1) + ty) * TX + tx]);
        rhs[v] = (divX + divY) + (ND == 3 ? divZ[v] : 0.0);
        R0[v] = S[v * RHW + oc];
      }
      stage_cell_epilogue<ND, EU, PRIM, ND == 3>(A, i, j, ND == 3 ? k : 0, R0, rhs, dt, cflv, errv, flags);
    }
  }

  if (aborted) {
    // a copy did not complete in time: report it, give the copies still in flight their
    // (bounded) time to land in this block's shared memory, leave
    if (tid == 0) {
      if (A.ctl) atomicOr(&A.ctl->dev_err, 1);
      for (int kp = k0 + waited; kp < k0 + issued; ++kp)
        mbar_wait(&mbar[(kp - k0) % NSLOT], (unsigned)(((kp - k0) / NSLOT) & 1));
    }
    __syncthreads();
    return;
  }
  const bool err_out = A.last_stage || A.err_low;
  if (RED && A.ctl && (A.cfl_mode || err_out)) {
    int nv = A.cfl_mode ? (M.vis ? 4 : (ND == 3 ? 3 : 1)) : 0;
    double vals[4] = {cflv[0], cflv[1], cflv[2], cflv[3]};
    if (err_out && !A.cfl_mode) { vals[0] = errv; nv = 1; }
    if (nv) block_reduce_emit<NT>(vals, nv, flags, err_out && !A.cfl_mode ? &A.ctl->err : A.ctl->invdt,
                                  &A.ctl->flags, sred);
  }
}

template <int ND, bool EU, bool PRIM, int TX, int TY, int MINB, int LIM, int NT = TX * TY, bool RED = true>
__global__ void __launch_bounds__(NT, MINB)
    tma_stage_kernel(const __grid_constant__ StageArgs A, const __grid_constant__ CUtensorMap tmap) {
  tma_stage_tile<ND, EU, PRIM, TX, TY, LIM, NT, RED>(A, &tmap, blockIdx.x, blockIdx.y, blockIdx.z);
}

// Batched ensemble on the TMA layout: one block per entry of the flattened queue of many
// independent grids, entry (grid, bx, byb, 0) the column of kchunk tiles that a block of the
// single-grid kernel computes; args[grid] are the grid's stage arguments and maps[grid] the
// tensor map of its stage input (global memory, 64-byte aligned, written by the host before
// the launch).
template <int ND, bool EU, bool PRIM, int TX, int TY, int MINB, int LIM, int NT = TX * TY, bool RED = true>
__global__ void __launch_bounds__(NT, MINB)
    batched_tma_stage_kernel(const StageArgs* __restrict__ args, const CUtensorMap* __restrict__ maps,
                             const int4* __restrict__ tiles) {
  // the grid's arguments are copied into shared memory once per block: the tile then reads
  // them at fixed shared offsets instead of through global-memory address arithmetic
  __shared__ StageArgs sA;
  static_assert(sizeof(StageArgs) % 8 == 0, "argument copy by 8-byte words");
  const int4 T = tiles[blockIdx.x];
  const CUtensorMap* map = maps + T.x;
  if (threadIdx.x == 0)
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
  {
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(args + T.x);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sA);
    for (int w = threadIdx.x; w < (int)(sizeof(StageArgs) / 8); w += NT) dst[w] = __ldg(src + w);
  }
  __syncthreads();
  tma_stage_tile<ND, EU, PRIM, TX, TY, LIM, NT, RED>(sA, map, T.y, T.z, T.w);
}

}  // namespace fgpu
