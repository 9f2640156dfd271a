// fgpu_kernels.cuh -- fused stage kernel and the boundary / reduction kernels.
//
// One launch of stage_kernel is one right-hand-side evaluation of fosite's
// ComputeRHS (timedisc_base.f90:1073-1271) fused with what consumes it:
//   * the stage input state is formed on the fly (base - sum coef*K), so the
//     Butcher stages of timedisc_rkfehlberg.f90:170-302 read their k-arrays
//     once and never materialise ctmp;
//   * ghost cells are synthesised in the tile loader (no ghost-fill pass);
//   * reconstruction (reconstruction_linear.f90:215-630), KT fluxes
//     (fluxes_kt.f90:109-208), flux divergence and geometric / point-mass
//     sources are computed per tile in shared memory;
//   * the result is either written as k_m (Butcher engine) or consumed by the
//     Shu-Osher update of timedisc_modeuler.f90:279-291;
//   * epilogues: CFL maximum (CalcTimestep), CheckData flags, the embedded
//     error norm (ComputeError) and the high-order solution.
// 2D meshes use one x-y tile per block; 3D meshes march a 2.5D x-y tile
// along z so each plane is loaded once.
#pragma once
#include "fgpu_device.cuh"

namespace fgpu {

enum { OUT_RHS = 0, OUT_SSPRK = 1 };

struct StageArgs {
  Grid g;
  PhysP ph;
  MetricP mt;
  StateRef in;
  int limiter;
  double theta;
  int constant_recon;
  double invd[3];
  int has_accel;
  int out_mode;
  double* out;             // k_m (OUT_RHS) or the new state (OUT_SSPRK)
  const double* y0;        // OUT_SSPRK: state at the start of the step (cold)
  int y0_roundtrip;        // cold is the CHECK_PMIN round trip of y0
  double eta;
  const double* dt_dev;    // device-resident dt, or null to use dt
  double dt;
  double* out_base;        // optional: write the (round-tripped) input state
  // Butcher last stage: high/low order combination and error norm
  int last_stage;
  int nstage;
  double bh_dt[FGPU_MAXK], bl_dt[FGPU_MAXK];
  double* out_high;
  double tol_rel;
  double tol_abs[FGPU_MAXV];
  // CFL/CheckData epilogue: 0 none, 1 on the OUT_SSPRK result, 2 on the input state, 3 CheckData
  // of the input state only (AcceptSolution's ComputeRHS inside a step)
  int cfl_mode;
  int cfl_roundtrip;       // the checked state gets the CHECK_PMIN round trip
  int checkdata;
  Ctl* ctl;
  int kchunk;
  // FARGO (2D isothermal): co-moving frame of the fluxes (SubtractBackgroundVelocityY after the
  // sources) and the Shu-Osher base states as chains of frame changes of the stored states
  const double* w_sub;
  Chain yn_chain, y0_chain;
  // adaptive modified Euler: a second Shu-Osher result from the same RHS,
  // out2 = yn - dt*rhs + eta2*(y0 - yn + dt*rhs) (the embedded lower-order solution,
  // timedisc_modeuler.f90:163-192), and the error norm of the new state against
  // err_low (ComputeError, timedisc_base.f90:1012-1053) reduced into ctl->err
  double* out2;
  double eta2;
  // Shu-Osher stage followed by another (primitive reconstruction): the new state's
  // primitive variables, which the next stage's stencil reads ready-made (its rin, ready = 1)
  // instead of converting every staged point; null = off
  double* out_prim;
  const double* err_low;
  Chain err_chain;         // FARGO: frame changes of err_low before the comparison
  // point-mass accretion: the boundary row of this RHS through the outbound x face,
  // (dy*dz)*xflux of the density (face 0 west) or -(dy*dz)*xflux (face 1 east), by j
  double* brow;
  int brow_face;
  double bdydz;
  // optional: the stage's reconstruction variables formed once per cell by form_kernel
  // (rin.ready = 1 for primitive reconstruction); the stencil then reads these instead of
  // forming base - sum coef*K and converting at every stencil point.  in stays the
  // stage state for the epilogues.
  StateRef rin;
  // optional: viscous source of the stage state, [ND momentum (+ energy)][n] (visc_kernel)
  const double* visc;
  // device-clock attempt slots: run only if the slot's actions include a gate bit
  int gate;
  // optional (Butcher stage m < M, OUT_RHS): the next stage's state (base and k_1..k_m, the
  // last being this stage's output) formed into fnext_out as its reconstruction variables
  StateRef fnext;
  double* fnext_out;
  // optional: the interface fluxes of this right-hand side, [3 directions][V][padded cells]
  // in fosite's xfluxdydz/yfluxdzdx/zfluxdxdy indexing (face between cells i and i+1 at i)
  double* flux_out;
};

// padded index of interior cell (i, j, k) (ghost layers of 2 in every active direction)
__device__ __forceinline__ long long padded_index(const Grid& g, int i, int j, int k, int nd) {
  const long long NXp = g.nx + 4, NYp = g.ny + 4;
  return (i + 2) + NXp * ((j + 2) + NYp * (long long)(nd == 3 ? k + 2 : 0));
}
// store F (V values) as the flux of direction d at the face after padded cell pc
template <int V>
__device__ __forceinline__ void store_flux(const StageArgs& A, int d, long long pc, long long npad, const double* F) {
#pragma unroll
  for (int v = 0; v < V; ++v) A.flux_out[((long long)d * V + v) * npad + pc] = F[v];
}

// block-wide max of up to 4 non-negative doubles + OR of flags, then one atomic per block;
// sred holds RED_STRIDE doubles per warp
constexpr int RED_STRIDE = 5;
template <int NT>
__device__ __forceinline__ void block_reduce_emit(double* vals, int nv, int flags, unsigned long long* dst,
                                                  int* dflags, double* sred) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int q = 0; q < nv; ++q) {
    double x = vals[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = dmax(x, __shfl_xor_sync(0xffffffffu, x, o));
    vals[q] = x;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) flags |= __shfl_xor_sync(0xffffffffu, flags, o);
  __syncthreads();
  if (lane == 0) {
    for (int q = 0; q < nv; ++q) sred[warp * RED_STRIDE + q] = vals[q];
    sred[warp * RED_STRIDE + 4] = __longlong_as_double((long long)flags);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    constexpr int NW = (NT + 31) / 32;
    int f = 0;
    for (int q = 0; q < nv; ++q) {
      double m = 0.0;
      for (int w = 0; w < NW; ++w) m = dmax(m, sred[w * RED_STRIDE + q]);
      if (dst) atomicMax(dst + q, (unsigned long long)__double_as_longlong(m));
    }
    for (int w = 0; w < NW; ++w) f |= (int)__double_as_longlong(sred[w * RED_STRIDE + 4]);
    if (f && dflags) atomicOr(dflags, f);
  }
}

// Shared memory of one stage tile (dynamic): reconstruction variables with the
// cross halo, x and y slopes, x and y interface fluxes.
template <int V, int TX, int TY>
constexpr size_t stage_smem_bytes() {
  return sizeof(double) * (size_t)V *
         ((size_t)(TY + 4) * (TX + 4) + (size_t)TY * (TX + 2) + (size_t)(TY + 2) * TX + (size_t)TY * (TX + 1) +
          (size_t)(TY + 1) * TX);
}

// One TX x TY tile (bx, by) of one grid, z chunk bz.  Shared by the single-grid
// kernel (arguments in the parameter space) and the batched kernel (per-grid
// arguments in global memory, tiles from a flattened queue).
__device__ __forceinline__ void prefetch_l2(const double* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// The per-cell part of one right-hand side after the flux divergence: the centre state as
// ComputeRHS sees it, geometric and external sources (timedisc_base.f90:1263-1267), and the
// stage's consumer (k_m and the next Butcher stage's state, the Shu-Osher update, the embedded
// solutions and error norm, CheckData and CFL partial maxima).  R0: the cell's reconstruction
// variables; rhs: (divX + divY) + divZ on entry, the full right-hand side after the sources.
// Shared by the stage kernels of every tile layout.
template <int ND, bool EU, bool PRIM, bool KSEQ = false>
__device__ __forceinline__ void stage_cell_epilogue(const StageArgs& A, const int i, const int j, const int k,
                                                    const double* R0, double* rhs, const double dt, double* cflv,
                                                    double& errv, int& flags) {
  using PH = Phys<ND, EU>;
  using CE = Cells<ND, EU>;
  constexpr int V = PH::V;
  constexpr bool FG = ND == 2;   // FARGO transforms are compiled for 2D meshes only
  const Grid& g = A.g;
  const PhysP& P = A.ph;
  const MetricP& M = A.mt;
  const bool roundtrip = EU && A.in.roundtrip;
  const int ip = i + 2;
  // the CHECK_PMIN round trip of a conservative state, P2C(MAX(C2P(c),pmin))
  auto rt_cons = [&](double* c) {
    double q[V];
    PH::c2p(c, q, P);
    if (EU) q[V - 1] = dmax(q[V - 1], P.pmin);
    PH::p2c(q, c, P);
  };
  const long long idx = CE::lin(g, i, j, k);
  // centre primitive / conservative state as ComputeRHS sees it
  double pc[V], cc[V];
  if (PRIM) {
#pragma unroll
    for (int v = 0; v < V; ++v) pc[v] = R0[v];
    // the sources read cvar itself (the stage state), which Prim2Cons(pvar) only
    // reproduces to rounding; after the CHECK_PMIN round trip cvar is Prim2Cons(pvar)
    if (!roundtrip && (M.curv || A.has_accel || A.out_base)) state_at<V>(A.in, g.n, idx, cc);
    else PH::p2c(pc, cc, P);
  } else {
#pragma unroll
    for (int v = 0; v < V; ++v) cc[v] = R0[v];
    if (roundtrip) {
      double u[V];
      state_at<V>(A.in, g.n, idx, u);
      PH::c2p(u, pc, P);
      pc[V - 1] = dmax(pc[V - 1], P.pmin);
    } else {
      PH::c2p(cc, pc, P);
    }
  }
  // with FARGO the sources see the real frame: cvar after AddBackgroundVelocityY and the
  // primitive state CenterBoundary derives from it
  const bool fsrc = FG && A.w_sub;
  if (fsrc) {
    state_at<V>(A.in, g.n, idx, cc);
    if (A.in.pre.n) apply_chain<V>(A.in.pre, cc, g, i, j);
    PH::c2p(cc, pc, P);
    if (roundtrip) {   // CHECK_PMIN of this ComputeRHS (FirstStep's CHECK_ALL)
      pc[V - 1] = dmax(pc[V - 1], P.pmin);
      PH::p2c(pc, cc, P);
    }
  }
  // geometric sources (physics_euler.f90:1706-1847 / physics_eulerisotherm.f90:689-832)
  double geo2 = 0.0;
  if (fsrc && g.fdir == 1) {
    // transport along x: geometric sources of the real frame, AddFargoSourcesX into the x
    // one (isothermal physics_eulerisotherm.f90:1462-1518; Euler physics_euler.f90:2267-2355
    // adds the energy term -vx*(tmp + GetGeometricalSourceX(vz = P = mz = 0)))
    const double vx = pc[1], vy = pc[2];
    const double cxyx = M.cxyx[ip], cyxy = M.cyxy[ip], czxz = M.czxz[ip], czyz = M.czyz[ip];
    double geo1 = 0.0;
    if (M.curv) {
      const double Pp = EU ? pc[V - 1] : pc[0] * (M.cs[ip] * M.cs[ip]);
      geo1 = cc[2] * (cyxy * vy - cxyx * vx) + (cyxy + czxz) * Pp;
      rhs[2] = rhs[2] - (cc[1] * (cxyx * vx - cyxy * vy) + (cxyx + czyz) * Pp);
    }
    const int jp = j + 2;
    const double tmp = cc[2] * 0.5 * (A.w_sub[jp + 1] - A.w_sub[jp - 1]) / M.dly[ip];
    geo1 = geo1 - tmp;
    rhs[1] = rhs[1] - geo1;
    if (EU) {
      const double cxzx = M.cxzx[ip];
      const double gx = cc[2] * (cyxy * vy - cxyx * vx) + 0.0 * (czxz * 0.0 - cxzx * vx) + (cyxy + czxz) * 0.0;
      const double geoE = 0.0 - vx * (tmp + gx);
      rhs[V - 1] = rhs[V - 1] - geoE;
    }
  } else if (M.curv && ND == 2 && fsrc) {
    double Pp = EU ? pc[V - 1] : pc[0] * (M.cs[ip] * M.cs[ip]);
    double vx = pc[1], vy = pc[2];
    double cxyx = M.cxyx[ip], cyxy = M.cyxy[ip], czxz = M.czxz[ip], czyz = M.czyz[ip];
    rhs[1] = rhs[1] - (cc[2] * (cyxy * vy - cxyx * vx) + (cyxy + czxz) * Pp);
    geo2 = cc[1] * (cxyx * vx - cyxy * vy) + (cxyx + czyz) * Pp;
  }
  if (fsrc && g.fdir != 1) {
    // AddFargoSourcesY into the geometric source (isothermal
    // physics_eulerisotherm.f90:1531-1586; Euler physics_euler.f90:2368-2455 adds the
    // energy term -vy*(tmp + GetGeometricalSourceY(vz = P = mz = 0)))
    const double tmp = cc[1] * 0.5 * (A.w_sub[ip + 1] - A.w_sub[ip - 1]) / M.dlx[ip];
    geo2 = geo2 - tmp;
    rhs[2] = rhs[2] - geo2;
    if (EU) {
      const double vx = pc[1], vy = pc[2];
      const double cxyx = M.cxyx[ip], cyxy = M.cyxy[ip], cyzy = M.cyzy[ip], czyz = M.czyz[ip];
      const double gy = 0.0 * (czyz * 0.0 - cyzy * vy) + cc[1] * (cxyx * vx - cyxy * vy) + (cxyx + czyz) * 0.0;
      const double geoE = 0.0 - vy * (tmp + gy);
      rhs[V - 1] = rhs[V - 1] - geoE;
    }
  } else if (!fsrc && M.curv) {
    double Pp = EU ? pc[V - 1] : pc[0] * (M.cs[ip] * M.cs[ip]);
    double vx = pc[1], vy = pc[2];
    double cxyx = M.cxyx[ip], cyxy = M.cyxy[ip], czxz = M.czxz[ip], czyz = M.czyz[ip];
    if (ND == 2) {
      double mx = cc[1], my = cc[2];
      rhs[1] = rhs[1] - (my * (cyxy * vy - cxyx * vx) + (cyxy + czxz) * Pp);
      rhs[2] = rhs[2] - (mx * (cxyx * vx - cyxy * vy) + (cxyx + czyz) * Pp);
    } else {
      double vz = pc[3], mx = cc[1], my = cc[2], mz = cc[3];
      double cxzx = M.cxzx[ip], cyzy = M.cyzy[ip];
      rhs[1] = rhs[1] - (my * (cyxy * vy - cxyx * vx) + mz * (czxz * vz - cxzx * vx) + (cyxy + czxz) * Pp);
      rhs[2] = rhs[2] - (mz * (czyz * vz - cyzy * vy) + mx * (cxyx * vx - cyxy * vy) + (cxyx + czyz) * Pp);
      rhs[3] = rhs[3] - (mx * (cxzx * vx - czxz * vz) + my * (cyzy * vy - czyz * vz) + (cxzx + cyzy) * Pp);
    }
  }
  // external sources (sources_generic.f90:220-261): point-mass gravity (gravity_pointmass.f90:
  // 263-282, physics ExternalSources) first in the list, then the viscous source of this
  // stage state (precomputed by visc_kernel); rhs = ... - (gravity + viscosity)
  if (A.has_accel || A.visc) {
    double sm[ND] = {}, se = 0.0;
    if (A.has_accel) {
      const double ax = M.accel[ip], ay = M.accel[M.nxp + ip];
      sm[0] = cc[0] * ax;
      sm[1] = cc[0] * ay;
      if (EU) se = cc[1] * ax + cc[2] * ay;
    }
    if (A.visc) {
#pragma unroll
      for (int m = 0; m < ND; ++m) {
        const double sv = __ldg(A.visc + (long long)m * g.n + idx);
        sm[m] = A.has_accel ? sm[m] + sv : sv;
      }
      if (EU) {
        const double sv = __ldg(A.visc + (long long)ND * g.n + idx);
        se = A.has_accel ? se + sv : sv;
      }
    }
#pragma unroll
    for (int m = 0; m < ND; ++m) rhs[1 + m] = rhs[1 + m] - sm[m];
    if (EU) rhs[V - 1] = rhs[V - 1] - se;
  }

  if (A.out_mode == OUT_RHS) {
#pragma unroll
    for (int v = 0; v < V; ++v) A.out[(long long)v * g.n + idx] = rhs[v];
    if (A.fnext_out) {
      // the next Butcher stage's state base - sum_q (a dt) k_q in the reference's order
      // (timedisc_rkfehlberg.f90:277-302), this stage's k from the registers, formed as
      // form_kernel would form it
      const StateRef& S = A.fnext;
      double u[V];
#pragma unroll
      for (int v = 0; v < V; ++v) u[v] = __ldg(S.base + (long long)v * g.n + idx);
      // the earlier stages' k: unrolled to the tableau limit, so that all loads issue together,
      // or (KSEQ: kernels short of registers, whose streams the L2 prefetch has brought in) one
      // k at a time
      auto kterm = [&](int q) {
        const double a = S.dt_dev ? S.coef[q] * *S.dt_dev : S.coef[q];
#pragma unroll
        for (int v = 0; v < V; ++v) u[v] = u[v] - a * __ldg(S.K[q] + (long long)v * g.n + idx);
      };
      if (KSEQ) {
#pragma unroll 1
        for (int q = 0; q + 1 < S.nk; ++q) kterm(q);
      } else {
#pragma unroll
        for (int q = 0; q < FGPU_MAXK - 1; ++q)
          if (q + 1 < S.nk) kterm(q);
      }
      {
        const double a = S.dt_dev ? S.coef[S.nk - 1] * *S.dt_dev : S.coef[S.nk - 1];
#pragma unroll
        for (int v = 0; v < V; ++v) u[v] = u[v] - a * rhs[v];
      }
      if (PRIM) {
        double p[V];
        PH::c2p(u, p, P);
#pragma unroll
        for (int v = 0; v < V; ++v) A.fnext_out[(long long)v * g.n + idx] = p[v];
      } else {
#pragma unroll
        for (int v = 0; v < V; ++v) A.fnext_out[(long long)v * g.n + idx] = u[v];
      }
    }
  } else {
    // Shu-Osher update y = yn - dt*rhs + eta*(y0 - yn + dt*rhs) (timedisc_modeuler.f90:289)
    double yn[V], y0[V], y[V];
    if (FG && A.yn_chain.n) {
      state_at<V>(A.in, g.n, idx, yn);
      apply_chain<V>(A.yn_chain, yn, g, i, j, rt_cons);
    } else if (!PRIM) {
#pragma unroll
      for (int v = 0; v < V; ++v) yn[v] = cc[v];
    } else if (roundtrip) {
#pragma unroll
      for (int v = 0; v < V; ++v) yn[v] = cc[v];
    } else {
      state_at<V>(A.in, g.n, idx, yn);
    }
#pragma unroll
    for (int v = 0; v < V; ++v) y0[v] = __ldg(A.y0 + (long long)v * g.n + idx);
    if (FG && A.y0_chain.n) apply_chain<V>(A.y0_chain, y0, g, i, j, rt_cons);
    if (EU && A.y0_roundtrip) {
      double q[V];
      PH::c2p(y0, q, P);
      q[V - 1] = dmax(q[V - 1], P.pmin);
      PH::p2c(q, y0, P);
    }
#pragma unroll
    for (int v = 0; v < V; ++v) {
      y[v] = yn[v] - dt * rhs[v] + A.eta * (y0[v] - yn[v] + dt * rhs[v]);
      A.out[(long long)v * g.n + idx] = y[v];
    }
    if (PRIM && A.out_prim) {
      // Cons2Prim of the new state, the conversion the next stage applies to its input
      double p[V];
      PH::c2p(y, p, P);
#pragma unroll
      for (int v = 0; v < V; ++v) A.out_prim[(long long)v * g.n + idx] = p[v];
    }
    if (A.out2) {
#pragma unroll
      for (int v = 0; v < V; ++v)
        A.out2[(long long)v * g.n + idx] = yn[v] - dt * rhs[v] + A.eta2 * (y0[v] - yn[v] + dt * rhs[v]);
    }
    if (A.err_low) {
      double l[V];
#pragma unroll
      for (int v = 0; v < V; ++v) l[v] = __ldg(A.err_low + (long long)v * g.n + idx);
      // FARGO: the low-order solution as its ComputeRHS framed it in place
      if (FG && A.err_chain.n) apply_chain<V>(A.err_chain, l, g, i, j);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const double e = fabs(y[v] - l[v]) / (A.tol_rel * fabs(y[v]) + A.tol_abs[v]);
        errv = dmax(errv, e);
      }
    }
    if (A.cfl_mode == 1) {
      double p[V], c[V];
      PH::c2p(y, p, P);
      if (EU && A.cfl_roundtrip) p[V - 1] = dmax(p[V - 1], P.pmin);
      double cs = EU ? PH::cs_of(p, P) : M.cs[ip];
      double v3[4];
      CE::cfl_cell(p, cs, M, ip, v3);
#pragma unroll
      for (int q = 0; q < 4; ++q) cflv[q] = dmax(cflv[q], v3[q]);
      if (EU && A.cfl_roundtrip) PH::p2c(p, c, P);
      else { for (int v = 0; v < V; ++v) c[v] = y[v]; }
      if ((A.checkdata & 0x01) && !(cs > 0.)) flags |= 0x01;
      if (EU && (A.checkdata & 0x02) && p[V - 1] < P.pmin) flags |= 0x02;
      if ((A.checkdata & 0x04) && p[0] < P.rhomin) flags |= 0x04;
      if (A.checkdata & 0x08)
        for (int v = 0; v < V; ++v) if (invalid_value(p[v]) || invalid_value(c[v])) flags |= 0x08;
    }
  }
  if (A.out_base) {
#pragma unroll
    for (int v = 0; v < V; ++v) A.out_base[(long long)v * g.n + idx] = cc[v];
    if (fsrc) {
      // FARGO: cvar after this ComputeRHS is co-moving (its SubtractBackgroundVelocity)
      double o[V];
#pragma unroll
      for (int v = 0; v < V; ++v) o[v] = cc[v];
      frame_change<V>(o, -1.0, A.w_sub[fargo_ix(g, i, j)], g.fdir);
#pragma unroll
      for (int v = 0; v < V; ++v) A.out_base[(long long)v * g.n + idx] = o[v];
    }
  }
  if (A.cfl_mode >= 2) {
    double cs = EU ? PH::cs_of(pc, P) : M.cs[ip];
    if (A.cfl_mode == 2) {
      double v3[4];
      CE::cfl_cell(pc, cs, M, ip, v3);
#pragma unroll
      for (int q = 0; q < 4; ++q) cflv[q] = dmax(cflv[q], v3[q]);
    }
    if ((A.checkdata & 0x01) && !(cs > 0.)) flags |= 0x01;
    if (EU && (A.checkdata & 0x02) && pc[V - 1] < P.pmin) flags |= 0x02;
    if ((A.checkdata & 0x04) && pc[0] < P.rhomin) flags |= 0x04;
    if (A.checkdata & 0x08)
      for (int v = 0; v < V; ++v) if (invalid_value(pc[v]) || invalid_value(cc[v])) flags |= 0x08;
  }
  if (A.last_stage) {
    // high/low order solutions and ComputeError (timedisc_rkfehlberg.f90:198-265,
    // timedisc_base.f90:1012-1053); base and the earlier k unrolled to the tableau limit
    // so that their loads issue together, this stage's k from the registers.  On the
    // device clock (in.dt_dev) bh_dt/bl_dt hold the weights, multiplied by *dt_dev here.
    const double* dtd = A.in.dt_dev;
    double hi[V], lo[V];
#pragma unroll
    for (int v = 0; v < V; ++v) hi[v] = lo[v] = __ldg(A.in.base + (long long)v * g.n + idx);
    auto kterm = [&](int q) {
      const double bh = dtd ? A.bh_dt[q] * *dtd : A.bh_dt[q];
      const double bl = dtd ? A.bl_dt[q] * *dtd : A.bl_dt[q];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const double kq = __ldg(A.in.K[q] + (long long)v * g.n + idx);
        lo[v] = lo[v] - bl * kq;
        hi[v] = hi[v] - bh * kq;
      }
    };
    if (KSEQ) {
#pragma unroll 1
      for (int q = 0; q + 1 < A.nstage; ++q) kterm(q);
    } else {
#pragma unroll
      for (int q = 0; q < FGPU_MAXK - 1; ++q)
        if (q + 1 < A.nstage) kterm(q);
    }
    {
      const int q = A.nstage - 1;
      const double bh = dtd ? A.bh_dt[q] * *dtd : A.bh_dt[q];
      const double bl = dtd ? A.bl_dt[q] * *dtd : A.bl_dt[q];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        lo[v] = lo[v] - bl * rhs[v];
        hi[v] = hi[v] - bh * rhs[v];
      }
    }
#pragma unroll
    for (int v = 0; v < V; ++v) {
      A.out_high[(long long)v * g.n + idx] = hi[v];
      const double e = fabs(hi[v] - lo[v]) / (A.tol_rel * fabs(hi[v]) + A.tol_abs[v]);
      errv = dmax(errv, e);
    }
  }
}

template <int ND, bool EU, bool PRIM, int TX, int TY>
__device__ __forceinline__ void stage_tile(const StageArgs& A, const int bx, const int by, const int bz) {
  using PH = Phys<ND, EU>;
  using CE = Cells<ND, EU>;
  constexpr int V = PH::V;
  constexpr int NT = TX * TY;
  constexpr int RW = TX + 4, RH = TY + 4;
  // dynamic shared memory, stage_smem_bytes<V, TX, TY>() bytes
  extern __shared__ __align__(16) double stage_smem[];
  double* const Rs = stage_smem;                    // [V][TY+4][TX+4]
  double* const Sx = Rs + V * RH * RW;              // [V][TY][TX+2]   x slopes
  double* const Sy = Sx + V * TY * (TX + 2);        // [V][TY+2][TX]   y slopes
  double* const Fx = Sy + V * (TY + 2) * TX;        // [V][TY][TX+1]   x fluxes
  double* const Fy = Fx + V * TY * (TX + 1);        // [V][TY+1][TX]   y fluxes
  __shared__ double sred[RED_STRIDE * ((NT + 31) / 32)];

  if (A.ctl && (A.ctl->stop | A.ctl->brk)) return;
  if (gated_out(A.ctl, A.gate)) return;
  const Grid& g = A.g;
  const PhysP& P = A.ph;
  const MetricP& M = A.mt;
  const double dt = A.dt_dev ? *A.dt_dev : A.dt;
  const bool roundtrip = EU && A.in.roundtrip;
  constexpr bool FG = ND == 2;   // FARGO transforms are compiled for 2D meshes only
  const int tid = threadIdx.x;
  const int tx = tid % TX, ty = tid / TX;
  const int i0 = bx * TX, j0 = by * TY;
  const int ex = min(TX, g.nx - i0), ey = min(TY, g.ny - j0);
  const bool own = tx < ex && ty < ey;
  const int i = i0 + tx, j = j0 + ty;
  int k0 = 0, k1 = 1;
  if (ND == 3) { k0 = bz * A.kchunk; k1 = min(g.nz, k0 + A.kchunk); }

  auto RS = [&](int v, int ly, int lx) -> double& { return Rs[(v * RH + ly) * RW + lx]; };
  auto SX = [&](int v, int r, int c) -> double& { return Sx[(v * TY + r) * (TX + 2) + c]; };
  auto SY = [&](int v, int r, int c) -> double& { return Sy[(v * (TY + 2) + r) * TX + c]; };
  auto FX = [&](int v, int r, int c) -> double& { return Fx[(v * TY + r) * (TX + 1) + c]; };
  auto FY = [&](int v, int r, int c) -> double& { return Fy[(v * (TY + 1) + r) * TX + c]; };

  // the CHECK_PMIN round trip of a conservative state, P2C(MAX(C2P(c),pmin))
  auto rt_cons = [&](double* c) {
    double q[V];
    PH::c2p(c, q, P);
    if (EU) q[V - 1] = dmax(q[V - 1], P.pmin);
    PH::p2c(q, c, P);
  };
  // reconstruction variables at a cross point (interior or face ghost)
  const StateRef& SR = A.rin.base ? A.rin : A.in;
  auto recon_at = [&](int gi, int gj, int gk, double* R) {
    double p[V];
    bool inx = gi >= 0 && gi < g.nx, iny = gj >= 0 && gj < g.ny, inz = gk >= 0 && gk < g.nz;
    if (inx && iny && inz) {
      double u[V];
      state_at<V>(SR, g.n, CE::lin(g, gi, gj, gk), u);
      if (PRIM && SR.ready) {
#pragma unroll
        for (int l = 0; l < V; ++l) R[l] = u[l];
        return;
      }
      if (FG && A.in.pre.n) apply_chain<V>(A.in.pre, u, g, gi, gj);
      if (PRIM) {
        PH::c2p(u, p, P);
        if (roundtrip) p[V - 1] = dmax(p[V - 1], P.pmin);
        if (FG && A.w_sub) sub_velocity(p, A.w_sub[fargo_ix(g, gi, gj)], g.fdir);
#pragma unroll
        for (int l = 0; l < V; ++l) R[l] = p[l];
      } else if (roundtrip) {
        PH::c2p(u, p, P);
        p[V - 1] = dmax(p[V - 1], P.pmin);
        PH::p2c(p, R, P);
        if (FG && A.w_sub) frame_change<V>(R, -1.0, A.w_sub[fargo_ix(g, gi, gj)], g.fdir);
      } else {
#pragma unroll
        for (int l = 0; l < V; ++l) R[l] = u[l];
        if (FG && A.w_sub) frame_change<V>(R, -1.0, A.w_sub[fargo_ix(g, gi, gj)], g.fdir);
      }
    } else {
      int d = !inx ? 0 : (!iny ? 1 : 2);
      CE::face_ghost_p(SR, g, P, M, d, gi, gj, gk, p);
      if (roundtrip) p[V - 1] = dmax(p[V - 1], P.pmin);
      if (PRIM) {
        if (FG && A.w_sub) sub_velocity(p, A.w_sub[fargo_ix(g, gi, gj)], g.fdir);
#pragma unroll
        for (int l = 0; l < V; ++l) R[l] = p[l];
      } else {
        PH::p2c(p, R, P);
        if (FG && A.w_sub) frame_change<V>(R, -1.0, A.w_sub[fargo_ix(g, gi, gj)], g.fdir);
      }
    }
  };

  const int ip = i + 2;   // padded i of the own cell
  // padded cells of one flux field (flux_out)
  const long long npad = (long long)(g.nx + 4) * (g.ny + 4) * (ND == 3 ? g.nz + 4 : 1);
  double cflv[4] = {0.0, 0.0, 0.0, 0.0};
  double errv = 0.0;
  int flags = 0;

  // z-direction state of the own column (3D): R at k, k+1, z-slope at k, flux at k-1/2
  double Rz0[V], Rz1[V], sz0[V], Fzm[V];
  if (ND == 3 && own) {
    double Ra[V], Rb[V];
    recon_at(i, j, k0 - 2, Ra);
    recon_at(i, j, k0 - 1, Rb);
    recon_at(i, j, k0, Rz0);
    recon_at(i, j, k0 + 1, Rz1);
    double szm[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      szm[v] = A.constant_recon ? 0.0 : slope(A.limiter, A.theta, A.invd[2], Ra[v], Rb[v], Rz0[v]);
      sz0[v] = A.constant_recon ? 0.0 : slope(A.limiter, A.theta, A.invd[2], Rb[v], Rz0[v], Rz1[v]);
    }
    double RL[V], RR[V];
    double oT = M.offzT[k0 - 1 + 2], oB = M.offzB[k0 + 2];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      RL[v] = A.constant_recon ? Rb[v] : Rb[v] + szm[v] * oT;
      RR[v] = A.constant_recon ? Rz0[v] : Rz0[v] + sz0[v] * oB;
    }
    kt_flux<ND, EU, PRIM>(2, RL, RR, EU ? 0.0 : M.cs[6 * M.nxp + ip], EU ? 0.0 : M.cs[5 * M.nxp + ip],
                          M.dAzB[ip], P, Fzm);
    if (A.flux_out && k0 == 0) store_flux<V>(A, 2, padded_index(g, i, j, k0 - 1, ND), npad, Fzm);
  }

  for (int k = k0; k < k1; ++k) {
    double divZ[V];
    if ((A.fnext_out || A.last_stage) && own) {
      // the stream the epilogue combines (base and the earlier stages' k of this cell, for the
      // next stage's state or the high/low-order solutions), fetched into L2 while the
      // plane's stencil runs
      const long long pidx = CE::lin(g, i, j, k);
      const StateRef& S = A.fnext_out ? A.fnext : A.in;
      const int nq = A.fnext_out ? S.nk - 1 : A.nstage - 1;
#pragma unroll
      for (int v = 0; v < V; ++v) prefetch_l2(S.base + (long long)v * g.n + pidx);
#pragma unroll 1
      for (int q = 0; q < nq; ++q)
#pragma unroll
        for (int v = 0; v < V; ++v) prefetch_l2(S.K[q] + (long long)v * g.n + pidx);
    }
    // ---- own cell: plane k into shared memory; z-flux at k+1/2
    if (own) {
      double Rc[V];
      if (ND == 3) {
        double Rz2[V], sz1[V], Fzp[V];
        recon_at(i, j, k + 2, Rz2);
#pragma unroll
        for (int v = 0; v < V; ++v)
          sz1[v] = A.constant_recon ? 0.0 : slope(A.limiter, A.theta, A.invd[2], Rz0[v], Rz1[v], Rz2[v]);
        double RL[V], RR[V];
        double oT = M.offzT[k + 2], oB = M.offzB[k + 1 + 2];
#pragma unroll
        for (int v = 0; v < V; ++v) {
          RL[v] = A.constant_recon ? Rz0[v] : Rz0[v] + sz0[v] * oT;
          RR[v] = A.constant_recon ? Rz1[v] : Rz1[v] + sz1[v] * oB;
        }
        kt_flux<ND, EU, PRIM>(2, RL, RR, EU ? 0.0 : M.cs[6 * M.nxp + ip], EU ? 0.0 : M.cs[5 * M.nxp + ip],
                              M.dAzB[ip], P, Fzp);
        if (A.flux_out) store_flux<V>(A, 2, padded_index(g, i, j, k, ND), npad, Fzp);
        double dV = M.dxdydV[ip];
#pragma unroll
        for (int v = 0; v < V; ++v) {
          divZ[v] = dV * (Fzp[v] - Fzm[v]);
          Rc[v] = Rz0[v];
          Rz0[v] = Rz1[v];
          Rz1[v] = Rz2[v];
          sz0[v] = sz1[v];
          Fzm[v] = Fzp[v];
        }
      } else {
        recon_at(i, j, k, Rc);
      }
#pragma unroll
      for (int v = 0; v < V; ++v) RS(v, ty + 2, tx + 2) = Rc[v];
    }
    // ---- x-y cross halo of plane k
    {
      const int H = 4 * (ex + ey);
      for (int h = tid; h < H; h += NT) {
        int lx, ly;
        if (h < 4 * ey) {
          int r = h >> 2, q = h & 3;
          ly = r;
          lx = q < 2 ? q - 2 : ex + (q - 2);
        } else {
          int hh = h - 4 * ey;
          int c = hh >> 2, q = hh & 3;
          lx = c;
          ly = q < 2 ? q - 2 : ey + (q - 2);
        }
        double R[V];
        recon_at(i0 + lx, j0 + ly, k, R);
#pragma unroll
        for (int v = 0; v < V; ++v) RS(v, ly + 2, lx + 2) = R[v];
      }
    }
    __syncthreads();

    double divX[V], divY[V];
    // ---- slopes of both directions in one phase (x: ey rows x ex+2 cells, y: ey+2 rows x ex cells)
    // work items are enumerated over the full tile shape (compile-time divisors) and the
    // ones outside a partial edge tile are skipped
    constexpr int NSX = TY * (TX + 2), NSY = (TY + 2) * TX;
    constexpr int RHW = RH * RW;
    if (!A.constant_recon) {
      // one code path for both directions (no divergence where a warp spans the x/y boundary)
      for (int t = tid; t < NSX + NSY; t += NT) {
        int cidx, step, sidx, sstride;
        double* Sout;
        double invd;
        if (t < NSX) {
          const int r = t / (TX + 2), c = t % (TX + 2) - 1;
          if (r >= ey || c > ex) continue;
          cidx = (r + 2) * RW + (c + 2); step = 1;
          Sout = Sx; sidx = r * (TX + 2) + (c + 1); sstride = TY * (TX + 2);
          invd = A.invd[0];
        } else {
          const int u = t - NSX;
          const int c = u % TX, r = u / TX - 1;
          if (c >= ex || r > ey) continue;
          cidx = (r + 2) * RW + (c + 2); step = RW;
          Sout = Sy; sidx = (r + 1) * TX + c; sstride = (TY + 2) * TX;
          invd = A.invd[1];
        }
#pragma unroll
        for (int v = 0; v < V; ++v) {
          const double* R = Rs + v * RHW + cidx;
          Sout[v * sstride + sidx] = slope(A.limiter, A.theta, invd, R[-step], R[0], R[step]);
        }
      }
      __syncthreads();
    }
    // ---- interface fluxes of both directions in one phase, one code path
    constexpr int NFX = TY * (TX + 1), NFY = (TY + 1) * TX;
    for (int t = tid; t < NFX + NFY; t += NT) {
      double RL[V], RR[V], F[V];
      int lidx, ridx, sL, sR, sstride, fstride, d;
      const double* S;
      double* Fout;
      double oL, oR, csL, csR, dA;
      const bool xf = t < NFX;
      int xr = 0, xfc = 0, yc = 0, yf = 0;
      if (xf) {
        const int r = t / (TX + 1), f = t % (TX + 1);
        if (r >= ey || f > ex) continue;
        const int gl = i0 + f - 1 + 2;   // padded i of the left cell
        oL = M.offxE[gl]; oR = M.offxW[gl + 1];
        lidx = (r + 2) * RW + (f + 1); ridx = lidx + 1;
        S = Sx; sL = r * (TX + 2) + f; sR = sL + 1; sstride = TY * (TX + 2);
        csL = EU ? 0.0 : M.cs[2 * M.nxp + gl]; csR = EU ? 0.0 : M.cs[1 * M.nxp + gl + 1];
        dA = M.dAxW[gl + 1];
        Fout = Fx + r * (TX + 1) + f; fstride = TY * (TX + 1);
        d = 0;
        xr = r; xfc = f;
      } else {
        const int u = t - NFX;
        const int c = u % TX, f = u / TX;
        if (c >= ex || f > ey) continue;
        yc = c; yf = f;
        const int gjl = j0 + f - 1 + 2;     // padded j of the lower cell
        const int gi = i0 + c + 2;          // padded i of the column
        oL = M.offyN[gjl]; oR = M.offyS[gjl + 1];
        lidx = (f + 1) * RW + (c + 2); ridx = lidx + RW;
        S = Sy; sL = f * TX + c; sR = sL + TX; sstride = (TY + 2) * TX;
        csL = EU ? 0.0 : M.cs[4 * M.nxp + gi]; csR = EU ? 0.0 : M.cs[3 * M.nxp + gi];
        dA = M.dAyS[gi];
        Fout = Fy + f * TX + c; fstride = (TY + 1) * TX;
        d = 1;
      }
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const double rl = Rs[v * RHW + lidx], rr = Rs[v * RHW + ridx];
        RL[v] = A.constant_recon ? rl : rl + S[v * sstride + sL] * oL;
        RR[v] = A.constant_recon ? rr : rr + S[v * sstride + sR] * oR;
      }
      kt_flux<ND, EU, PRIM>(d, RL, RR, csL, csR, dA, P, F);
#pragma unroll
      for (int v = 0; v < V; ++v) Fout[v * fstride] = F[v];
      if (A.flux_out)
        store_flux<V>(A, d, xf ? padded_index(g, i0 + xfc - 1, j0 + xr, k, ND) : padded_index(g, i0 + yc, j0 + yf - 1, k, ND),
                      npad, F);
      // boundary row of ComputeRHS (timedisc_base.f90:1224-1231) for the accretion bookkeeping
      if (ND == 2 && xf && A.brow && ((A.brow_face == 0 && i0 + xfc == 0) || (A.brow_face == 1 && i0 + xfc == g.nx)))
        A.brow[j0 + xr] = (A.brow_face == 0 ? A.bdydz : -A.bdydz) * F[0];
    }
    __syncthreads();

    if (own) {
      {
        double dV = M.dydzdV[ip];
#pragma unroll
        for (int v = 0; v < V; ++v) divX[v] = dV * (FX(v, ty, tx + 1) - FX(v, ty, tx));
      }
      double dV = M.dzdxdV[ip];
#pragma unroll
      for (int v = 0; v < V; ++v) divY[v] = dV * (FY(v, ty + 1, tx) - FY(v, ty, tx));
      double R0[V], rhs[V];
#pragma unroll
      for (int v = 0; v < V; ++v) R0[v] = RS(v, ty + 2, tx + 2);
#pragma unroll
      for (int v = 0; v < V; ++v) rhs[v] = (divX[v] + divY[v]) + (ND == 3 ? divZ[v] : 0.0);
      stage_cell_epilogue<ND, EU, PRIM>(A, i, j, k, R0, rhs, dt, cflv, errv, flags);
    }
    // no barrier between the planes of one tile: a thread writes only its own cell and the
    // halo of the next plane, and every reader of this plane has passed the flux barrier
  }

  const bool err_out = A.last_stage || A.err_low;
  if (A.ctl && (A.cfl_mode || err_out)) {
    int nv = A.cfl_mode ? (M.vis ? 4 : (ND == 3 ? 3 : 1)) : 0;
    double vals[4] = {cflv[0], cflv[1], cflv[2], cflv[3]};
    if (err_out && !A.cfl_mode) { vals[0] = errv; nv = 1; }
    if (nv) block_reduce_emit<NT>(vals, nv, flags, err_out && !A.cfl_mode ? &A.ctl->err : A.ctl->invdt,
                                  &A.ctl->flags, sred);
  }
  // the next tile of a persistent block may place its halo where this tile had cells
  __syncthreads();
}

template <int ND, bool EU, bool PRIM, int TX, int TY, int MINB = 1>
__global__ void __launch_bounds__(TX* TY, MINB) stage_kernel(const __grid_constant__ StageArgs A) {
  stage_tile<ND, EU, PRIM, TX, TY>(A, blockIdx.x, blockIdx.y, blockIdx.z);
}

// Batched ensemble: one persistent launch over the flattened tile queue of
// many independent grids; tile t = (grid, bx, by, bz), args[grid] its stage.
template <int ND, bool EU, bool PRIM, int TX, int TY, int MINB = 1>
__global__ void __launch_bounds__(TX* TY, MINB) batched_stage_kernel(const StageArgs* __restrict__ args,
                                                                      const int4* __restrict__ tiles, int ntiles) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int4 T = tiles[t];
    stage_tile<ND, EU, PRIM, TX, TY>(args[T.x], T.y, T.z, T.w);
  }
}

}  // namespace fgpu
