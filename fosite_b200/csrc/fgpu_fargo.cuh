// fgpu_fargo.cuh -- FARGO transport (fosite fargo types 1 and 2, 2D x-y meshes)
// along y (direction 2) or x (direction 1): the background velocity of
// CalcBackgroundVelocity and the shift + upwind residual advection of
// FargoAdvectionY / FargoAdvectionX, with the CFL / CheckData pass of the
// step's closing ComputeRHS + CalcTimestep fused into the advection.
#pragma once
#include "fgpu_kernels.cuh"

namespace fgpu {

struct FargoWArgs {
  Grid g;
  PhysP ph;
  MetricP mt;
  StateRef in;            // state whose real frame is in + in.pre
  const double* w_prev;   // background velocity of the last ComputeRHS (pvar round trip), or null
  const double* wfac;     // wfactor, by padded i (direction 2) or padded j (direction 1)
  double* w_out;          // new background velocity, indexed like wfac
  Ctl* ctl;
  int gate;               // device-clock attempt slots: run only with one of these action bits
};

// CalcBackgroundVelocity for direction 2 (timedisc_base.f90:2243-2326):
//   w(i) = SUM_j pvar(i,j,vy)*wfactor(i) / JNUM over the interior j, for every
//   padded column i (the x-ghost columns come from the boundary fill).
// pvar is the primitive state of the last ComputeRHS after its
// SubtractBackgroundVelocityY and this routine's AddBackgroundVelocityY, i.e.
// (vy - w_prev) + w_prev.  The sum runs in j order like the reference loop, so
// the result is bitwise reproducible: a block owns FW_WX columns; per chunk of FW_RC
// rows (one chunk for up to 512 rows) its FW_NT threads evaluate the terms in parallel
// into shared memory, each thread FW_RC / (FW_NT / FW_WX) rows of one column with their
// loads in flight together, then one thread per column adds the chunk's terms in order
// (shared-memory loads issued ahead of the dependent adds).
constexpr int FW_WX = 8, FW_NT = 512, FW_RC = 512;
template <bool EU>
__device__ __forceinline__ void fargo_w_body(const FargoWArgs& A, const int bx) {
  using CE = Cells<2, EU>;
  constexpr int RPT = FW_RC / (FW_NT / FW_WX);   // rows per thread and chunk
  __shared__ double terms[FW_RC][FW_WX];
  if (A.ctl && (A.ctl->stop | A.ctl->brk)) return;
  if (gated_out(A.ctl, A.gate)) return;
  const Grid& g = A.g;
  const int tx = threadIdx.x % FW_WX, ty = threadIdx.x / FW_WX;
  const int ip = bx * FW_WX + tx;
  const bool valid = ip < g.nx + 4;
  const int i = ip - 2;
  const bool ghost = i < 0 || i >= g.nx;
  const double wf = valid ? A.wfac[ip] : 0.0;
  const double wp = (valid && A.w_prev) ? A.w_prev[ip] : 0.0;
  double wi = 0.0;
  for (int j0 = 0; j0 < g.ny; j0 += FW_RC) {
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
      const int q = ty + (FW_NT / FW_WX) * r, j = j0 + q;
      double t = 0.0;
      if (valid && j < g.ny) {
        double p[Phys<2, EU>::V];
        if (ghost) CE::face_ghost_p(A.in, g, A.ph, A.mt, 0, i, j, 0, p);
        else CE::interior_p(A.in, g, A.ph, i, j, 0, p);
        double vy = p[2];
        if (A.w_prev) vy = (vy - wp) + wp;
        t = vy * wf;
      }
      terms[q][tx] = t;
    }
    __syncthreads();
    if (ty == 0 && valid) {
      const int nq = min(FW_RC, g.ny - j0);
      int q = 0;
      for (; q + 8 <= nq; q += 8) {
        double t[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) t[u] = terms[q + u][tx];
#pragma unroll
        for (int u = 0; u < 8; ++u) wi = wi + t[u];
      }
      for (; q < nq; ++q) wi = wi + terms[q][tx];
    }
    __syncthreads();
  }
  if (ty == 0 && valid) A.w_out[ip] = wi / (double)g.ny;
}
template <bool EU>
__global__ void __launch_bounds__(FW_NT) fargo_w_kernel(const __grid_constant__ FargoWArgs A) {
  fargo_w_body<EU>(A, blockIdx.x);
}

// The same sums for a single grid in two passes, so that the terms (a cell's primitive
// velocity, or an absorbing / reflecting ghost of a boundary column, which costs many times an
// interior term) spread over every SM: fargo_w_terms_kernel writes term (ip, j) to a scratch
// array, one per thread; fargo_w_sum_kernel adds each column's terms in j order, a block per
// FS_WX columns staging FS_RC rows at a time in shared memory, one thread per column adding.
template <bool EU>
__global__ void __launch_bounds__(256) fargo_w_terms_kernel(const __grid_constant__ FargoWArgs A,
                                                            double* __restrict__ terms) {
  using CE = Cells<2, EU>;
  if (A.ctl && (A.ctl->stop | A.ctl->brk)) return;
  if (gated_out(A.ctl, A.gate)) return;
  const Grid& g = A.g;
  const int nxp = g.nx + 4;
  const long long t = blockIdx.x * 256LL + threadIdx.x;
  if (t >= (long long)nxp * g.ny) return;
  const int ip = (int)(t % nxp), j = (int)(t / nxp);
  const int i = ip - 2;
  double p[Phys<2, EU>::V];
  if (i < 0 || i >= g.nx) CE::face_ghost_p(A.in, g, A.ph, A.mt, 0, i, j, 0, p);
  else CE::interior_p(A.in, g, A.ph, i, j, 0, p);
  double vy = p[2];
  if (A.w_prev) {
    const double wp = A.w_prev[ip];
    vy = (vy - wp) + wp;
  }
  terms[t] = vy * A.wfac[ip];
}
constexpr int FS_WX = 8, FS_NT = 1024, FS_RC = 512;
__global__ void __launch_bounds__(FS_NT) fargo_w_sum_kernel(const __grid_constant__ FargoWArgs A,
                                                            const double* __restrict__ terms) {
  __shared__ double st[FS_RC * FS_WX];
  if (A.ctl && (A.ctl->stop | A.ctl->brk)) return;
  if (gated_out(A.ctl, A.gate)) return;
  const Grid& g = A.g;
  const int nxp = g.nx + 4;
  const int c0 = blockIdx.x * FS_WX;
  double wi = 0.0;
  for (int j0 = 0; j0 < g.ny; j0 += FS_RC) {
    const int nq = min(FS_RC, g.ny - j0);
#pragma unroll 4
    for (int e = threadIdx.x; e < FS_RC * FS_WX; e += FS_NT) {
      const int q = e / FS_WX, c = e % FS_WX;
      st[e] = (q < nq && c0 + c < nxp) ? __ldg(terms + (long long)(j0 + q) * nxp + c0 + c) : 0.0;
    }
    __syncthreads();
    if (threadIdx.x < FS_WX) {
      const int c = threadIdx.x;
      int q = 0;
      for (; q + 8 <= nq; q += 8) {
        double t[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) t[u] = st[(q + u) * FS_WX + c];
#pragma unroll
        for (int u = 0; u < 8; ++u) wi = wi + t[u];
      }
      for (; q < nq; ++q) wi = wi + st[q * FS_WX + c];
    }
    __syncthreads();
  }
  if (threadIdx.x < FS_WX && c0 + (int)threadIdx.x < nxp) A.w_out[c0 + threadIdx.x] = wi / (double)g.ny;
}

// CalcBackgroundVelocity for direction 1 (timedisc_base.f90:2262-2282):
//   w(j) = SUM_i pvar(i,j,vx)*wfactor(j) / INUM over the interior i, for every padded row j
// (the y-ghost rows come from the boundary fill), with vx = (vx - w_prev) + w_prev as for
// direction 2.  A block owns FX_WY rows; per chunk of FX_WX columns its threads evaluate the
// terms in parallel into shared memory (coalesced along x), then one thread per row adds
// them in i order, so the sum rounds like the reference loop.
constexpr int FX_WX = 32, FX_WY = 8;
template <bool EU>
__device__ __forceinline__ void fargo_w_x_body(const FargoWArgs& A, const int bx) {
  using CE = Cells<2, EU>;
  __shared__ double terms[FX_WY][FX_WX + 1];
  if (A.ctl && (A.ctl->stop | A.ctl->brk)) return;
  if (gated_out(A.ctl, A.gate)) return;
  const Grid& g = A.g;
  const int tx = threadIdx.x % FX_WX, ty = threadIdx.x / FX_WX;
  const int jp = bx * FX_WY + ty;
  const bool valid = jp < g.ny + 4;
  const int j = jp - 2;
  const bool ghost = j < 0 || j >= g.ny;
  const double wf = valid ? A.wfac[jp] : 0.0;
  const double wp = (valid && A.w_prev) ? A.w_prev[jp] : 0.0;
  double wi = 0.0;
  for (int i0 = 0; i0 < g.nx; i0 += FX_WX) {
    const int i = i0 + tx;
    double t = 0.0;
    if (valid && i < g.nx) {
      double p[Phys<2, EU>::V];
      if (ghost) CE::face_ghost_p(A.in, g, A.ph, A.mt, 1, i, j, 0, p);
      else CE::interior_p(A.in, g, A.ph, i, j, 0, p);
      double vx = p[1];
      if (A.w_prev) vx = (vx - wp) + wp;
      t = vx * wf;
    }
    terms[ty][tx] = t;
    __syncthreads();
    if (tx == 0 && valid) {
      const int nq = min(FX_WX, g.nx - i0);
      for (int q = 0; q < nq; ++q) wi = wi + terms[ty][q];
    }
    __syncthreads();
  }
  if (tx == 0 && valid) A.w_out[jp] = wi / (double)g.nx;
}
template <bool EU>
__global__ void __launch_bounds__(FX_WX* FX_WY) fargo_w_x_kernel(const __grid_constant__ FargoWArgs A) {
  fargo_w_x_body<EU>(A, blockIdx.x);
}

struct FargoAdvArgs {
  Grid g;
  PhysP ph;
  MetricP mt;
  StateRef in;           // co-moving state after the last stage (no frame changes)
  const double* w;       // background velocity, by padded i (direction 2) or padded j (direction 1)
  double* out;           // advected state (must not alias in.base)
  Ctl* ctl;              // dt/time source and CFL / CheckData sink
  int checkdata;
  int chunk;             // rows of one thread
  double dt_host;        // > 0: the transport's dt (IntegrationStep's this%dt); else (time+dt)-time of ctl
  int dt_ctl;            // 1: the transport's dt is ctl->dt (an embedded scheme's closed step)
  int gate;              // device-clock attempt slots: run only with one of these action bits
};

__device__ __forceinline__ double fargo_minmod(double a, double b) {
  return fsign1(a) * fsign1(b) > 0. ? fsign(dmin(fabs(a), fabs(b)), a) : 0.;
}

// FargoAdvectionY (timedisc_base.f90:1935-2069) for the interior cells:
//   delxy = w*dt/dly, shift = NINT(delxy), delxy -= shift;
//   residual transport with minmod-limited upwind fluxes
//     flux(j) = q(j) + dql(j)/2*(1-d)      (d > 0)
//             = q(j+1) - dql(j+1)/2*(1+d)  (d <= 0)
//     q(j)   -= d*(flux(j) - flux(j-1))
//   then the integer shift CSHIFT(q, -shift) over the interior rows.
// dt is IntegrationStep's (time+dt)-time.  The y ghosts of the input come from
// the boundary fill of the co-moving state (CenterBoundary before the
// transport).  Each result cell depends on rows j-2..j+2 only, so a thread
// transports a run of rows of one column with a 5-row register window and
// writes each result to its shifted row.  The same pass evaluates the closing
// ComputeRHS's CheckData (real frame) and CalcTimestep's wave speeds
// (co-moving frame) of the interior cells.
template <bool EU, int TX, int TY>
__device__ __forceinline__ void fargo_advect_body(const FargoAdvArgs& A, const int bx, const int by) {
  using PH = Phys<2, EU>;
  using CE = Cells<2, EU>;
  constexpr int V = PH::V;
  constexpr int NT = TX * TY;
  __shared__ double sred[RED_STRIDE * ((NT + 31) / 32)];
  if (A.ctl->stop | A.ctl->brk) return;
  if (gated_out(A.ctl, A.gate)) return;
  const Grid& g = A.g;
  const PhysP& P = A.ph;
  const MetricP& M = A.mt;
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  const int i = bx * TX + tx;
  const int j0 = (by * TY + ty) * A.chunk;
  const int j1 = min(g.ny, j0 + A.chunk);
  double cflv = 0.0, cflvis = 0.0;
  int flags = 0;
  if (i < g.nx && j0 < g.ny) {
    const int ip = i + 2;
    const double w = A.w[ip];
    const double dte = A.dt_ctl ? A.ctl->dt : (A.dt_host > 0. ? A.dt_host : (A.ctl->time + A.ctl->dt) - A.ctl->time);
    double d = w * dte / M.dly[ip];
    const double sh = round(d);   // NINT: half away from zero
    const int s = (int)sh;
    d = d - (double)s;
    const double cs = M.cs[ip];
    auto load = [&](int jj, double* c) {
      if (jj >= 0 && jj < g.ny) {
        state_at<V>(A.in, g.n, CE::lin(g, i, jj, 0), c);
      } else {
        double p[V];
        CE::face_ghost_p(A.in, g, P, M, 1, i, jj, 0, p);
        PH::p2c(p, c, P);
      }
    };
    double q[5][V];
#pragma unroll
    for (int r = 0; r < 4; ++r) load(j0 - 2 + r, q[r]);
    for (int j = j0; j < j1; ++j) {
      load(j + 2, q[4]);
      double u[V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        double a0 = q[1][v] - q[0][v], a1 = q[2][v] - q[1][v];
        double a2 = q[3][v] - q[2][v], a3 = q[4][v] - q[3][v];
        double fl, fr;   // flux(j-1), flux(j)
        if (d > 0.) {
          fl = q[1][v] + .5 * fargo_minmod(a0, a1) * (1. - d);
          fr = q[2][v] + .5 * fargo_minmod(a1, a2) * (1. - d);
        } else {
          fl = q[2][v] - .5 * fargo_minmod(a1, a2) * (1. + d);
          fr = q[3][v] - .5 * fargo_minmod(a2, a3) * (1. + d);
        }
        u[v] = q[2][v] - d * (fr - fl);
      }
      int jd = (j + s) % g.ny;
      if (jd < 0) jd += g.ny;
      const long long o = CE::lin(g, i, jd, 0);
#pragma unroll
      for (int v = 0; v < V; ++v) A.out[(long long)v * g.n + o] = u[v];
      // closing ComputeRHS: AddBackgroundVelocityY, CenterBoundary's Cons2Prim, CheckData;
      // CalcTimestep on the co-moving primitive state
      double c[V], p[V];
#pragma unroll
      for (int v = 0; v < V; ++v) c[v] = u[v];
      frame_change<V>(c, 1.0, w, 2);
      PH::c2p(c, p, P);
      const double csc = EU ? PH::cs_of(p, P) : cs;
      if ((A.checkdata & 0x01) && !(csc > 0.)) flags |= 0x01;
      if (EU && (A.checkdata & 0x02) && p[V - 1] < P.pmin) flags |= 0x02;
      if ((A.checkdata & 0x04) && p[0] < P.rhomin) flags |= 0x04;
      if (A.checkdata & 0x08)
        for (int v = 0; v < V; ++v) if (invalid_value(p[v]) || invalid_value(c[v])) flags |= 0x08;
      p[2] = p[2] - w;
      double v3[4];
      CE::cfl_cell(p, csc, M, ip, v3);
      cflv = dmax(cflv, v3[0]);
      cflvis = dmax(cflvis, v3[3]);
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int v = 0; v < V; ++v) q[r][v] = q[r + 1][v];
    }
  }
  double vals[4] = {cflv, 0.0, 0.0, cflvis};
  block_reduce_emit<NT>(vals, M.vis ? 4 : 1, flags, A.ctl->invdt, &A.ctl->flags, sred);
}
template <bool EU, int TX, int TY>
__global__ void __launch_bounds__(TX* TY) fargo_advect_kernel(const __grid_constant__ FargoAdvArgs A) {
  fargo_advect_body<EU, TX, TY>(A, blockIdx.x, blockIdx.y);
}

// FargoAdvectionX (timedisc_base.f90:1779-1914) for the interior cells, the same transport
// along x with w(j): delxy = w*dt/dlx(IMIN), shift = NINT(delxy), delxy -= shift; the
// minmod-limited upwind residual step over i, then CSHIFT(q, -shift) over the interior
// columns.  The x ghosts of the input come from the boundary fill of the co-moving state.
// One thread per cell reads its five-cell window along x (adjacent threads, adjacent i) and
// writes the result to its shifted column; the closing ComputeRHS's CheckData and
// CalcTimestep see that cell at the shifted column (its metric and sound speed).
template <bool EU>
__device__ __forceinline__ void fargo_advect_x_body(const FargoAdvArgs& A, const int b, const int nb) {
  using PH = Phys<2, EU>;
  using CE = Cells<2, EU>;
  constexpr int V = PH::V;
  __shared__ double sred[RED_STRIDE * 8];
  if (A.ctl->stop | A.ctl->brk) return;
  if (gated_out(A.ctl, A.gate)) return;
  const Grid& g = A.g;
  const PhysP& P = A.ph;
  const MetricP& M = A.mt;
  double cflv = 0.0, cflvis = 0.0;
  int flags = 0;
  const double dte = A.dt_ctl ? A.ctl->dt : (A.dt_host > 0. ? A.dt_host : (A.ctl->time + A.ctl->dt) - A.ctl->time);
  const double dlx0 = M.dlx[2];   // dlx(IMIN, j): the metric depends on i only
  for (long long t = b * 256LL + threadIdx.x; t < g.n; t += (long long)nb * 256) {
    const int i = (int)(t % g.nx), j = (int)(t / g.nx);
    const double w = A.w[j + 2];
    double d = w * dte / dlx0;
    const double sh = round(d);   // NINT: half away from zero
    const int s = (int)sh;
    d = d - (double)s;
    auto load = [&](int ii, double* c) {
      if (ii >= 0 && ii < g.nx) {
        state_at<V>(A.in, g.n, CE::lin(g, ii, j, 0), c);
      } else {
        double p[V];
        CE::face_ghost_p(A.in, g, P, M, 0, ii, j, 0, p);
        PH::p2c(p, c, P);
      }
    };
    double q[5][V];
#pragma unroll
    for (int r = 0; r < 5; ++r) load(i - 2 + r, q[r]);
    double u[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      double a0 = q[1][v] - q[0][v], a1 = q[2][v] - q[1][v];
      double a2 = q[3][v] - q[2][v], a3 = q[4][v] - q[3][v];
      double fl, fr;   // flux(i-1), flux(i)
      if (d > 0.) {
        fl = q[1][v] + .5 * fargo_minmod(a0, a1) * (1. - d);
        fr = q[2][v] + .5 * fargo_minmod(a1, a2) * (1. - d);
      } else {
        fl = q[2][v] - .5 * fargo_minmod(a1, a2) * (1. + d);
        fr = q[3][v] - .5 * fargo_minmod(a2, a3) * (1. + d);
      }
      u[v] = q[2][v] - d * (fr - fl);
    }
    int id = (i + s) % g.nx;
    if (id < 0) id += g.nx;
    const long long o = CE::lin(g, id, j, 0);
#pragma unroll
    for (int v = 0; v < V; ++v) A.out[(long long)v * g.n + o] = u[v];
    // closing ComputeRHS: AddBackgroundVelocityX, CenterBoundary's Cons2Prim, CheckData;
    // CalcTimestep on the co-moving primitive state, at the cell's new column
    const int ipd = id + 2;
    double c[V], p[V];
#pragma unroll
    for (int v = 0; v < V; ++v) c[v] = u[v];
    frame_change<V>(c, 1.0, w, 1);
    PH::c2p(c, p, P);
    const double csc = EU ? PH::cs_of(p, P) : M.cs[ipd];
    if ((A.checkdata & 0x01) && !(csc > 0.)) flags |= 0x01;
    if (EU && (A.checkdata & 0x02) && p[V - 1] < P.pmin) flags |= 0x02;
    if ((A.checkdata & 0x04) && p[0] < P.rhomin) flags |= 0x04;
    if (A.checkdata & 0x08)
      for (int v = 0; v < V; ++v) if (invalid_value(p[v]) || invalid_value(c[v])) flags |= 0x08;
    p[1] = p[1] - w;
    double v3[4];
    CE::cfl_cell(p, csc, M, ipd, v3);
    cflv = dmax(cflv, v3[0]);
    cflvis = dmax(cflvis, v3[3]);
  }
  double vals[4] = {cflv, 0.0, 0.0, cflvis};
  block_reduce_emit<256>(vals, M.vis ? 4 : 1, flags, A.ctl->invdt, &A.ctl->flags, sred);
}
template <bool EU>
__global__ void __launch_bounds__(256) fargo_advect_x_kernel(const __grid_constant__ FargoAdvArgs A) {
  fargo_advect_x_body<EU>(A, blockIdx.x, gridDim.x);
}

// Batches of FARGO grids: the same passes over per-member argument tables, one block per
// (member, block) entry of a block table (x: member, y/z: block coordinates or, along x, the
// block and the member's block count); every FARGO member of a batch transports along the
// same direction (DIR)
template <bool EU, int DIR>
__global__ void __launch_bounds__(DIR == 1 ? 256 : FW_NT) batched_fargo_w_kernel(const FargoWArgs* __restrict__ args,
                                                                                 const int4* __restrict__ blocks) {
  const int4 T = blocks[blockIdx.x];
  if constexpr (DIR == 1) fargo_w_x_body<EU>(args[T.x], T.y);
  else fargo_w_body<EU>(args[T.x], T.y);
}
constexpr int FA_TX = 32, FA_TY = 4;   // the along-y transport's block of a batch
template <bool EU, int DIR>
__global__ void __launch_bounds__(DIR == 1 ? 256 : FA_TX* FA_TY) batched_fargo_advect_kernel(
    const FargoAdvArgs* __restrict__ args, const int4* __restrict__ blocks) {
  const int4 T = blocks[blockIdx.x];
  if constexpr (DIR == 1) fargo_advect_x_body<EU>(args[T.x], T.y, T.z);
  else fargo_advect_body<EU, FA_TX, FA_TY>(args[T.x], T.y, T.z);
}

// out = the frame-change chain C applied to every interior cell of the conservative state in
// (2D): the in-place Add/SubtractBackgroundVelocity calls that IntegrationStep makes on cvar
template <int V>
__global__ void __launch_bounds__(256) fargo_chain_copy_kernel(const double* __restrict__ in, double* __restrict__ out,
                                                               Grid g, Chain C, const Ctl* ctl, int gate) {
  if (ctl && gate && (ctl->stop | ctl->brk)) return;
  if (gated_out(ctl, gate)) return;
  for (long long t = blockIdx.x * 256LL + threadIdx.x; t < g.n; t += (long long)gridDim.x * 256) {
    const int i = (int)(t % g.nx), j = (int)(t / g.nx);
    double c[V];
#pragma unroll
    for (int v = 0; v < V; ++v) c[v] = in[(long long)v * g.n + t];
    apply_chain<V>(C, c, g, i, j);
#pragma unroll
    for (int v = 0; v < V; ++v) out[(long long)v * g.n + t] = c[v];
  }
}

}  // namespace fgpu
