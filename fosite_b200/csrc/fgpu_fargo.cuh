// fgpu_fargo.cuh -- FARGO transport along y (fosite fargo type 1, 2D x-y
// meshes, isothermal physics): the background velocity w(i) of
// CalcBackgroundVelocity and the shift + upwind residual advection of
// FargoAdvectionY, with the CFL / CheckData pass of the step's closing
// ComputeRHS + CalcTimestep fused into the advection.
#pragma once
#include "fgpu_kernels.cuh"

namespace fgpu {

struct FargoWArgs {
  Grid g;
  PhysP ph;
  MetricP mt;
  StateRef in;            // state whose real frame is in + in.pre
  const double* w_prev;   // background velocity of the last ComputeRHS (pvar round trip), or null
  const double* wfac;     // wfactor(i), by padded i
  double* w_out;          // new background velocity, by padded i
  Ctl* ctl;
};

// CalcBackgroundVelocity for direction 2 (timedisc_base.f90:2243-2326):
//   w(i) = SUM_j pvar(i,j,vy)*wfactor(i) / JNUM over the interior j, for every
//   padded column i (the x-ghost columns come from the boundary fill).
// pvar is the primitive state of the last ComputeRHS after its
// SubtractBackgroundVelocityY and this routine's AddBackgroundVelocityY, i.e.
// (vy - w_prev) + w_prev.  The sum runs in j order like the reference loop, so
// the result is bitwise reproducible: a block owns WX columns; per chunk of WR
// rows its threads evaluate the WR x WX terms in parallel into shared memory,
// then one thread per column adds them in order.
constexpr int FW_WX = 8, FW_WY = 32, FW_RPT = 4, FW_WR = FW_WY * FW_RPT;
template <bool EU>
__global__ void __launch_bounds__(FW_WX* FW_WY) fargo_w_kernel(const __grid_constant__ FargoWArgs A) {
  using CE = Cells<2, EU>;
  __shared__ double terms[FW_WR][FW_WX + 1];
  if (A.ctl && (A.ctl->stop | A.ctl->brk)) return;
  const Grid& g = A.g;
  const int tx = threadIdx.x % FW_WX, ty = threadIdx.x / FW_WX;
  const int ip = blockIdx.x * FW_WX + tx;
  const bool valid = ip < g.nx + 4;
  const int i = ip - 2;
  const bool ghost = i < 0 || i >= g.nx;
  const double wf = valid ? A.wfac[ip] : 0.0;
  const double wp = (valid && A.w_prev) ? A.w_prev[ip] : 0.0;
  double wi = 0.0;
  for (int j0 = 0; j0 < g.ny; j0 += FW_WR) {
#pragma unroll
    for (int r = 0; r < FW_RPT; ++r) {
      const int q = ty + FW_WY * r, j = j0 + q;
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
      const int nq = min(FW_WR, g.ny - j0);
      for (int q = 0; q < nq; ++q) wi = wi + terms[q][tx];
    }
    __syncthreads();
  }
  if (ty == 0 && valid) A.w_out[ip] = wi / (double)g.ny;
}

struct FargoAdvArgs {
  Grid g;
  PhysP ph;
  MetricP mt;
  StateRef in;           // co-moving state after the last stage (no frame changes)
  const double* w;       // background velocity, by padded i
  double* out;           // advected state (must not alias in.base)
  Ctl* ctl;              // dt/time source and CFL / CheckData sink
  int checkdata;
  int chunk;             // rows of one thread
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
__global__ void __launch_bounds__(TX* TY) fargo_advect_kernel(const __grid_constant__ FargoAdvArgs A) {
  using PH = Phys<2, EU>;
  using CE = Cells<2, EU>;
  constexpr int V = PH::V;
  constexpr int NT = TX * TY;
  __shared__ double sred[RED_STRIDE * ((NT + 31) / 32)];
  if (A.ctl->stop | A.ctl->brk) return;
  const Grid& g = A.g;
  const PhysP& P = A.ph;
  const MetricP& M = A.mt;
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  const int i = blockIdx.x * TX + tx;
  const int j0 = (blockIdx.y * TY + ty) * A.chunk;
  const int j1 = min(g.ny, j0 + A.chunk);
  double cflv = 0.0, cflvis = 0.0;
  int flags = 0;
  if (i < g.nx && j0 < g.ny) {
    const int ip = i + 2;
    const double w = A.w[ip];
    const double dte = (A.ctl->time + A.ctl->dt) - A.ctl->time;
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
      frame_change<V>(c, 1.0, w);
      PH::c2p(c, p, P);
      const double csc = EU ? PH::cs_of(p, P) : cs;
      if ((A.checkdata & 0x01) && !(csc > 0.)) flags |= 0x01;
      if (EU && (A.checkdata & 0x02) && p[V - 1] < P.pmin) flags |= 0x02;
      if ((A.checkdata & 0x04) && p[0] < P.rhomin) flags |= 0x04;
      if (A.checkdata & 0x08)
        for (int v = 0; v < V; ++v) if (!isfinite(p[v]) || !isfinite(c[v])) flags |= 0x08;
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

}  // namespace fgpu
