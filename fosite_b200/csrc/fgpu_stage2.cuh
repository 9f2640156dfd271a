// fgpu_stage2.cuh -- the fused stage kernel, warp-shuffle layout.
//
// Each block owns a window of 32 x NW points (columns -1..30, rows -1..NW-2
// of its output tile); thread (lane, warp) holds one point.  The output tile
// is 30 x (NW-2) cells.  Per plane:
//   x: every lane reconstructs the west and east faces of its point, the
//      west-face data moves one lane left with __shfl_down, the KT flux of the
//      interface (c, c+1) is formed in registers and the flux of (c-1, c)
//      arrives with __shfl_up -- no shared memory, no barrier;
//   y: every column thread writes its south-face data to shared memory, the
//      thread below forms the KT flux of the interface, one more exchange gives
//      the divergence (two barriers);
//   z (3D): a register window along the marching direction.
// The arithmetic per face/interface is the same code as kt_flux, so results
// are bit-identical to the tile kernel.
#pragma once
#include "fgpu_kernels.cuh"

namespace fgpu {

template <int ND, bool EU, bool PRIM>
struct FaceOps {
  using PH = Phys<ND, EU>;
  static constexpr int V = PH::V;
  static constexpr int FD = 2 * V + 2;   // cons, physical flux, min(0,u-cs), max(0,u+cs)

  // face data of one reconstructed face state for transport along d
  static __device__ __forceinline__ void face(int d, const double* Rf, double cs_iso, const PhysP& P, double* fd) {
    double p[V], c[V];
    if (PRIM) {
#pragma unroll
      for (int l = 0; l < V; ++l) p[l] = Rf[l];
      PH::p2c(p, c, P);
    } else {
#pragma unroll
      for (int l = 0; l < V; ++l) c[l] = Rf[l];
      PH::c2p(c, p, P);
    }
    double cs = EU ? PH::cs_of(p, P) : cs_iso;
    int vn = 1 + d;
    double u = p[vn];
    double f[V];
    f[0] = p[0] * u;
    if (EU) {
      double Pp = p[V - 1];
#pragma unroll
      for (int m = 1; m <= ND; ++m) f[m] = (m == vn) ? c[m] * u + Pp : c[m] * u;
      f[V - 1] = (c[V - 1] + Pp) * u;
    } else {
#pragma unroll
      for (int m = 1; m <= ND; ++m) f[m] = (m == vn) ? c[m] * u + p[0] * cs * cs : c[m] * u;
    }
#pragma unroll
    for (int l = 0; l < V; ++l) { fd[l] = c[l]; fd[V + l] = f[l]; }
    fd[2 * V] = dmin(0., u - cs);
    fd[2 * V + 1] = dmax(0., u + cs);
  }
  // KT flux from the plus face of the left cell (L) and the minus face of the right cell (R)
  static __device__ __forceinline__ void kt(const double* L, const double* R, double dA, double* F) {
    double am = dmin(dmin(0.0, R[2 * V]), L[2 * V]);
    double ap = dmax(dmax(0.0, R[2 * V + 1]), L[2 * V + 1]);
    double fac = dA / (ap - am);
    double amap = am * ap;
#pragma unroll
    for (int l = 0; l < V; ++l) F[l] = fac * (ap * L[V + l] - am * R[V + l] + amap * (R[l] - L[l]));
  }
};

__device__ __forceinline__ double shfl_down1(double x) { return __shfl_down_sync(0xffffffffu, x, 1); }
__device__ __forceinline__ double shfl_up1(double x) { return __shfl_up_sync(0xffffffffu, x, 1); }

template <int ND, bool EU, bool PRIM, int NW>
__global__ void __launch_bounds__(32 * NW, 2) stage2_kernel(const __grid_constant__ StageArgs A) {
  using PH = Phys<ND, EU>;
  using CE = Cells<ND, EU>;
  using FO = FaceOps<ND, EU, PRIM>;
  constexpr int V = PH::V;
  constexpr int FD = FO::FD;
  constexpr int NT = 32 * NW;
  constexpr int TXO = 30, TYO = NW - 2;
  constexpr int RW = 34, RH = NW + 2;           // R window: columns -2..31, rows -2..NW-1
  __shared__ double Rs[V * RH * RW];
  __shared__ double Fy[FD * NW * TXO];          // south-face data of rows -1..NW-2
  __shared__ double Gy[V * (NW - 1) * TXO];     // y fluxes of interfaces (r, r+1), r = -1..NW-3
  __shared__ double sred[RED_STRIDE * NW];

  if (A.ctl && (A.ctl->stop | A.ctl->brk)) return;
  const Grid& g = A.g;
  const PhysP& P = A.ph;
  const MetricP& M = A.mt;
  const double dt = A.dt_dev ? *A.dt_dev : A.dt;
  const bool roundtrip = EU && A.in.roundtrip;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int c = lane - 1, r = w - 1;              // the thread's point within the tile
  const int i0 = blockIdx.x * TXO, j0 = blockIdx.y * TYO;
  const int exo = min(TXO, g.nx - i0), eyo = min(TYO, g.ny - j0);
  const int gi = i0 + c, gj = j0 + r;
  // the point is needed if it lies in the cross-shaped stencil region of the output tile
  const bool inx = c >= 0 && c < exo, iny = r >= 0 && r < eyo;
  const bool needed = (inx && r >= -2 && r <= eyo + 1) || (iny && c >= -2 && c <= exo + 1);
  const bool out = inx && iny;
  const int ip = gi + 2;
  const bool inxy = gi >= 0 && gi < g.nx && gj >= 0 && gj < g.ny;   // z window only for in-domain columns
  int k0 = 0, k1 = 1;
  if (ND == 3) { k0 = blockIdx.z * A.kchunk; k1 = min(g.nz, k0 + A.kchunk); }

  auto RS = [&](int v, int rr, int cc) -> double& { return Rs[(v * RH + (rr + 2)) * RW + (cc + 2)]; };

  auto recon_at = [&](int xi, int xj, int xk, double* R) {
    double p[V];
    bool ix = xi >= 0 && xi < g.nx, iy = xj >= 0 && xj < g.ny, iz = xk >= 0 && xk < g.nz;
    if (ix && iy && iz) {
      double u[V];
      state_at<V>(A.in, g.n, CE::lin(g, xi, xj, xk), u);
      if (PRIM) {
        PH::c2p(u, p, P);
        if (roundtrip) p[V - 1] = dmax(p[V - 1], P.pmin);
#pragma unroll
        for (int l = 0; l < V; ++l) R[l] = p[l];
      } else if (roundtrip) {
        PH::c2p(u, p, P);
        p[V - 1] = dmax(p[V - 1], P.pmin);
        PH::p2c(p, R, P);
      } else {
#pragma unroll
        for (int l = 0; l < V; ++l) R[l] = u[l];
      }
    } else {
      int d = !ix ? 0 : (!iy ? 1 : 2);
      CE::face_ghost_p(A.in, g, P, M, d, xi, xj, xk, p);
      if (roundtrip) p[V - 1] = dmax(p[V - 1], P.pmin);
      if (PRIM) {
#pragma unroll
        for (int l = 0; l < V; ++l) R[l] = p[l];
      } else {
        PH::p2c(p, R, P);
      }
    }
  };

  double cflv[3] = {0.0, 0.0, 0.0};
  double errv = 0.0;
  int flags = 0;

  // 3D register window of the own column: R(k), R(k+1); for output cells also the
  // z-slope at k and the z-flux at k-1/2
  double Rz0[V], Rz1[V], sz0[V], Fzm[V];
  if (ND == 3 && needed && inxy) {
    recon_at(gi, gj, k0, Rz0);
    recon_at(gi, gj, k0 + 1, Rz1);
    if (out) {
      double Ra[V], Rb[V], szm[V];
      recon_at(gi, gj, k0 - 2, Ra);
      recon_at(gi, gj, k0 - 1, Rb);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        szm[v] = A.constant_recon ? 0.0 : slope(A.limiter, A.theta, A.invd[2], Ra[v], Rb[v], Rz0[v]);
        sz0[v] = A.constant_recon ? 0.0 : slope(A.limiter, A.theta, A.invd[2], Rb[v], Rz0[v], Rz1[v]);
      }
      double oT = M.offzT[k0 - 1 + 2], oB = M.offzB[k0 + 2];
      double FL[FD], FR[FD], Rf[V];
#pragma unroll
      for (int v = 0; v < V; ++v) Rf[v] = A.constant_recon ? Rb[v] : Rb[v] + szm[v] * oT;
      FO::face(2, Rf, EU ? 0.0 : M.cs[6 * M.nxp + ip], P, FL);
#pragma unroll
      for (int v = 0; v < V; ++v) Rf[v] = A.constant_recon ? Rz0[v] : Rz0[v] + sz0[v] * oB;
      FO::face(2, Rf, EU ? 0.0 : M.cs[5 * M.nxp + ip], P, FR);
      FO::kt(FL, FR, M.dAzB[ip], Fzm);
    }
  }

  for (int k = k0; k < k1; ++k) {
    double Rc[V], divZ[V];
    // ---- own point of plane k (and the z-flux at k+1/2 for output cells)
    if (needed) {
      if (ND == 3 && inxy) {
        double Rz2[V];
        recon_at(gi, gj, k + 2, Rz2);
        if (out) {
          double sz1[V];
#pragma unroll
          for (int v = 0; v < V; ++v)
            sz1[v] = A.constant_recon ? 0.0 : slope(A.limiter, A.theta, A.invd[2], Rz0[v], Rz1[v], Rz2[v]);
          double oT = M.offzT[k + 2], oB = M.offzB[k + 1 + 2];
          double FL[FD], FR[FD], Rf[V], Fzp[V];
#pragma unroll
          for (int v = 0; v < V; ++v) Rf[v] = A.constant_recon ? Rz0[v] : Rz0[v] + sz0[v] * oT;
          FO::face(2, Rf, EU ? 0.0 : M.cs[6 * M.nxp + ip], P, FL);
#pragma unroll
          for (int v = 0; v < V; ++v) Rf[v] = A.constant_recon ? Rz1[v] : Rz1[v] + sz1[v] * oB;
          FO::face(2, Rf, EU ? 0.0 : M.cs[5 * M.nxp + ip], P, FR);
          FO::kt(FL, FR, M.dAzB[ip], Fzp);
          double dV = M.dxdydV[ip];
#pragma unroll
          for (int v = 0; v < V; ++v) {
            divZ[v] = dV * (Fzp[v] - Fzm[v]);
            sz0[v] = sz1[v];
            Fzm[v] = Fzp[v];
          }
        }
#pragma unroll
        for (int v = 0; v < V; ++v) {
          Rc[v] = Rz0[v];
          Rz0[v] = Rz1[v];
          Rz1[v] = Rz2[v];
        }
      } else {
        recon_at(gi, gj, k, Rc);
      }
#pragma unroll
      for (int v = 0; v < V; ++v) RS(v, r, c) = Rc[v];
    }
    // ---- extra halo points of plane k: column -2 (and 31), row -2 (and NW-1)
    {
      const bool right = exo == TXO, top = eyo == TYO;
      const int nl = eyo, nr = right ? eyo : 0, nb = exo, nt = top ? exo : 0;
      const int H = nl + nr + nb + nt;
      for (int h = tid; h < H; h += NT) {
        int cc, rr;
        if (h < nl) { cc = -2; rr = h; }
        else if (h < nl + nr) { cc = TXO + 1; rr = h - nl; }
        else if (h < nl + nr + nb) { cc = h - nl - nr; rr = -2; }
        else { cc = h - nl - nr - nb; rr = TYO + 1; }
        double R[V];
        recon_at(i0 + cc, j0 + rr, k, R);
#pragma unroll
        for (int v = 0; v < V; ++v) RS(v, rr, cc) = R[v];
      }
    }
    __syncthreads();

    // ---- x direction in registers (rows with output cells)
    double divX[V];
    if (iny) {
      double R[V], sx[V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        R[v] = RS(v, r, c);
        sx[v] = A.constant_recon ? 0.0
                                 : slope(A.limiter, A.theta, A.invd[0], RS(v, r, c - 1), R[v], RS(v, r, c + 1));
      }
      const int ipc = min(max(ip, 0), M.nxp - 2);   // lanes beyond the tile compute unused values
      double Rf[V], Fw[FD], Fn[FD], Fe[FD], F[V];
      double oW = M.offxW[ipc], oE = M.offxE[ipc];
#pragma unroll
      for (int v = 0; v < V; ++v) Rf[v] = A.constant_recon ? R[v] : R[v] + sx[v] * oW;
      FO::face(0, Rf, EU ? 0.0 : M.cs[1 * M.nxp + ipc], P, Fw);
#pragma unroll
      for (int q = 0; q < FD; ++q) Fn[q] = shfl_down1(Fw[q]);
#pragma unroll
      for (int v = 0; v < V; ++v) Rf[v] = A.constant_recon ? R[v] : R[v] + sx[v] * oE;
      FO::face(0, Rf, EU ? 0.0 : M.cs[2 * M.nxp + ipc], P, Fe);
      FO::kt(Fe, Fn, M.dAxW[ipc + 1], F);          // interface (c, c+1)
      double dV = M.dydzdV[ipc];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        double Fm = shfl_up1(F[v]);                 // interface (c-1, c)
        divX[v] = dV * (F[v] - Fm);
      }
    }

    // ---- y direction: south-face data through shared memory
    double Fnorth[FD];
    const bool ycol = inx && r <= eyo;
    if (ycol) {
      double R[V], sy[V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        R[v] = RS(v, r, c);
        sy[v] = A.constant_recon ? 0.0
                                 : slope(A.limiter, A.theta, A.invd[1], RS(v, r - 1, c), R[v], RS(v, r + 1, c));
      }
      double Rf[V], Fs[FD];
      double oS = M.offyS[gj + 2], oN = M.offyN[gj + 2];
#pragma unroll
      for (int v = 0; v < V; ++v) Rf[v] = A.constant_recon ? R[v] : R[v] + sy[v] * oS;
      FO::face(1, Rf, EU ? 0.0 : M.cs[3 * M.nxp + ip], P, Fs);
#pragma unroll
      for (int q = 0; q < FD; ++q) Fy[(q * NW + (r + 1)) * TXO + c] = Fs[q];
#pragma unroll
      for (int v = 0; v < V; ++v) Rf[v] = A.constant_recon ? R[v] : R[v] + sy[v] * oN;
      FO::face(1, Rf, EU ? 0.0 : M.cs[4 * M.nxp + ip], P, Fnorth);
    }
    __syncthreads();
    if (ycol && r < eyo) {
      double Fup[FD], G[V];
#pragma unroll
      for (int q = 0; q < FD; ++q) Fup[q] = Fy[(q * NW + (r + 2)) * TXO + c];
      FO::kt(Fnorth, Fup, M.dAyS[ip], G);          // interface (r, r+1)
#pragma unroll
      for (int v = 0; v < V; ++v) Gy[(v * (NW - 1) + (r + 1)) * TXO + c] = G[v];
    }
    __syncthreads();

    // ---- output cells: divergence, sources, stage update, epilogues
    if (out) {
      double divY[V];
      double dVy = M.dzdxdV[ip];
#pragma unroll
      for (int v = 0; v < V; ++v)
        divY[v] = dVy * (Gy[(v * (NW - 1) + (r + 1)) * TXO + c] - Gy[(v * (NW - 1) + r) * TXO + c]);
      const long long idx = CE::lin(g, gi, gj, k);
      double pc[V], cc[V];
      if (PRIM) {
#pragma unroll
        for (int v = 0; v < V; ++v) pc[v] = Rc[v];
        // the sources read cvar itself (see stage_tile)
        if (!roundtrip && (M.curv || A.has_accel || A.out_base)) state_at<V>(A.in, g.n, idx, cc);
        else PH::p2c(pc, cc, P);
      } else {
#pragma unroll
        for (int v = 0; v < V; ++v) cc[v] = Rc[v];
        if (roundtrip) {
          double u[V];
          state_at<V>(A.in, g.n, idx, u);
          PH::c2p(u, pc, P);
          pc[V - 1] = dmax(pc[V - 1], P.pmin);
        } else {
          PH::c2p(cc, pc, P);
        }
      }
      double rhs[V];
#pragma unroll
      for (int v = 0; v < V; ++v) rhs[v] = (divX[v] + divY[v]) + (ND == 3 ? divZ[v] : 0.0);
      if (M.curv) {
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
      if (A.has_accel) {
        double ax = M.accel[ip], ay = M.accel[M.nxp + ip];
        rhs[1] = rhs[1] - cc[0] * ax;
        rhs[2] = rhs[2] - cc[0] * ay;
        if (EU) rhs[V - 1] = rhs[V - 1] - (cc[1] * ax + cc[2] * ay);
      }
      if (A.out_mode == OUT_RHS) {
#pragma unroll
        for (int v = 0; v < V; ++v) A.out[(long long)v * g.n + idx] = rhs[v];
      } else {
        double yn[V], y0[V], y[V];
        if (!PRIM || roundtrip) {
#pragma unroll
          for (int v = 0; v < V; ++v) yn[v] = cc[v];
        } else {
          state_at<V>(A.in, g.n, idx, yn);
        }
#pragma unroll
        for (int v = 0; v < V; ++v) y0[v] = __ldg(A.y0 + (long long)v * g.n + idx);
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
        if (A.cfl_mode == 1) {
          double p[V], cv[V];
          PH::c2p(y, p, P);
          if (EU && A.cfl_roundtrip) p[V - 1] = dmax(p[V - 1], P.pmin);
          double cs = EU ? PH::cs_of(p, P) : M.cs[ip];
          double v3[4];
          CE::cfl_cell(p, cs, M, ip, v3);
#pragma unroll
          for (int q = 0; q < 3; ++q) cflv[q] = dmax(cflv[q], v3[q]);
          if (EU && A.cfl_roundtrip) PH::p2c(p, cv, P);
          else {
#pragma unroll
            for (int v = 0; v < V; ++v) cv[v] = y[v];
          }
          if ((A.checkdata & 0x01) && !(cs > 0.)) flags |= 0x01;
          if (EU && (A.checkdata & 0x02) && p[V - 1] < P.pmin) flags |= 0x02;
          if ((A.checkdata & 0x04) && p[0] < P.rhomin) flags |= 0x04;
          if (A.checkdata & 0x08)
            for (int v = 0; v < V; ++v) if (invalid_value(p[v]) || invalid_value(cv[v])) flags |= 0x08;
        }
      }
      if (A.out_base) {
#pragma unroll
        for (int v = 0; v < V; ++v) A.out_base[(long long)v * g.n + idx] = cc[v];
      }
      if (A.cfl_mode == 2) {
        double cs = EU ? PH::cs_of(pc, P) : M.cs[ip];
        double v3[4];
        CE::cfl_cell(pc, cs, M, ip, v3);
#pragma unroll
        for (int q = 0; q < 3; ++q) cflv[q] = dmax(cflv[q], v3[q]);
        if ((A.checkdata & 0x01) && !(cs > 0.)) flags |= 0x01;
        if (EU && (A.checkdata & 0x02) && pc[V - 1] < P.pmin) flags |= 0x02;
        if ((A.checkdata & 0x04) && pc[0] < P.rhomin) flags |= 0x04;
        if (A.checkdata & 0x08)
          for (int v = 0; v < V; ++v) if (invalid_value(pc[v]) || invalid_value(cc[v])) flags |= 0x08;
      }
      if (A.last_stage) {
#pragma unroll
        for (int v = 0; v < V; ++v) {
          double b = __ldg(A.in.base + (long long)v * g.n + idx);
          double h = b, l = b;
          for (int q = 0; q < A.nstage - 1; ++q) {
            double kq = __ldg(A.in.K[q] + (long long)v * g.n + idx);
            l = l - A.bl_dt[q] * kq;
            h = h - A.bh_dt[q] * kq;
          }
          l = l - A.bl_dt[A.nstage - 1] * rhs[v];
          h = h - A.bh_dt[A.nstage - 1] * rhs[v];
          A.out_high[(long long)v * g.n + idx] = h;
          double e = fabs(h - l) / (A.tol_rel * fabs(h) + A.tol_abs[v]);
          errv = dmax(errv, e);
        }
      }
    }
    __syncthreads();
  }

  if (A.ctl && (A.cfl_mode || A.last_stage)) {
    int nv = A.cfl_mode ? (ND == 3 ? 3 : 1) : 0;
    double vals[3] = {cflv[0], cflv[1], cflv[2]};
    if (A.last_stage && !A.cfl_mode) { vals[0] = errv; nv = 1; }
    if (nv) block_reduce_emit<NT>(vals, nv, flags, A.last_stage && !A.cfl_mode ? &A.ctl->err : A.ctl->invdt,
                                  &A.ctl->flags, sred);
  }
}

}  // namespace fgpu
