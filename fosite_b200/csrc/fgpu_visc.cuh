// fgpu_visc.cuh -- viscous source of one stage state (sources_viscosity.f90).
//
// sources_viscosity.f90:484-507 ExternalSources: CalcStresses
// (physics_eulerisotherm.f90:1023-1198) builds the stress tensor
//   T = eta (grad v + grad v^T) + mu_b (div v) I
// at the cell centres of the interior and one ghost layer from the ghost-padded
// primitive velocity (CenterBoundary + SetCornerEdges, lab frame with FARGO);
// ViscositySources (physics_eulerisotherm.f90:982-1017, physics_euler.f90:
// 1887-1943) takes its curvilinear divergence from face averages
// (mesh_midpoint.f90:156-630) and, for ideal gas, the heating div(v.T).
//
// One block owns a TX x TY (x TZ) tile of interior cells and works in three
// shared-memory phases: the velocities of the cells within two steps (L1) of the
// tile, the stress tensor within one step, then the divergences of its own
// cells.  The result [ND momentum (+ energy)][n] is read by the stage kernel
// of the same state, which subtracts it with the other external sources.
//
// MOLECULAR viscosity is constant; ALPHA, BETA and POWERLAW keep a dynamic
// viscosity per padded cell that visc_update_kernel refreshes from the state
// whenever a right-hand side (or CalcTimestep) comes at a new time, as
// UpdateViscosity does, and visc_cfl_kernel evaluates their time-step limit.
#pragma once
#include "fgpu_kernels.cuh"

namespace fgpu {

struct ViscArgs {
  Grid g;
  PhysP ph;
  MetricP mt;
  StateRef in;             // the stage state as the stencil reads it (rin or in)
  double eta;              // MOLECULAR: dynamic viscosity (dynconst)
  double mub;              // MOLECULAR: bulk viscosity (bulkconst)
  const double* dynvis;    // other models: dynamic viscosity by padded cell (bulk = -2/3 of it)
  double* out;
  const Ctl* ctl;          // device-clock attempt slots: gate bits (0 = always run)
  int gate;
};

// index of a cell of the ghost-padded grid (coordinates -2 .. n+1; 2D meshes have no z ghosts)
template <int ND>
__device__ __forceinline__ long long pad_index(const Grid& g, int i, int j, int k) {
  return (long long)(i + 2) + (long long)(g.nx + 4) * ((long long)(j + 2) + (long long)(g.ny + 4) * (ND == 3 ? k + 2 : 0));
}

// Density and velocity of an interior cell of a stage state, as Cells::interior_p gives them
// (the FARGO frame chain without round trips, then Cons2Prim's m * (1/rho)), reading only the
// density and momentum fields (the velocity of a formed primitive state directly)
template <int ND>
__device__ __forceinline__ void interior_rv(const StateRef& S, const Grid& g, long long idx, int i, int j, double* rv) {
  const long long n = g.n;
  const double* b = S.base + idx;
#pragma unroll
  for (int v = 0; v <= ND; ++v) rv[v] = __ldg(b + (long long)v * n);
#pragma unroll 1
  for (int q = 0; q < S.nk; ++q) {
    const double* kq = S.K[q] + idx;
    const double a = S.dt_dev ? S.coef[q] * *S.dt_dev : S.coef[q];
#pragma unroll
    for (int v = 0; v <= ND; ++v) rv[v] = rv[v] - a * __ldg(kq + (long long)v * n);
  }
  if (S.ready) return;
  if (ND == 2 && S.pre.n) {
    // the frame changes of the momentum along the transport (the energy is not read)
    const int ix = fargo_ix(g, i, j);
    double m = g.fdir == 1 ? rv[1] : rv[2];
    for (int q = 0; q < S.pre.n; ++q) m = m + S.pre.s[q] * (rv[0] * S.pre.w[q][ix]);
    if (g.fdir == 1) rv[1] = m;
    else rv[2] = m;
  }
  const double inv_rho = 1. / rv[0];
#pragma unroll
  for (int m = 1; m <= ND; ++m) rv[m] = rv[m] * inv_rho;
}

// mesh_midpoint.f90:586-630 Divergence3D, arguments in the reference's order,
// evaluated left to right like the reference's expression
__device__ __forceinline__ double div3d(double aW, double aE, double aS, double aN, double aB, double aT,
                                        double dydzdV, double dxdzdV, double dxdydV,
                                        double cxyx, double cxzx, double cyxy, double czxz,
                                        double TxxW, double TxxE, double TxyS, double TxyN, double TxzB, double TxzT,
                                        double TyxC, double TzxC, double TyyC, double TzzC) {
  return dydzdV * (aE * TxxE - aW * TxxW) + dxdzdV * (aN * TxyN - aS * TxyS) + dxdydV * (aT * TxzT - aB * TxzB) +
         cxyx * TyxC + cxzx * TzxC - cyxy * TyyC - czxz * TzzC;
}

template <int ND, int TX, int TY, int TZ>
struct ViscTile {
  static constexpr int HZ = ND == 3 ? 2 : 0, HB = ND == 3 ? 1 : 0;
  static constexpr int VX = TX + 4, VY = TY + 4, VZ = TZ + 2 * HZ;   // velocity box
  static constexpr int BX = TX + 2, BY = TY + 2, BZ = TZ + 2 * HB;   // stress box
  static constexpr int NB = ND == 3 ? 6 : 3;                          // xx yy (zz) xy (xz yz)
  static constexpr size_t SMEM = sizeof(double) * ((size_t)ND * VX * VY * VZ + (size_t)NB * BX * BY * BZ);
};

// steps outside [0, e) along one axis
__device__ __forceinline__ int outside(int a, int e) { return a < 0 ? -a : (a >= e ? a - e + 1 : 0); }

template <int ND, bool EU, int TX, int TY, int TZ>
__global__ void __launch_bounds__(TX* TY* TZ) visc_kernel(const __grid_constant__ ViscArgs A) {
  using CE = Cells<ND, EU>;
  using L = ViscTile<ND, TX, TY, TZ>;
  constexpr int V = Phys<ND, EU>::V;
  constexpr int NT = TX * TY * TZ;
  constexpr int VX = L::VX, VY = L::VY, VZ = L::VZ, BX = L::BX, BY = L::BY, BZ = L::BZ;
  extern __shared__ __align__(16) double visc_smem[];
  if (A.gate && (A.ctl->stop | A.ctl->brk)) return;
  if (gated_out(A.ctl, A.gate)) return;
  double* const Vs = visc_smem;                     // [ND][VZ][VY][VX]
  double* const Ts = Vs + ND * VX * VY * VZ;        // [NB][BZ][BY][BX]
  const Grid& g = A.g;
  const MetricP& M = A.mt;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY, k0 = ND == 3 ? blockIdx.z * TZ : 0;
  const int ex = min(TX, g.nx - i0), ey = min(TY, g.ny - j0), ez = ND == 3 ? min(TZ, g.nz - k0) : 1;
  auto VV = [&](int m, int a, int b, int c) -> double& {   // velocity at tile-local (a, b, c)
    return Vs[((m * VZ + (c + L::HZ)) * VY + (b + 2)) * VX + (a + 2)];
  };
  auto TT = [&](int q, int a, int b, int c) -> double& {   // stress component q at tile-local (a, b, c)
    return Ts[((q * BZ + (c + L::HB)) * BY + (b + 1)) * BX + (a + 1)];
  };

  // ---- phase 1: primitive velocity of the ghost-padded state within two steps of the tile
  for (int t = threadIdx.x; t < VX * VY * VZ; t += NT) {
    const int lx = t % VX, r = t / VX, ly = r % VY, lz = r / VY;
    const int a = lx - 2, b = ly - 2, c = lz - L::HZ;
    const int ox = outside(a, ex), oy = outside(b, ey), oz = ND == 3 ? outside(c, ez) : 0;
    if (ox + oy + oz > 2) continue;
    const int gi = i0 + a, gj = j0 + b, gk = ND == 3 ? k0 + c : 0;
    double p[V];
    if (gi >= 0 && gi < g.nx && gj >= 0 && gj < g.ny && gk >= 0 && gk < g.nz)
      interior_rv<ND>(A.in, g, CE::lin(g, gi, gj, gk), gi, gj, p);
    else
      CE::cell_p(A.in, g, A.ph, M, gi, gj, gk, p);
#pragma unroll
    for (int m = 0; m < ND; ++m) Vs[((m * VZ + lz) * VY + ly) * VX + lx] = p[1 + m];
  }
  __syncthreads();

  // ---- phase 2: CalcStresses within one step of the tile (the interior and the first ghost layer)
  for (int t = threadIdx.x; t < BX * BY * BZ; t += NT) {
    const int lx = t % BX, r = t / BX, ly = r % BY, lz = r / BY;
    const int a = lx - 1, b = ly - 1, c = lz - L::HB;
    if (outside(a, ex) + outside(b, ey) + (ND == 3 ? outside(c, ez) : 0) > 1) continue;
    const int ip = i0 + a + 2;
    const double dlx = M.dlx[ip], dly = M.dly[ip];
    const double cxyx = M.cxyx[ip], cyxy = M.cyxy[ip];
    double eta = A.eta, mub = A.mub;
    if (A.dynvis) {
      eta = A.dynvis[pad_index<ND>(g, i0 + a, j0 + b, ND == 3 ? k0 + c : 0)];
      mub = -2. / 3. * eta;
    }
    const double vx = VV(0, a, b, c), vy = VV(1, a, b, c);
    const double vxW = VV(0, a - 1, b, c), vxE = VV(0, a + 1, b, c), vxS = VV(0, a, b - 1, c), vxN = VV(0, a, b + 1, c);
    const double vyW = VV(1, a - 1, b, c), vyE = VV(1, a + 1, b, c), vyS = VV(1, a, b - 1, c), vyN = VV(1, a, b + 1, c);
    if (ND == 2) {
      // VectorDivergence2D_1 of v (mesh_midpoint.f90:156-183) times the bulk viscosity
      const double tb = mub * div3d(M.dAxW[ip], M.dAxE[ip], M.dAyS[ip], M.dAyS[ip], 0.0, 0.0, M.dydzdV[ip],
                                      M.dzdxdV[ip], 0.0, 0.0, 0.0, 0.0, 0.0, 0.5 * (vxW + vx), 0.5 * (vxE + vx),
                                      0.5 * (vyS + vy), 0.5 * (vyN + vy), 0.0, 0.0, 0.0, 0.0, 0.0, 0.0);
      TT(0, a, b, c) = eta * ((vxE - vxW) / dlx + 2.0 * cxyx * vy) + tb;
      TT(1, a, b, c) = eta * ((vyN - vyS) / dly + 2.0 * cyxy * vx) + tb;
      TT(2, a, b, c) = eta * (0.5 * ((vyE - vyW) / dlx + (vxN - vxS) / dly) - cxyx * vx - cyxy * vy);
    } else {
      const double dlz = M.dlz[ip];
      const double cxzx = M.cxzx[ip], cyzy = M.cyzy[ip], czxz = M.czxz[ip], czyz = M.czyz[ip];
      const double vz = VV(2, a, b, c);
      const double vxB = VV(0, a, b, c - 1), vxT = VV(0, a, b, c + 1), vyB = VV(1, a, b, c - 1), vyT = VV(1, a, b, c + 1);
      const double vzW = VV(2, a - 1, b, c), vzE = VV(2, a + 1, b, c), vzS = VV(2, a, b - 1, c), vzN = VV(2, a, b + 1, c);
      const double vzB = VV(2, a, b, c - 1), vzT = VV(2, a, b, c + 1);
      // VectorDivergence3D (mesh_midpoint.f90:474-502)
      const double tb = mub * div3d(M.dAxW[ip], M.dAxE[ip], M.dAyS[ip], M.dAyS[ip], M.dAzB[ip], M.dAzB[ip],
                                      M.dydzdV[ip], M.dzdxdV[ip], M.dxdydV[ip], 0.0, 0.0, 0.0, 0.0,
                                      0.5 * (vxW + vx), 0.5 * (vxE + vx), 0.5 * (vyS + vy), 0.5 * (vyN + vy),
                                      0.5 * (vzB + vz), 0.5 * (vzT + vz), 0.0, 0.0, 0.0, 0.0);
      TT(0, a, b, c) = eta * ((vxE - vxW) / dlx + 2.0 * cxyx * vy + 2.0 * cxzx * vz) + tb;
      TT(1, a, b, c) = eta * ((vyN - vyS) / dly + 2.0 * cyxy * vx + 2.0 * cyzy * vz) + tb;
      TT(2, a, b, c) = eta * ((vzT - vzB) / dlz + 2.0 * czxz * vx + 2.0 * czyz * vy) + tb;
      TT(3, a, b, c) = eta * (0.5 * ((vyE - vyW) / dlx + (vxN - vxS) / dly) - cxyx * vx - cyxy * vy);
      TT(4, a, b, c) = eta * (0.5 * ((vzE - vzW) / dlx + (vxT - vxB) / dlz) - czxz * vz - cxzx * vx);
      TT(5, a, b, c) = eta * (0.5 * ((vyT - vyB) / dlz + (vzN - vzS) / dly) - czyz * vz - cyzy * vy);
    }
  }
  __syncthreads();

  // ---- phase 3: tensor divergence (and the heating) of the own cell
  const int a = threadIdx.x % TX, b = (threadIdx.x / TX) % TY, c = ND == 3 ? threadIdx.x / (TX * TY) : 0;
  if (a >= ex || b >= ey || c >= ez) return;
  const int ip = i0 + a + 2;
  const long long idx = CE::lin(g, i0 + a, j0 + b, k0 + c);
  const double aW = M.dAxW[ip], aE = M.dAxE[ip], aS = M.dAyS[ip];
  const double dydzdV = M.dydzdV[ip], dzdxdV = M.dzdxdV[ip];
  const double cxyx = M.cxyx[ip], cyxy = M.cyxy[ip];
  double sv[ND + 1];
  if (ND == 2) {
    const double xx = TT(0, a, b, c), yy = TT(1, a, b, c), xy = TT(2, a, b, c);
    // TensorDivergence2D_1 (mesh_midpoint.f90:283-323) with Tyx = Txy
    sv[0] = div3d(aW, aE, aS, aS, 0.0, 0.0, dydzdV, dzdxdV, 0.0, cxyx, 0.0, cyxy, 0.0,
                  0.5 * (TT(0, a - 1, b, c) + xx), 0.5 * (TT(0, a + 1, b, c) + xx),
                  0.5 * (TT(2, a, b - 1, c) + xy), 0.5 * (TT(2, a, b + 1, c) + xy), 0.0, 0.0, xy, 0.0, yy, 0.0);
    sv[1] = div3d(aW, aE, aS, aS, 0.0, 0.0, dydzdV, dzdxdV, 0.0, -cxyx, 0.0, -cyxy, 0.0,
                  0.5 * (TT(2, a - 1, b, c) + xy), 0.5 * (TT(2, a + 1, b, c) + xy),
                  0.5 * (TT(1, a, b - 1, c) + yy), 0.5 * (TT(1, a, b + 1, c) + yy), 0.0, 0.0, xx, 0.0, xy, 0.0);
    if (EU) {
      // div(v.T): (vx Txx + vy Txy, vx Txy + vy Tyy) at the neighbours along their own axis
      auto ex_ = [&](int da, int db) {
        return VV(0, a + da, b + db, c) * TT(0, a + da, b + db, c) + VV(1, a + da, b + db, c) * TT(2, a + da, b + db, c);
      };
      auto ey_ = [&](int da, int db) {
        return VV(0, a + da, b + db, c) * TT(2, a + da, b + db, c) + VV(1, a + da, b + db, c) * TT(1, a + da, b + db, c);
      };
      const double tx = ex_(0, 0), ty = ey_(0, 0);
      sv[2] = div3d(aW, aE, aS, aS, 0.0, 0.0, dydzdV, dzdxdV, 0.0, 0.0, 0.0, 0.0, 0.0,
                    0.5 * (ex_(-1, 0) + tx), 0.5 * (ex_(1, 0) + tx), 0.5 * (ey_(0, -1) + ty), 0.5 * (ey_(0, 1) + ty),
                    0.0, 0.0, 0.0, 0.0, 0.0, 0.0);
    }
  } else {
    const double aB = M.dAzB[ip], dxdydV = M.dxdydV[ip];
    const double cxzx = M.cxzx[ip], cyzy = M.cyzy[ip], czxz = M.czxz[ip], czyz = M.czyz[ip];
    const double xx = TT(0, a, b, c), yy = TT(1, a, b, c), zz = TT(2, a, b, c);
    const double xy = TT(3, a, b, c), xz = TT(4, a, b, c), yz = TT(5, a, b, c);
    // TensorDivergence3D (mesh_midpoint.f90:508-580) with Tyx = Txy, Tzx = Txz, Tzy = Tyz
    sv[0] = div3d(aW, aE, aS, aS, aB, aB, dydzdV, dzdxdV, dxdydV, cxyx, cxzx, cyxy, czxz,
                  0.5 * (TT(0, a - 1, b, c) + xx), 0.5 * (TT(0, a + 1, b, c) + xx),
                  0.5 * (TT(3, a, b - 1, c) + xy), 0.5 * (TT(3, a, b + 1, c) + xy),
                  0.5 * (TT(4, a, b, c - 1) + xz), 0.5 * (TT(4, a, b, c + 1) + xz), xy, xz, yy, zz);
    sv[1] = div3d(aW, aE, aS, aS, aB, aB, dydzdV, dzdxdV, dxdydV, -cxyx, cyzy, -cyxy, czyz,
                  0.5 * (TT(3, a - 1, b, c) + xy), 0.5 * (TT(3, a + 1, b, c) + xy),
                  0.5 * (TT(1, a, b - 1, c) + yy), 0.5 * (TT(1, a, b + 1, c) + yy),
                  0.5 * (TT(5, a, b, c - 1) + yz), 0.5 * (TT(5, a, b, c + 1) + yz), xx, yz, xy, zz);
    sv[2] = div3d(aW, aE, aS, aS, aB, aB, dydzdV, dzdxdV, dxdydV, czyz, -cxzx, cyzy, -czxz,
                  0.5 * (TT(4, a - 1, b, c) + xz), 0.5 * (TT(4, a + 1, b, c) + xz),
                  0.5 * (TT(5, a, b - 1, c) + yz), 0.5 * (TT(5, a, b + 1, c) + yz),
                  0.5 * (TT(2, a, b, c - 1) + zz), 0.5 * (TT(2, a, b, c + 1) + zz), yz, xx, yy, xz);
    if (EU) {
      // v.T rows: (xx xy xz), (xy yy yz), (xz yz zz)
      auto row = [&](int q0, int q1, int q2, int da, int db, int dc) {
        return VV(0, a + da, b + db, c + dc) * TT(q0, a + da, b + db, c + dc) +
               VV(1, a + da, b + db, c + dc) * TT(q1, a + da, b + db, c + dc) +
               VV(2, a + da, b + db, c + dc) * TT(q2, a + da, b + db, c + dc);
      };
      const double tx = row(0, 3, 4, 0, 0, 0), ty = row(3, 1, 5, 0, 0, 0), tz = row(4, 5, 2, 0, 0, 0);
      sv[3] = div3d(aW, aE, aS, aS, aB, aB, dydzdV, dzdxdV, dxdydV, 0.0, 0.0, 0.0, 0.0,
                    0.5 * (row(0, 3, 4, -1, 0, 0) + tx), 0.5 * (row(0, 3, 4, 1, 0, 0) + tx),
                    0.5 * (row(3, 1, 5, 0, -1, 0) + ty), 0.5 * (row(3, 1, 5, 0, 1, 0) + ty),
                    0.5 * (row(4, 5, 2, 0, 0, -1) + tz), 0.5 * (row(4, 5, 2, 0, 0, 1) + tz), 0.0, 0.0, 0.0, 0.0);
    }
  }
#pragma unroll
  for (int m = 0; m < ND + (EU ? 1 : 0); ++m) A.out[(long long)m * g.n + idx] = sv[m];
}

// ---------------------------------------------------------------- ALPHA / BETA / POWERLAW
// sources_viscosity.f90:359-453 UpdateViscosity on the ghost-padded stage state: only when the
// right-hand side's time differs from the last update's, or is 0.  The time is the host value t
// or, on the device clock, *t_dev + zeta * *dt_dev (the reference's time + zeta*dt).
struct VisUpdArgs {
  Grid g;
  PhysP ph;
  MetricP mt;
  StateRef in;
  int model;                 // FGPU_VIS_ALPHA / _BETA / _POWERLAW
  double dynconst, power;
  const double* ephir;       // [ndim][npad] ephi/r in curvilinear components
  const double* rad;         // [npad] Mesh%radius at the bary centres
  double* dynvis;            // [npad]
  const double* vis_time;    // time of the last update (initially -1)
  double t;
  const double* t_dev;
  const double* dt_dev;
  double zeta;
  long long npad;
  const Ctl* ctl;            // device clock: nothing to do once the run has stopped or broken
  int gate;                  // device-clock attempt slots (ACT_* bits)
};

__device__ __forceinline__ double vis_rhs_time(const VisUpdArgs& A) {
  return A.t_dev ? *A.t_dev + A.zeta * *A.dt_dev : A.t;
}

template <int ND, bool EU>
__global__ void __launch_bounds__(256) visc_update_kernel(const __grid_constant__ VisUpdArgs A) {
  using CE = Cells<ND, EU>;
  constexpr int V = Phys<ND, EU>::V;
  if (A.ctl && (A.ctl->stop | A.ctl->brk)) return;
  if (gated_out(A.ctl, A.gate)) return;
  const double t = vis_rhs_time(A);
  if (!(t != *A.vis_time || t == 0.0)) return;
  const int NXp = A.g.nx + 4, NYp = A.g.ny + 4;
  for (long long q = blockIdx.x * 256LL + threadIdx.x; q < A.npad; q += (long long)gridDim.x * 256) {
    const int px = (int)(q % NXp), py = (int)((q / NXp) % NYp), pz = (int)(q / ((long long)NXp * NYp));
    const int gi = px - 2, gj = py - 2, gk = ND == 3 ? pz - 2 : 0;
    double p[V];
    if (gi >= 0 && gi < A.g.nx && gj >= 0 && gj < A.g.ny && gk >= 0 && gk < A.g.nz)
      interior_rv<ND>(A.in, A.g, CE::lin(A.g, gi, gj, gk), gi, gj, p);
    else
      CE::cell_p(A.in, A.g, A.ph, A.mt, gi, gj, gk, p);
    double om = A.ephir[q] * p[1];
#pragma unroll
    for (int l = 1; l < ND; ++l) om = om + A.ephir[(long long)l * A.npad + q] * p[1 + l];
    om = om + 0.0;   // Mesh%Omega of a non-rotating frame
    const double r = A.rad[q];
    double eta;
    if (A.model == 2) {
      const double cs = A.mt.cs[px];
      eta = A.dynconst * p[0] * (cs * cs) / fabs(om);
    } else if (A.model == 3) {
      eta = A.dynconst * p[0] * (r * r) * fabs(om);
    } else {
      eta = A.dynconst * p[0] * pow(r * r * fabs(om), A.power);
    }
    A.dynvis[q] = eta;
  }
}

// records the update's time (after visc_update_kernel, whose blocks all read the old value)
__global__ void visc_time_kernel(VisUpdArgs A, double* vis_time) {
  if (A.ctl && (A.ctl->stop | A.ctl->brk)) return;
  if (gated_out(A.ctl, A.gate)) return;
  *vis_time = vis_rhs_time(A);
}

// The viscous time-step limit of sources_viscosity.f90:511-581 with the cell dynamic viscosity,
// over every cell of the ghost-padded state (CalcTimestep's this%pvar): the maximum of
// sum_d (max wave speed_d + 2 kinvis/dl_d)/dl_d goes to ctl->invdt[3]
struct VisCflArgs {
  Grid g;
  PhysP ph;
  MetricP mt;
  StateRef in;
  int roundtrip;             // the checked state gets the CHECK_PMIN clamp (ideal gas)
  const double* dynvis;
  long long npad;
  Ctl* ctl;
  int gate;
};

template <int ND, bool EU>
__global__ void __launch_bounds__(256) visc_cfl_kernel(const __grid_constant__ VisCflArgs A) {
  using PH = Phys<ND, EU>;
  using CE = Cells<ND, EU>;
  constexpr int V = PH::V;
  __shared__ double sred[RED_STRIDE * 8];
  if (A.ctl->stop | A.ctl->brk) return;
  if (gated_out(A.ctl, A.gate)) return;
  const MetricP& M = A.mt;
  const int NXp = A.g.nx + 4, NYp = A.g.ny + 4;
  double mx = 0.0;
  for (long long q = blockIdx.x * 256LL + threadIdx.x; q < A.npad; q += (long long)gridDim.x * 256) {
    const int px = (int)(q % NXp), py = (int)((q / NXp) % NYp), pz = (int)(q / ((long long)NXp * NYp));
    double p[V];
    CE::cell_p(A.in, A.g, A.ph, M, px - 2, py - 2, ND == 3 ? pz - 2 : 0, p);
    if (EU && A.roundtrip) p[V - 1] = dmax(p[V - 1], A.ph.pmin);
    const double cs = EU ? PH::cs_of(p, A.ph) : M.cs[px];
    const double dl[3] = {M.dlx[px], M.dly[px], ND == 3 ? M.dlz[px] : 1.0};
    const double kinvis = A.dynvis[q] / p[0];
    double s = 0.0;
#pragma unroll
    for (int m = 0; m < ND; ++m) {
      const double v = p[1 + m];
      const double w = dmax(dmax(0., v + cs), -dmin(0., v - cs));
      const double term = (w + 2.0 * kinvis / dl[m]) / dl[m];
      s = m == 0 ? term : s + term;
    }
    mx = dmax(mx, s);
  }
  double vals[4] = {0.0, 0.0, 0.0, mx};
  block_reduce_emit<256>(vals, 4, 0, A.ctl->invdt, nullptr, sred);
}

}  // namespace fgpu
