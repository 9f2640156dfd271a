// fgpu_visc.cuh -- viscous source of one stage state (MOLECULAR model).
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
#pragma once
#include "fgpu_device.cuh"

namespace fgpu {

struct ViscArgs {
  Grid g;
  PhysP ph;
  MetricP mt;
  StateRef in;      // the stage state as the stencil reads it (rin or in)
  double eta;       // dynamic viscosity (dynconst)
  double mub;       // bulk viscosity (bulkconst)
  double* out;
};

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
    if (outside(a, ex) + outside(b, ey) + (ND == 3 ? outside(c, ez) : 0) > 2) continue;
    double p[V];
    CE::cell_p(A.in, g, A.ph, M, i0 + a, j0 + b, ND == 3 ? k0 + c : 0, p);
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
    const double vx = VV(0, a, b, c), vy = VV(1, a, b, c);
    const double vxW = VV(0, a - 1, b, c), vxE = VV(0, a + 1, b, c), vxS = VV(0, a, b - 1, c), vxN = VV(0, a, b + 1, c);
    const double vyW = VV(1, a - 1, b, c), vyE = VV(1, a + 1, b, c), vyS = VV(1, a, b - 1, c), vyN = VV(1, a, b + 1, c);
    if (ND == 2) {
      // VectorDivergence2D_1 of v (mesh_midpoint.f90:156-183) times the bulk viscosity
      const double tb = A.mub * div3d(M.dAxW[ip], M.dAxE[ip], M.dAyS[ip], M.dAyS[ip], 0.0, 0.0, M.dydzdV[ip],
                                      M.dzdxdV[ip], 0.0, 0.0, 0.0, 0.0, 0.0, 0.5 * (vxW + vx), 0.5 * (vxE + vx),
                                      0.5 * (vyS + vy), 0.5 * (vyN + vy), 0.0, 0.0, 0.0, 0.0, 0.0, 0.0);
      TT(0, a, b, c) = A.eta * ((vxE - vxW) / dlx + 2.0 * cxyx * vy) + tb;
      TT(1, a, b, c) = A.eta * ((vyN - vyS) / dly + 2.0 * cyxy * vx) + tb;
      TT(2, a, b, c) = A.eta * (0.5 * ((vyE - vyW) / dlx + (vxN - vxS) / dly) - cxyx * vx - cyxy * vy);
    } else {
      const double dlz = M.dlz[ip];
      const double cxzx = M.cxzx[ip], cyzy = M.cyzy[ip], czxz = M.czxz[ip], czyz = M.czyz[ip];
      const double vz = VV(2, a, b, c);
      const double vxB = VV(0, a, b, c - 1), vxT = VV(0, a, b, c + 1), vyB = VV(1, a, b, c - 1), vyT = VV(1, a, b, c + 1);
      const double vzW = VV(2, a - 1, b, c), vzE = VV(2, a + 1, b, c), vzS = VV(2, a, b - 1, c), vzN = VV(2, a, b + 1, c);
      const double vzB = VV(2, a, b, c - 1), vzT = VV(2, a, b, c + 1);
      // VectorDivergence3D (mesh_midpoint.f90:474-502)
      const double tb = A.mub * div3d(M.dAxW[ip], M.dAxE[ip], M.dAyS[ip], M.dAyS[ip], M.dAzB[ip], M.dAzB[ip],
                                      M.dydzdV[ip], M.dzdxdV[ip], M.dxdydV[ip], 0.0, 0.0, 0.0, 0.0,
                                      0.5 * (vxW + vx), 0.5 * (vxE + vx), 0.5 * (vyS + vy), 0.5 * (vyN + vy),
                                      0.5 * (vzB + vz), 0.5 * (vzT + vz), 0.0, 0.0, 0.0, 0.0);
      TT(0, a, b, c) = A.eta * ((vxE - vxW) / dlx + 2.0 * cxyx * vy + 2.0 * cxzx * vz) + tb;
      TT(1, a, b, c) = A.eta * ((vyN - vyS) / dly + 2.0 * cyxy * vx + 2.0 * cyzy * vz) + tb;
      TT(2, a, b, c) = A.eta * ((vzT - vzB) / dlz + 2.0 * czxz * vx + 2.0 * czyz * vy) + tb;
      TT(3, a, b, c) = A.eta * (0.5 * ((vyE - vyW) / dlx + (vxN - vxS) / dly) - cxyx * vx - cyxy * vy);
      TT(4, a, b, c) = A.eta * (0.5 * ((vzE - vzW) / dlx + (vxT - vxB) / dlz) - czxz * vz - cxzx * vx);
      TT(5, a, b, c) = A.eta * (0.5 * ((vyT - vyB) / dlz + (vzN - vzS) / dly) - czyz * vz - cyzy * vy);
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

}  // namespace fgpu
