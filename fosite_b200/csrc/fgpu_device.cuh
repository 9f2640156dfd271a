// fgpu_device.cuh -- device-side physics, boundary synthesis and KT flux
// building blocks of the fused finite-volume stage kernels (sm_100a, FP64).
//
// State layout in HBM: interior cells only, structure of arrays, one field of
// n = nx*ny*nz doubles per variable, i fastest (the interior block of fosite's
// marray data4d).  Ghost cells are never stored: every kernel that needs a
// ghost value synthesises it from interior cells with the boundary rules of
// boundary_generic.f90:287-763 (CenterBoundary + SetCornerEdges).
//
// Metric factors of the supported geometries (cartesian, cylindrical,
// logcylindrical) depend on the first coordinate only, so they live in 1-D
// arrays indexed by the ghost-padded i (i + 2).
#pragma once
#include <cstdint>
#include <cfloat>

#define FGPU_MAXK 7
#define FGPU_MAXV 5

namespace fgpu {

struct PhysP {
  double gamma, gm1, pmin, rhomin, tiny2;   // tiny2 = 2*TINY(1.0)
  double inv_gm1;                            // 1/(gamma-1), used by the product build only
};

struct Grid {
  int nx, ny, nz;      // interior cells (nz = 1 in 2D)
  long long n;         // nx*ny*nz
  int bc[6];           // boundary type per face (W,E,S,N,B,T)
  int fdir;            // FARGO transport direction: 1 along x (w by padded j), 2 along y (w by padded i)
};

// CheckData's CHECK_INVALID test of one value (timedisc_base.f90:1716-1725): NaN or above
// HUGE (negative infinity passes, as in the reference)
__device__ __forceinline__ bool invalid_value(double x) { return x != x || x > DBL_MAX; }

// FARGO: index of a cell's background velocity (padded j for transport along x, padded i
// along y); the transported momentum is component fdir of the state (1 x, 2 y)
__device__ __forceinline__ int fargo_ix(const Grid& g, int i, int j) { return (g.fdir == 1 ? j : i) + 2; }

struct MetricP {
  const double *dAxW, *dAyS, *dAzB;          // face area factors (dAxdydz(i,W) ...)
  const double *dydzdV, *dzdxdV, *dxdydV;
  const double *cxyx, *cxzx, *cyxy, *cyzy, *czxz, *czyz;
  const double *dlx, *dly, *dlz;
  const double *offxW, *offxE;               // reconstruction offsets, by padded i
  const double *offyS, *offyN;               // by padded j
  const double *offzB, *offzT;               // by padded k
  const double *accel;                       // [ndim][nx+4] point-mass acceleration or null
  const double *cs;                          // [7][nx+4] isothermal sound speed: C,W,E,S,N,B,T
  const double *dAxE;                        // dAxdydz(i,E) (the N/S and T/B areas share the centre's x)
  int nxp;                                   // nx + 4
  int curv;                                  // geometric sources active
  int vis;                                   // molecular viscosity: viscous time-step limit in cfl_cell
  double vis_eta;                            // its constant dynamic viscosity
};

// A sequence of FARGO frame changes of the momentum along the transport,
// m = m + s_q*(rho*w_q), applied in order.  It reproduces the in-place
// Add/SubtractBackgroundVelocityX/Y calls (physics_eulerisotherm.f90:1229-1413)
// that IntegrationStep and ComputeRHS make on cvar (timedisc_base.f90:662-674,
// 1096-1121, 1190-1208): every stored state is kept untransformed and the
// transforms are replayed pointwise where the state is read, so the rounding of
// each in-place update is reproduced.
struct Chain {
  int n;
  const double* w[4];   // background velocity by fargo_ix
  double s[4];          // +1 add, -1 subtract
  int rt;               // k > 0: the CHECK_PMIN round trip P2C(MAX(C2P(c),pmin)) before element k-1
                        // (k = n+1: after the last); 0: none
};

// The stage input state at a cell: base - coef[0]*K[0] - coef[1]*K[1] - ...
// evaluated in that order (timedisc_rkfehlberg.f90:277-302); nk = 0 for a
// plain state.  roundtrip = 1 applies fosite's CHECK_PMIN pass of the
// end-of-step ComputeRHS (timedisc_base.f90:1150-1164): p = MAX(C2P(u),pmin),
// c = P2C(p).
struct StateRef {
  const double* base;
  const double* K[FGPU_MAXK];
  double coef[FGPU_MAXK];
  int nk;
  int roundtrip;
  // FARGO (2D isothermal): frame changes applied to the state before the
  // boundary fill, i.e. the real-frame cvar that CenterBoundary sees
  Chain pre;
  // 1: base holds primitive variables already formed from a stage state (nk = 0)
  int ready;
  // device clock: coef[q] holds the tableau entry, multiplied by *dt_dev when read
  const double* dt_dev;
};

// One frame change of a conservative 2D state c by s*w (s = +1 add, -1 subtract).  With
// the energy (V = 4, ideal gas) the energy goes first, with the old momentum:
// E + s*w*(m + s*rho*w/2), then m + s*rho*w (physics_euler.f90:2003-2047, 2159-2203);
// multiplying by s = +-1 is exact, so both signs round like the reference's two forms.
// The momentum component is fdir (1 x, 2 y), selected without indexing the array.
template <int V>
__device__ __forceinline__ void frame_change(double* c, double s, double w, int fdir) {
  const double m = fdir == 1 ? c[1] : c[2];
  if (V == 4) c[3] = c[3] + s * (w * (m + s * (0.5 * c[0] * w)));
  const double mn = m + s * (c[0] * w);
  if (fdir == 1) c[1] = mn;
  else c[2] = mn;
}
// the velocity component along the transport of a primitive state, minus w
__device__ __forceinline__ void sub_velocity(double* p, double w, int fdir) {
  if (fdir == 1) p[1] = p[1] - w;
  else p[2] = p[2] - w;
}
// apply a frame-change chain to the conservative state c of cell (i, j) (0-based interior
// coordinates; rt_fn performs the round trip on c when the chain has one)
template <int V, class RT>
__device__ __forceinline__ void apply_chain(const Chain& C, double* c, const Grid& g, int i, int j, RT&& rt_fn) {
  const int ix = fargo_ix(g, i, j);
  for (int q = 0; q < C.n; ++q) {
    if (C.rt == q + 1) rt_fn(c);
    frame_change<V>(c, C.s[q], C.w[q][ix], g.fdir);
  }
  if (C.rt == C.n + 1) rt_fn(c);
}
// chains without a round trip (the frame of a stage input)
template <int V>
__device__ __forceinline__ void apply_chain(const Chain& C, double* c, const Grid& g, int i, int j) {
  apply_chain<V>(C, c, g, i, j, [](double*) {});
}

// Device control block for device-resident stepping.
struct Ctl {
  unsigned long long invdt[4];   // CFL partial maxima (bits of non-negative doubles); [3] viscous
  unsigned long long err;        // error-norm partial maximum
  int flags;                     // CheckData failures (FGPU_CHECK_* bits)
  unsigned int blocks_done;      // last-block detection of the boundary kernel
  double time, dt, dtold, dtmin, stoptime, tout, cfl, dtlimit;
  long long iter;
  int stop, brk, dtcause, pad;
  double cvis;                   // viscous Courant number (vis = 1)
  int vis, pad2;
  // embedded Runge-Kutta schemes on the device clock: the IntegrationStep sub-step loop
  // (timedisc_base.f90:649-750) as a state machine, one attempt per replayed slot
  double t_loc;                  // the loop's time t
  double d_att;                  // the attempt's dt (d)
  double dtold_att;              // dt of the last attempt (dtold)
  double maxerrold, last_err;    // AdjustTimestep's memory, the last error norm
  long long n_adj;               // rejected attempts
  long long steps_left;          // fosite steps still to run
  int act;                       // this slot's actions (ACT_* bits)
  int phase;                     // 0: next slot starts a fosite step, 1: inside IntegrationStep
  int rhs_done;                  // AcceptSolution evaluated the RHS at t (rhs_done_at_t)
  int checkflags;                // CheckData failures seen (FGPU_CHECK_* bits)
  double time_prev, dt_prev, dtold_prev;   // the step's time, dt, dtold before a slot closed it
  int dev_err;                   // a kernel's bounded wait ran out (its results are void)
  int pad3;
};

// actions of a device-clock attempt slot, decided by bt_decide_kernel
// (ACT_BRK: CheckData failed inside the step; the slot ends with a break; ACT_OPEN: the slot
// opens a fosite step; ACT_ENDNC: the step closes without AcceptSolution's RHS at its end)
enum { ACT_ATTEMPT = 1, ACT_REJECT = 2, ACT_SUB = 4, ACT_END = 8, ACT_COPY = 16, ACT_BRK = 32, ACT_OPEN = 64,
       ACT_ENDNC = 128 };
// a kernel of a slot runs only if the slot's actions include one of its gate bits
__device__ __forceinline__ bool gated_out(const Ctl* c, int gate) {
  return gate && c && !(c->act & gate);
}

enum { BC_NOGRAD = 0x01, BC_PERIODIC = 0x02, BC_REFLECTING = 0x03, BC_AXIS = 0x04, BC_ABSORBING = 0x0D };
enum { LIM_MINMOD = 1, LIM_MC = 2, LIM_SWEBY = 3, LIM_SUPERBEE = 4, LIM_OSPRE = 5, LIM_VANLEER = 7, LIM_NOLIMIT = 8 };
// kernel-internal code: MC with theta = 1 (the products theta*difference are exact and skipped)
enum { LIM_MC1 = 102 };

__device__ __forceinline__ double fsign1(double b) { return signbit(b) ? -1.0 : 1.0; }
__device__ __forceinline__ double fsign(double a, double b) { return signbit(b) ? -fabs(a) : fabs(a); }
// Fortran MIN/MAX on non-NaN operands.  The --fmad=false build keeps the
// compare-and-select form (the operand returned for +0/-0 ties is the first,
// as in the oracle); the product build uses the native FP64 min/max.
#ifdef FGPU_EXACT
__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double dmax(double a, double b) { return b > a ? b : a; }
#else
__device__ __forceinline__ double dmin(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ double dmax(double a, double b) { return fmax(a, b); }
#endif

// ---------------------------------------------------------------- physics
// Variables: 0 density, 1..ND velocity/momentum, ND+1 pressure/energy (Euler).
template <int ND, bool EU>
struct Phys {
  static constexpr int V = EU ? ND + 2 : ND + 1;

  // Cons2Prim (physics_euler.f90:3064-3100, physics_eulerisotherm.f90:2831-2856)
  static __device__ __forceinline__ void c2p(const double* c, double* p, const PhysP& P) {
    double inv_rho = 1. / c[0];
    p[0] = c[0];
#pragma unroll
    for (int m = 1; m <= ND; ++m) p[m] = c[m] * inv_rho;
    if (EU) {
      double s = c[1] * c[1] + c[2] * c[2];
      if (ND == 3) s = s + c[3] * c[3];
      p[V - 1] = P.gm1 * (c[V - 1] - 0.5 * inv_rho * s);
    }
  }
  // Prim2Cons (physics_euler.f90:3103-3117, physics_eulerisotherm.f90:2858-2892)
  static __device__ __forceinline__ void p2c(const double* p, double* c, const PhysP& P) {
    c[0] = p[0];
#pragma unroll
    for (int m = 1; m <= ND; ++m) c[m] = p[0] * p[m];
    if (EU) {
      double s = p[1] * p[1] + p[2] * p[2];
      if (ND == 3) s = s + p[3] * p[3];
#ifdef FGPU_EXACT
      c[V - 1] = p[V - 1] / P.gm1 + 0.5 * p[0] * s;
#else
      c[V - 1] = p[V - 1] * P.inv_gm1 + 0.5 * p[0] * s;
#endif
    }
  }
  // GetSoundSpeed (physics_euler.f90:2682-2689): sqrt(MAX(2 TINY, gamma*p/rho)).
  // The product build evaluates sqrt(s/rho) as s*rsqrt(s*rho) with s = gamma*p (one
  // reciprocal square root instead of a division and a square root; within a few ulp).
  static __device__ __forceinline__ double cs_of(const double* p, const PhysP& P) {
#ifdef FGPU_EXACT
    return sqrt(dmax(P.tiny2, P.gamma * p[V - 1] / p[0]));
#else
    const double s = P.gamma * p[V - 1];
    const double q = s * p[0];
    if (s > P.tiny2 * p[0] && q > 1e-300 && q < 1e300) return s * rsqrt(q);
    return sqrt(dmax(P.tiny2, s / p[0]));
#endif
  }
};

// ---------------------------------------------------------------- limiters
// reconstruction_linear.f90:645-733; returns the limited difference (times invd by caller)
__device__ __forceinline__ double limit2(int lim, double theta, double a1, double a2) {
  switch (lim) {
    case LIM_MINMOD: {
#ifdef FGPU_EXACT
      if (fsign1(a1) * fsign1(a2) > 0) return fsign(dmin(fabs(a1), fabs(a2)), a1);
      return 0.;
#else
      // the same value for non-zero differences (see MONOCENT in slope)
      const double lo = dmin(a1, a2), hi = dmax(a1, a2);
      return lo > 0. ? lo : (hi < 0. ? hi : 0.);
#endif
    }
    case LIM_SWEBY:
    case LIM_SUPERBEE: {
      double p = lim == LIM_SWEBY ? theta : 2.0;
      if (fsign1(a1) * fsign1(a2) > 0)
        return fsign(dmax(dmin(p * fabs(a1), fabs(a2)), dmin(fabs(a1), p * fabs(a2))), a1);
      return 0.;
    }
    case LIM_OSPRE:
      return 1.5 * a1 * a2 * (a1 + a2) / (a1 * (a1 + 0.5 * a2) + a2 * (a2 + 0.5 * a1) + DBL_MIN);
    case LIM_VANLEER: {
      double b1 = fabs(a1), b2 = fabs(a2);
      return (a1 * b2 + a2 * b1) / (b1 + b2 + DBL_MIN);
    }
    case LIM_NOLIMIT:
      return 0.5 * (a1 + a2);
    default:
      return 0.;
  }
}
// slope of q0 with neighbours qm, qp (MONOCENT uses minmod3 of three differences)
__device__ __forceinline__ double slope(int lim, double theta, double invd, double qm, double q0, double qp) {
  if (lim == LIM_MC || lim == LIM_MC1) {
    double a1 = lim == LIM_MC1 ? q0 - qm : theta * (q0 - qm), a2 = lim == LIM_MC1 ? qp - q0 : theta * (qp - q0);
    double a3 = 0.5 * (qp - qm);
#ifdef FGPU_EXACT
    double r = 0.;
    if (((fsign1(a1) * fsign1(a2)) > 0) && ((fsign1(a2) * fsign1(a3)) > 0))
      r = fsign(dmin(dmin(fabs(a1), fabs(a2)), fabs(a3)), a1);
#else
    // same value as the sign-test form for all non-zero slopes: the smallest of three
    // positive differences, the largest of three negative ones, else zero (the sign of
    // a zero result may differ)
    const double lo = dmin(dmin(a1, a2), a3), hi = dmax(dmax(a1, a2), a3);
    const double r = lo > 0. ? lo : (hi < 0. ? hi : 0.);
#endif
    return invd * r;
  }
  return invd * limit2(lim, theta, q0 - qm, qp - q0);
}

// ---------------------------------------------------------------- state access
template <int V>
__device__ __forceinline__ void state_at(const StateRef& S, long long n, long long idx, double* u) {
  const double* b = S.base + idx;
#pragma unroll
  for (int v = 0; v < V; ++v) u[v] = __ldg(b + (long long)v * n);
  // one k-array at a time, in the reference's accumulation order; only the
  // stage's own arrays are touched (no predicated loads of unused slots)
#pragma unroll 1
  for (int q = 0; q < S.nk; ++q) {
    const double* kq = S.K[q] + idx;
    const double a = S.dt_dev ? S.coef[q] * *S.dt_dev : S.coef[q];
    double t[V];
#pragma unroll
    for (int v = 0; v < V; ++v) t[v] = __ldg(kq + (long long)v * n);
#pragma unroll
    for (int v = 0; v < V; ++v) u[v] = u[v] - a * t[v];
  }
}

// Boundary-aware primitive state of any cell of the ghost-padded grid, as
// CenterBoundary + SetCornerEdges leave it (before the CHECK_PMIN clamp).
// Indices are 0-based interior coordinates, ghosts are -2..-1 and n..n+1.
template <int ND, bool EU>
struct Cells {
  using PH = Phys<ND, EU>;
  static constexpr int V = PH::V;

  static __device__ __forceinline__ long long lin(const Grid& g, int i, int j, int k) {
    return (long long)i + (long long)g.nx * ((long long)j + (long long)g.ny * k);
  }
  static __device__ __forceinline__ void interior_p(const StateRef& S, const Grid& g, const PhysP& P,
                                                    int i, int j, int k, double* p) {
    double u[V];
    state_at<V>(S, g.n, lin(g, i, j, k), u);
    if (S.ready) {
#pragma unroll
      for (int l = 0; l < V; ++l) p[l] = u[l];
      return;
    }
    if (ND == 2 && S.pre.n) apply_chain<V>(S.pre, u, g, i, j);
    PH::c2p(u, p, P);
  }

  // Face ghost: exactly one of (i,j,k) outside the interior, in direction d.
  // boundary_periodic.f90:73-116, boundary_reflecting.f90:89-204,
  // boundary_nogradients.f90:75-125, boundary_absorbing.f90:114-211.
  static __device__ __noinline__ void face_ghost_p(const StateRef& S, const Grid& g, const PhysP& P, const MetricP& M,
                                      int d, int i, int j, int k, double* p) {
    int ijk[3] = {i, j, k};
    int nd = d == 0 ? g.nx : d == 1 ? g.ny : g.nz;
    int x = ijk[d];
    bool lo = x < 0;
    int s = lo ? -x : x - (nd - 1);   // ghost depth 1 or 2
    int face = 2 * d + (lo ? 0 : 1);
    int type = g.bc[face];
    int vn = 1 + d;                   // normal velocity slot (x-y / x-y-z meshes)
    if (type == BC_PERIODIC) {
      ijk[d] = lo ? nd - s : s - 1;
      interior_p(S, g, P, ijk[0], ijk[1], ijk[2], p);
    } else if (type == BC_REFLECTING || type == BC_AXIS) {
      ijk[d] = lo ? s - 1 : nd - s;
      interior_p(S, g, P, ijk[0], ijk[1], ijk[2], p);
      p[vn] = -p[vn];
      // AXIS (boundary_axis.f90, physics_eulerisotherm.f90:1701-1760 AxisMasks): on the
      // curvilinear meshes here the azimuth is the second coordinate, whose velocity is
      // reflected too at the x faces
      if (type == BC_AXIS && d == 0 && M.curv) p[2] = -p[2];
    } else if (type == BC_NOGRAD) {
      ijk[d] = lo ? 0 : nd - 1;
      interior_p(S, g, P, ijk[0], ijk[1], ijk[2], p);
    } else {   // BC_ABSORBING: characteristic extrapolation into the first ghost layer, copied outward
      int i1 = lo ? 0 : nd - 1, i2 = lo ? 1 : nd - 2;
      int iL = i1 < i2 ? i1 : i2, iR = i1 < i2 ? i2 : i1;
      int delta = lo ? -1 : 1;
      double p1[V], p2[V];
      ijk[d] = i1; interior_p(S, g, P, ijk[0], ijk[1], ijk[2], p1);
      ijk[d] = i2; interior_p(S, g, P, ijk[0], ijk[1], ijk[2], p2);
      const double* pL = (iL == i1) ? p1 : p2;
      const double* pR = (iR == i1) ? p1 : p2;
      double lam[V], xv[V];
      if (!EU) {
        // iso: physics_eulerisotherm.f90:1764-2220, elementals :2895-2970
        int ip1 = (d == 0 ? i1 : ijk[0]) + 2;                 // padded i of the boundary cell
        int ipR = (d == 0 ? iR : ijk[0]) + 2;
        double cs1 = M.cs[0 * M.nxp + ip1];
        double csf = M.cs[(1 + 2 * d) * M.nxp + ipR];          // fcsound(iR, west/south/bottom)
        double v = p1[vn];
        lam[0] = v - cs1;
#pragma unroll
        for (int t = 1; t < V - 1; ++t) lam[t] = v;
        lam[V - 1] = v + cs1;
        double dlnrho = log(pR[0] / pL[0]);
        double ducs = (pR[vn] - pL[vn]) / csf;
        xv[0] = dlnrho - ducs;
        xv[V - 1] = dlnrho + ducs;
        int t = 1;
#pragma unroll
        for (int m = 1; m <= ND; ++m)
          if (m != vn) { xv[t] = pR[m] - pL[m]; ++t; }
      } else {
        // Euler: physics_euler.f90:743-1265, elementals :2799-2890
        double cs = PH::cs_of(p1, P);
        double v = p1[vn];
        double l1 = v - cs, l3 = v + cs;
        lam[0] = l1;
#pragma unroll
        for (int t = 1; t < V - 1; ++t) lam[t] = v;
        lam[V - 1] = l3;
        double dlnP = log(pR[V - 1] / pL[V - 1]);
        double gdu = 2 * P.gamma * (pR[vn] - pL[vn]) / (l3 - l1);
        xv[0] = dlnP - gdu;
        xv[1] = dlnP - P.gamma * log(pR[0] / pL[0]);
        int t = 2;
#pragma unroll
        for (int m = 1; m <= ND; ++m)
          if (m != vn) { xv[t] = pR[m] - pL[m]; ++t; }
        xv[V - 1] = dlnP + gdu;
      }
#pragma unroll
      for (int l = 0; l < V; ++l)
        if (lo ? (lam[l] >= 0.0) : (lam[l] <= 0.0)) xv[l] = 0.0;
      if (!EU) {
        int ip1 = (d == 0 ? i1 : ijk[0]) + 2;
        double csf = M.cs[(1 + 2 * d + (lo ? 0 : 1)) * M.nxp + ip1];
        p[0] = p1[0] * exp(delta * 0.5 * (xv[V - 1] + xv[0]));
        p[vn] = p1[vn] + delta * 0.5 * csf * (xv[V - 1] - xv[0]);
        int t = 1;
#pragma unroll
        for (int m = 1; m <= ND; ++m)
          if (m != vn) { p[m] = p1[m] + delta * xv[t]; ++t; }
      } else {
        double dlnP = 0.5 * (xv[V - 1] + xv[0]);
        double rho2 = p1[0] * exp(delta / P.gamma * (dlnP - xv[1]));
        double P2 = p1[V - 1] * exp(delta * dlnP);
        double pa[V];
        pa[0] = p1[0] + rho2;
        pa[V - 1] = p1[V - 1] + P2;
        double cs = PH::cs_of(pa, P);
        p[0] = rho2;
        p[V - 1] = P2;
        p[vn] = p1[vn] + 0.5 * delta * cs / P.gamma * (xv[V - 1] - xv[0]);
        int t = 2;
#pragma unroll
        for (int m = 1; m <= ND; ++m)
          if (m != vn) { p[m] = p1[m] + delta * xv[t]; ++t; }
      }
    }
  }

  // Any cell of the padded grid (interior, face ghost, edge or corner), following
  // SetCornerEdges (boundary_generic.f90:434-763) for GNUM = 2.  No clamp.
  static __device__ void cell_p(const StateRef& S, const Grid& g, const PhysP& P, const MetricP& M,
                                int i, int j, int k, double* p) {
    int ijk[3] = {i, j, k};
    int nn[3] = {g.nx, g.ny, g.nz};
    int gd[3], depth[3], ng = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      depth[d] = ijk[d] < 0 ? -ijk[d] : (ijk[d] >= nn[d] ? ijk[d] - nn[d] + 1 : 0);
      if (depth[d] > 0) gd[ng++] = d;
    }
    auto bnd = [&](int d) { return ijk[d] < 0 ? 0 : nn[d] - 1; };
    if (ng == 0) { interior_p(S, g, P, i, j, k, p); return; }
    if (ng == 1) { face_ghost_p(S, g, P, M, gd[0], i, j, k, p); return; }
    if (ng == 2) { edge_p(S, g, P, M, gd[0], gd[1], ijk, depth, p); return; }
    // three ghost directions (3D)
    if (depth[0] == depth[1] && depth[1] == depth[2]) {
      double a[V], b[V], c[V];
      int q[3];
      q[0] = ijk[0]; q[1] = bnd(1); q[2] = bnd(2); face_ghost_p(S, g, P, M, 0, q[0], q[1], q[2], a);
      q[0] = bnd(0); q[1] = ijk[1]; q[2] = bnd(2); face_ghost_p(S, g, P, M, 1, q[0], q[1], q[2], b);
      q[0] = bnd(0); q[1] = bnd(1); q[2] = ijk[2]; face_ghost_p(S, g, P, M, 2, q[0], q[1], q[2], c);
#pragma unroll
      for (int l = 0; l < V; ++l) p[l] = (a[l] + b[l] + c[l]) / 3.0;
      return;
    }
    // y-z pass over all i (the last writer of cells ghost in all directions)
    int q[3] = {ijk[0], ijk[1], ijk[2]};
    int dq[3] = {depth[0], depth[1], depth[2]};
    if (depth[1] == depth[2]) {
      double a[V], b[V];
      q[1] = bnd(1); dq[1] = 0; edge_p(S, g, P, M, 0, 2, q, dq, a);   // (ghost x, bnd y, ghost z)
      q[1] = ijk[1]; dq[1] = depth[1]; q[2] = bnd(2); dq[2] = 0;
      edge_p(S, g, P, M, 0, 1, q, dq, b);                              // (ghost x, ghost y, bnd z)
#pragma unroll
      for (int l = 0; l < V; ++l) p[l] = 0.5 * (a[l] + b[l]);
    } else if (depth[1] < depth[2]) {
      q[1] = bnd(1); dq[1] = 0; edge_p(S, g, P, M, 0, 2, q, dq, p);
    } else {
      q[2] = bnd(2); dq[2] = 0; edge_p(S, g, P, M, 0, 1, q, dq, p);
    }
  }

  // cell ghost in exactly the two directions d1 < d2
  static __device__ void edge_p(const StateRef& S, const Grid& g, const PhysP& P, const MetricP& M,
                                int d1, int d2, const int* ijk, const int* depth, double* p) {
    int nn[3] = {g.nx, g.ny, g.nz};
    int q[3] = {ijk[0], ijk[1], ijk[2]};
    int b1 = ijk[d1] < 0 ? 0 : nn[d1] - 1, b2 = ijk[d2] < 0 ? 0 : nn[d2] - 1;
    int a = depth[d1], b = depth[d2];
    if (a == b) {
      double x[V], y[V];
      q[d2] = b2; face_ghost_p(S, g, P, M, d1, q[0], q[1], q[2], x);
      q[d2] = ijk[d2]; q[d1] = b1; face_ghost_p(S, g, P, M, d2, q[0], q[1], q[2], y);
#pragma unroll
      for (int l = 0; l < V; ++l) p[l] = 0.5 * (x[l] + y[l]);
    } else if (a > b) {
      q[d2] = b2; face_ghost_p(S, g, P, M, d1, q[0], q[1], q[2], p);
    } else {
      q[d1] = b1; face_ghost_p(S, g, P, M, d2, q[0], q[1], q[2], p);
    }
  }

  // CFL contribution of one cell (CalcWaveSpeeds_center + CalcTimestep,
  // physics_eulerisotherm.f90:530-552, timedisc_base.f90:860-893).
  // ip = padded i; out[0] = 2D sum or x; out[1], out[2] for 3D; out[3] the inverse
  // viscous time step of sources_viscosity.f90:532-575, sum over the directions of
  // (max wave speed + 2*kinvis/dl)/dl with kinvis = dynvis/density (0 without viscosity).
  static __device__ __forceinline__ void cfl_cell(const double* p, double cs, const MetricP& M, int ip, double* out) {
    double dl[3] = {M.dlx[ip], M.dly[ip], ND == 3 ? M.dlz[ip] : 1.0};
    double w[3], a[3];
#pragma unroll
    for (int m = 0; m < ND; ++m) {
      double v = p[1 + m];
      double mn = dmin(0., v - cs), mx = dmax(0., v + cs);
      w[m] = dmax(mx, -mn);
      a[m] = w[m] / dl[m];
    }
    if (ND == 2) { out[0] = a[0] + a[1]; out[1] = 0.0; out[2] = 0.0; }
    else { out[0] = a[0]; out[1] = a[1]; out[2] = a[2]; }
    out[3] = 0.0;
    if (M.vis) {
      const double kinvis = M.vis_eta / p[0];
      double s = (w[0] + 2.0 * kinvis / dl[0]) / dl[0];
#pragma unroll
      for (int m = 1; m < ND; ++m) s = s + (w[m] + 2.0 * kinvis / dl[m]) / dl[m];
      out[3] = s;
    }
  }
};

// ---------------------------------------------------------------- KT flux
// fluxes_kt.f90:126-207 with CalcWaveSpeeds_faces (physics_eulerisotherm.f90:
// 555-686) and CalcFluxes{X,Y,Z}/SetFlux (physics_euler.f90:492-742,
// physics_eulerisotherm.f90:835-979).  RL: reconstructed variables on the
// plus face of the left cell, RR: on the minus face of the right cell.
// DC >= 0: the direction is DC, known at compile time (d_rt is ignored).
template <int ND, bool EU, bool PRIM, int DC = -1>
__device__ __forceinline__ void kt_flux(int d_rt, const double* RL, const double* RR, double csL_iso, double csR_iso,
                                        double dA, const PhysP& P, double* F) {
  using PH = Phys<ND, EU>;
  constexpr int V = PH::V;
  const int d = DC >= 0 ? DC : d_rt;
  double pL[V], cL[V], pR[V], cR[V];
  if (PRIM) {
#pragma unroll
    for (int l = 0; l < V; ++l) { pL[l] = RL[l]; pR[l] = RR[l]; }
    PH::p2c(pL, cL, P);
    PH::p2c(pR, cR, P);
  } else {
#pragma unroll
    for (int l = 0; l < V; ++l) { cL[l] = RL[l]; cR[l] = RR[l]; }
    PH::c2p(cL, pL, P);
    PH::c2p(cR, pR, P);
  }
  double csL = EU ? PH::cs_of(pL, P) : csL_iso;
  double csR = EU ? PH::cs_of(pR, P) : csR_iso;
  const int vn = 1 + d;
  // the normal velocity by selection (d may be a run-time value: no indexed register arrays)
  auto normal = [&](const double* q) {
    return ND == 3 ? (vn == 1 ? q[1] : (vn == 2 ? q[2] : q[3])) : (vn == 1 ? q[1] : q[2]);
  };
  double uL = normal(pL), uR = normal(pR);
#ifdef FGPU_EXACT
  double am = dmin(dmin(0.0, dmin(0., uR - csR)), dmin(0., uL - csL));
  double ap = dmax(dmax(0.0, dmax(0., uR + csR)), dmax(0., uL + csL));
#else
  // the same extrema with two native min/max each (a zero result may differ in sign, which
  // no flux component sees: it enters as a product and in ap - am)
  double am = dmin(0.0, dmin(uR - csR, uL - csL));
  double ap = dmax(0.0, dmax(uR + csR, uL + csL));
#endif
  double fL[V], fR[V];
  fL[0] = pL[0] * uL;
  fR[0] = pR[0] * uR;
  if (EU) {
    double PL = pL[V - 1], PR = pR[V - 1];
#pragma unroll
    for (int m = 1; m <= ND; ++m) {
      fL[m] = (m == vn) ? cL[m] * uL + PL : cL[m] * uL;
      fR[m] = (m == vn) ? cR[m] * uR + PR : cR[m] * uR;
    }
    fL[V - 1] = (cL[V - 1] + PL) * uL;
    fR[V - 1] = (cR[V - 1] + PR) * uR;
  } else {
#pragma unroll
    for (int m = 1; m <= ND; ++m) {
      fL[m] = (m == vn) ? cL[m] * uL + pL[0] * csL * csL : cL[m] * uL;
      fR[m] = (m == vn) ? cR[m] * uR + pR[0] * csR * csR : cR[m] * uR;
    }
  }
  double fac = dA / (ap - am);
  double amap = am * ap;
#pragma unroll
  for (int l = 0; l < V; ++l) F[l] = fac * (ap * fL[l] - am * fR[l] + amap * (cR[l] - cL[l]));
}

}  // namespace fgpu
