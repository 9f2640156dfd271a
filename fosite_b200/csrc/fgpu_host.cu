// fgpu_host.cu -- C ABI of the B200 backend (include/fosite_gpu.h): config
// validation, host-side metric precompute, device memory, and the two time
// integration drivers:
//   * Shu-Osher "modified Euler" (timedisc_modeuler.f90, fixed step): fully
//     device-resident -- dt, time and the stop/break flags live in a device
//     control block, each step is a fixed kernel sequence replayed from a
//     captured CUDA graph;
//   * embedded Butcher engine (timedisc_rkfehlberg.f90 with the Dormand-Prince,
//     Fehlberg, Cash-Karp and SSPRK tableaus): one stage kernel per stage, the
//     accept/reject logic of IntegrationStep (timedisc_base.f90:649-750) runs on
//     the host after one 8-byte read of the error norm per attempt.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <cmath>
#include <cfloat>
#include <cstring>
#include <cstdio>
#include <string>
#include <vector>
#include <algorithm>
#include <map>
#include <mutex>
#include <type_traits>
#include <cstdlib>
#include "../../include/fosite_gpu.h"
#include "fgpu_kernels_misc.cuh"
#include "fgpu_fargo.cuh"
#include "fgpu_visc.cuh"
#include "fgpu_ddmath.h"
#include "fgpu_bt.cuh"
#include "fgpu_tma_launch.h"
#include "fgpu_stage_launch.h"

using namespace fgpu;

namespace {

std::string g_create_error;

struct Tableau {
  int m = 0, order = 0;
  std::vector<double> A, bh, bl, c;
};

bool make_tableau(int method, int order, Tableau& T) {
  auto set = [&](int m, int o, std::initializer_list<double> bh, std::initializer_list<double> bl,
                 std::initializer_list<double> c, std::initializer_list<double> a) {
    T.m = m; T.order = o; T.bh = bh; T.bl = bl; T.c = c; T.A = a;
  };
  // timedisc_dormand_prince.f90:91-114
  if (method == FGPU_DORMAND_PRINCE && order == 5) {
    set(7, 5, {35./384., 0., 500./1113., 125./192., -2187./6784., 11./84., 0.},
        {5179./57600., 0., 7571./16695., 393./640., -92097./339200., 187./2100., 1./40.},
        {0., .2, 3./10., 4./5., 8./9., 1., 1.},
        {0., 0., 0., 0., 0., 0., 0.,
         .2, 0., 0., 0., 0., 0., 0.,
         3./40., 9./40., 0., 0., 0., 0., 0.,
         44./45., -56./15., 32./9., 0., 0., 0., 0.,
         19372./6561., -25360./2187., 64448./6561., -212./729., 0., 0., 0.,
         9017./3168., -355./33., 46732./5247., 49./176., -5103./18656., 0., 0.,
         35./384., 0., 500./1113., 125./192., -2187./6784., 11./84., 0.});
    return true;
  }
  // timedisc_rkfehlberg.f90:305-335
  if (method == FGPU_RK_FEHLBERG && order == 3) {
    set(3, 3, {1.0/6.0, 2.0/3.0, 1.0/6.0}, {0.0, 1.0, 0.0}, {0.0, 0.5, 1.0},
        {0.0, 0.0, 0.0, 0.5, 0.0, 0.0, -1.0, 2.0, 0.0});
    return true;
  }
  if (method == FGPU_RK_FEHLBERG && order == 5) {
    set(6, 5, {16.0/135.0, 0.0, 6656.0/12825.0, 28561.0/56430.0, -9.0/50.0, 2.0/55.0},
        {25.0/216.0, 0.0, 1408.0/2565.0, 2197.0/4104.0, -0.2, 0.0},
        {0.0, 0.25, 3.0/8.0, 12.0/13.0, 1.0, 0.5},
        {0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
         0.25, 0.0, 0.0, 0.0, 0.0, 0.0,
         3.0/32.0, 9.0/32.0, 0.0, 0.0, 0.0, 0.0,
         1932.0/2197.0, -7200.0/2197.0, 7296.0/2197.0, 0.0, 0.0, 0.0,
         439.0/216.0, -8.0, 3680.0/513.0, -845.0/4104.0, 0.0, 0.0,
         -8.0/27.0, 2.0, -3544.0/2565.0, 1859.0/4104.0, -11.0/40.0, 0.0});
    return true;
  }
  // timedisc_cashkarp.f90:95-117
  if (method == FGPU_CASH_KARP && order == 5) {
    set(6, 5, {37.0/378.0, 0.0, 250.0/621.0, 125.0/594.0, 0.0, 512.0/1771.0},
        {2825.0/27648.0, 0.0, 18575.0/48384.0, 13525.0/55296.0, 277.0/14336.0, 0.25},
        {0.0, 0.2, 0.3, 0.6, 1.0, 7.0/8.0},
        {0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
         0.2, 0.0, 0.0, 0.0, 0.0, 0.0,
         0.075, 0.225, 0.0, 0.0, 0.0, 0.0,
         0.3, -0.9, 1.2, 0.0, 0.0, 0.0,
         -11.0/54.0, 2.5, -70.0/27.0, 35.0/27.0, 0.0, 0.0,
         1631.0/55296.0, 175.0/512.0, 575.0/13824.0, 44275.0/110592.0, 253.0/4096.0, 0.0});
    return true;
  }
  // timedisc_ssprk.f90:93-126
  if (method == FGPU_SSPRK && order == 3) {
    set(3, 3, {1./6., 1./6., 2./3.}, {0.5, 0.5, 0.}, {0., 1., 0.5},
        {0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.25, 0.25, 0.0});
    return true;
  }
  if (method == FGPU_SSPRK && order == 5) {
    set(5, 5, {0.17279, 0.094505, 0.12947, 0.29899, 0.30424},
        {0.12293, 0.31981, -0.15316, 0.31887, 0.39155},
        {0., 0.36717, 0.58522, 0.44156, 0.8464},
        {0., 0., 0., 0., 0.,
         0.36717, 0., 0., 0., 0.,
         0.26802, 0.3172, 0., 0., 0.,
         0.11606, 0.13735, 0.18816, 0., 0.,
         0.11212, 0.13269, 0.18178, 0.4198, 0.});
    return true;
  }
  return false;
}

}  // namespace

struct fgpu_handle {
  fgpu_config cfg;
  std::string err;
  int device = 0;
  cudaStream_t stream = nullptr;
  int nd = 2, V = 4;
  bool euler = true, prim = false, roundtrip_cfg = false, curv = false, has_accel = false;
  Grid g;
  PhysP ph;
  MetricP mt;
  double invd[3];
  double* d_metric = nullptr;
  std::vector<double> h_metric;
  int nxp = 0;
  // state buffers: [0] P (stored state), then scheme-specific
  std::vector<double*> buf;
  double* d_pad = nullptr;      // padded download scratch (2 * npad * V)
  double* d_flux = nullptr;     // interface fluxes of the last fgpu_compute_rhs (3 * V * padded cells)
  bool flux_valid = false;
  long long npad = 0;
  Ctl* d_ctl = nullptr;
  Ctl* h_ctl = nullptr;         // pinned
  // timedisc
  bool butcher = false;
  int order = 3;
  Tableau T;
  double tol_rel, beta, cfl, dtlimit, stoptime, tout;
  double tol_abs[FGPU_MAXVAR];
  // host-side bookkeeping (Butcher engine) / mirror of the control block
  double time = 0, dt = 0, dtold = 0, dtmin = 0, maxerrold = 0, last_err = 0;
  int dtcause = 0;
  bool brk = false;
  long long iter = -1, n_adj = 0;
  int checkflags = 0;
  bool first_done = false;
  bool pre_rt = false;          // buffer P holds a state whose fosite cvar is its CHECK_PMIN round trip
                                // (after FirstStep's CHECK_ALL, and after steps when checkdata has PMIN)
  // graph of G Shu-Osher steps
  cudaGraphExec_t graph = nullptr;
  // device-clock embedded schemes: the captured attempt slot (fgpu_bt.cuh)
  cudaGraphExec_t bt_graph = nullptr;
  int kernels_per_slot = 0;
  int graph_steps = 0;
  // launch shape
  int tile_x = 32, tile_y = 8, kchunk = 16;
  bool adaptive_me = false;     // modified Euler with embedded error control (tol_rel < 1)
  bool materialize = true;      // Butcher stages: form the stage's reconstruction variables once per cell
  bool fuse_form = true;        // ... stage m's kernel forms stage m+1's (buffers alternate), only stage 2 by form_kernel
  bool fuse_end = true;         // the last stage's kernel also forms the high/low-order solutions and the error norm
  // fixed-step Shu-Osher with primitive reconstruction: stage n < order also writes the
  // primitive variables of its result (d_pform[(n-1)%2]), which stage n+1's stencil reads
  bool so_form = false;
  double* d_pform[2] = {nullptr, nullptr};
  double* d_ready = nullptr;    // ... into this array (one state)
  int variant = 0;              // stage kernel layout: 0 shared-memory tile, 1 warp-shuffle window,
                                // 2/3 tile with a register cap for more resident blocks, 4 taller tile,
                                // 6 tile with TMA-staged planes (fgpu_tma.cuh), 7 its 32 x 4 form (2D)
  // tensor maps of the stage inputs the TMA layout has read (by base pointer and tile shape)
  struct TmapEntry { const double* base; int tx, ty; CUtensorMap map; };
  std::vector<TmapEntry> tmaps;
  // instrumentation
  cudaStream_t own_stream = nullptr;
  bool profiling = false;
  struct Timed { cudaEvent_t a, b; double bytes; int stage; };
  std::vector<Timed> timed;
  fgpu_stats stats;
  int kernels_per_step = 0;
  // FARGO transport (type 1, direction 2): d_w = [w | w_new], each by padded i.
  // fargo_phase 0: before FirstStep; 1: after FirstStep (the stored state is
  // FirstStep's real-frame cvar); 2: after a step (the stored state is the
  // transported state, w the background velocity of its closing ComputeRHS)
  bool fargo = false;
  int fdir = 2;                 // transport along x (1, w by padded j) or y (2, w by padded i)
  int nw = 0;                   // padded length of w along the other direction
  double* d_w = nullptr;        // [w | w_new | wfactor of direction 1]
  double* d_fw_terms = nullptr; // direction 2: the background-velocity sum's terms [ny][nx+4]
  int fargo_phase = 0;
  bool fargo_tmp_fresh = true;  // Butcher + FARGO: the stage vectors' frame flags are still unset
  // point-mass accretion: d_acc = [bx (ny) | bxold (ny) | brow (ny) | mass, mdot]
  bool accrete = false;
  int acc_face = 0;             // 0 west, 1 east
  double* d_acc = nullptr;
  double dxyz[3] = {1.0, 1.0, 1.0};
  // viscosity: model, constants and the viscous source of the current stage state; the
  // ALPHA/BETA/POWERLAW models keep the dynamic viscosity by padded cell with the time of
  // its last update (sources_viscosity.f90:359-453)
  bool vis = false;
  int vis_model = 0;
  double vis_eta = 0.0, vis_mub = 0.0, cvis = 0.5, vis_power = 0.0;
  double* d_visc = nullptr;     // [nd (+1 energy)][n]
  double* d_dynvis = nullptr;   // [npad]
  double* d_ephir = nullptr;    // [nd][npad]
  double* d_visrad = nullptr;   // [npad]
  double* d_vistime = nullptr;  // 1 double, initially -1
  long long npad_vis = 0;
};

// The time of a right-hand side evaluation, for the viscosity update: a host value, or on the
// device clock the control block's time + zeta*dt
// device clock (time + zeta*dt), or on the attempt clock of the device-clock embedded
// schemes (t + zeta*d of the IntegrationStep loop)
struct RhsTime {
  bool dev = false;
  bool attempt = false;
  double t = 0.0;
  double zeta = 0.0;
  static RhsTime host(double t) { RhsTime r; r.t = t; return r; }
  static RhsTime device(double zeta) { RhsTime r; r.dev = true; r.zeta = zeta; return r; }
  static RhsTime att(double zeta) { RhsTime r; r.dev = true; r.attempt = true; r.zeta = zeta; return r; }
};

namespace {

int set_err(fgpu_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg; else g_create_error = msg;
  return code;
}
// Slot budget of the device-clock loops (attempt slots replayed before a call gives up with
// FGPU_ETIMEOUT); FGPU_SLOT_CAP overrides the computed budget (tests force the timeout path).
long long slot_cap(long long computed) {
  if (const char* e = std::getenv("FGPU_SLOT_CAP")) return std::atoll(e);
  return computed;
}
#define CUDA_TRY(h, call)                                                                    \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return set_err(h, e_ == cudaErrorMemoryAllocation ? FGPU_ENOMEM : FGPU_ECUDA,          \
                     std::string(#call) + ": " + cudaGetErrorString(e_));                    \
  } while (0)

// ---------------------------------------------------------------- metric
// Restatement of mesh_base.f90:570-729 and mesh_midpoint.f90:97-145 for
// geometries whose scale factors depend on the first coordinate only.
void scale(int geo, double gp, double x, double& hx, double& hy, double& hz) {
  if (geo == FGPU_CYLINDRICAL) { hx = 1.0; hy = x; hz = 1.0; }
  else if (geo == FGPU_LOGCYLINDRICAL) { hx = gp * std::exp(x); hy = hx; hz = 1.0; }
  else { hx = hy = hz = 1.0; }
}

enum { M_dAxW, M_dAyS, M_dAzB, M_dydzdV, M_dzdxdV, M_dxdydV, M_cxyx, M_cxzx, M_cyxy, M_cyzy, M_czxz, M_czyz,
       M_dlx, M_dly, M_dlz, M_offxW, M_offxE, M_accel0, M_accel1, M_wfac, M_dAxE, M_cs0, M_NI = M_cs0 + 7 };

int build_metric(fgpu_handle* h) {
  const fgpu_config& c = h->cfg;
  int nx = c.inum, ny = c.jnum, nz = c.knum;
  double dx = (c.xmax - c.xmin) / nx, mdx = dx;
  double dy = (c.ymax - c.ymin) / ny, mdy = dy;
  double dz = (c.zmax - c.zmin) / nz, mdz = dz;
  if (dx < 2 * DBL_EPSILON) { if (nx == 1) { dx = 1.0; mdx = 0.0; } else return set_err(h, FGPU_EBADCFG, "INUM > 1 conflicts with zero x-extent"); }
  if (dy < 2 * DBL_EPSILON) { if (ny == 1) { dy = 1.0; mdy = 0.0; } else return set_err(h, FGPU_EBADCFG, "JNUM > 1 conflicts with zero y-extent"); }
  if (dz < 2 * DBL_EPSILON) { if (nz == 1) { dz = 1.0; mdz = 0.0; } else return set_err(h, FGPU_EBADCFG, "KNUM > 1 conflicts with zero z-extent"); }
  h->invd[0] = 1. / dx; h->invd[1] = 1. / dy; h->invd[2] = 1. / dz;
  h->dxyz[0] = dx; h->dxyz[1] = dy; h->dxyz[2] = dz;
  int nxp = nx + 4, nyp = ny + 4, nzp = nz + 4;
  h->nxp = nxp;
  // layout: M_NI arrays of nxp, then offyS, offyN (nyp), offzB, offzT (nzp)
  size_t base_y = (size_t)M_NI * nxp;
  size_t total = base_y + 2 * (size_t)nyp + 2 * (size_t)nzp;
  std::vector<double>& m = h->h_metric;
  m.assign(total, 0.0);
  auto A = [&](int which, int ip) -> double& { return m[(size_t)which * nxp + ip]; };
  int geo = c.geometry;
  double gp = c.gparam;
  // the centre z coordinate of a 2D mesh (KNUM = 1): zmin + 0.5*0
  double zc2d = c.zmin + ((double)(2 * 1 - 1) * 0.5) * mdz;
  for (int ip = 0; ip < nxp; ++ip) {
    int I = ip - 1;   // fosite 1-based index
    double x = c.xmin + ((double)(2 * I - 1) * 0.5) * mdx;
    double xw = x + (-0.5 * mdx), xe = x + 0.5 * mdx;
    double hxc, hyc, hzc, hxw, hyw, hzw, hxe, hye, hze;
    scale(geo, gp, x, hxc, hyc, hzc);
    scale(geo, gp, xw, hxw, hyw, hzw);
    scale(geo, gp, xe, hxe, hye, hze);
    // S/N/B/T faces share the centre's first coordinate
    double sqrtg = hxc * (hyc * hzc);
    double volume = sqrtg * dx * dy * dz;
    double dxdydV = dx * dy / (volume + DBL_MIN);
    double dydzdV = dy * dz / (volume + DBL_MIN);
    double dzdxdV = dz * dx / (volume + DBL_MIN);
    A(M_dAxW, ip) = hyw * hzw;
    A(M_dAxE, ip) = hye * hze;
    A(M_dAyS, ip) = hzc * hxc;
    A(M_dAzB, ip) = hxc * hyc;
    A(M_dydzdV, ip) = dydzdV;
    A(M_dzdxdV, ip) = dzdxdV;
    A(M_dxdydV, ip) = dxdydV;
    A(M_cyxy, ip) = 0.5 * (hze + hzw) * (hye - hyw) * dydzdV;
    A(M_cyzy, ip) = 0.5 * (hxc + hxc) * (hyc - hyc) * dxdydV;
    A(M_cxyx, ip) = 0.5 * (hzc + hzc) * (hxc - hxc) * dzdxdV;
    A(M_cxzx, ip) = 0.5 * (hyc + hyc) * (hxc - hxc) * dxdydV;
    A(M_czxz, ip) = 0.5 * (hye + hyw) * (hze - hzw) * dydzdV;
    A(M_czyz, ip) = 0.5 * (hxc + hxc) * (hzc - hzc) * dzdxdV;
    A(M_dlx, ip) = hxc * dx;
    A(M_dly, ip) = hyc * dy;
    A(M_dlz, ip) = hzc * dz;
    A(M_offxW, ip) = xw - x;
    A(M_offxE, ip) = xe - x;
    // FARGO wfactor (timedisc_base.f90:433-441): the narrowest y-width of the cell over its
    // W/E and B/T faces relative to the width through the centre
    {
      auto mn = [](double a, double b) { return b < a ? b : a; };
      A(M_wfac, ip) = mn(mn(hyw, hye), mn(hyc, hyc)) / hyc;
    }
    if (h->has_accel) {
      // gravity_pointmass.f90:263-282 with the point mass at the origin, NEWTON potential
      double r, posx;
      if (geo == FGPU_LOGCYLINDRICAL) { double rr = gp * std::exp(x); r = std::sqrt(rr * rr + zc2d * zc2d); posx = r; }
      else { r = std::sqrt(x * x + zc2d * zc2d); posx = r; }
      double om2 = 1. / std::max(10 * DBL_MIN, ((r * ((r - 0.0) * (r - 0.0))) + 0.0 * 0.0 * 0.0) / (c.gn * c.pm_mass));
      A(M_accel0, ip) = -om2 * posx;
      A(M_accel1, ip) = -om2 * 0.0;
    }
    if (!h->euler && c.csiso > 0.0)
      for (int q = 0; q < 7; ++q) A(M_cs0 + q, ip) = c.csiso;
  }
  for (int jp = 0; jp < nyp; ++jp) {
    int J = jp - 1;
    double y = c.ymin + ((double)(2 * J - 1) * 0.5) * mdy;
    m[base_y + jp] = (y + (-0.5 * mdy)) - y;
    m[base_y + nyp + jp] = (y + 0.5 * mdy) - y;
  }
  for (int kp = 0; kp < nzp; ++kp) {
    int K = kp - 1;
    double z = c.zmin + ((double)(2 * K - 1) * 0.5) * mdz;
    m[base_y + 2 * nyp + kp] = (z + (-0.5 * mdz)) - z;
    m[base_y + 2 * nyp + nzp + kp] = (z + 0.5 * mdz) - z;
  }
  return FGPU_OK;
}

// Cell geometry of the ALPHA/BETA/POWERLAW viscosities by padded cell: Mesh%radius at the
// bary centres (geometry_*.f90 Radius) and ephi/r in curvilinear components
// (sources_viscosity.f90:186-226: -y/r^2, x/r^2 from Convert2Cartesian of the bary centres,
// geometry_cylindrical.f90:446-455 / geometry_logcylindrical.f90:344-356, converted back with
// geometry_cylindrical.f90:485-494; Cartesian meshes use them as they are)
int upload_visc_geometry(fgpu_handle* h) {
  const fgpu_config& c = h->cfg;
  const int nx = c.inum, ny = c.jnum, nz = c.knum, nd = h->nd;
  const long long NXp = nx + 4, NYp = ny + 4, NZp = nd == 3 ? nz + 4 : 1;
  const long long npad = NXp * NYp * NZp;
  const double mdx = (c.xmax - c.xmin) / nx, mdy = (c.ymax - c.ymin) / ny;
  double mdz = (c.zmax - c.zmin) / nz;
  if (mdz < 2 * DBL_EPSILON && nz == 1) mdz = 0.0;
  std::vector<double> eph((size_t)nd * npad), rad((size_t)npad);
  for (long long kp = 0; kp < NZp; ++kp)
    for (long long jp = 0; jp < NYp; ++jp)
      for (long long ip = 0; ip < NXp; ++ip) {
        const long long q = ip + NXp * (jp + NYp * kp);
        const int I = (int)ip - 1, J = (int)jp - 1, K = nd == 3 ? (int)kp - 1 : 1;
        const double x1 = c.xmin + ((double)(2 * I - 1) * 0.5) * mdx;
        const double x2 = c.ymin + ((double)(2 * J - 1) * 0.5) * mdy;
        const double x3 = c.zmin + ((double)(2 * K - 1) * 0.5) * mdz;
        double X, Y, r;
        if (c.geometry == FGPU_CYLINDRICAL) {
          X = x1 * std::cos(x2); Y = x1 * std::sin(x2); r = std::sqrt(x1 * x1 + x3 * x3);
        } else if (c.geometry == FGPU_LOGCYLINDRICAL) {
          const double rr = c.gparam * std::exp(x1);
          X = rr * std::cos(x2); Y = rr * std::sin(x2); r = std::sqrt(rr * rr + x3 * x3);
        } else {
          X = x1; Y = x2; r = std::sqrt(x1 * x1 + x2 * x2 + x3 * x3);
        }
        const double r2 = r * r;
        const double ex = -Y / r2, ey = X / r2, ez = 0.0;
        double e[3];
        if (c.geometry == FGPU_CARTESIAN) { e[0] = ex; e[1] = ey; e[2] = ez; }
        else {
          e[0] = ex * std::cos(x2) + ey * std::sin(x2);
          e[1] = -ex * std::sin(x2) + ey * std::cos(x2);
          e[2] = ez;
        }
        for (int l = 0; l < nd; ++l) eph[(size_t)l * npad + q] = e[l];
        rad[q] = r;
      }
  h->npad_vis = npad;
  CUDA_TRY(h, cudaMalloc(&h->d_ephir, sizeof(double) * eph.size()));
  CUDA_TRY(h, cudaMalloc(&h->d_visrad, sizeof(double) * rad.size()));
  CUDA_TRY(h, cudaMalloc(&h->d_dynvis, sizeof(double) * npad));
  CUDA_TRY(h, cudaMalloc(&h->d_vistime, sizeof(double)));
  CUDA_TRY(h, cudaMemcpy(h->d_ephir, eph.data(), sizeof(double) * eph.size(), cudaMemcpyHostToDevice));
  CUDA_TRY(h, cudaMemcpy(h->d_visrad, rad.data(), sizeof(double) * rad.size(), cudaMemcpyHostToDevice));
  std::vector<double> dv((size_t)npad, c.dynconst);
  CUDA_TRY(h, cudaMemcpy(h->d_dynvis, dv.data(), sizeof(double) * npad, cudaMemcpyHostToDevice));
  const double t0 = -1.0;   // sources_viscosity.f90:256-258
  CUDA_TRY(h, cudaMemcpy(h->d_vistime, &t0, sizeof(double), cudaMemcpyHostToDevice));
  return FGPU_OK;
}

int upload_metric(fgpu_handle* h) {
  size_t bytes = h->h_metric.size() * sizeof(double);
  if (!h->d_metric) CUDA_TRY(h, cudaMalloc(&h->d_metric, bytes));
  CUDA_TRY(h, cudaMemcpyAsync(h->d_metric, h->h_metric.data(), bytes, cudaMemcpyHostToDevice, h->stream));
  int nxp = h->nxp, nyp = h->cfg.jnum + 4, nzp = h->cfg.knum + 4;
  const double* b = h->d_metric;
  auto P = [&](int which) { return b + (size_t)which * nxp; };
  MetricP& M = h->mt;
  M.dAxW = P(M_dAxW); M.dAyS = P(M_dAyS); M.dAzB = P(M_dAzB);
  M.dydzdV = P(M_dydzdV); M.dzdxdV = P(M_dzdxdV); M.dxdydV = P(M_dxdydV);
  M.cxyx = P(M_cxyx); M.cxzx = P(M_cxzx); M.cyxy = P(M_cyxy); M.cyzy = P(M_cyzy); M.czxz = P(M_czxz); M.czyz = P(M_czyz);
  M.dlx = P(M_dlx); M.dly = P(M_dly); M.dlz = P(M_dlz);
  M.offxW = P(M_offxW); M.offxE = P(M_offxE);
  size_t base_y = (size_t)M_NI * nxp;
  M.offyS = b + base_y; M.offyN = b + base_y + nyp;
  M.offzB = b + base_y + 2 * nyp; M.offzT = b + base_y + 2 * nyp + nzp;
  M.accel = h->has_accel ? P(M_accel0) : nullptr;
  M.cs = P(M_cs0);
  M.dAxE = P(M_dAxE);
  M.nxp = nxp;
  M.curv = h->curv ? 1 : 0;
  // the fused CFL epilogues add the viscous limit of the constant model; the other models
  // evaluate it in visc_cfl_kernel after their end-of-step update
  M.vis = h->vis && h->vis_model == FGPU_VIS_MOLECULAR ? 1 : 0;
  M.vis_eta = h->vis_eta;
  return FGPU_OK;
}

// ---------------------------------------------------------------- launchers
// (the shared-memory stage layouts are launched through fgpu_stage_launch.h, the TMA-staged
// ones through fgpu_tma_launch.h)
void configure_stage_kernels(int nd, bool e, bool p) {
  if (nd == 2) {
    legacy_stage_configure_2d(e, p);
    tma_stage_configure_2d(e, p);
  } else {
    legacy_stage_configure_3d(e, p);
    tma_stage_configure_3d(e, p);
  }
}

// cuTensorMapEncodeTiled from the driver (no link against libcuda)
PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// Tensor map of a state (V fields of n doubles, i fastest) for boxes of (tx+4) x (ty+4) cells
// of one plane and every variable: dims (nx, ny, [nz,] V); cached per handle by base pointer.
const CUtensorMap* stage_tmap(fgpu_handle* h, const double* base, int tx, int ty) {
  for (const auto& e : h->tmaps)
    if (e.base == base && e.tx == tx && e.ty == ty) return &e.map;
  PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
  if (!enc) return nullptr;
  const Grid& g = h->g;
  fgpu_handle::TmapEntry e;
  e.base = base; e.tx = tx; e.ty = ty;
  cuuint64_t dims[4], strides[3];
  cuuint32_t box[4], es[4] = {1, 1, 1, 1};
  int rank;
  if (h->nd == 3) {
    rank = 4;
    dims[0] = g.nx; dims[1] = g.ny; dims[2] = g.nz; dims[3] = h->V;
    strides[0] = 8ull * g.nx; strides[1] = 8ull * g.nx * g.ny; strides[2] = 8ull * g.n;
    box[0] = tx + 4; box[1] = ty + 4; box[2] = 1; box[3] = h->V;
  } else {
    rank = 3;
    dims[0] = g.nx; dims[1] = g.ny; dims[2] = h->V;
    strides[0] = 8ull * g.nx; strides[1] = 8ull * g.n;
    box[0] = tx + 4; box[1] = ty + 4; box[2] = h->V;
  }
  CUresult r = enc(&e.map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, rank, const_cast<double*>(base), dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return nullptr;
  h->tmaps.push_back(e);
  return &h->tmaps.back().map;
}

// The TMA layout serves stages whose input is a plain or formed state (no k-sums at the stencil
// points) without viscous source or accretion rows, on meshes whose x extent is even (16-byte
// strides of the tensor map); FARGO frame changes on 2D meshes.
bool tma_eligible(const fgpu_handle* h, const StageArgs& A) {
  const StateRef& S = A.rin.base ? A.rin : A.in;
  const bool frames = h->fargo || A.w_sub || S.pre.n || A.in.pre.n || A.yn_chain.n || A.y0_chain.n || A.err_chain.n;
  return h->g.nx % 2 == 0 && (!frames || h->nd == 2) && !h->vis && !A.visc && !A.brow && !A.flux_out && S.nk == 0 &&
         (S.pre.n == 0 || &S == &A.in) && tmap_encoder() != nullptr;
}

template <int ND, bool EU, bool PRIM>
int launch_stage_t(fgpu_handle* h, StageArgs& A) {
  A.kchunk = h->kchunk;
  const Grid& g = h->g;
  if ((h->variant == 6 || (h->variant == 7 && ND == 2)) && tma_eligible(h, A)) {
    const StateRef& SR = A.rin.base ? A.rin : A.in;
    const int ty = h->variant == 7 ? 4 : kTmaTY;
    const CUtensorMap* map = stage_tmap(h, SR.base, kTmaTX, ty);
    if (!map) return set_err(h, FGPU_ECUDA, "cuTensorMapEncodeTiled failed for a stage input");
    const bool crec = A.constant_recon != 0;
    if (ND == 3) CUDA_TRY(h, tma_stage_launch_3d(EU, PRIM, A.limiter, crec, g, h->kchunk, h->stream, A, *map));
    else CUDA_TRY(h, tma_stage_launch_2d(EU, PRIM, A.limiter, crec, ty, g, h->stream, A, *map));
    return FGPU_OK;
  }
  // the warp-shuffle layout implements neither FARGO frame changes, the accretion rows, the
  // viscous source, the device-clock gates, the next Butcher stage's state formation nor the
  // CheckData-only epilogue
  // (a variant-6 launch that the TMA layout does not serve runs on the base tile)
  const int variant =
      (h->variant == 1 && (h->fargo || h->accrete || h->vis || A.gate || A.fnext_out || A.cfl_mode == 3 ||
                           A.flux_out || A.out_prim))
          ? 0 : (h->variant >= 6 ? 0 : h->variant);
  if (ND == 3) CUDA_TRY(h, legacy_stage_launch_3d(EU, PRIM, variant, g, h->kchunk, h->stream, A));
  else CUDA_TRY(h, legacy_stage_launch_2d(EU, PRIM, variant, g, h->stream, A));
  CUDA_TRY(h, cudaGetLastError());
  return FGPU_OK;
}

int launch_stage_raw(fgpu_handle* h, StageArgs& A) {
  bool e = h->euler, p = h->prim;
  if (h->nd == 2) {
    if (e) return p ? launch_stage_t<2, true, true>(h, A) : launch_stage_t<2, true, false>(h, A);
    return p ? launch_stage_t<2, false, true>(h, A) : launch_stage_t<2, false, false>(h, A);
  }
  if (e) return p ? launch_stage_t<3, true, true>(h, A) : launch_stage_t<3, true, false>(h, A);
  return p ? launch_stage_t<3, false, true>(h, A) : launch_stage_t<3, false, false>(h, A);
}

template <int ND, bool EU>
int launch_misc_t(fgpu_handle* h, int which, BndArgs& B) {
  if (which == 0) {
    long long blocks = std::min<long long>((B.nghost + 255) / 256, 4096);
    if (blocks < 1) blocks = 1;
    boundary_kernel<ND, EU><<<(unsigned)blocks, 256, 0, h->stream>>>(B);
  } else if (which == 1) {
    long long blocks = std::min<long long>((h->g.n + 255) / 256, 148 * 16);
    interior_cfl_kernel<ND, EU><<<(unsigned)blocks, 256, 0, h->stream>>>(B);
  } else {
    long long blocks = std::min<long long>((h->g.n + 255) / 256, 148 * 16);
    pack_interior_kernel<ND, EU><<<(unsigned)blocks, 256, 0, h->stream>>>(B);
  }
  CUDA_TRY(h, cudaGetLastError());
  return FGPU_OK;
}
int launch_misc_raw(fgpu_handle* h, int which, BndArgs& B) {
  if (h->nd == 2) return h->euler ? launch_misc_t<2, true>(h, which, B) : launch_misc_t<2, false>(h, which, B);
  return h->euler ? launch_misc_t<3, true>(h, which, B) : launch_misc_t<3, false>(h, which, B);
}
// Algorithmic HBM arrays of one stage launch: the stencil input arrays once,
// the start-of-step state for the Shu-Osher update, and every output written.
double stage_bytes(const fgpu_handle* h, const StageArgs& A) {
  int arrays = 1 + A.in.nk;
  if (A.out_mode == OUT_SSPRK) arrays += 1;
  arrays += 1;
  if (A.out_base) arrays += 1;
  if (A.last_stage && A.out_high) arrays += 1;
  double bytes = (double)arrays * h->V * (double)h->g.n * 8.0;
  if (A.visc) bytes += (double)(h->nd + (h->euler ? 1 : 0)) * (double)h->g.n * 8.0;
  return bytes;
}

template <class F>
// kind: 0 boundary/reduction/transfer kernels, 1 stage kernel, 2 stage-state formation
int timed_launch(fgpu_handle* h, int kind, double bytes, F&& fn) {
  h->stats.launches += 1;
  if (kind == 1) h->stats.stage_launches += 1;
  if (!h->profiling) return fn();
  fgpu_handle::Timed t;
  t.bytes = bytes;
  t.stage = kind;
  CUDA_TRY(h, cudaEventCreate(&t.a));
  CUDA_TRY(h, cudaEventCreate(&t.b));
  CUDA_TRY(h, cudaEventRecord(t.a, h->stream));
  int rc = fn();
  CUDA_TRY(h, cudaEventRecord(t.b, h->stream));
  h->timed.push_back(t);
  return rc;
}

// Viscous source of the stage state of A into h->d_visc (sources_viscosity.f90:484-507); the
// stage kernel reads it.  Tiles: 2D 32 x 8, 3D 8 x 8 x 4.
template <int ND> struct ViscShape;
template <> struct ViscShape<2> { static constexpr int TX = 32, TY = 8, TZ = 1; };
template <> struct ViscShape<3> { static constexpr int TX = 8, TY = 8, TZ = 4; };
template <int ND, bool EU>
void configure_visc_t() {
  using S = ViscShape<ND>;
  cudaFuncSetAttribute(visc_kernel<ND, EU, S::TX, S::TY, S::TZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)ViscTile<ND, S::TX, S::TY, S::TZ>::SMEM);
}
void configure_visc(int nd, bool e) {
  if (nd == 2) e ? configure_visc_t<2, true>() : configure_visc_t<2, false>();
  else e ? configure_visc_t<3, true>() : configure_visc_t<3, false>();
}
template <int ND, bool EU>
void launch_visc_t(fgpu_handle* h, const ViscArgs& V) {
  using S = ViscShape<ND>;
  const Grid& g = h->g;
  dim3 grid((g.nx + S::TX - 1) / S::TX, (g.ny + S::TY - 1) / S::TY, ND == 3 ? (g.nz + S::TZ - 1) / S::TZ : 1);
  visc_kernel<ND, EU, S::TX, S::TY, S::TZ>
      <<<grid, S::TX * S::TY * S::TZ, ViscTile<ND, S::TX, S::TY, S::TZ>::SMEM, h->stream>>>(V);
}
// UpdateViscosity of the state S at the time `when` (ALPHA/BETA/POWERLAW): the conditional
// update of the cell viscosities, then the record of its time
template <int ND, bool EU>
void launch_visc_update_t(fgpu_handle* h, const VisUpdArgs& U) {
  const unsigned blocks = (unsigned)std::min<long long>((U.npad + 255) / 256, 148 * 8);
  visc_update_kernel<ND, EU><<<blocks, 256, 0, h->stream>>>(U);
  visc_time_kernel<<<1, 1, 0, h->stream>>>(U, h->d_vistime);
}
int launch_visc_update(fgpu_handle* h, const StateRef& S, const RhsTime& when, int gate = 0) {
  if (!h->vis || h->vis_model == FGPU_VIS_MOLECULAR) return FGPU_OK;
  VisUpdArgs U;
  std::memset(&U, 0, sizeof(U));
  U.g = h->g; U.ph = h->ph; U.mt = h->mt;
  U.in = S;
  U.model = h->vis_model;
  U.dynconst = h->vis_eta;
  U.power = h->vis_power;
  U.ephir = h->d_ephir;
  U.rad = h->d_visrad;
  U.dynvis = h->d_dynvis;
  U.vis_time = h->d_vistime;
  U.t = when.t;
  if (when.dev) {
    U.t_dev = when.attempt ? &h->d_ctl->t_loc : &h->d_ctl->time;
    U.dt_dev = when.attempt ? &h->d_ctl->d_att : &h->d_ctl->dt;
    U.zeta = when.zeta;
    U.ctl = h->d_ctl;
  }
  U.gate = gate;
  U.npad = h->npad_vis;
  return timed_launch(h, 0, 0.0, [&] {
    if (h->nd == 2) h->euler ? launch_visc_update_t<2, true>(h, U) : launch_visc_update_t<2, false>(h, U);
    else h->euler ? launch_visc_update_t<3, true>(h, U) : launch_visc_update_t<3, false>(h, U);
    CUDA_TRY(h, cudaGetLastError());
    return FGPU_OK;
  });
}
// CalcTimestep's viscous limit for ALPHA/BETA/POWERLAW: UpdateViscosity at the state's time,
// then the reduction over the padded cells into ctl->invdt[3]
int launch_visc_cfl(fgpu_handle* h, const StateRef& S, bool roundtrip, const RhsTime& when, int gate = 0) {
  if (!h->vis || h->vis_model == FGPU_VIS_MOLECULAR) return FGPU_OK;
  if (int rc = launch_visc_update(h, S, when, gate)) return rc;
  VisCflArgs C;
  std::memset(&C, 0, sizeof(C));
  C.g = h->g; C.ph = h->ph; C.mt = h->mt;
  C.in = S;
  C.roundtrip = roundtrip ? 1 : 0;
  C.dynvis = h->d_dynvis;
  C.npad = h->npad_vis;
  C.ctl = h->d_ctl;
  C.gate = gate;
  const unsigned blocks = (unsigned)std::min<long long>((C.npad + 255) / 256, 148 * 8);
  return timed_launch(h, 0, 0.0, [&] {
    if (h->nd == 2) {
      if (h->euler) visc_cfl_kernel<2, true><<<blocks, 256, 0, h->stream>>>(C);
      else visc_cfl_kernel<2, false><<<blocks, 256, 0, h->stream>>>(C);
    } else {
      if (h->euler) visc_cfl_kernel<3, true><<<blocks, 256, 0, h->stream>>>(C);
      else visc_cfl_kernel<3, false><<<blocks, 256, 0, h->stream>>>(C);
    }
    CUDA_TRY(h, cudaGetLastError());
    return FGPU_OK;
  });
}

int launch_visc(fgpu_handle* h, const StateRef& S, int gate = 0) {
  ViscArgs V;
  std::memset(&V, 0, sizeof(V));
  V.g = h->g; V.ph = h->ph; V.mt = h->mt;
  V.in = S;
  V.eta = h->vis_eta;
  V.mub = h->vis_mub;
  V.dynvis = h->vis_model == FGPU_VIS_MOLECULAR ? nullptr : h->d_dynvis;
  V.out = h->d_visc;
  V.ctl = h->d_ctl;
  V.gate = gate;
  // algorithmic bytes: the state read once, the source written once
  const double bytes = (double)(h->V + h->nd + (h->euler ? 1 : 0)) * (double)h->g.n * 8.0;
  return timed_launch(h, 1, bytes, [&] {
    if (h->nd == 2) h->euler ? launch_visc_t<2, true>(h, V) : launch_visc_t<2, false>(h, V);
    else h->euler ? launch_visc_t<3, true>(h, V) : launch_visc_t<3, false>(h, V);
    CUDA_TRY(h, cudaGetLastError());
    return FGPU_OK;
  });
}

// One right-hand side evaluation (stage kernel) at the time `when`, preceded by the viscous
// source of its state when the viscosity is on
int launch_stage(fgpu_handle* h, StageArgs& A, const RhsTime& when = RhsTime()) {
  if (h->vis) {
    const StateRef& S = A.rin.base ? A.rin : A.in;
    if (int rc = launch_visc_update(h, S, when, A.gate)) return rc;
    if (int rc = launch_visc(h, S, A.gate)) return rc;
    A.visc = h->d_visc;
  }
  return timed_launch(h, true, stage_bytes(h, A), [&] { return launch_stage_raw(h, A); });
}
int launch_misc(fgpu_handle* h, int which, BndArgs& B) {
  return timed_launch(h, false, 0.0, [&] { return launch_misc_raw(h, which, B); });
}

template <int ND, bool EU>
void launch_form_t(fgpu_handle* h, const StateRef& S, double* out, unsigned blocks, int gate) {
  if (h->prim) form_kernel<ND, EU, true><<<blocks, 256, 0, h->stream>>>(S, h->g, h->ph, out, h->d_ctl, gate);
  else form_kernel<ND, EU, false><<<blocks, 256, 0, h->stream>>>(S, h->g, h->ph, out, h->d_ctl, gate);
}
int launch_form(fgpu_handle* h, const StateRef& S, double* out, int gate = 0) {
  unsigned blocks = (unsigned)std::min<long long>((h->g.n + 255) / 256, 148 * 8);
  if (h->nd == 2) h->euler ? launch_form_t<2, true>(h, S, out, blocks, gate) : launch_form_t<2, false>(h, S, out, blocks, gate);
  else h->euler ? launch_form_t<3, true>(h, S, out, blocks, gate) : launch_form_t<3, false>(h, S, out, blocks, gate);
  CUDA_TRY(h, cudaGetLastError());
  return FGPU_OK;
}

int launch_roundtrip(fgpu_handle* h, const double* in, double* out) {
  long long blocks = std::min<long long>((h->g.n + 255) / 256, 148 * 16);
  if (h->nd == 2) {
    if (h->euler) roundtrip_kernel<2, true><<<(unsigned)blocks, 256, 0, h->stream>>>(in, out, h->g.n, h->ph);
  } else {
    if (h->euler) roundtrip_kernel<3, true><<<(unsigned)blocks, 256, 0, h->stream>>>(in, out, h->g.n, h->ph);
  }
  if (!h->euler) CUDA_TRY(h, cudaMemcpyAsync(out, in, sizeof(double) * h->V * h->g.n, cudaMemcpyDeviceToDevice, h->stream));
  CUDA_TRY(h, cudaGetLastError());
  return FGPU_OK;
}

long long ghost_count(const fgpu_handle* h) {
  long long NXp = h->g.nx + 4, NYp = h->g.ny + 4, NZp = h->nd == 3 ? h->g.nz + 4 : 1;
  return NXp * NYp * NZp - h->g.n;
}

StateRef plain_state(const double* s, bool roundtrip) {
  StateRef S;
  std::memset(&S, 0, sizeof(S));
  S.base = s;
  S.nk = 0;
  S.roundtrip = roundtrip ? 1 : 0;
  return S;
}

StageArgs base_args(fgpu_handle* h) {
  StageArgs A;
  std::memset(&A, 0, sizeof(A));
  A.g = h->g; A.ph = h->ph; A.mt = h->mt;
  A.limiter = h->cfg.limiter; A.theta = h->cfg.theta;
  A.constant_recon = h->cfg.order == FGPU_CONSTANT ? 1 : 0;
  for (int d = 0; d < 3; ++d) A.invd[d] = h->invd[d];
  A.has_accel = h->has_accel ? 1 : 0;
  A.checkdata = h->cfg.checkdata;
  A.ctl = h->d_ctl;
  A.tol_rel = h->tol_rel;
  for (int v = 0; v < FGPU_MAXV; ++v) A.tol_abs[v] = h->tol_abs[v];
  if (h->accrete) {
    A.brow = h->d_acc + 2 * (size_t)h->g.ny;
    A.brow_face = h->acc_face;
    A.bdydz = h->dxyz[1] * h->dxyz[2];
  }
  return A;
}

// Butcher stage m's formed input (reconstruction variables), alternating between two buffers
// when the stage kernels form the next stage's state (fuse_form)
double* stage_rbuf(const fgpu_handle* h, int m) {
  return h->buf[2 + h->T.m + (h->fuse_form ? (m % 2) : 0)];
}
// let stage m (< M) form stage m+1's state: base - sum_{q<=m} (a_{m+1,q} dt) k_q into its buffer;
// coefficients times dt on the host (dt_dev null) or, on the device clock, times *dt_dev
void set_fnext(const fgpu_handle* h, StageArgs& A, int m, double dtv, const double* dt_dev) {
  const Tableau& T = h->T;
  if (!h->fuse_form || m >= T.m) return;
  StateRef& S = A.fnext;
  std::memset(&S, 0, sizeof(S));
  S.base = h->buf[1];
  S.nk = m;
  for (int q = 0; q < m; ++q) {
    S.K[q] = h->buf[2 + q];
    S.coef[q] = dt_dev ? T.A[m * T.m + q] : T.A[m * T.m + q] * dtv;
  }
  S.dt_dev = dt_dev;
  A.fnext_out = stage_rbuf(h, m + 1);
}

// the last Butcher stage's epilogue: high/low-order solutions (the high one into out_high) and
// the error norm; weights times dt on the host, or (dtv = 0, device clock) the bare weights
// that the kernel multiplies by *in.dt_dev
void set_last_stage(const fgpu_handle* h, StageArgs& A, double* out_high, double dtv) {
  const Tableau& T = h->T;
  A.last_stage = 1;
  A.nstage = T.m;
  for (int q = 0; q < T.m; ++q) {
    A.bh_dt[q] = A.in.dt_dev ? T.bh[q] : T.bh[q] * dtv;
    A.bl_dt[q] = A.in.dt_dev ? T.bl[q] : T.bl[q] * dtv;
  }
  A.out_high = out_high;
}

BndArgs bnd_args(fgpu_handle* h, const double* state, bool roundtrip, int finalize) {
  BndArgs B;
  std::memset(&B, 0, sizeof(B));
  B.g = h->g; B.ph = h->ph; B.mt = h->mt;
  B.in = plain_state(state, roundtrip);
  B.roundtrip = roundtrip ? 1 : 0;
  B.checkdata = h->cfg.checkdata;
  B.ctl = h->d_ctl;
  B.finalize = finalize;
  B.nghost = ghost_count(h);
  return B;
}

int read_ctl(fgpu_handle* h) {
  CUDA_TRY(h, cudaMemcpyAsync(h->h_ctl, h->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return FGPU_OK;
}
int write_ctl(fgpu_handle* h) {
  CUDA_TRY(h, cudaMemcpyAsync(h->d_ctl, h->h_ctl, sizeof(Ctl), cudaMemcpyHostToDevice, h->stream));
  return FGPU_OK;
}
double ctl_invdt(const fgpu_handle* h) {
  const Ctl* c = h->h_ctl;
  auto D = [](unsigned long long b) { double d; std::memcpy(&d, &b, 8); return d; };
  if (h->nd == 2) return D(c->invdt[0]);
  double ix = D(c->invdt[0]), iy = D(c->invdt[1]), iz = D(c->invdt[2]);
  return std::max(std::max(iy, iz), ix);
}
// CalcTimestep's closing arithmetic on the host: the CFL step (timedisc_base.f90:885-900),
// then the sources list (sources_generic.f90:264-293) with the viscous limit of
// sources_viscosity.f90:576-580; *cause receives the dtcause
double ctl_dt(const fgpu_handle* h, int* cause) {
  double dt = h->cfl / ctl_invdt(h);
  *cause = FGPU_DTCAUSE_CFL;
  if (h->vis) {
    double iv;
    std::memcpy(&iv, &h->h_ctl->invdt[3], 8);
    const double dtv = iv > DBL_MIN ? h->cvis / iv : DBL_MAX;
    if (dtv < dt) *cause = FGPU_DTCAUSE_VISCOSITY;
    dt = std::min(dt, dtv);
  }
  return dt;
}

// ---------------------------------------------------------------- Shu-Osher (device clock)
// eta(n,order) and zeta(n,order), timedisc_modeuler.f90:74-77
const double kEta[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.5, 0.0}, {0.0, 0.75, 1.0 / 3.0}};
const double kZeta[3][3] = {{0.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 1.0, 0.5}};
// time of the right-hand side read by Shu-Osher stage n: the previous step's closing
// ComputeRHS at time (n = 1), else the one after update n-1 at time + zeta(n-1)*dt
// (timedisc_modeuler.f90:150-158)
double stage_zeta(const fgpu_handle* h, int n) { return n == 1 ? 0.0 : kZeta[h->order - 1][n - 2]; }

// Arguments of Shu-Osher stage n (1-based) of one grid: stage 1 reads the
// stored state P (with the CHECK_PMIN round trip of the last ComputeRHS),
// stages alternate between the scratch states A and B, the last stage writes P
// and reduces the CFL of the new state (order 1 goes through A and a copy).
StageArgs shu_osher_stage(fgpu_handle* h, int n) {
  double* P = h->buf[0];
  double* Abuf = h->buf[1];
  double* Bbuf = h->buf[2];
  const double* in = n == 1 ? P : ((n - 1) % 2 == 1 ? Abuf : Bbuf);
  StageArgs A = base_args(h);
  A.in = plain_state(in, n == 1 && h->pre_rt);
  A.out_mode = OUT_SSPRK;
  A.eta = kEta[h->order - 1][n - 1];
  A.y0 = P;
  A.y0_roundtrip = h->pre_rt ? 1 : 0;
  A.dt_dev = &h->d_ctl->dt;
  A.out = (n == h->order && h->order > 1) ? P : ((n % 2 == 1) ? Abuf : Bbuf);
  if (n == h->order) { A.cfl_mode = 1; A.cfl_roundtrip = h->roundtrip_cfg ? 1 : 0; }
  if (h->so_form) {
    // the primitive form of A (stage 1's result) and B (stage 2's) beside the states
    if (n < h->order) A.out_prim = h->d_pform[(n - 1) % 2];
    if (n >= 2) {
      A.rin = plain_state(h->d_pform[(n - 2) % 2], false);
      A.rin.ready = 1;
    }
  }
  return A;
}

// accretion bookkeeping after Shu-Osher stage n (no-op without accretion)
int launch_accrete(fgpu_handle* h, int n) {
  if (!h->accrete) return FGPU_OK;
  AccArgs C;
  std::memset(&C, 0, sizeof(C));
  const size_t ny = (size_t)h->g.ny;
  C.bx = h->d_acc;
  C.bxold = h->d_acc + ny;
  C.brow = h->d_acc + 2 * ny;
  C.grav = h->d_acc + 3 * ny;
  C.ny = h->g.ny;
  C.eta = kEta[h->order - 1][n - 1];
  C.dt = &h->d_ctl->dt;
  C.last = n == h->order ? 1 : 0;
  C.accel = h->d_metric + (size_t)M_accel0 * h->nxp;   // accel0 and accel1 are adjacent
  C.naccel = 2 * h->nxp;
  C.ctl = h->d_ctl;
  return timed_launch(h, 0, 0.0, [&] {
    accrete_kernel<<<1, 256, 0, h->stream>>>(C);
    CUDA_TRY(h, cudaGetLastError());
    return FGPU_OK;
  });
}

int enqueue_shu_osher_step(fgpu_handle* h) {
  for (int n = 1; n <= h->order; ++n) {
    StageArgs A = shu_osher_stage(h, n);
    if (int rc = launch_stage(h, A, RhsTime::device(stage_zeta(h, n)))) return rc;
    if (int rc = launch_accrete(h, n)) return rc;
  }
  if (h->order == 1)
    CUDA_TRY(h, cudaMemcpyAsync(h->buf[0], h->buf[1], sizeof(double) * h->V * h->g.n, cudaMemcpyDeviceToDevice,
                                h->stream));
  // the closing ComputeRHS at time + dt (AcceptSolution) updates the viscosity that
  // CalcTimestep then reads
  if (int rc = launch_visc_cfl(h, plain_state(h->buf[0], h->roundtrip_cfg), h->roundtrip_cfg, RhsTime::device(1.0)))
    return rc;
  BndArgs B = bnd_args(h, h->buf[0], h->roundtrip_cfg, FIN_STEP);
  h->pre_rt = h->roundtrip_cfg;   // the end-of-step ComputeRHS uses the checkdata mask
  return launch_misc(h, 0, B);
}

// ---------------------------------------------------------------- FARGO (device clock)
Chain chain_add(Chain c, const double* w, double sgn) {
  c.w[c.n] = w;
  c.s[c.n] = sgn;
  c.n += 1;
  return c;
}
Chain chain_none() {
  Chain c;
  std::memset(&c, 0, sizeof(c));
  return c;
}
// Frame changes that turn the stored state into the real-frame cvar of the last
// ComputeRHS: none after FirstStep, AddBackgroundVelocityY(w) after a step.
Chain fargo_pre(const fgpu_handle* h) {
  return h->fargo_phase == 2 ? chain_add(chain_none(), h->d_w, 1.0) : chain_none();
}
const double* fargo_wfac(const fgpu_handle* h) {
  return h->fdir == 1 ? h->d_w + 2 * (size_t)h->nw : h->d_metric + (size_t)M_wfac * h->nxp;
}

int launch_fargo_w(fgpu_handle* h, const StateRef& in, const double* w_prev, double* w_out, int gate = 0) {
  FargoWArgs F;
  std::memset(&F, 0, sizeof(F));
  F.gate = gate;
  F.g = h->g; F.ph = h->ph; F.mt = h->mt;
  F.in = in;
  F.w_prev = w_prev;
  F.wfac = fargo_wfac(h);
  F.w_out = w_out;
  F.ctl = h->d_ctl;
  return timed_launch(h, false, 0.0, [&] {
    if (h->fdir == 1) {
      unsigned blocks = (unsigned)((h->g.ny + 4 + FX_WY - 1) / FX_WY);
      if (h->euler) fargo_w_x_kernel<true><<<blocks, FX_WX * FX_WY, 0, h->stream>>>(F);
      else fargo_w_x_kernel<false><<<blocks, FX_WX * FX_WY, 0, h->stream>>>(F);
    } else {
      const long long nt = (long long)(h->g.nx + 4) * h->g.ny;
      const unsigned tb = (unsigned)((nt + 255) / 256), sb = (unsigned)((h->g.nx + 4 + FS_WX - 1) / FS_WX);
      if (h->euler) fargo_w_terms_kernel<true><<<tb, 256, 0, h->stream>>>(F, h->d_fw_terms);
      else fargo_w_terms_kernel<false><<<tb, 256, 0, h->stream>>>(F, h->d_fw_terms);
      fargo_w_sum_kernel<<<sb, FS_NT, 0, h->stream>>>(F, h->d_fw_terms);
    }
    CUDA_TRY(h, cudaGetLastError());
    return FGPU_OK;
  });
}

int launch_fargo_advect_args(fgpu_handle* h, const FargoAdvArgs& X) {
  return timed_launch(h, false, 0.0, [&] {
    if (h->fdir == 1) {
      const unsigned blocks = (unsigned)std::min<long long>((h->g.n + 255) / 256, 148 * 8);
      if (h->euler) fargo_advect_x_kernel<true><<<blocks, 256, 0, h->stream>>>(X);
      else fargo_advect_x_kernel<false><<<blocks, 256, 0, h->stream>>>(X);
    } else {
      constexpr int TX = 32, TY = 4;
      dim3 grid((h->g.nx + TX - 1) / TX, (h->g.ny + TY * X.chunk - 1) / (TY * X.chunk));
      if (h->euler) fargo_advect_kernel<true, TX, TY><<<grid, TX * TY, 0, h->stream>>>(X);
      else fargo_advect_kernel<false, TX, TY><<<grid, TX * TY, 0, h->stream>>>(X);
    }
    CUDA_TRY(h, cudaGetLastError());
    return FGPU_OK;
  });
}

// The arguments of one FARGO step's passes (shared by the single-grid step and batches):
// the background velocity of the step, stage n of the Shu-Osher update, the advection and the
// closing ghost-cell pass.  W is the background velocity of the last ComputeRHS, Wn the step's.
struct FargoStep {
  double* P;
  const double* W;
  double* Wn;
  bool dyn;        // type 1: w_new computed from the state; type 2: the user's w stays
  Chain pre;       // the stored state's frame (the last ComputeRHS's AddBackgroundVelocity)
};
FargoStep fargo_step_of(fgpu_handle* h) {
  FargoStep F;
  F.P = h->buf[0];
  F.W = h->d_w;
  F.dyn = h->cfg.fargo_method == 1;
  F.Wn = F.dyn ? h->d_w + h->nw : h->d_w;
  F.pre = fargo_pre(h);
  return F;
}
FargoWArgs fargo_w_args(fgpu_handle* h, const FargoStep& F) {
  FargoWArgs X;
  std::memset(&X, 0, sizeof(X));
  X.g = h->g; X.ph = h->ph; X.mt = h->mt;
  X.in = plain_state(F.P, false);
  X.in.pre = F.pre;
  X.w_prev = F.W;
  X.wfac = fargo_wfac(h);
  X.w_out = F.Wn;
  X.ctl = h->d_ctl;
  return X;
}
StageArgs fargo_stage_args(fgpu_handle* h, const FargoStep& F, int n) {
  double* Abuf = h->buf[1];
  double* Bbuf = h->buf[2];
  // after FirstStep an ideal-gas cvar is the CHECK_ALL round trip of the stored state
  Chain cold = chain_add(F.pre, F.W, -1.0);
  if (h->pre_rt) cold.rt = 1;
  const double* in = n == 1 ? F.P : ((n - 1) % 2 == 1 ? Abuf : Bbuf);
  StageArgs A = base_args(h);
  A.in = plain_state(in, n == 1 && h->pre_rt);
  if (n == 1) {
    A.in.pre = F.pre;
    A.w_sub = F.W;
    // type 1: CalcBackgroundVelocity adds w and the step subtracts w_new; type 2: cvar
    // is already co-moving, the step's SubtractBackgroundVelocity does nothing
    A.yn_chain = F.dyn ? chain_add(chain_add(cold, F.W, 1.0), F.Wn, -1.0) : cold;
  } else {
    A.in.pre = chain_add(chain_none(), F.Wn, 1.0);
    A.w_sub = F.Wn;
    A.yn_chain = chain_add(A.in.pre, F.Wn, -1.0);
  }
  A.out_mode = OUT_SSPRK;
  A.eta = kEta[h->order - 1][n - 1];
  A.y0 = F.P;
  A.y0_chain = cold;
  A.dt_dev = &h->d_ctl->dt;
  A.out = (n % 2 == 1) ? Abuf : Bbuf;
  return A;
}
// the last stage's result, which the advection transports into P
const double* fargo_last_stage_out(const fgpu_handle* h) { return (h->order % 2 == 1) ? h->buf[1] : h->buf[2]; }
FargoAdvArgs fargo_adv_args(fgpu_handle* h, const FargoStep& F) {
  FargoAdvArgs X;
  std::memset(&X, 0, sizeof(X));
  X.g = h->g; X.ph = h->ph; X.mt = h->mt;
  X.in = plain_state(fargo_last_stage_out(h), false);
  X.w = F.Wn;
  X.out = F.P;
  X.ctl = h->d_ctl;
  X.checkdata = h->cfg.checkdata;
  X.chunk = 8;
  return X;
}
BndArgs fargo_closing_bnd(fgpu_handle* h, const FargoStep& F) {
  BndArgs B = bnd_args(h, F.P, false, FIN_STEP);
  B.in.pre = chain_add(chain_none(), F.Wn, 1.0);
  B.w_sub = F.Wn;
  return B;
}

// One fosite%Step with FARGO transport (timedisc_base.f90:649-750 with the
// modified-Euler SolveODE, timedisc_modeuler.f90:279-291):
//   CalcBackgroundVelocity -> w_new; the Shu-Osher stages on the co-moving
//   state; FargoAdvection; the closing ComputeRHS's CheckData and
//   CalcTimestep.  The in-place frame changes of cvar are carried as chains:
//   fosite's cvar at stage 1 is pre + [-w, +w, -w_new] applied to the stored
//   state, cold is pre + [-w], later stages read the previous stage's result
//   with [+w_new] (ComputeRHS's AddBackgroundVelocity) and their Shu-Osher
//   base is [+w_new, -w_new].
int enqueue_fargo_step(fgpu_handle* h) {
  const FargoStep F = fargo_step_of(h);
  if (F.dyn) {
    const FargoWArgs X = fargo_w_args(h, F);
    if (int rc = launch_fargo_w(h, X.in, X.w_prev, X.w_out)) return rc;
  }
  for (int n = 1; n <= h->order; ++n) {
    StageArgs A = fargo_stage_args(h, F, n);
    if (int rc = launch_stage(h, A)) return rc;
    if (int rc = launch_accrete(h, n)) return rc;
  }
  if (int rc = launch_fargo_advect_args(h, fargo_adv_args(h, F))) return rc;
  BndArgs B = fargo_closing_bnd(h, F);
  if (int rc = launch_misc(h, 0, B)) return rc;
  if (F.dyn) CUDA_TRY(h, cudaMemcpyAsync(h->d_w, F.Wn, sizeof(double) * h->nw, cudaMemcpyDeviceToDevice, h->stream));
  h->fargo_phase = 2;
  h->pre_rt = h->roundtrip_cfg;
  return FGPU_OK;
}

int enqueue_step(fgpu_handle* h) { return h->fargo ? enqueue_fargo_step(h) : enqueue_shu_osher_step(h); }

int build_graph(fgpu_handle* h, int steps) {
  if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
  cudaGraph_t gr;
  fgpu_stats saved = h->stats;
  CUDA_TRY(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  int rc = 0;
  for (int s = 0; s < steps && !rc; ++s) rc = enqueue_step(h);
  cudaError_t e = cudaStreamEndCapture(h->stream, &gr);
  h->kernels_per_step = (int)((h->stats.launches - saved.launches) / steps);
  h->stats = saved;
  if (rc) return rc;
  if (e != cudaSuccess) return set_err(h, FGPU_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&h->graph, gr, 0);
  cudaGraphDestroy(gr);
  if (e != cudaSuccess) return set_err(h, FGPU_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  h->graph_steps = steps;
  return FGPU_OK;
}

void sync_from_ctl(fgpu_handle* h) {
  const Ctl* c = h->h_ctl;
  h->time = c->time; h->dt = c->dt; h->dtold = c->dtold; h->dtmin = c->dtmin;
  h->iter = c->iter; h->dtcause = c->dtcause; h->brk = c->brk != 0; h->checkflags = c->flags;
}

// ---------------------------------------------------------------- Butcher engine (host clock)
int enqueue_k1(fgpu_handle* h, bool from_pre, bool cfl, bool rt, int checkdata, double t) {
  // ComputeRHS of the current state into K1.  from_pre: the stored state in P
  // gets the end-of-step CHECK_ALL treatment and its round trip goes to the
  // base buffer (cold = cvar); otherwise RejectSolution's CHECK_NOTHING RHS of base.
  double* P = h->buf[0];
  double* base = h->buf[1];
  double* K1 = h->buf[2];
  StageArgs A = base_args(h);
  A.out_mode = OUT_RHS;
  A.out = K1;
  if (from_pre) {
    A.in = plain_state(P, rt);
    A.out_base = base;
    A.checkdata = checkdata;
    if (cfl) A.cfl_mode = 2;
    else if (checkdata) A.cfl_mode = 3;   // AcceptSolution's ComputeRHS inside the step
  } else {
    A.in = plain_state(base, false);
  }
  return launch_stage(h, A, RhsTime::host(t));
}

double adjust_timestep(fgpu_handle* h, double maxerr, double dtold_) {
  // timedisc_base.f90:759-814
  double dtnew, dttmp;
  if (h->tol_rel >= 1.0) return DBL_MAX;
  // correctly rounded exp/log (fgpu_ddmath.h): the device controller computes the same values
  if (maxerr > 0.) dttmp = 0.9 * dtold_ * ddm::exp_cr(-ddm::log_cr(maxerr) / h->T.order);
  else dttmp = 4. * dtold_;
  if (h->maxerrold > 0.) dtnew = dttmp * ddm::exp_cr(-h->beta * ddm::log_cr(h->maxerrold / maxerr));
  else dtnew = dttmp;
  if (maxerr < 1.0) {
    dtnew = std::min(dtnew, 4. * dtold_);
    if (dtnew < dtold_) h->dtcause = FGPU_DTCAUSE_SMALLERR;
  } else {
    if (dtnew > dtold_) dtnew = dttmp;
    dtnew = std::max(dtnew, 0.25 * dtold_);
  }
  h->maxerrold = maxerr;
  return dtnew;
}

// One attempt of the adaptive modified Euler scheme (timedisc_modeuler.f90:125-195,
// tol_rel < 1).  At an attempt's start cvar = cold = base and rhs = k1:
//   s1 = update(eta1, base, base, k1)                     (pointwise)
//   order 3: s2 = update(eta2, base, s1, rhs(s1)), low = update(1/2, base, s1, rhs(s1))
//            P  = update(eta3, base, s2, rhs(s2)),  err = ComputeError(P, low)
//   order 2: P  = update(eta2, base, s1, rhs(s1)),  err = ComputeError(P, s1)
const double* fargo_wn(const fgpu_handle* h);
double* bt_cvar(const fgpu_handle* h);

int modeuler_attempt(fgpu_handle* h, double t, double dtv, double& err) {
  // timedisc_modeuler.f90:125-195 with tol_rel < 1: cvar -> ctmp (stage 1), the RHS of ctmp,
  // cvar and the embedded solution from it, the RHS of cvar, cvar (stage 3); with FARGO each
  // ComputeRHS frames its state vector in place (AddBackgroundVelocity only once the vector
  // carries the frame flag) and the updates read the framed vectors
  double* P = h->buf[0];
  double* base = h->buf[1];      // cold
  double* cv = bt_cvar(h);       // cvar (cold itself without FARGO)
  double* K1 = h->buf[2];
  double* S1 = h->buf[3];
  double* S2 = h->buf[4];
  double* LO = h->buf[5];
  const int ord = h->order;
  h->stats.attempts += 1;
  {
    const long long n = (long long)h->V * h->g.n;
    unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 148 * 8);
    const double e1 = kEta[ord - 1][0];
    int rc = timed_launch(h, 0, 0.0, [&] {
      shu_osher_update_kernel<<<blocks, 256, 0, h->stream>>>(base, cv, K1, S1, n, e1, dtv, nullptr, nullptr, 0);
      CUDA_TRY(h, cudaGetLastError());
      return FGPU_OK;
    });
    if (rc) return rc;
  }
  for (int n = 2; n <= ord; ++n) {
    StageArgs A = base_args(h);
    A.in = plain_state(n == 2 ? S1 : S2, false);
    if (h->fargo) {
      // n = 2 reads ctmp (its own frame flag), n = 3 cvar
      const Chain pre = (n == 2 && h->fargo_tmp_fresh) ? chain_none() : chain_add(chain_none(), fargo_wn(h), 1.0);
      A.in.pre = pre;
      A.w_sub = fargo_wn(h);
      A.yn_chain = chain_add(pre, fargo_wn(h), -1.0);
      // order 2 compares with ctmp itself, which this stage's ComputeRHS framed
      if (n == ord && ord == 2) A.err_chain = A.yn_chain;
      if (n == 2) h->fargo_tmp_fresh = false;
    }
    A.out_mode = OUT_SSPRK;
    A.eta = kEta[ord - 1][n - 1];
    A.y0 = base;
    A.dt = dtv;
    if (n == ord) {
      A.out = P;
      A.err_low = ord == 3 ? LO : S1;
    } else {
      A.out = S2;
      A.out2 = LO;
      A.eta2 = kEta[1][1];   // the second-order solution from the same RHS
    }
    if (int rc = launch_stage(h, A, RhsTime::host(t + kZeta[ord - 1][n - 2] * dtv))) return rc;
  }
  if (int rc = read_ctl(h)) return rc;
  double e;
  std::memcpy(&e, &h->h_ctl->err, 8);
  h->h_ctl->err = 0ULL;
  CUDA_TRY(h, cudaMemsetAsync(&h->d_ctl->err, 0, sizeof(unsigned long long), h->stream));
  err = e;
  return FGPU_OK;
}

// FARGO with a Butcher scheme: the background velocity of the step (w_new for type 1) and the
// attempt base cvar, which differs from cold once a ComputeRHS has framed it (the spare
// formed-state buffer; cold stays in buf[1])
const double* fargo_wn(const fgpu_handle* h) { return h->cfg.fargo_method == 1 ? h->d_w + h->nw : h->d_w; }
double* bt_cvar(const fgpu_handle* h) { return h->fargo ? h->buf[2 + h->T.m] : h->buf[1]; }

int launch_fargo_chain_copy(fgpu_handle* h, const double* in, double* out, const Chain& C, int gate = 0) {
  const unsigned blocks = (unsigned)std::min<long long>((h->g.n + 255) / 256, 148 * 8);
  const Ctl* ctl = gate ? h->d_ctl : nullptr;
  return timed_launch(h, false, 0.0, [&] {
    switch (h->V) {
      case 3: fargo_chain_copy_kernel<3><<<blocks, 256, 0, h->stream>>>(in, out, h->g, C, ctl, gate); break;
      default: fargo_chain_copy_kernel<4><<<blocks, 256, 0, h->stream>>>(in, out, h->g, C, ctl, gate); break;
    }
    CUDA_TRY(h, cudaGetLastError());
    return FGPU_OK;
  });
}

// ComputeRHS of a FARGO state vector into k1 (timedisc_base.f90:1096-1121,1190-1208): in gets
// AddBackgroundVelocity (pre) before the boundary fill and SubtractBackgroundVelocity(w) after
// the sources; cvar after the call (co-moving) goes to out_base
int enqueue_k1_fargo(fgpu_handle* h, const double* in, const Chain& pre, bool rt, int checkdata, double* out_base,
                     double t, bool check = false) {
  StageArgs A = base_args(h);
  A.out_mode = OUT_RHS;
  A.out = h->buf[2];
  A.in = plain_state(in, rt);
  A.in.pre = pre;
  A.w_sub = fargo_wn(h);
  A.out_base = out_base;
  A.checkdata = checkdata;
  if (check && checkdata) A.cfl_mode = 3;
  return launch_stage(h, A, RhsTime::host(t));
}

// CheckData of AcceptSolution's ComputeRHS inside a step: a failure breaks the step's loop
// before the next attempt (timedisc_base.f90:676,926-931)
int read_substep_check(fgpu_handle* h) {
  if (!h->cfg.checkdata) return FGPU_OK;
  if (int rc = read_ctl(h)) return rc;
  if (h->h_ctl->flags) {
    h->checkflags |= h->h_ctl->flags;
    h->brk = true;
    h->h_ctl->flags = 0;
    CUDA_TRY(h, cudaMemsetAsync(&h->d_ctl->flags, 0, sizeof(int), h->stream));
  }
  return FGPU_OK;
}

int butcher_attempt(fgpu_handle* h, double t, double dtv, double& err) {
  if (h->adaptive_me) return modeuler_attempt(h, t, dtv, err);
  const Tableau& T = h->T;
  double* P = h->buf[0];
  double* base = bt_cvar(h);
  h->stats.attempts += 1;
  for (int m = 2; m <= T.m; ++m) {
    StageArgs A = base_args(h);
    A.in.base = base;
    A.in.nk = m - 1;
    A.in.roundtrip = 0;
    for (int q = 0; q < m - 1; ++q) {
      A.in.K[q] = h->buf[2 + q];
      A.in.coef[q] = T.A[(m - 1) * T.m + q] * dtv;
    }
    if (h->fargo) {
      // ComputeRHS(ptmp, ctmp): AddBackgroundVelocity(w) acts only once the stage vectors carry
      // the frame flag, i.e. not on the first ComputeRHS of the run (physics_eulerisotherm.f90:
      // 1279-1299); SubtractBackgroundVelocity(w) always
      A.in.pre = h->fargo_tmp_fresh ? chain_none() : chain_add(chain_none(), fargo_wn(h), 1.0);
      A.w_sub = fargo_wn(h);
      h->fargo_tmp_fresh = false;
    }
    if (h->materialize) {
      // the stage state's reconstruction variables once per cell, read by the stencil
      // (formed by the previous stage's kernel when fuse_form, else by form_kernel)
      double* R = stage_rbuf(h, m);
      StateRef S = A.in;
      if (m == 2 || !h->fuse_form)
        if (int rc = timed_launch(h, 2, 0.0, [&] { return launch_form(h, S, R); })) return rc;
      A.rin = plain_state(R, false);
      A.rin.ready = h->prim ? 1 : 0;
    }
    A.out_mode = OUT_RHS;
    A.out = h->buf[2 + m - 1];
    set_fnext(h, A, m, dtv, nullptr);
    const bool fused_end = m == T.m && (!h->materialize || h->fuse_end);
    if (fused_end) set_last_stage(h, A, P, dtv);
    // timedisc_rkfehlberg.f90:195: ComputeRHS at t + c(m)*dt
    if (int rc = launch_stage(h, A, RhsTime::host(t + T.c[m - 1] * dtv))) return rc;
    if (m == T.m && !fused_end) {
      // the high/low combination and error norm as a streaming pass (the stencil kernel
      // keeps its registers for the stencil)
      CombineArgs Cb;
      std::memset(&Cb, 0, sizeof(Cb));
      Cb.base = base;
      for (int q = 0; q < T.m; ++q) {
        Cb.K[q] = h->buf[2 + q];
        Cb.bh_dt[q] = T.bh[q] * dtv;
        Cb.bl_dt[q] = T.bl[q] * dtv;
      }
      Cb.nstage = T.m;
      Cb.out_high = P;
      Cb.tol_rel = h->tol_rel;
      for (int v = 0; v < FGPU_MAXV; ++v) Cb.tol_abs[v] = h->tol_abs[v];
      Cb.n = h->g.n;
      Cb.ctl = h->d_ctl;
      const unsigned blocks = (unsigned)std::min<long long>((h->g.n + 255) / 256, 148 * 8);
      // algorithmic bytes: the new state written (base and k reads are counted with the stage)
      int rc = timed_launch(h, 2, (double)h->V * h->g.n * 8.0, [&] {
        switch (h->V) {
          case 3: combine_kernel<3><<<blocks, 256, 0, h->stream>>>(Cb); break;
          case 4: combine_kernel<4><<<blocks, 256, 0, h->stream>>>(Cb); break;
          default: combine_kernel<5><<<blocks, 256, 0, h->stream>>>(Cb); break;
        }
        CUDA_TRY(h, cudaGetLastError());
        return FGPU_OK;
      });
      if (rc) return rc;
    }
  }
  if (int rc = read_ctl(h)) return rc;
  double e;
  std::memcpy(&e, &h->h_ctl->err, 8);
  h->h_ctl->err = 0ULL;
  CUDA_TRY(h, cudaMemsetAsync(&h->d_ctl->err, 0, sizeof(unsigned long long), h->stream));
  err = e;
  return FGPU_OK;
}

int finish_cfl_host(fgpu_handle* h, const double* state, bool roundtrip, double& dtcfl, int checkdata, int& cause,
                    bool interior = false) {
  BndArgs B = bnd_args(h, state, roundtrip, FIN_NONE);
  B.checkdata = checkdata;
  if (h->fargo) { B.in.pre = fargo_pre(h); B.w_sub = h->d_w; }
  // interior cells too (the stage kernels' CFL epilogue sees the real frame only)
  if (interior)
    if (int rc = launch_misc(h, 1, B)) return rc;
  if (int rc = launch_misc(h, 0, B)) return rc;
  if (int rc = launch_visc_cfl(h, plain_state(state, roundtrip), roundtrip, RhsTime::host(h->time))) return rc;
  if (int rc = read_ctl(h)) return rc;
  dtcfl = ctl_dt(h, &cause);
  h->checkflags |= h->h_ctl->flags;
  if (h->h_ctl->flags) h->brk = true;
  h->h_ctl->flags = 0;
  h->h_ctl->invdt[0] = h->h_ctl->invdt[1] = h->h_ctl->invdt[2] = h->h_ctl->invdt[3] = 0ULL;
  CUDA_TRY(h, cudaMemsetAsync(h->d_ctl, 0, sizeof(unsigned long long) * 4, h->stream));
  CUDA_TRY(h, cudaMemsetAsync(&h->d_ctl->flags, 0, sizeof(int), h->stream));
  return FGPU_OK;
}

int butcher_integration_step(fgpu_handle* h) {
  // timedisc_base.f90:649-750 IntegrationStep
  if (h->fargo) {
    // CalcBackgroundVelocity (type 1: w_new from the real-frame state of the last ComputeRHS)
    // adds w to cvar, SubtractBackgroundVelocity(w_new) takes it to the new co-moving frame;
    // cold is not touched (timedisc_base.f90:661-674)
    double* W = h->d_w;
    const double* Wn = fargo_wn(h);
    if (h->cfg.fargo_method == 1) {
      StateRef S = plain_state(h->buf[0], false);
      S.pre = fargo_pre(h);
      if (int rc = launch_fargo_w(h, S, W, h->d_w + h->nw)) return rc;
      if (int rc = launch_fargo_chain_copy(h, h->buf[1], bt_cvar(h), chain_add(chain_add(chain_none(), W, 1.0), Wn, -1.0)))
        return rc;
    } else {
      CUDA_TRY(h, cudaMemcpyAsync(bt_cvar(h), h->buf[1], sizeof(double) * h->V * h->g.n, cudaMemcpyDeviceToDevice,
                                  h->stream));
    }
  }
  double t = h->time, d = h->dt;
  if (d < h->dtmin && h->dtcause != FGPU_DTCAUSE_FILEIO) h->dtmin = d;
  double dtold_ = 0.0;
  bool rhs_done_at_t = false;   // AcceptSolution already evaluated ComputeRHS(checkdatabm)
  while (!h->brk && t + d <= h->time + h->dt) {
    dtold_ = d;
    double e = 0.0;
    if (int rc = butcher_attempt(h, t, d, e)) return rc;
    h->last_err = e;
    d = adjust_timestep(h, e, d);
    rhs_done_at_t = false;
    if (e != e) h->brk = true;
    else if (e > DBL_MAX) h->brk = true;
    else if (e >= 1.0) {   // RejectSolution: cvar = cold, RHS with CHECK_NOTHING
      if (h->fargo) {
        // the RHS frames cvar (cold + w_new - w_new), cold keeps its data
        const Chain pre = chain_add(chain_none(), fargo_wn(h), 1.0);
        if (int rc = enqueue_k1_fargo(h, h->buf[1], pre, false, FGPU_CHECK_NOTHING, bt_cvar(h), t)) return rc;
      } else if (int rc = enqueue_k1(h, false, false, false, h->cfg.checkdata, t)) {
        return rc;
      }
      h->n_adj++;
      h->dtcause = FGPU_DTCAUSE_ERRADJ;
      if (d < h->dtmin) h->dtmin = d;
    } else {               // AcceptSolution
      t = t + dtold_;
      if (t < h->time + h->dt) {
        if (h->fargo) {
          // cold = cvar = the accepted state framed by this ComputeRHS
          const Chain pre = chain_add(chain_none(), fargo_wn(h), 1.0);
          if (int rc = enqueue_k1_fargo(h, h->buf[0], pre, h->roundtrip_cfg, h->cfg.checkdata, h->buf[1], t, true))
            return rc;
          CUDA_TRY(h, cudaMemcpyAsync(bt_cvar(h), h->buf[1], sizeof(double) * h->V * h->g.n, cudaMemcpyDeviceToDevice,
                                      h->stream));
        } else if (int rc = enqueue_k1(h, true, false, h->roundtrip_cfg, h->cfg.checkdata, t)) {
          return rc;
        }
        if (int rc = read_substep_check(h)) return rc;
        // on a break the stored state is the accepted solution; with this ComputeRHS's round
        // trip it gives cvar and pvar as fosite leaves them
        if (h->brk) h->pre_rt = h->roundtrip_cfg;
        rhs_done_at_t = true;
      }
      h->iter++;
      h->stats.cell_updates += h->g.n;
    }
    if (d < h->dtlimit) h->brk = true;
  }
  if (!h->brk && h->fargo) {
    const double dt_step = t - h->time;
    h->dt = dt_step;
    h->time = t;
    h->dtold = d;
    // CenterBoundary + FargoAdvection of cvar (the accepted state, or its framed copy in cold
    // when AcceptSolution already evaluated the RHS), Convert2Primitive and the closing
    // ComputeRHS (timedisc_base.f90:727-744); the advection pass also reduces the interior
    // CFL (co-moving) and CheckData (real frame) of the closing ComputeRHS
    const double* Wn = fargo_wn(h);
    double* src = rhs_done_at_t ? h->buf[1] : h->buf[0];
    double* dst = rhs_done_at_t ? h->buf[0] : bt_cvar(h);   // then copied into P (fixed buffers)
    FargoAdvArgs X;
    std::memset(&X, 0, sizeof(X));
    X.g = h->g; X.ph = h->ph; X.mt = h->mt;
    X.in = plain_state(src, false);
    X.w = Wn;
    X.out = dst;
    X.ctl = h->d_ctl;
    X.checkdata = h->cfg.checkdata;
    X.chunk = 8;
    X.dt_host = dt_step;
    if (int rc = launch_fargo_advect_args(h, X)) return rc;
    if (!rhs_done_at_t)
      CUDA_TRY(h, cudaMemcpyAsync(h->buf[0], dst, sizeof(double) * h->V * h->g.n, cudaMemcpyDeviceToDevice, h->stream));
    const Chain pre = chain_add(chain_none(), Wn, 1.0);
    if (int rc = enqueue_k1_fargo(h, h->buf[0], pre, false, h->cfg.checkdata, h->buf[1], h->time)) return rc;
    if (h->cfg.fargo_method == 1)
      CUDA_TRY(h, cudaMemcpyAsync(h->d_w, Wn, sizeof(double) * h->nw, cudaMemcpyDeviceToDevice, h->stream));
    h->fargo_phase = 2;
    h->pre_rt = false;
    return FGPU_OK;
  }
  if (!h->brk) {
    h->dt = t - h->time;
    h->time = t;
    h->dtold = d;
    if (rhs_done_at_t) {
      // the state in base already went through one CHECK_ALL ComputeRHS; fosite applies a second one
      CUDA_TRY(h, cudaMemcpyAsync(h->buf[0], h->buf[1], sizeof(double) * h->V * h->g.n, cudaMemcpyDeviceToDevice,
                                  h->stream));
    }
    if (int rc = enqueue_k1(h, true, true, h->roundtrip_cfg, h->cfg.checkdata, h->time)) return rc;
    h->pre_rt = h->roundtrip_cfg;
  }
  return FGPU_OK;
}

int validate(fgpu_handle* h) {
  const fgpu_config& c = h->cfg;
  if (c.inum < 2 || c.jnum < 2 || c.knum < 1)
    return set_err(h, FGPU_EUNSUPPORTED, "meshes must be 2D (x-y) or 3D; 1D and collapsed-x/y meshes are not supported");
  h->nd = c.knum > 1 ? 3 : 2;
  if (c.physics != FGPU_EULER && c.physics != FGPU_EULER_ISOTHERM) return set_err(h, FGPU_EBADCFG, "unknown physics");
  h->euler = c.physics == FGPU_EULER;
  h->V = 1 + h->nd + (h->euler ? 1 : 0);
  if (c.geometry != FGPU_CARTESIAN && c.geometry != FGPU_CYLINDRICAL && c.geometry != FGPU_LOGCYLINDRICAL)
    return set_err(h, FGPU_EUNSUPPORTED, "geometry not supported (cartesian, cylindrical, logcylindrical)");
  if (c.fluxtype != FGPU_KT) return set_err(h, FGPU_EBADCFG, "only KT fluxes exist");
  if (c.order != FGPU_CONSTANT && c.order != FGPU_LINEAR) return set_err(h, FGPU_EBADCFG, "reconstruction order must be CONSTANT or LINEAR");
  if (c.order == FGPU_LINEAR && (c.limiter < 1 || c.limiter > 8)) return set_err(h, FGPU_EBADCFG, "Unknown limiter");
  if (c.order == FGPU_LINEAR && c.limiter == FGPU_PP) return set_err(h, FGPU_EUNSUPPORTED, "PP limiter currently not supported.");
  h->prim = c.variables == FGPU_PRIMITIVE;
  for (int f = 0; f < 6; ++f) {
    if (h->nd == 2 && f >= 4) continue;
    int t = c.bc[f];
    if (t != FGPU_PERIODIC && t != FGPU_REFLECTING && t != FGPU_ABSORBING && t != FGPU_NO_GRADIENTS &&
        t != FGPU_AXIS)
      return set_err(h, FGPU_EUNSUPPORTED, "boundary condition not supported (periodic, reflecting, axis, absorbing, no_gradients)");
  }
  for (int d = 0; d < h->nd; ++d)
    if ((c.bc[2 * d] == FGPU_PERIODIC) != (c.bc[2 * d + 1] == FGPU_PERIODIC))
      return set_err(h, FGPU_EBADCFG, "periodic boundaries must be paired");
  h->curv = c.geometry != FGPU_CARTESIAN;
  if (c.pointmass) {
    if (c.geometry == FGPU_CARTESIAN || h->nd != 2)
      return set_err(h, FGPU_EUNSUPPORTED, "point mass supported on 2D cylindrical/logcylindrical meshes");
    h->has_accel = true;
  }
  if (!h->euler && c.csiso < 0.0) return set_err(h, FGPU_EBADCFG, "negative isothermal sound speed");
  // timedisc
  h->tol_rel = c.tol_rel; h->beta = c.beta; h->cfl = c.cfl; h->stoptime = c.stoptime;
  h->dtlimit = c.dtlimit > 0 ? c.dtlimit : DBL_EPSILON * c.stoptime;
  h->tout = c.tout > 0 ? c.tout : c.stoptime;
  for (int v = 0; v < FGPU_MAXVAR; ++v) h->tol_abs[v] = c.tol_abs[v];
  if (c.method == FGPU_MODIFIED_EULER) {
    h->butcher = false;
    h->order = c.tdorder ? c.tdorder : 3;
    if (h->order < 1 || h->order > 3) return set_err(h, FGPU_EBADCFG, "time order must be one of 1,2,3");
    if (h->order == 1) { h->tol_rel = 10.0; for (int v = 0; v < FGPU_MAXVAR; ++v) h->tol_abs[v] = 1.0; }
    if (h->tol_rel < 1.0) {
      // embedded error control (timedisc_modeuler.f90:163-192): the host-controlled attempt
      // engine of the Butcher schemes with Shu-Osher attempts; buffers P, base, k1, the
      // stage-1 state, the stage-2 state, the embedded solution and one spare
      h->butcher = true;
      h->adaptive_me = true;
      h->T.m = 4;
      h->T.order = h->order;
    }
  } else {
    h->butcher = true;
    int ord = c.tdorder ? c.tdorder : 5;
    if (!make_tableau(c.method, ord, h->T)) return set_err(h, FGPU_EBADCFG, "unknown timedisc method/order");
    h->order = ord;
    if (h->tol_rel > 1.0) return set_err(h, FGPU_EUNSUPPORTED, "embedded RK with disabled step control is not supported");
  }
  if (c.tol_rel < 0.0) return set_err(h, FGPU_EBADCFG, "error tolerance levels must be greater than 0");
  if (c.stoptime <= 0.0) return set_err(h, FGPU_EBADCFG, "stoptime must be positive");
  if (c.tmin > 1.e-10 && (c.checkdata & FGPU_CHECK_TMIN) && h->euler)
    return set_err(h, FGPU_EUNSUPPORTED, "CHECK_TMIN with tmin > 1e-10 is not supported");
  h->roundtrip_cfg = h->euler && (c.checkdata & FGPU_CHECK_PMIN);
  if (c.pm_outbound != 0) {
    if (!c.pointmass) return set_err(h, FGPU_EBADCFG, "accretion needs the point mass");
    if (c.pm_outbound != 1 && c.pm_outbound != 2)
      return set_err(h, FGPU_EUNSUPPORTED, "accretion through the x boundaries only (outbound 1 or 2)");
    if (h->butcher) return set_err(h, FGPU_EUNSUPPORTED, "accretion with the fixed-step modified Euler scheme only");
    h->accrete = true;
    h->acc_face = c.pm_outbound - 1;
  }
  if (c.fargo_method != 0) {
    if (c.fargo_method != 1 && c.fargo_method != 2)
      return set_err(h, FGPU_EUNSUPPORTED, "fargo: types 1 (computed) and 2 (user-supplied) background velocity only; "
                                           "type 3 needs the shearing-box sources");
    if (c.fargo_direction != 1 && c.fargo_direction != 2)
      return set_err(h, FGPU_EUNSUPPORTED, "fargo: transport along x (direction 1) or y (direction 2) only");
    if (h->nd != 2) return set_err(h, FGPU_EUNSUPPORTED, "fargo: 2D x-y meshes only");
    if (c.fargo_direction == 1 && h->accrete)
      return set_err(h, FGPU_EUNSUPPORTED, "fargo along x with point-mass accretion through the x boundaries");
    h->fdir = c.fargo_direction;
    if (h->roundtrip_cfg)
      return set_err(h, FGPU_EUNSUPPORTED, "fargo with ideal-gas physics: checkdata without CHECK_PMIN "
                                           "(its round trip sits between the frame changes)");
    h->fargo = true;
  }
  if (c.vismodel != 0) {
    // sources_viscosity.f90:132-266
    if (c.vismodel < FGPU_VIS_MOLECULAR || c.vismodel > FGPU_VIS_ALPHA_ALT)
      return set_err(h, FGPU_EBADCFG, "Viscosity prescription not supported.");
    if (c.vismodel == FGPU_VIS_ALPHA_ALT)
      return set_err(h, FGPU_EUNSUPPORTED, "alternative alpha-viscosity currently not supported");
    if (c.vismodel == FGPU_VIS_ALPHA && h->euler)
      return set_err(h, FGPU_EUNSUPPORTED, "viscosity: ALPHA with isothermal physics only");
    if (c.vismodel != FGPU_VIS_MOLECULAR && c.fargo_method != 0)
      return set_err(h, FGPU_EUNSUPPORTED, "viscosity: ALPHA/BETA/POWERLAW without fargo");
    h->vis = true;
    h->vis_model = c.vismodel;
    h->vis_power = c.vis_exponent;
    h->vis_eta = c.dynconst;
    h->vis_mub = std::isnan(c.bulkconst) ? -2. / 3. * c.dynconst : c.bulkconst;
    h->cvis = c.cvis;
  }
  return FGPU_OK;
}

}  // namespace

// ======================================================================= C ABI
// The grid reads the whole array `passes` times (grid-stride, 16-byte loads that bypass L1, so
// every pass comes from L2); the sums go to out only if they are non-zero (the array holds
// zeros), which keeps the loads without writing.
__global__ void __launch_bounds__(512) l2_read_probe_kernel(const double2* __restrict__ a, size_t n2, int passes,
                                                            double* out) {
  double s0 = 0.0, s1 = 0.0;
  const size_t stride = (size_t)gridDim.x * 512;
  for (int p = 0; p < passes; ++p)
#pragma unroll 4
    for (size_t q = (size_t)blockIdx.x * 512 + threadIdx.x; q < n2; q += stride) {
      const double2 v = __ldcg(a + q);
      s0 += v.x;
      s1 += v.y;
    }
  if (s0 + s1 != 0.0) out[threadIdx.x] = s0 + s1;
}

extern "C" {

void fgpu_config_init(fgpu_config* c) {
  std::memset(c, 0, sizeof(*c));
  c->inum = c->jnum = c->knum = 1;
  c->geometry = FGPU_CARTESIAN;
  c->gparam = 1.0;
  c->physics = FGPU_EULER;
  c->gamma = 1.4;
  c->gn = 1.0;
  c->fluxtype = FGPU_KT;
  c->order = FGPU_LINEAR;
  c->variables = FGPU_CONSERVATIVE;
  c->limiter = FGPU_MINMOD;
  c->theta = 1.0;
  for (int f = 0; f < 6; ++f) c->bc[f] = FGPU_PERIODIC;
  c->method = FGPU_MODIFIED_EULER;
  c->cfl = 0.4;
  c->stoptime = 1.0;
  c->tol_rel = 0.01;
  c->beta = 0.08;
  for (int v = 0; v < FGPU_MAXVAR; ++v) c->tol_abs[v] = 0.001;
  c->checkdata = FGPU_CHECK_ALL;
  c->pmin = c->rhomin = c->tmin = DBL_MIN;
  c->pm_mass = 1.0;
  // sources_viscosity.f90:150-166
  c->dynconst = 0.1;
  c->bulkconst = std::nan("");
  c->cvis = 0.5;
}

int fgpu_create(const fgpu_config* cfg, int device, fgpu_handle** out) {
  if (!cfg || !out) return set_err(nullptr, FGPU_EARG, "null argument");
  *out = nullptr;
  fgpu_handle* h = new fgpu_handle();
  std::memset(&h->stats, 0, sizeof(h->stats));
  h->cfg = *cfg;
  int rc = validate(h);
  if (!rc) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) rc = set_err(h, FGPU_ECUDA, "no CUDA device");
  }
  if (!rc) {
    if (device >= 0) { if (cudaSetDevice(device) != cudaSuccess) rc = set_err(h, FGPU_ECUDA, "cudaSetDevice failed"); }
    cudaGetDevice(&h->device);
  }
  if (!rc) {
    // FGPU_STAGE_VARIANT / FGPU_KCHUNK force a stage-kernel layout and z chunk (the tuner's choice otherwise)
    if (const char* e = std::getenv("FGPU_STAGE_VARIANT")) h->variant = std::max(0, std::min(7, std::atoi(e)));
    if (const char* e = std::getenv("FGPU_KCHUNK")) { int v = std::atoi(e); if (v > 0) h->kchunk = v; }
    if (const char* e = std::getenv("FGPU_MATERIALIZE")) h->materialize = std::atoi(e) != 0;
    if (const char* e = std::getenv("FGPU_FUSE_FORM")) h->fuse_form = std::atoi(e) != 0;
    if (const char* e = std::getenv("FGPU_FUSE_END")) h->fuse_end = std::atoi(e) != 0;
    // FGPU_FORM_SO=0 converts every staged point of the Shu-Osher stages instead
    h->so_form = true;
    if (const char* e = std::getenv("FGPU_FORM_SO")) h->so_form = std::atoi(e) != 0;
    // FARGO with a Butcher scheme: the stencil forms each stage state with its frame changes
    if (h->fargo && h->butcher) h->materialize = false;
    h->fuse_form = h->fuse_form && h->materialize;
  }
  if (!rc) configure_stage_kernels(h->nd, h->euler, h->prim);
  if (!rc && h->vis) configure_visc(h->nd, h->euler);
  if (!rc) rc = build_metric(h);
  if (!rc) {
    h->g.nx = cfg->inum; h->g.ny = cfg->jnum; h->g.nz = h->nd == 3 ? cfg->knum : 1;
    h->g.n = (long long)h->g.nx * h->g.ny * h->g.nz;
    for (int f = 0; f < 6; ++f) h->g.bc[f] = cfg->bc[f];
    h->g.fdir = h->fdir;
    h->ph.gamma = cfg->gamma; h->ph.gm1 = cfg->gamma - 1.; h->ph.pmin = cfg->pmin; h->ph.rhomin = cfg->rhomin;
    h->ph.tiny2 = 2.0 * DBL_MIN;
    h->ph.inv_gm1 = 1.0 / h->ph.gm1;
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) rc = set_err(h, FGPU_ECUDA, "stream");
  }
  if (!rc) rc = upload_metric(h);
  if (!rc) {
    // Butcher: P, base, k1..km, formed stage state(s)
    int nbuf = h->butcher ? 2 + h->T.m + 1 + (h->fuse_form ? 1 : 0) : 3;
    size_t bytes = sizeof(double) * h->V * h->g.n;
    for (int b = 0; b < nbuf && !rc; ++b) {
      double* p = nullptr;
      cudaError_t e = cudaMalloc(&p, bytes);
      if (e != cudaSuccess) { rc = set_err(h, FGPU_ENOMEM, "device memory for state arrays"); break; }
      cudaMemsetAsync(p, 0, bytes, h->stream);
      h->buf.push_back(p);
    }
  }
  // the primitive forms of the Shu-Osher stage results (fixed step, primitive reconstruction,
  // no frame changes, accretion rows or viscous source between the stages)
  h->so_form = h->so_form && h->prim && !h->butcher && !h->adaptive_me && !h->fargo && !h->accrete && !h->vis &&
               h->order >= 2;
  for (int b = 0; b < (h->order >= 3 ? 2 : 1) && !rc && h->so_form; ++b) {
    size_t bytes = sizeof(double) * h->V * h->g.n;
    if (cudaMalloc(&h->d_pform[b], bytes) != cudaSuccess) rc = set_err(h, FGPU_ENOMEM, "device memory for state arrays");
    else cudaMemsetAsync(h->d_pform[b], 0, bytes, h->stream);
  }
  if (!rc && h->accrete) {
    size_t na = 3 * (size_t)h->g.ny + 2;
    if (cudaMalloc(&h->d_acc, sizeof(double) * na) != cudaSuccess) rc = set_err(h, FGPU_ENOMEM, "accretion arrays");
    else {
      std::vector<double> a(na, 0.0);
      a[3 * (size_t)h->g.ny] = cfg->pm_mass;
      cudaMemcpy(h->d_acc, a.data(), sizeof(double) * na, cudaMemcpyHostToDevice);
    }
  }
  if (!rc && h->vis) {
    size_t bytes = sizeof(double) * (h->nd + (h->euler ? 1 : 0)) * h->g.n;
    if (cudaMalloc(&h->d_visc, bytes) != cudaSuccess) rc = set_err(h, FGPU_ENOMEM, "viscous source array");
    else cudaMemsetAsync(h->d_visc, 0, bytes, h->stream);
    if (!rc && h->vis_model != FGPU_VIS_MOLECULAR) rc = upload_visc_geometry(h);
  }
  if (!rc && h->fargo) {
    h->nw = h->fdir == 1 ? h->g.ny + 4 : h->nxp;
    if (cudaMalloc(&h->d_w, sizeof(double) * 3 * h->nw) != cudaSuccess ||
        (h->fdir != 1 && cudaMalloc(&h->d_fw_terms, sizeof(double) * (size_t)h->nxp * h->g.ny) != cudaSuccess))
      rc = set_err(h, FGPU_ENOMEM, "fargo arrays");
    else cudaMemsetAsync(h->d_w, 0, sizeof(double) * 3 * h->nw, h->stream);
    if (!rc && h->fdir == 1) {
      // wfactor(j) (timedisc_base.f90:435-441): the narrowest x-width of the first interior
      // column over its S/N and B/T faces relative to the width through the centre; those
      // faces share the centre's x, and the scale factors depend on x only
      const fgpu_config& c = h->cfg;
      const double x = c.xmin + ((double)(2 * 1 - 1) * 0.5) * ((c.xmax - c.xmin) / c.inum);
      double hxc, hyc, hzc;
      scale(c.geometry, c.gparam, x, hxc, hyc, hzc);
      auto mn = [](double a, double b) { return b < a ? b : a; };
      std::vector<double> wf((size_t)h->nw, mn(mn(hxc, hxc), mn(hxc, hxc)) / hxc);
      // on the handle's stream, after its memset (a pageable source is staged before the call returns)
      if (cudaMemcpyAsync(h->d_w + 2 * (size_t)h->nw, wf.data(), sizeof(double) * wf.size(), cudaMemcpyHostToDevice,
                          h->stream) != cudaSuccess)
        rc = set_err(h, FGPU_ECUDA, "fargo wfactor upload");
    }
  }
  if (!rc) {
    if (cudaMalloc(&h->d_ctl, sizeof(Ctl)) != cudaSuccess) rc = set_err(h, FGPU_ENOMEM, "control block");
    else if (cudaMallocHost(&h->h_ctl, sizeof(Ctl)) != cudaSuccess) rc = set_err(h, FGPU_ENOMEM, "pinned control block");
  }
  if (!rc) {
    std::memset(h->h_ctl, 0, sizeof(Ctl));
    h->h_ctl->stoptime = h->stoptime; h->h_ctl->tout = h->tout; h->h_ctl->cfl = h->cfl;
    h->h_ctl->dtlimit = h->dtlimit; h->h_ctl->dt = h->stoptime; h->h_ctl->dtmin = h->stoptime;
    h->h_ctl->iter = -1;
    h->h_ctl->vis = h->vis ? 1 : 0; h->h_ctl->cvis = h->cvis;
    rc = write_ctl(h);
    h->dt = h->stoptime; h->dtold = h->dt; h->dtmin = h->dt;
  }
  if (!rc) {
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) rc = set_err(h, FGPU_ECUDA, cudaGetErrorString(e));
  }
  if (rc) { g_create_error = h->err; fgpu_destroy(h); return rc; }
  *out = h;
  return FGPU_OK;
}

void fgpu_destroy(fgpu_handle* h) {
  if (!h) return;
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->graph) cudaGraphExecDestroy(h->graph);
  if (h->bt_graph) cudaGraphExecDestroy(h->bt_graph);
  for (double* p : h->buf) cudaFree(p);
  for (double* p : h->d_pform) if (p) cudaFree(p);
  if (h->d_pad) cudaFree(h->d_pad);
  if (h->d_flux) cudaFree(h->d_flux);
  if (h->d_metric) cudaFree(h->d_metric);
  if (h->d_w) cudaFree(h->d_w);
  if (h->d_fw_terms) cudaFree(h->d_fw_terms);
  if (h->d_acc) cudaFree(h->d_acc);
  if (h->d_visc) cudaFree(h->d_visc);
  if (h->d_dynvis) cudaFree(h->d_dynvis);
  if (h->d_ephir) cudaFree(h->d_ephir);
  if (h->d_visrad) cudaFree(h->d_visrad);
  if (h->d_vistime) cudaFree(h->d_vistime);
  if (h->d_ctl) cudaFree(h->d_ctl);
  if (h->h_ctl) cudaFreeHost(h->h_ctl);
  if (h->own_stream) h->stream = h->own_stream;
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

int fgpu_last_error(const fgpu_handle* h, char* buf, int len) {
  const std::string& s = h ? h->err : g_create_error;
  if (buf && len > 0) {
    int n = std::min<int>((int)s.size(), len - 1);
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return (int)s.size();
}

int64_t fgpu_cell_count(const fgpu_handle* h) {
  return (int64_t)(h->g.nx + 4) * (h->g.ny + 4) * (h->nd == 3 ? h->g.nz + 4 : 1);
}
int64_t fgpu_state_size(const fgpu_handle* h) { return fgpu_cell_count(h) * h->V; }
int fgpu_vnum(const fgpu_handle* h) { return h->V; }

int fgpu_get_mesh(fgpu_handle* h, int which, double* out, int64_t n) {
  if (!h || !out) return FGPU_EARG;
  if (n < fgpu_cell_count(h)) return set_err(h, FGPU_EARG, "output too small");
  const fgpu_config& c = h->cfg;
  int NXp = h->g.nx + 4, NYp = h->g.ny + 4, NZp = h->nd == 3 ? h->g.nz + 4 : 1;
  double mdx = (c.xmax - c.xmin) / c.inum, mdy = (c.ymax - c.ymin) / c.jnum, mdz = (c.zmax - c.zmin) / c.knum;
  if (mdz < 2 * DBL_EPSILON && c.knum == 1) mdz = 0.0;
  for (int kp = 0; kp < NZp; ++kp)
    for (int jp = 0; jp < NYp; ++jp)
      for (int ip = 0; ip < NXp; ++ip) {
        int I = ip - 1, J = jp - 1, K = h->nd == 3 ? kp - 1 : 1;
        double x = c.xmin + ((double)(2 * I - 1) * 0.5) * mdx;
        double y = c.ymin + ((double)(2 * J - 1) * 0.5) * mdy;
        double z = c.zmin + ((double)(2 * K - 1) * 0.5) * mdz;
        double v;
        switch (which) {
          case FGPU_MESH_X: v = x; break;
          case FGPU_MESH_Y: v = y; break;
          case FGPU_MESH_Z: v = z; break;
          case FGPU_MESH_RADIUS:
            if (c.geometry == FGPU_LOGCYLINDRICAL) { double r = c.gparam * std::exp(x); v = std::sqrt(r * r + z * z); }
            else if (c.geometry == FGPU_CYLINDRICAL) v = std::sqrt(x * x + z * z);
            else v = std::sqrt(x * x + y * y + z * z);
            break;
          default: return set_err(h, FGPU_EARG, "unknown mesh array");
        }
        out[ip + (long long)NXp * (jp + (long long)NYp * kp)] = v;
      }
  return FGPU_OK;
}

int fgpu_set_sound_speeds(fgpu_handle* h, const double* bcc, int64_t nb, const double* fcs, int64_t nf) {
  if (!h) return FGPU_EARG;
  if (h->euler) return set_err(h, FGPU_EBADCFG, "sound speeds are computed for ideal-gas physics");
  long long nc = fgpu_cell_count(h);
  int nfaces = 2 * h->nd;
  if (nb < nc || nf < nc * nfaces) return set_err(h, FGPU_EARG, "sound speed arrays too small");
  int NXp = h->g.nx + 4, NYp = h->g.ny + 4, NZp = h->nd == 3 ? h->g.nz + 4 : 1;
  // the profiles must depend on the first coordinate only
  for (int q = 0; q <= nfaces; ++q) {
    const double* a = q == 0 ? bcc : fcs + (long long)(q - 1) * nc;
    for (int kp = 0; kp < NZp; ++kp)
      for (int jp = 0; jp < NYp; ++jp)
        for (int ip = 0; ip < NXp; ++ip) {
          double v = a[ip + (long long)NXp * (jp + (long long)NYp * kp)];
          double r = a[ip + (long long)NXp * (2 + (long long)NYp * (h->nd == 3 ? 2 : 0))];
          if (v != r) return set_err(h, FGPU_EUNSUPPORTED, "sound speed profiles that vary along y or z are not supported");
        }
  }
  int row = NXp * (2 + NYp * (h->nd == 3 ? 2 : 0));
  for (int ip = 0; ip < NXp; ++ip) {
    h->h_metric[(size_t)(M_cs0 + 0) * NXp + ip] = bcc[row + ip];
    for (int q = 0; q < nfaces; ++q) h->h_metric[(size_t)(M_cs0 + 1 + q) * NXp + ip] = fcs[(long long)q * nc + row + ip];
    if (h->nd == 2) {   // B/T profiles unused in 2D
      h->h_metric[(size_t)(M_cs0 + 5) * NXp + ip] = bcc[row + ip];
      h->h_metric[(size_t)(M_cs0 + 6) * NXp + ip] = bcc[row + ip];
    }
  }
  int rc = upload_metric(h);
  if (rc) return rc;
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return FGPU_OK;
}

int fgpu_upload_state(fgpu_handle* h, int which, const double* data, int64_t n) {
  if (!h || !data) return FGPU_EARG;
  if (n < fgpu_state_size(h)) return set_err(h, FGPU_EARG, "state array too small");
  if (which != FGPU_CVAR && which != FGPU_PVAR) return set_err(h, FGPU_EARG, "upload CVAR or PVAR");
  long long nc = fgpu_cell_count(h);
  if (!h->d_pad) CUDA_TRY(h, cudaMalloc(&h->d_pad, sizeof(double) * 2 * nc * h->V));
  CUDA_TRY(h, cudaMemcpyAsync(h->d_pad, data, sizeof(double) * nc * h->V, cudaMemcpyHostToDevice, h->stream));
  long long blocks = std::min<long long>((h->g.n + 255) / 256, 148 * 16);
  int prim = which == FGPU_PVAR;
  h->stats.launches += 1;
  if (h->nd == 2) {
    if (h->euler) unpack_kernel<2, true><<<(unsigned)blocks, 256, 0, h->stream>>>(h->d_pad, h->buf[0], h->g, nc, prim, h->ph);
    else unpack_kernel<2, false><<<(unsigned)blocks, 256, 0, h->stream>>>(h->d_pad, h->buf[0], h->g, nc, prim, h->ph);
  } else {
    if (h->euler) unpack_kernel<3, true><<<(unsigned)blocks, 256, 0, h->stream>>>(h->d_pad, h->buf[0], h->g, nc, prim, h->ph);
    else unpack_kernel<3, false><<<(unsigned)blocks, 256, 0, h->stream>>>(h->d_pad, h->buf[0], h->g, nc, prim, h->ph);
  }
  CUDA_TRY(h, cudaGetLastError());
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  h->pre_rt = false;
  // FARGO: after FirstStep an uploaded cvar is in the co-moving frame (what fgpu_download
  // returns); it takes the place of the transported state of the last step
  if (h->fargo && h->fargo_phase >= 1) h->fargo_phase = 2;
  return FGPU_OK;
}

int fgpu_download(fgpu_handle* h, int which, double* out, int64_t n) {
  if (!h || !out) return FGPU_EARG;
  long long nc = fgpu_cell_count(h);
  if (which == FGPU_RHS) {
    if (n < nc * h->V) return set_err(h, FGPU_EARG, "output too small");
    // the RHS of the last fgpu_compute_rhs lives in a stage scratch buffer
    const double* src = h->butcher ? h->buf[2 + h->T.m - 1] : h->buf[1];
    std::vector<double> tmp((size_t)h->V * h->g.n);
    CUDA_TRY(h, cudaMemcpyAsync(tmp.data(), src, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    std::memset(out, 0, sizeof(double) * nc * h->V);
    int NXp = h->g.nx + 4, NYp = h->g.ny + 4, kofs = h->nd == 3 ? 2 : 0;
    for (int l = 0; l < h->V; ++l)
      for (int k = 0; k < h->g.nz; ++k)
        for (int j = 0; j < h->g.ny; ++j)
          for (int i = 0; i < h->g.nx; ++i)
            out[(i + 2) + (long long)NXp * ((j + 2) + (long long)NYp * (k + kofs)) + nc * l] =
                tmp[i + (long long)h->g.nx * (j + (long long)h->g.ny * k) + h->g.n * l];
    return FGPU_OK;
  }
  if (which == FGPU_XFLUX || which == FGPU_YFLUX || which == FGPU_ZFLUX) {
    if (n < nc * h->V) return set_err(h, FGPU_EARG, "output too small");
    if (!h->flux_valid) return set_err(h, FGPU_EARG, "no fluxes: call fgpu_compute_rhs first");
    const int d = which - FGPU_XFLUX;
    if (d >= h->nd) return set_err(h, FGPU_EARG, "no such direction on this mesh");
    CUDA_TRY(h, cudaMemcpyAsync(out, h->d_flux + (size_t)d * h->V * nc, sizeof(double) * nc * h->V,
                                cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return FGPU_OK;
  }
  if (which == FGPU_BCCSOUND) {
    if (n < nc) return set_err(h, FGPU_EARG, "output too small");
    std::vector<double> pv((size_t)nc * h->V);
    int rc = fgpu_download(h, FGPU_PVAR, pv.data(), (int64_t)pv.size());
    if (rc) return rc;
    int NXp = h->g.nx + 4;
    for (long long x = 0; x < nc; ++x) {
      if (h->euler) out[x] = std::sqrt(std::max(2.0 * DBL_MIN, h->cfg.gamma * pv[x + nc * (h->V - 1)] / pv[x]));
      else out[x] = h->h_metric[(size_t)M_cs0 * NXp + (x % NXp)];
    }
    return FGPU_OK;
  }
  if (which != FGPU_CVAR && which != FGPU_PVAR) return set_err(h, FGPU_EARG, "unknown array");
  if (n < nc * h->V) return set_err(h, FGPU_EARG, "output too small");
  if (!h->d_pad) CUDA_TRY(h, cudaMalloc(&h->d_pad, sizeof(double) * 2 * nc * h->V));
  CUDA_TRY(h, cudaMemsetAsync(h->d_pad, 0, sizeof(double) * 2 * nc * h->V, h->stream));
  bool rt = h->pre_rt;
  BndArgs B = bnd_args(h, h->buf[0], rt, FIN_NONE);
  if (h->fargo) { B.in.pre = fargo_pre(h); B.w_sub = h->d_w; }
  B.ctl = nullptr;
  B.out_p = h->d_pad;
  B.out_c = h->d_pad + nc * h->V;
  B.npad = nc;
  if (int rc = launch_misc(h, 2, B)) return rc;
  if (int rc = launch_misc(h, 0, B)) return rc;
  CUDA_TRY(h, cudaMemcpyAsync(out, which == FGPU_PVAR ? B.out_p : B.out_c, sizeof(double) * nc * h->V,
                              cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return FGPU_OK;
}

int fgpu_first_step(fgpu_handle* h) {
  if (!h) return FGPU_EARG;
  if (h->first_done) return set_err(h, FGPU_EBADCFG, "FirstStep should only be called once.");
  h->first_done = true;
  h->iter = 0;
  h->time = h->cfg.starttime;
  // fosite%FirstStep's ComputeRHS checks with CHECK_ALL whatever the checkdata mask
  // (fosite.f90:315-321): ideal-gas states get the CHECK_PMIN round trip here
  const bool rt_first = h->euler;
  if (h->butcher) {
    double dtc;
    int cause = 0;
    if (h->fargo) {
      // FirstStep's CenterBoundary + CalcBackgroundVelocity (the state carries no frame yet),
      // then its ComputeRHS: no AddBackgroundVelocity, SubtractBackgroundVelocity(w) after the
      // sources; cold = that co-moving cvar; CalcTimestep on the co-moving state
      if (h->cfg.fargo_method == 1)
        if (int rc = launch_fargo_w(h, plain_state(h->buf[0], false), nullptr, h->d_w)) return rc;
      CUDA_TRY(h, cudaMemcpyAsync(h->d_w + h->nw, h->d_w, sizeof(double) * h->nw, cudaMemcpyDeviceToDevice, h->stream));
      h->fargo_phase = 1;
      if (int rc = enqueue_k1_fargo(h, h->buf[0], chain_none(), rt_first, FGPU_CHECK_ALL, h->buf[1], h->time)) return rc;
      if (int rc = finish_cfl_host(h, h->buf[0], rt_first, dtc, FGPU_CHECK_ALL, cause, true)) return rc;
    } else {
      if (int rc = enqueue_k1(h, true, true, rt_first, FGPU_CHECK_ALL, h->time)) return rc;
      if (int rc = finish_cfl_host(h, h->buf[0], rt_first, dtc, FGPU_CHECK_ALL, cause)) return rc;
    }
    h->dt = dtc;
    h->dtcause = cause;
    h->pre_rt = rt_first;
    if (h->brk) return set_err(h, FGPU_BREAK, "FirstStep: Initial data invalid!");
    // first fosite%Step clip happens in fgpu_step
    return FGPU_OK;
  }
  // device clock: interior + boundary CFL, finalize computes dt and the clip for step 1
  Ctl* c = h->h_ctl;
  std::memset(c, 0, sizeof(Ctl));
  c->stoptime = h->stoptime; c->tout = h->tout; c->cfl = h->cfl; c->dtlimit = h->dtlimit;
  c->time = h->cfg.starttime; c->dtmin = h->stoptime; c->iter = 0;
  c->vis = h->vis ? 1 : 0; c->cvis = h->cvis;
  if (int rc = write_ctl(h)) return rc;
  BndArgs B = bnd_args(h, h->buf[0], rt_first, FIN_FIRST);
  B.checkdata = FGPU_CHECK_ALL;
  if (h->fargo) {
    // FirstStep's CenterBoundary + CalcBackgroundVelocity (fosite.f90:315-321), then the
    // CFL of its ComputeRHS on the co-moving state
    if (h->cfg.fargo_method == 1)
      if (int rc = launch_fargo_w(h, plain_state(h->buf[0], false), nullptr, h->d_w)) return rc;
    CUDA_TRY(h, cudaMemcpyAsync(h->d_w + h->nw, h->d_w, sizeof(double) * h->nw, cudaMemcpyDeviceToDevice, h->stream));
    B.w_sub = h->d_w;
    h->fargo_phase = 1;
  }
  if (int rc = launch_misc(h, 1, B)) return rc;
  if (int rc = launch_visc_cfl(h, plain_state(h->buf[0], rt_first), rt_first, RhsTime::host(h->time))) return rc;
  if (int rc = launch_misc(h, 0, B)) return rc;
  if (int rc = read_ctl(h)) return rc;
  sync_from_ctl(h);
  h->pre_rt = rt_first;
  if (h->brk) return set_err(h, FGPU_BREAK, "FirstStep: Initial data invalid!");
  return FGPU_OK;
}

// ---------------------------------------------------------------- embedded schemes (device clock)
// One attempt slot (fgpu_bt.cuh): open a step if due, one attempt with dt read on the device,
// the decision, then the RHS of the restored (reject) or advanced (accepted sub-step) state,
// or the step's closing: cvar from AcceptSolution, the closing RHS with CheckData and the
// CFL reduction, and CalcTimestep.  Every kernel after bt_begin runs only when its action
// bit is set; the sequence is what butcher_integration_step and butcher_step enqueue.
static int enqueue_bt_slot(fgpu_handle* h) {
  const Tableau& T = h->T;
  double* P = h->buf[0];
  double* base = h->buf[1];
  double* K1 = h->buf[2];
  Ctl* c = h->d_ctl;
  const double* d_att = &c->d_att;
  auto one = [&](auto&& launch) {
    return timed_launch(h, 0, 0.0, [&] {
      launch();
      CUDA_TRY(h, cudaGetLastError());
      return FGPU_OK;
    });
  };
  if (int rc = one([&] { bt_begin_kernel<<<1, 1, 0, h->stream>>>(c); })) return rc;
  // FARGO (after the run's first step, which the host loop takes): cvar of the attempts lives
  // apart from cold; every ComputeRHS adds and subtracts the step's background velocity
  const bool fg = h->fargo;
  double* CV = bt_cvar(h);
  const double* Wn = fg ? fargo_wn(h) : nullptr;
  const Chain addWn = fg ? chain_add(chain_none(), Wn, 1.0) : chain_none();
  const bool dyn = fg && h->cfg.fargo_method == 1;
  if (fg) {
    // IntegrationStep's opening: CalcBackgroundVelocity (type 1) and cvar = cold + w - w_new
    if (dyn) {
      const FargoStep F = fargo_step_of(h);
      if (int rc = launch_fargo_w(h, fargo_w_args(h, F).in, F.W, F.Wn, ACT_OPEN)) return rc;
      if (int rc = launch_fargo_chain_copy(h, base, CV, chain_add(chain_add(chain_none(), h->d_w, 1.0), Wn, -1.0),
                                           ACT_OPEN))
        return rc;
    } else if (int rc = launch_fargo_chain_copy(h, base, CV, chain_none(), ACT_OPEN)) {
      return rc;
    }
  }
  if (h->adaptive_me) {
    double* S1 = h->buf[3];
    double* S2 = h->buf[4];
    double* LO = h->buf[5];
    const int ord = h->order;
    const long long n = (long long)h->V * h->g.n;
    const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 148 * 8);
    const double e1 = kEta[ord - 1][0];
    if (int rc = one([&] {
          shu_osher_update_kernel<<<blocks, 256, 0, h->stream>>>(base, CV, K1, S1, n, e1, 0.0, d_att, c, ACT_ATTEMPT);
        }))
      return rc;
    for (int m = 2; m <= ord; ++m) {
      StageArgs A = base_args(h);
      A.in = plain_state(m == 2 ? S1 : S2, false);
      if (fg) {
        // every ComputeRHS frames its vector in place; the updates read the framed vectors
        A.in.pre = addWn;
        A.w_sub = Wn;
        A.yn_chain = chain_add(addWn, Wn, -1.0);
        if (m == ord && ord == 2) A.err_chain = A.yn_chain;
      }
      A.out_mode = OUT_SSPRK;
      A.eta = kEta[ord - 1][m - 1];
      A.y0 = base;
      A.dt_dev = d_att;
      if (m == ord) {
        A.out = P;
        A.err_low = ord == 3 ? LO : S1;
      } else {
        A.out = S2;
        A.out2 = LO;
        A.eta2 = kEta[1][1];
      }
      A.gate = ACT_ATTEMPT;
      if (int rc = launch_stage(h, A, RhsTime::att(kZeta[ord - 1][m - 2]))) return rc;
    }
  } else if (fg) {
    // stage states formed in the stencil from cvar with their frame chain; the last stage
    // forms the high/low-order solutions and the error norm
    for (int m = 2; m <= T.m; ++m) {
      StageArgs A = base_args(h);
      A.in.base = CV;
      A.in.nk = m - 1;
      A.in.roundtrip = 0;
      for (int q = 0; q < m - 1; ++q) {
        A.in.K[q] = h->buf[2 + q];
        A.in.coef[q] = T.A[(m - 1) * T.m + q];
      }
      A.in.dt_dev = d_att;
      A.in.pre = addWn;
      A.w_sub = Wn;
      A.out_mode = OUT_RHS;
      A.out = h->buf[2 + m - 1];
      if (m == T.m) set_last_stage(h, A, P, 0.0);
      A.gate = ACT_ATTEMPT;
      if (int rc = launch_stage(h, A, RhsTime::att(T.c[m - 1]))) return rc;
    }
  } else {
    for (int m = 2; m <= T.m; ++m) {
      StageArgs A = base_args(h);
      A.in.base = base;
      A.in.nk = m - 1;
      A.in.roundtrip = 0;
      for (int q = 0; q < m - 1; ++q) {
        A.in.K[q] = h->buf[2 + q];
        A.in.coef[q] = T.A[(m - 1) * T.m + q];
      }
      A.in.dt_dev = d_att;
      double* R = stage_rbuf(h, m);
      StateRef S = A.in;
      if (m == 2 || !h->fuse_form)
        if (int rc = timed_launch(h, 2, 0.0, [&] { return launch_form(h, S, R, ACT_ATTEMPT); })) return rc;
      A.rin = plain_state(R, false);
      A.rin.ready = h->prim ? 1 : 0;
      A.out_mode = OUT_RHS;
      A.out = h->buf[2 + m - 1];
      set_fnext(h, A, m, 0.0, d_att);
      if (m == T.m && h->fuse_end) set_last_stage(h, A, P, 0.0);
      A.gate = ACT_ATTEMPT;
      if (int rc = launch_stage(h, A, RhsTime::att(T.c[m - 1]))) return rc;
    }
  }
  if (h->butcher && !h->fuse_end && !fg) {
    CombineArgs Cb;
    std::memset(&Cb, 0, sizeof(Cb));
    Cb.base = base;
    for (int q = 0; q < T.m; ++q) {
      Cb.K[q] = h->buf[2 + q];
      Cb.bh_dt[q] = T.bh[q];
      Cb.bl_dt[q] = T.bl[q];
    }
    Cb.nstage = T.m;
    Cb.out_high = P;
    Cb.tol_rel = h->tol_rel;
    for (int v = 0; v < FGPU_MAXV; ++v) Cb.tol_abs[v] = h->tol_abs[v];
    Cb.n = h->g.n;
    Cb.ctl = c;
    Cb.dt_dev = d_att;
    Cb.gate = ACT_ATTEMPT;
    const unsigned blocks = (unsigned)std::min<long long>((h->g.n + 255) / 256, 148 * 8);
    if (int rc = timed_launch(h, 2, (double)h->V * h->g.n * 8.0, [&] {
          switch (h->V) {
            case 3: combine_kernel<3><<<blocks, 256, 0, h->stream>>>(Cb); break;
            case 4: combine_kernel<4><<<blocks, 256, 0, h->stream>>>(Cb); break;
            default: combine_kernel<5><<<blocks, 256, 0, h->stream>>>(Cb); break;
          }
          CUDA_TRY(h, cudaGetLastError());
          return FGPU_OK;
        }))
      return rc;
  }
  BtParams bp;
  bp.order = T.order;
  bp.beta = h->beta;
  bp.tol_rel = h->tol_rel;
  if (int rc = one([&] { bt_decide_kernel<<<1, 1, 0, h->stream>>>(c, bp); })) return rc;
  {   // RejectSolution: the RHS of cold (CHECK_NOTHING); with FARGO it frames cvar
    StageArgs A = base_args(h);
    A.out_mode = OUT_RHS;
    A.out = K1;
    A.in = plain_state(base, false);
    if (fg) { A.in.pre = addWn; A.w_sub = Wn; A.out_base = CV; }
    A.gate = ACT_REJECT;
    if (int rc = launch_stage(h, A, RhsTime::att(0.0))) return rc;
  }
  {   // AcceptSolution inside the step: the RHS at t with the checkdata mask, cold = cvar
    StageArgs A = base_args(h);
    A.out_mode = OUT_RHS;
    A.out = K1;
    A.in = plain_state(P, h->roundtrip_cfg);
    A.out_base = base;
    A.checkdata = h->cfg.checkdata;
    if (h->cfg.checkdata) A.cfl_mode = 3;
    if (fg) { A.in.pre = addWn; A.w_sub = Wn; }
    A.gate = ACT_SUB;
    if (int rc = launch_stage(h, A, RhsTime::att(0.0))) return rc;
    if (h->cfg.checkdata)
      if (int rc = one([&] { bt_subcheck_kernel<<<1, 1, 0, h->stream>>>(c); })) return rc;
    if (fg) {   // cvar = cold
      const long long n = (long long)h->V * h->g.n;
      const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 148 * 8);
      if (int rc = one([&] { gated_copy_kernel<<<blocks, 256, 0, h->stream>>>(base, CV, n, c, ACT_SUB); })) return rc;
    }
  }
  if (fg) {
    // the closing (timedisc_base.f90:727-744): FargoAdvection of cvar (AcceptSolution's framed
    // copy in cold when it evaluated the RHS at the step's end, else the accepted state), the
    // closing ComputeRHS (its CheckData and the interior CFL come from the advection pass),
    // the ghost cells' CFL, w = w_new and CalcTimestep
    const long long n = (long long)h->V * h->g.n;
    const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 148 * 8);
    const FargoStep F = fargo_step_of(h);
    FargoAdvArgs X = fargo_adv_args(h, F);
    X.w = Wn;
    X.dt_ctl = 1;
    X.in = plain_state(base, false); X.out = P; X.gate = ACT_COPY;
    if (int rc = launch_fargo_advect_args(h, X)) return rc;
    X.in = plain_state(P, false); X.out = CV; X.gate = ACT_ENDNC;
    if (int rc = launch_fargo_advect_args(h, X)) return rc;
    if (int rc = one([&] { gated_copy_kernel<<<blocks, 256, 0, h->stream>>>(CV, P, n, c, ACT_ENDNC); })) return rc;
    StageArgs A = base_args(h);
    A.out_mode = OUT_RHS;
    A.out = K1;
    A.in = plain_state(P, false);
    A.in.pre = addWn;
    A.w_sub = Wn;
    A.out_base = base;
    A.gate = ACT_END;
    if (int rc = launch_stage(h, A, RhsTime::att(0.0))) return rc;
    BndArgs B = bnd_args(h, P, false, FIN_NONE);
    B.in.pre = addWn;
    B.w_sub = Wn;
    B.checkdata = h->cfg.checkdata;
    B.gate = ACT_END;
    if (int rc = launch_misc(h, 0, B)) return rc;
    if (dyn) {
      const long long nw = h->nw;
      double* W = h->d_w;
      if (int rc = one([&] { gated_copy_kernel<<<1, 256, 0, h->stream>>>(Wn, W, nw, c, ACT_END); })) return rc;
    }
    const int nd = h->nd;
    return one([&] { bt_finish_kernel<<<1, 1, 0, h->stream>>>(c, nd); });
  }
  {   // the closing: cvar as AcceptSolution's ComputeRHS left it, then IntegrationStep's RHS
    const long long n = (long long)h->V * h->g.n;
    const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 148 * 8);
    if (int rc = one([&] { gated_copy_kernel<<<blocks, 256, 0, h->stream>>>(base, P, n, c, ACT_COPY); })) return rc;
    StageArgs A = base_args(h);
    A.out_mode = OUT_RHS;
    A.out = K1;
    A.in = plain_state(P, h->roundtrip_cfg);
    A.out_base = base;
    A.checkdata = h->cfg.checkdata;
    A.cfl_mode = 2;
    A.gate = ACT_END;
    if (int rc = launch_stage(h, A, RhsTime::att(0.0))) return rc;
  }
  BndArgs B = bnd_args(h, P, h->roundtrip_cfg, FIN_NONE);
  B.checkdata = h->cfg.checkdata;
  B.gate = ACT_END;
  if (int rc = launch_misc(h, 0, B)) return rc;
  if (int rc = launch_visc_cfl(h, plain_state(P, h->roundtrip_cfg), h->roundtrip_cfg, RhsTime::att(0.0), ACT_END))
    return rc;
  const int nd = h->nd;
  return one([&] { bt_finish_kernel<<<1, 1, 0, h->stream>>>(c, nd); });
}

// n fosite steps of an embedded scheme on the device clock: the host state goes into the
// control block, attempt slots are replayed (a captured graph) in chunks with one control-
// block read per chunk, and the state comes back.  Results equal n calls of butcher_step.
static int bt_run(fgpu_handle* h, int64_t n, int64_t* done) {
  Ctl* c = h->h_ctl;
  std::memset(c, 0, sizeof(Ctl));
  c->time = h->time; c->dt = h->dt; c->dtold = h->dtold; c->dtmin = h->dtmin;
  c->stoptime = h->stoptime; c->tout = h->tout; c->cfl = h->cfl; c->dtlimit = h->dtlimit;
  c->iter = h->iter; c->brk = h->brk ? 1 : 0; c->dtcause = h->dtcause;
  c->cvis = h->cvis; c->vis = h->vis ? 1 : 0;
  c->maxerrold = h->maxerrold; c->last_err = h->last_err; c->n_adj = h->n_adj;
  c->checkflags = h->checkflags;
  c->steps_left = n;
  if (int rc = write_ctl(h)) return rc;
  if (!h->bt_graph && !h->profiling) {
    cudaGraph_t gr;
    fgpu_stats saved = h->stats;
    CUDA_TRY(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_bt_slot(h);
    cudaError_t e = cudaStreamEndCapture(h->stream, &gr);
    h->kernels_per_slot = (int)(h->stats.launches - saved.launches);
    h->stats = saved;
    if (rc) return rc;
    if (e != cudaSuccess) return set_err(h, FGPU_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&h->bt_graph, gr, 0);
    cudaGraphDestroy(gr);
    if (e != cudaSuccess) return set_err(h, FGPU_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  }
  const long long it0 = h->iter, adj0 = h->n_adj;
  long long slots = 0;
  const long long cap = slot_cap(64 * (long long)n + 64);   // every attempt either advances t or shrinks dt 4x
  bool stalled = false;
  while (true) {
    // as many slots as steps are left (most steps take one attempt), at most 8 per read
    const int CH = (int)std::max<long long>(1, std::min<long long>(8, c->steps_left));
    for (int k = 0; k < CH; ++k) {
      if (h->profiling) {
        if (int rc = enqueue_bt_slot(h)) return rc;
      } else {
        CUDA_TRY(h, cudaGraphLaunch(h->bt_graph, h->stream));
        h->stats.launches += h->kernels_per_slot;
      }
    }
    slots += CH;
    if (int rc = read_ctl(h)) return rc;
    if (c->steps_left <= 0 || c->stop || c->brk) break;
    if (slots > cap) { stalled = true; break; }
  }
  h->time = c->time; h->dt = c->dt; h->dtold = c->dtold; h->dtmin = c->dtmin;
  h->iter = c->iter; h->brk = c->brk != 0; h->dtcause = c->dtcause;
  h->maxerrold = c->maxerrold; h->last_err = c->last_err; h->n_adj = c->n_adj;
  h->checkflags = c->checkflags;
  const int64_t steps = n - c->steps_left;
  // after a completed step, or a break inside one (the stored state then went through that
  // step's ComputeRHS with the configured checks)
  if (steps > 0 || h->brk) h->pre_rt = h->roundtrip_cfg;
  h->stats.attempts += (h->iter - it0) + (h->n_adj - adj0);
  h->stats.cell_updates += (h->iter - it0) * h->g.n;
  if (done) *done = steps;
  // no progress within the slot budget: the bookkeeping above is the device's, the call ends
  if (stalled) return set_err(h, FGPU_ETIMEOUT, "device-clock step loop: no progress");
  if (h->brk) return FGPU_BREAK;
  if (c->stop) return FGPU_STOPTIME;
  return FGPU_OK;
}

// the device clock serves embedded schemes whose stage states are formed by form_kernel;
// FGPU_BUTCHER_HOST=1 keeps the host-controlled loop
static bool bt_device(const fgpu_handle* h) {
  // (FARGO with an embedded scheme forms its stage states in the stencil)
  if (!h->materialize && !h->fargo) return false;
  const char* e = std::getenv("FGPU_BUTCHER_HOST");
  return !(e && std::atoi(e) != 0);
}

static int butcher_step(fgpu_handle* h) {
  // fosite%Step (fosite.f90:367-464) around the Butcher IntegrationStep
  if (std::fabs(h->stoptime - h->time) <= 1.0E-05 * h->stoptime) return FGPU_STOPTIME;
  if ((h->time + h->dt) / h->tout > 1.0) { h->dt = h->tout - h->time; h->dtcause = FGPU_DTCAUSE_FILEIO; }
  else if ((h->time + 1.5 * h->dt) / h->tout > 1.0) { h->dt = 0.5 * (h->tout - h->time); h->dtcause = FGPU_DTCAUSE_FILEIO; }
  if (int rc = butcher_integration_step(h)) return rc;
  if (h->brk) return FGPU_BREAK;
  double dtc;
  int cause = 0;
  if (int rc = finish_cfl_host(h, h->buf[0], h->roundtrip_cfg, dtc, h->cfg.checkdata, cause)) return rc;
  if (h->brk) return FGPU_BREAK;
  h->dt = dtc;
  h->dtcause = cause;
  return FGPU_OK;
}

int fgpu_run(fgpu_handle* h, int64_t n, int64_t* done) {
  if (!h) return FGPU_EARG;
  if (!h->first_done) { int rc = fgpu_first_step(h); if (rc) return rc; }
  int64_t k = 0;
  if (h->butcher) {
    if (n > 0 && bt_device(h) && h->fargo && (h->fargo_tmp_fresh || h->fargo_phase < 2)) {
      // the run's first FARGO step (its stage vectors' first frame flag, the frame of the
      // state FirstStep left) on the host loop, the rest on the device clock
      if (int rc = butcher_step(h)) { if (done) *done = 0; return rc; }
      int64_t d2 = 0;
      const int rc = n > 1 ? bt_run(h, n - 1, &d2) : FGPU_OK;
      if (done) *done = 1 + d2;
      return rc;
    }
    if (n > 0 && bt_device(h)) return bt_run(h, n, done);
    int rc = FGPU_OK;
    for (; k < n; ++k) {
      rc = butcher_step(h);
      if (rc) break;
    }
    if (done) *done = k;
    return rc;
  }
  // device clock: graph of G steps, replayed
  long long it0 = h->iter;
  if (n > 0 && ((h->fargo && h->fargo_phase < 2) || h->pre_rt != h->roundtrip_cfg)) {
    // the first step after FirstStep has its own frame chains (FARGO) or round trip
    // (FirstStep checks with CHECK_ALL): direct launches, the graph covers the rest
    if (int rc = enqueue_step(h)) return rc;
    n -= 1;
  }
  const int G = 16;
  int64_t full = n / G, rest = n % G;
  if (h->profiling) { rest += full * G; full = 0; }   // per-launch timing needs direct launches
  if (full > 0) {
    if (h->graph_steps != G) { if (int rc = build_graph(h, G)) return rc; }
    for (int64_t r = 0; r < full; ++r) {
      CUDA_TRY(h, cudaGraphLaunch(h->graph, h->stream));
      h->stats.launches += (int64_t)h->kernels_per_step * G;
      h->stats.stage_launches += (int64_t)h->order * G;
    }
  }
  for (int64_t r = 0; r < rest; ++r) { if (int rc = enqueue_step(h)) return rc; }
  if (int rc = read_ctl(h)) return rc;
  sync_from_ctl(h);
  h->stats.attempts += h->iter - it0;
  h->stats.cell_updates += (h->iter - it0) * h->g.n;
  if (done) *done = h->iter - it0;
  if (h->brk) return FGPU_BREAK;
  if (h->h_ctl->stop) return FGPU_STOPTIME;
  return FGPU_OK;
}

int fgpu_step(fgpu_handle* h) {
  if (!h) return FGPU_EARG;
  if (!h->first_done) { int rc = fgpu_first_step(h); if (rc) return rc; }
  if (h->butcher) return butcher_step(h);
  if (h->h_ctl->stop || h->h_ctl->brk) return h->h_ctl->brk ? FGPU_BREAK : FGPU_STOPTIME;
  int64_t d = 0;
  return fgpu_run(h, 1, &d);
}

int fgpu_compute_rhs(fgpu_handle* h) {
  if (!h) return FGPU_EARG;
  // ComputeRHS(CHECK_NOTHING) of fosite's current cvar
  double* P = h->buf[0];
  const double* src = P;
  // K_m and K_(m-1) of the Butcher engine are recomputed by every attempt,
  // so between steps they are free scratch (m >= 3 for all tableaus)
  double* out = h->butcher ? h->buf[2 + h->T.m - 1] : h->buf[1];
  double* scratch = h->butcher ? h->buf[2 + h->T.m - 2] : h->buf[2];
  if (h->pre_rt) {
    if (int rc = launch_roundtrip(h, P, scratch)) return rc;
    src = scratch;
  }
  StageArgs A = base_args(h);
  A.in = plain_state(src, false);
  if (h->fargo) {
    // fosite's cvar is pre + [-w]; ComputeRHS adds w back before the boundary fill.
    // The stored state is left as it is (the reference's in-place round trip is not applied).
    if (h->fargo_phase >= 1) A.in.pre = chain_add(chain_add(fargo_pre(h), h->d_w, -1.0), h->d_w, 1.0);
    A.w_sub = h->d_w;
  }
  A.out_mode = OUT_RHS;
  A.out = out;
  A.ctl = nullptr;
  // the interface fluxes too, for fgpu_download(FGPU_XFLUX..ZFLUX)
  const size_t nflux = 3 * (size_t)h->V * (size_t)fgpu_cell_count(h);
  if (!h->d_flux) CUDA_TRY(h, cudaMalloc(&h->d_flux, sizeof(double) * nflux));
  CUDA_TRY(h, cudaMemsetAsync(h->d_flux, 0, sizeof(double) * nflux, h->stream));
  A.flux_out = h->d_flux;
  if (int rc = launch_stage(h, A, RhsTime::host(h->time))) return rc;
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  h->flux_valid = true;
  return FGPU_OK;
}

int fgpu_set_output_time(fgpu_handle* h, double tout) {
  if (!h) return FGPU_EARG;
  if (!(tout > 0.0)) return set_err(h, FGPU_EARG, "output time must be positive");
  h->tout = tout;
  return FGPU_OK;
}

int fgpu_calc_timestep(fgpu_handle* h, double* dt) {
  if (!h || !dt) return FGPU_EARG;
  bool rt = h->pre_rt;
  Ctl save = *h->h_ctl;
  if (int rc = read_ctl(h)) return rc;
  save = *h->h_ctl;
  h->h_ctl->invdt[0] = h->h_ctl->invdt[1] = h->h_ctl->invdt[2] = h->h_ctl->invdt[3] = 0ULL;
  h->h_ctl->flags = 0;
  h->h_ctl->stop = 0; h->h_ctl->brk = 0;
  if (int rc = write_ctl(h)) return rc;
  BndArgs B = bnd_args(h, h->buf[0], rt, FIN_NONE);
  if (h->fargo) { B.in.pre = fargo_pre(h); B.w_sub = h->d_w; }
  if (int rc = launch_misc(h, 1, B)) return rc;
  if (int rc = launch_misc(h, 0, B)) return rc;
  if (int rc = launch_visc_cfl(h, plain_state(h->buf[0], rt), rt, RhsTime::host(h->time))) return rc;
  if (int rc = read_ctl(h)) return rc;
  int cause = 0;
  *dt = ctl_dt(h, &cause);
  *h->h_ctl = save;
  return write_ctl(h);
}

int fgpu_get_status(fgpu_handle* h, fgpu_status* st) {
  if (!h || !st) return FGPU_EARG;
  std::memset(st, 0, sizeof(*st));
  st->time = h->time; st->dt = h->dt; st->dtold = h->dtold; st->dtmin = h->dtmin; st->maxerr = h->last_err;
  st->iter = h->iter; st->n_adj = h->n_adj; st->dtcause = h->dtcause; st->brk = h->brk ? 1 : 0;
  st->checkflags = h->checkflags;
  return FGPU_OK;
}

int fgpu_set_fargo_velocity(fgpu_handle* h, const double* w, int64_t n) {
  if (!h || !w) return FGPU_EARG;
  if (!h->fargo || h->cfg.fargo_method != 2)
    return set_err(h, FGPU_EBADCFG, "the background velocity is supplied for fargo type 2 only");
  if (h->first_done) return set_err(h, FGPU_EBADCFG, "set the fargo background velocity before the first step");
  if (n < h->nw)
    return set_err(h, FGPU_EARG, "background velocity array too small (inum+4 values along y, jnum+4 along x)");
  CUDA_TRY(h, cudaMemcpyAsync(h->d_w, w, sizeof(double) * h->nw, cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(h, cudaMemcpyAsync(h->d_w + h->nw, w, sizeof(double) * h->nw, cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return FGPU_OK;
}

int fgpu_get_pointmass(fgpu_handle* h, double* mass, double* mdot) {
  if (!h || !mass || !mdot) return FGPU_EARG;
  if (!h->accrete) { *mass = h->cfg.pm_mass; *mdot = 0.0; return FGPU_OK; }
  double g[2];
  CUDA_TRY(h, cudaMemcpyAsync(g, h->d_acc + 3 * (size_t)h->g.ny, sizeof(g), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  *mass = g[0];
  *mdot = g[1];
  return FGPU_OK;
}

int fgpu_synchronize(fgpu_handle* h) {
  if (!h) return FGPU_EARG;
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return FGPU_OK;
}

int fgpu_set_stream(fgpu_handle* h, void* stream) {
  if (!h) return FGPU_EARG;
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if (!h->own_stream) h->own_stream = h->stream;
  h->stream = stream ? (cudaStream_t)stream : h->own_stream;
  return FGPU_OK;
}

int fgpu_measure_l2_read(int device, int mb, int passes, double* gbs) {
  if (!gbs || mb < 1 || mb > 64 || passes < 1) return FGPU_EARG;
  if (cudaSetDevice(device) != cudaSuccess) return FGPU_ECUDA;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const size_t n2 = (size_t)mb * (1u << 20) / 16;
  double2* a = nullptr;
  double* out = nullptr;
  if (cudaMalloc(&a, n2 * 16) != cudaSuccess) return FGPU_ENOMEM;
  if (cudaMalloc(&out, sizeof(double) * 1024) != cudaSuccess) { cudaFree(a); return FGPU_ENOMEM; }
  cudaMemset(a, 0, n2 * 16);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const unsigned blocks = (unsigned)(4 * sms);
  l2_read_probe_kernel<<<blocks, 512>>>(a, n2, passes, out);
  cudaEventRecord(e0);
  l2_read_probe_kernel<<<blocks, 512>>>(a, n2, passes, out);
  cudaEventRecord(e1);
  cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(a);
  cudaFree(out);
  if (e != cudaSuccess || ms <= 0.f) return FGPU_ECUDA;
  *gbs = (double)n2 * 16.0 * passes / (ms * 1e-3) / 1e9;
  return FGPU_OK;
}

int fgpu_set_profiling(fgpu_handle* h, int on) {
  if (!h) return FGPU_EARG;
  h->profiling = on != 0;
  return FGPU_OK;
}

int fgpu_get_stats(fgpu_handle* h, fgpu_stats* st) {
  if (!h || !st) return FGPU_EARG;
  if (!h->timed.empty()) {
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    for (auto& t : h->timed) {
      float ms = 0.f;
      CUDA_TRY(h, cudaEventElapsedTime(&ms, t.a, t.b));
      if (t.stage) { h->stats.stage_ms += ms; h->stats.stage_bytes += t.bytes; }
      else h->stats.other_ms += ms;
      if (t.stage == 2) h->stats.form_ms += ms;
      cudaEventDestroy(t.a);
      cudaEventDestroy(t.b);
    }
    h->timed.clear();
  }
  *st = h->stats;
  return FGPU_OK;
}

int fgpu_reset_stats(fgpu_handle* h) {
  if (!h) return FGPU_EARG;
  fgpu_stats tmp;
  int rc = fgpu_get_stats(h, &tmp);
  std::memset(&h->stats, 0, sizeof(h->stats));
  return rc;
}

}  // extern "C"

// ======================================================================= batched ensembles, autotuner
#include "fgpu_batch.cuh"

// ======================================================================= allocation-free CFL time step
// Callers that must not allocate device memory after start-up -- code running
// inside a memory-capped service, a real-time loop that forbids cudaMalloc, or
// a host that hands the solver a fixed memory pool -- get one entry point that
// uses only this file-scope scratch array: the 1-D metric of the mesh and the
// reduction control block live here instead of in per-handle allocations.
namespace {

constexpr size_t kNoallocScratchBytes = 1u << 20;   // 1 MiB, held by every device that loads the library
static __device__ __align__(256) double g_noalloc_scratch[kNoallocScratchBytes / sizeof(double)];

constexpr int kMaxDevices = 64;
double* g_noalloc_ptr[kMaxDevices] = {nullptr};
std::mutex g_noalloc_mutex;

// per-device set-up: the device address of the scratch array, taken with the device current
int noalloc_scratch(int dev, double** ptr) {
  if (dev < 0 || dev >= kMaxDevices) return FGPU_EARG;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    double* p = nullptr;
    if (cudaGetSymbolAddress((void**)&p, g_noalloc_scratch) != cudaSuccess || !p) return FGPU_ECUDA;
    g_noalloc_ptr[dev] = p;
  }
  *ptr = g_noalloc_ptr[dev];
  return FGPU_OK;
}

// The Cartesian metric of the allocation-free CFL call in its scratch array: the constant
// factors by array (vals) and the reconstruction offsets x_face - x_centre of x, y and z in the
// operation order of build_metric (mesh_midpoint.f90:97-145), evaluated without contraction so
// that they equal the host's values bit for bit.
struct NoallocMetric {
  double vals[M_NI];
  double lo[3], d[3];
  int np[3];
};
__global__ void noalloc_metric_kernel(double* dm, const NoallocMetric m) {
  const int nxp = m.np[0], nyp = m.np[1], nzp = m.np[2];
  const int total = M_NI * nxp + 2 * nyp + 2 * nzp;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    int q, ip, dir, east;
    if (t < M_NI * nxp) {
      q = t / nxp; ip = t % nxp;
      if (q != M_offxW && q != M_offxE) { dm[t] = m.vals[q]; continue; }
      dir = 0; east = q == M_offxE;
    } else {
      int u = t - M_NI * nxp;
      if (u < 2 * nyp) { dir = 1; east = u / nyp; ip = u % nyp; }
      else { u -= 2 * nyp; dir = 2; east = u / nzp; ip = u % nzp; }
    }
    const double h = m.d[dir];
    const double x = __dadd_rn(m.lo[dir], __dmul_rn(__dmul_rn((double)(2 * (ip - 1) - 1), 0.5), h));
    const double f = east ? __dadd_rn(x, __dmul_rn(0.5, h)) : __dadd_rn(x, __dmul_rn(-0.5, h));
    dm[t] = __dsub_rn(f, x);
  }
}

__global__ void noalloc_finalize_kernel(const Ctl* c, int nd, double cfl, double* dt_out) {
  auto D = [](unsigned long long b) { return __longlong_as_double((long long)b); };
  double invdt = nd == 2 ? D(c->invdt[0]) : dmax(dmax(D(c->invdt[1]), D(c->invdt[2])), D(c->invdt[0]));
  *dt_out = cfl / invdt;
}

template <int ND, bool EU>
void noalloc_launch(const BndArgs& B, long long n, cudaStream_t s, int nd, double cfl, double* dt_out) {
  long long b1 = std::min<long long>((n + 255) / 256, 148 * 16);
  interior_cfl_kernel<ND, EU><<<(unsigned)b1, 256, 0, s>>>(B);
  long long b2 = std::min<long long>((B.nghost + 255) / 256, 4096);
  boundary_kernel<ND, EU><<<(unsigned)(b2 < 1 ? 1 : b2), 256, 0, s>>>(B);
  noalloc_finalize_kernel<<<1, 1, 0, s>>>(B.ctl, nd, cfl, dt_out);
}

}  // namespace

extern "C" int fgpu_calc_timestep_noalloc(const fgpu_config* cfg, const double* d_cvar, double* d_dt, void* stream) {
  if (!cfg || !d_cvar || !d_dt) return FGPU_EARG;
  const fgpu_config& c = *cfg;
  if (c.geometry != FGPU_CARTESIAN || c.pointmass || c.fargo_method || c.vismodel) return FGPU_EUNSUPPORTED;
  if (c.inum < 2 || c.jnum < 2 || c.knum < 1) return FGPU_EUNSUPPORTED;
  bool euler = c.physics == FGPU_EULER;
  if (!euler && !(c.physics == FGPU_EULER_ISOTHERM && c.csiso > 0.0)) return FGPU_EUNSUPPORTED;
  int nd = c.knum > 1 ? 3 : 2;
  for (int f = 0; f < 2 * nd; ++f) {
    int t = c.bc[f];
    if (t != FGPU_PERIODIC && t != FGPU_REFLECTING && t != FGPU_ABSORBING && t != FGPU_NO_GRADIENTS &&
        t != FGPU_AXIS)
      return FGPU_EUNSUPPORTED;
  }
  int nxp = c.inum + 4, nyp = c.jnum + 4, nzp = c.knum + 4;
  size_t ctl_doubles = (sizeof(Ctl) + 255) / 256 * 256 / sizeof(double);
  size_t metric_doubles = (size_t)M_NI * nxp + 2 * (size_t)nyp + 2 * (size_t)nzp;
  if ((ctl_doubles + metric_doubles) * sizeof(double) > kNoallocScratchBytes) return FGPU_EARG;   // mesh too large
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return FGPU_ECUDA;
  double* scratch = nullptr;
  if (int rc = noalloc_scratch(dev, &scratch)) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  Ctl* ctl = (Ctl*)scratch;
  double* dm = scratch + ctl_doubles;

  // Cartesian metric (mesh_base.f90:570-601, mesh_midpoint.f90:97-145 with h = 1): the constant
  // factors computed here, the reconstruction offsets by a kernel, all in the scratch array
  double dx = (c.xmax - c.xmin) / c.inum, dy = (c.ymax - c.ymin) / c.jnum, dz = (c.zmax - c.zmin) / c.knum;
  double mdx = dx, mdy = dy, mdz = dz;
  if (dz < 2 * DBL_EPSILON && c.knum == 1) { dz = 1.0; mdz = 0.0; }
  double volume = 1.0 * dx * dy * dz;
  NoallocMetric nm;
  for (int q = 0; q < M_NI; ++q) nm.vals[q] = 0.0;
  nm.vals[M_dAxW] = 1.0 * 1.0; nm.vals[M_dAxE] = 1.0 * 1.0; nm.vals[M_dAyS] = 1.0 * 1.0; nm.vals[M_dAzB] = 1.0 * 1.0;
  nm.vals[M_dxdydV] = dx * dy / (volume + DBL_MIN);
  nm.vals[M_dydzdV] = dy * dz / (volume + DBL_MIN);
  nm.vals[M_dzdxdV] = dz * dx / (volume + DBL_MIN);
  nm.vals[M_dlx] = 1.0 * dx; nm.vals[M_dly] = 1.0 * dy; nm.vals[M_dlz] = 1.0 * dz;
  for (int q = 0; q < 7; ++q) nm.vals[M_cs0 + q] = euler ? 0.0 : c.csiso;
  nm.lo[0] = c.xmin; nm.lo[1] = c.ymin; nm.lo[2] = c.zmin;
  nm.d[0] = mdx; nm.d[1] = mdy; nm.d[2] = mdz;
  nm.np[0] = nxp; nm.np[1] = nyp; nm.np[2] = nzp;
  const size_t by = (size_t)M_NI * nxp;
  {
    const int total = M_NI * nxp + 2 * nyp + 2 * nzp;
    noalloc_metric_kernel<<<(total + 255) / 256, 256, 0, s>>>(dm, nm);
  }
  // the reduction slots must start at zero on every call
  if (cudaMemsetAsync(ctl, 0, sizeof(Ctl), s) != cudaSuccess) return FGPU_ECUDA;

  BndArgs B;
  std::memset(&B, 0, sizeof(B));
  B.g.nx = c.inum; B.g.ny = c.jnum; B.g.nz = nd == 3 ? c.knum : 1;
  B.g.n = (long long)B.g.nx * B.g.ny * B.g.nz;
  for (int f = 0; f < 6; ++f) B.g.bc[f] = c.bc[f];
  B.ph.gamma = c.gamma; B.ph.gm1 = c.gamma - 1.; B.ph.pmin = c.pmin; B.ph.rhomin = c.rhomin; B.ph.tiny2 = 2.0 * DBL_MIN;
  B.ph.inv_gm1 = 1.0 / B.ph.gm1;
  MetricP& M = B.mt;
  auto P = [&](int which) { return dm + (size_t)which * nxp; };
  M.dAxW = P(M_dAxW); M.dAyS = P(M_dAyS); M.dAzB = P(M_dAzB);
  M.dydzdV = P(M_dydzdV); M.dzdxdV = P(M_dzdxdV); M.dxdydV = P(M_dxdydV);
  M.cxyx = P(M_cxyx); M.cxzx = P(M_cxzx); M.cyxy = P(M_cyxy); M.cyzy = P(M_cyzy); M.czxz = P(M_czxz); M.czyz = P(M_czyz);
  M.dlx = P(M_dlx); M.dly = P(M_dly); M.dlz = P(M_dlz);
  M.offxW = P(M_offxW); M.offxE = P(M_offxE);
  M.offyS = dm + by; M.offyN = dm + by + nyp; M.offzB = dm + by + 2 * nyp; M.offzT = dm + by + 2 * nyp + nzp;
  M.accel = nullptr; M.cs = P(M_cs0); M.nxp = nxp; M.curv = 0;
  B.in.base = d_cvar; B.in.nk = 0; B.in.roundtrip = 0;
  B.roundtrip = 0;
  B.checkdata = 0;
  B.ctl = ctl;
  B.finalize = FIN_NONE;
  B.nghost = (long long)nxp * nyp * (nd == 3 ? nzp : 1) - B.g.n;
  if (nd == 2) { if (euler) noalloc_launch<2, true>(B, B.g.n, s, nd, c.cfl, d_dt); else noalloc_launch<2, false>(B, B.g.n, s, nd, c.cfl, d_dt); }
  else { if (euler) noalloc_launch<3, true>(B, B.g.n, s, nd, c.cfl, d_dt); else noalloc_launch<3, false>(B, B.g.n, s, nd, c.cfl, d_dt); }
  return cudaGetLastError() == cudaSuccess ? FGPU_OK : FGPU_ECUDA;
}
