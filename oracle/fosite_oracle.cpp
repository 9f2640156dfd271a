// fosite_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A serial CPU restatement of fosite 0.8.3's explicit finite-volume time step,
// used exclusively as the parity checker of the B200 backend (tests, smoke
// and the bench's CPU baseline leg).  It is never linked into the product
// library and the product never calls it.
//
// The code keeps the reference's data layout (ghost-padded, Fortran order,
// i fastest, Mesh%IGMIN..IGMAX etc.) and its loop order and operation order,
// so that -- compiled with -ffp-contract=off like the reference's gfortran
// build without FMA (CMakeLists.txt:168-171) -- it reproduces the reference's
// arithmetic.  Each routine names the reference lines it restates.
//
// The step-size controller's EXP and LOG are evaluated correctly rounded (binary128,
// then rounded once), the values glibc's libm gave before version 2.28 and gives
// since then in all but about one argument in a thousand.
//
// Parity is pinned by the reference's own metamorphic test assertions
// (tests/KHI2D.f90:81-150 transposition symmetry to TINY, conservation on
// periodic boxes); the reference ships no golden vectors and cannot be
// compiled here (no Fortran compiler), so bit-for-bit agreement with a
// Fortran build is unverified.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <cfloat>
#include <vector>
#include <string>
#include <algorithm>
#include <quadmath.h>
#include "../include/fosite_gpu.h"

// Data-parallel loops (every iteration writes its own elements, no reductions) run on the
// host's cores when built with OpenMP; the arithmetic of each element is unchanged, so the
// results are the same bit for bit at any thread count.  Reductions stay serial.
#ifdef _OPENMP
#include <omp.h>
#define PAR_FOR _Pragma("omp parallel for schedule(static)")
#define PAR_FOR2 _Pragma("omp parallel for collapse(2) schedule(static)")
#define PAR_FOR3 _Pragma("omp parallel for collapse(3) schedule(static)")
#else
#define PAR_FOR
#define PAR_FOR2
#define PAR_FOR3
#endif

namespace {

const double TINY_ = DBL_MIN;     // Fortran TINY(1.0) for REAL(8)
const double HUGE_ = DBL_MAX;
const double EPS_ = DBL_EPSILON;
const double PI_ = 3.1415926535897932384626433832795028842;

inline double fsign(double a, double b) { return std::signbit(b) ? -std::fabs(a) : std::fabs(a); }
inline double fmin2(double a, double b) { return b < a ? b : a; }
inline double fmax2(double a, double b) { return b > a ? b : a; }

struct Oracle {
  fgpu_config cfg;
  std::string err;
  // ---- mesh (mesh/mesh_base.f90:446-729) ----
  int INUM, JNUM, KNUM, GINUM, GJNUM, GKNUM;
  int IMIN, IMAX, JMIN, JMAX, KMIN, KMAX, IGMIN, IGMAX, JGMIN, JGMAX, KGMIN, KGMAX;
  int IP1, IM1, JP1, JM1, KP1, KM1;
  int NDIMS, NFACES, NI, NJ, NK;
  long NC;
  int dirs[3];          // active directions (0=x,1=y,2=z)
  int VDIM, VNUM;
  bool euler;
  int PRESSURE;         // 0-based index of pressure/energy, -1 for isothermal
  double dx, dy, dz, invdx, invdy, invdz, mesh_dx, mesh_dy, mesh_dz;
  std::vector<double> cx, cy, cz;            // centre coordinates per index
  std::vector<double> hfx, hfy, hfz;         // scale factors at 6 faces (NC*6)
  std::vector<double> hcx, hcy, hcz;         // scale factors at centres
  std::vector<double> volume, dxdydV, dydzdV, dzdxdV, dlx, dly, dlz;
  std::vector<double> cxyx, cxzx, cyxy, cyzy, czxz, czyz;
  std::vector<double> dAx, dAy, dAz;         // dAxdydz etc, NC*2
  std::vector<double> rdx;                   // reconstruction offsets NC*NFACES
  std::vector<double> radius, posvec;        // NC, NC*3
  // ---- physics ----
  std::vector<double> bccsound, fcsound;     // NC, NC*NFACES
  // ---- state ----
  std::vector<double> pvar, cvar, ptmp, ctmp, cold, rhs, geo_src, src, cerr;
  std::vector<std::vector<double>> coeff;    // Butcher k_m (coeff[0] aliases rhs semantics)
  std::vector<double> xflux, yflux, zflux;   // NC*VNUM
  std::vector<double> slopes;                // NC*NDIMS*VNUM
  std::vector<double> fprim, fcons, pfluxes; // NC*NFACES*VNUM
  std::vector<double> minwav, maxwav;        // NC*NDIMS
  std::vector<double> tmpw, tmpw1;           // NC
  std::vector<double> accel;                 // NC*VDIM
  bool have_accel = false;
  // point-mass accretion: x-boundary fluxes (fluxes_base.f90:73-76 bxflux/bxfold, indexed
  // [((l*2 + face)*KNUM + k)*JNUM + j]) and the point mass (gravity_pointmass.f90:383-428)
  int outbound = 0;                          // fosite numbering: 1 WEST, 2 EAST
  std::vector<double> bxf, bxo;
  double pm_cur = 0.0, mdot = 0.0;
  // ---- timedisc ----
  int order, m_stages;
  bool butcher;
  std::vector<double> A, b_high, b_low, c_coef;  // Butcher tableau (m x m row-major)
  double time, dt, dtold, dtmin, maxerrold, stoptime, cfl, dtlimit, tol_rel, beta;
  std::vector<double> tol_abs;
  int dtcause, dtmincause, checkdatabm;
  bool brk = false;
  int64_t iter = -1, n_adj = 0;
  double last_err = 0;
  int checkflags = 0;
  // ---- fargo (direction 1: transport along x, w by (j,k); direction 2: along y, w by (i,k)) ----
  int fargo = 0, fdir = 2;
  std::vector<double> w, wfactor, delxy, fdq, fdql, fflux;
  std::vector<int> shift;
  // fargo_transformation_applied flags of each state vector (physics_eulerisotherm.f90:124):
  // cvar/pvar and the Butcher stage vectors ctmp/ptmp; assignments between state vectors copy
  // data only (marray_compound.f90:118-229), Convert2Primitive copies c's flag to p (:338)
  bool c_trans = false, p_trans = false, ct_trans = false, pt_trans = false;
  bool& cflag(const std::vector<double>& cv) { return &cv == &ctmp ? ct_trans : c_trans; }
  bool& pflag(const std::vector<double>& pv) { return &pv == &ptmp ? pt_trans : p_trans; }
  // ---- viscosity (sources_viscosity.f90) ----
  int vismodel = 0;
  double dynconst = 0.0, bulkconst = 0.0, power = 0.0, cvis = 0.5;
  double vis_time = -1.0;                                     // InitSources: time of the last update
  std::vector<double> dynvis, bulkvis, kinvis, ephir;         // NC, NC, NC, NC*VDIM
  std::vector<double> btxx, btxy, btxz, btyy, btyz, btzz;   // stress tensor (InitSources: zero)
  std::vector<double> vtmp, vtmp1, vtmp2;                     // Physics%tmp, tmp1, tmp2

  long id(int i, int j, int k) const {
    return (long)(i - IGMIN) + (long)NI * ((long)(j - JGMIN) + (long)NJ * (long)(k - KGMIN));
  }
  double& V(std::vector<double>& a, int i, int j, int k, int l) { return a[id(i, j, k) + NC * l]; }
  double& F(std::vector<double>& a, int i, int j, int k, int n, int l) {
    return a[id(i, j, k) + NC * ((long)n + (long)NFACES * l)];
  }

  int vel(int m) const { return 1 + m; }   // 0-based variable index of velocity slot m

  // ---------------------------------------------------------------- init
  int init(const fgpu_config* c) {
    cfg = *c;
    INUM = cfg.inum; JNUM = cfg.jnum; KNUM = cfg.knum;
    if (INUM < 1 || JNUM < 1 || KNUM < 1) { err = "bad resolution"; return FGPU_EBADCFG; }
    GINUM = INUM > 1 ? 2 : 0; GJNUM = JNUM > 1 ? 2 : 0; GKNUM = KNUM > 1 ? 2 : 0;
    IP1 = INUM > 1; IM1 = -IP1; JP1 = JNUM > 1; JM1 = -JP1; KP1 = KNUM > 1; KM1 = -KP1;
    IMIN = 1; IMAX = INUM; JMIN = 1; JMAX = JNUM; KMIN = 1; KMAX = KNUM;
    IGMIN = IMIN - GINUM; IGMAX = IMAX + GINUM; JGMIN = JMIN - GJNUM; JGMAX = JMAX + GJNUM;
    KGMIN = KMIN - GKNUM; KGMAX = KMAX + GKNUM;
    NI = IGMAX - IGMIN + 1; NJ = JGMAX - JGMIN + 1; NK = KGMAX - KGMIN + 1;
    NC = (long)NI * NJ * NK;
    NDIMS = 0;
    if (INUM > 1) dirs[NDIMS++] = 0;
    if (JNUM > 1) dirs[NDIMS++] = 1;
    if (KNUM > 1) dirs[NDIMS++] = 2;
    if (NDIMS == 0) { err = "no active direction"; return FGPU_EBADCFG; }
    NFACES = 2 * NDIMS;
    VDIM = NDIMS;
    euler = (cfg.physics == FGPU_EULER);
    if (!euler && cfg.physics != FGPU_EULER_ISOTHERM) { err = "unknown physics"; return FGPU_EBADCFG; }
    VNUM = 1 + VDIM + (euler ? 1 : 0);
    PRESSURE = euler ? VNUM - 1 : -1;
    if (cfg.geometry != FGPU_CARTESIAN && cfg.geometry != FGPU_CYLINDRICAL &&
        cfg.geometry != FGPU_LOGCYLINDRICAL) { err = "unsupported geometry"; return FGPU_EUNSUPPORTED; }
    if (cfg.order == FGPU_LINEAR && (cfg.limiter < 1 || cfg.limiter > 8)) { err = "Unknown limiter"; return FGPU_EBADCFG; }
    if (cfg.order == FGPU_LINEAR && cfg.limiter == FGPU_PP) { err = "PP limiter currently not supported."; return FGPU_EUNSUPPORTED; }
    build_mesh();
    // physics arrays
    bccsound.assign(NC, 0.0); fcsound.assign(NC * NFACES, 0.0);
    if (!euler && cfg.csiso > 0.0) { std::fill(bccsound.begin(), bccsound.end(), cfg.csiso);
                                     std::fill(fcsound.begin(), fcsound.end(), cfg.csiso); }
    long NS = NC * VNUM;
    pvar.assign(NS, 0); cvar.assign(NS, 0); ptmp.assign(NS, 0); ctmp.assign(NS, 0); cold.assign(NS, 0);
    rhs.assign(NS, 0); geo_src.assign(NS, 0); src.assign(NS, 0); cerr.assign(NS, 0);
    xflux.assign(NS, 0); yflux.assign(NS, 0); zflux.assign(NS, 0);
    slopes.assign(NC * NDIMS * VNUM, 0.0);
    fprim.assign(NC * NFACES * VNUM, 0); fcons.assign(NC * NFACES * VNUM, 0); pfluxes.assign(NC * NFACES * VNUM, 0);
    minwav.assign(NC * NDIMS, 0); maxwav.assign(NC * NDIMS, 0); tmpw.assign(NC, 0); tmpw1.assign(NC, 0);
    // timedisc (timedisc_base.f90:285-350, timedisc_modeuler.f90:97-123)
    time = cfg.starttime; stoptime = cfg.stoptime; dt = stoptime; dtold = dt; dtmin = dt; dtmincause = -99;
    cfl = cfg.cfl; dtlimit = cfg.dtlimit; tol_rel = cfg.tol_rel; beta = cfg.beta;
    tol_abs.assign(cfg.tol_abs, cfg.tol_abs + VNUM);
    checkdatabm = cfg.checkdata; maxerrold = 0.0; dtcause = 0;
    if (int rc = setup_timedisc()) return rc;
    // sources
    if (cfg.pointmass) { if (int rc = setup_pointmass()) return rc; }
    if (cfg.pm_outbound) {
      if (!cfg.pointmass) { err = "accretion needs the point mass"; return FGPU_EBADCFG; }
      if (cfg.pm_outbound != 1 && cfg.pm_outbound != 2) { err = "accretion through the x boundaries only"; return FGPU_EUNSUPPORTED; }
      if (cfg.geometry != FGPU_CYLINDRICAL && cfg.geometry != FGPU_LOGCYLINDRICAL) { err = "geometry does not support accretion"; return FGPU_EUNSUPPORTED; }
      if (butcher || tol_rel < 1.0) { err = "accretion with the fixed-step modified Euler scheme only"; return FGPU_EUNSUPPORTED; }
      outbound = cfg.pm_outbound;
      bxf.assign((size_t)VNUM * 2 * KNUM * JNUM, 0.0);
      bxo = bxf;
      pm_cur = cfg.pm_mass;
      mdot = 0.0;
    }
    // viscosity (sources_viscosity.f90:132-266)
    if (cfg.vismodel) {
      if (VDIM < 2) { err = "viscosity is currently not supported in 1D physics"; return FGPU_EBADCFG; }
      if (cfg.vismodel < FGPU_VIS_MOLECULAR || cfg.vismodel > FGPU_VIS_ALPHA_ALT) { err = "Viscosity prescription not supported."; return FGPU_EBADCFG; }
      if (cfg.vismodel == FGPU_VIS_ALPHA_ALT) { err = "alternative alpha-viscosity currently not supported"; return FGPU_EUNSUPPORTED; }
      if (cfg.vismodel == FGPU_VIS_ALPHA && euler) { err = "viscosity: ALPHA with isothermal physics only"; return FGPU_EUNSUPPORTED; }
      if (cfg.vismodel != FGPU_VIS_MOLECULAR && cfg.fargo_method) { err = "viscosity: ALPHA/BETA/POWERLAW without fargo"; return FGPU_EUNSUPPORTED; }
      if (NDIMS == 2 && !(dirs[0] == 0 && dirs[1] == 1)) { err = "viscosity: 2D x-y and 3D meshes only"; return FGPU_EUNSUPPORTED; }
      vismodel = cfg.vismodel;
      dynconst = cfg.dynconst;
      bulkconst = std::isnan(cfg.bulkconst) ? -2. / 3. * dynconst : cfg.bulkconst;
      power = cfg.vis_exponent;
      cvis = cfg.cvis;
      dynvis.assign(NC, dynconst); bulkvis.assign(NC, bulkconst); kinvis.assign(NC, 0.0);
      if (vismodel != FGPU_VIS_MOLECULAR) build_ephir();
      btxx.assign(NC, 0.0); btxy.assign(NC, 0.0); btxz.assign(NC, 0.0);
      btyy.assign(NC, 0.0); btyz.assign(NC, 0.0); btzz.assign(NC, 0.0);
      vtmp.assign(NC, 0.0); vtmp1.assign(NC, 0.0); vtmp2.assign(NC, 0.0);
    }
    // fargo (timedisc_base.f90:369-452)
    fargo = cfg.fargo_method;
    if (fargo) {
      // types 1 (w computed every step) and 2 (w supplied by the user, fixed); type 3
      // (shearing box) needs the shearing-box sources
      if (fargo != 1 && fargo != 2) { err = "fargo: types 1 and 2 only"; return FGPU_EUNSUPPORTED; }
      if (euler && (cfg.checkdata & FGPU_CHECK_PMIN)) { err = "fargo with ideal-gas physics: checkdata without CHECK_PMIN"; return FGPU_EUNSUPPORTED; }
      if ((cfg.fargo_direction != 1 && cfg.fargo_direction != 2) || NDIMS < 2) { err = "fargo: directions 1 and 2 only"; return FGPU_EUNSUPPORTED; }
      if (NDIMS != 2 || dirs[0] != 0 || dirs[1] != 1) { err = "fargo: 2D x-y meshes only"; return FGPU_EUNSUPPORTED; }
      fdir = cfg.fargo_direction;
      if (fdir == 1 && outbound) { err = "fargo along x with point-mass accretion"; return FGPU_EUNSUPPORTED; }
      const long nw = (long)(fdir == 1 ? NJ : NI) * NK;   // timedisc_base.f90:377-403
      w.assign(nw, 0.0); wfactor.assign(nw, 0.0); delxy.assign(nw, 0.0);
      shift.assign(nw, 0);
      fdq.assign(NC, 0.0); fdql.assign(NC, 0.0); fflux.assign(NC, 0.0);
      if (fargo == 1) {   // timedisc_base.f90:428-452
        if (fdir == 1) {
          for (int k = KGMIN; k <= KGMAX; ++k)
            for (int j = JGMIN; j <= JGMAX; ++j) {
              long c0 = id(IMIN, j, k);
              double a = fmin2(hfx[c0 * 6 + 2], hfx[c0 * 6 + 3]);
              double b = fmin2(hfx[c0 * 6 + 4], hfx[c0 * 6 + 5]);
              wfactor[widx(j, k)] = fmin2(a, b) / hcx[c0];
            }
        } else {
          for (int k = KGMIN; k <= KGMAX; ++k)
            for (int i = IGMIN; i <= IGMAX; ++i) {
              long c0 = id(i, JMIN, k);
              double a = fmin2(hfy[c0 * 6 + 0], hfy[c0 * 6 + 1]);
              double b = fmin2(hfy[c0 * 6 + 4], hfy[c0 * 6 + 5]);
              wfactor[widx(i, k)] = fmin2(a, b) / hcy[c0];
            }
        }
      }
    }
    return FGPU_OK;
  }

  // scale factors (mesh/geometry_*.f90 ScaleFactors)
  void scale(double x, double y, double z, double& hx, double& hy, double& hz) const {
    (void)y; (void)z;
    switch (cfg.geometry) {
      case FGPU_CYLINDRICAL: hx = 1.0; hy = x; hz = 1.0; break;
      case FGPU_LOGCYLINDRICAL: hx = cfg.gparam * std::exp(x); hy = hx; hz = 1.0; break;
      default: hx = 1.0; hy = 1.0; hz = 1.0;
    }
  }
  void radius_posvec(double x, double y, double z, double& r, double* pv) const {
    switch (cfg.geometry) {
      case FGPU_CYLINDRICAL: r = std::sqrt(x * x + z * z); pv[0] = r; pv[1] = 0.0; pv[2] = z; break;
      case FGPU_LOGCYLINDRICAL: { double rr = cfg.gparam * std::exp(x); r = std::sqrt(rr * rr + z * z);
                                  pv[0] = r; pv[1] = 0.0; pv[2] = z; } break;
      default: r = std::sqrt(x * x + y * y + z * z); pv[0] = x; pv[1] = y; pv[2] = z;
    }
  }

  void build_mesh() {
    // mesh_base.f90:570-601
    dx = (cfg.xmax - cfg.xmin) / INUM; mesh_dx = dx;
    dy = (cfg.ymax - cfg.ymin) / JNUM; mesh_dy = dy;
    dz = (cfg.zmax - cfg.zmin) / KNUM; mesh_dz = dz;
    if (dx < 2 * EPS_) { dx = 1.0; mesh_dx = 0.0; }
    if (dy < 2 * EPS_) { dy = 1.0; mesh_dy = 0.0; }
    if (dz < 2 * EPS_) { dz = 1.0; mesh_dz = 0.0; }
    invdx = 1. / dx; invdy = 1. / dy; invdz = 1. / dz;
    cx.resize(NI); cy.resize(NJ); cz.resize(NK);
    for (int i = IGMIN; i <= IGMAX; ++i) cx[i - IGMIN] = cfg.xmin + ((double)(2 * i - 1) * 0.5) * mesh_dx;
    for (int j = JGMIN; j <= JGMAX; ++j) cy[j - JGMIN] = cfg.ymin + ((double)(2 * j - 1) * 0.5) * mesh_dy;
    for (int k = KGMIN; k <= KGMAX; ++k) cz[k - KGMIN] = cfg.zmin + ((double)(2 * k - 1) * 0.5) * mesh_dz;
    double cf[6][3] = {{-0.5 * mesh_dx, 0, 0}, {0.5 * mesh_dx, 0, 0}, {0, -0.5 * mesh_dy, 0},
                       {0, 0.5 * mesh_dy, 0}, {0, 0, -0.5 * mesh_dz}, {0, 0, 0.5 * mesh_dz}};
    hfx.assign(NC * 6, 0); hfy.assign(NC * 6, 0); hfz.assign(NC * 6, 0);
    hcx.assign(NC, 0); hcy.assign(NC, 0); hcz.assign(NC, 0);
    volume.assign(NC, 0); dxdydV.assign(NC, 0); dydzdV.assign(NC, 0); dzdxdV.assign(NC, 0);
    dlx.assign(NC, 0); dly.assign(NC, 0); dlz.assign(NC, 0);
    cxyx.assign(NC, 0); cxzx.assign(NC, 0); cyxy.assign(NC, 0); cyzy.assign(NC, 0); czxz.assign(NC, 0); czyz.assign(NC, 0);
    dAx.assign(NC * 2, 0); dAy.assign(NC * 2, 0); dAz.assign(NC * 2, 0);
    rdx.assign(NC * NFACES, 0); radius.assign(NC, 0); posvec.assign(NC * 3, 0);
    for (int k = KGMIN; k <= KGMAX; ++k)
      for (int j = JGMIN; j <= JGMAX; ++j)
        for (int i = IGMIN; i <= IGMAX; ++i) {
          long c = id(i, j, k);
          double x = cx[i - IGMIN], y = cy[j - JGMIN], z = cz[k - KGMIN];
          double fx[6], fy[6], fz[6];
          for (int n = 0; n < 6; ++n) { fx[n] = x + cf[n][0]; fy[n] = y + cf[n][1]; fz[n] = z + cf[n][2]; }
          scale(x, y, z, hcx[c], hcy[c], hcz[c]);
          for (int n = 0; n < 6; ++n) scale(fx[n], fy[n], fz[n], hfx[c * 6 + n], hfy[c * 6 + n], hfz[c * 6 + n]);
          double sqrtg = hcx[c] * (hcy[c] * hcz[c]);
          // mesh_midpoint.f90:97-145
          double* hX = &hfx[c * 6]; double* hY = &hfy[c * 6]; double* hZ = &hfz[c * 6];
          dAx[c * 2 + 0] = hY[0] * hZ[0]; dAx[c * 2 + 1] = hY[1] * hZ[1];
          dAy[c * 2 + 0] = hZ[2] * hX[2]; dAy[c * 2 + 1] = hZ[3] * hX[3];
          dAz[c * 2 + 0] = hX[4] * hY[4]; dAz[c * 2 + 1] = hX[5] * hY[5];
          volume[c] = sqrtg * dx * dy * dz;
          dxdydV[c] = dx * dy / (volume[c] + TINY_);
          dydzdV[c] = dy * dz / (volume[c] + TINY_);
          dzdxdV[c] = dz * dx / (volume[c] + TINY_);
          cyxy[c] = 0.5 * (hZ[1] + hZ[0]) * (hY[1] - hY[0]) * dydzdV[c];
          cyzy[c] = 0.5 * (hX[5] + hX[4]) * (hY[5] - hY[4]) * dxdydV[c];
          cxyx[c] = 0.5 * (hZ[3] + hZ[2]) * (hX[3] - hX[2]) * dzdxdV[c];
          cxzx[c] = 0.5 * (hY[5] + hY[4]) * (hX[5] - hX[4]) * dxdydV[c];
          czxz[c] = 0.5 * (hY[1] + hY[0]) * (hZ[1] - hZ[0]) * dydzdV[c];
          czyz[c] = 0.5 * (hX[3] + hX[2]) * (hZ[3] - hZ[2]) * dzdxdV[c];
          dlx[c] = hcx[c] * dx; dly[c] = hcy[c] * dy; dlz[c] = hcz[c] * dz;
          // reconstruction offsets (reconstruction_linear.f90:155-177)
          int m = 0;
          if (INUM > 1) { rdx[c + NC * m] = fx[0] - x; rdx[c + NC * (m + 1)] = fx[1] - x; m += 2; }
          if (JNUM > 1) { rdx[c + NC * m] = fy[2] - y; rdx[c + NC * (m + 1)] = fy[3] - y; m += 2; }
          if (KNUM > 1) { rdx[c + NC * m] = fz[4] - z; rdx[c + NC * (m + 1)] = fz[5] - z; }
          radius_posvec(x, y, z, radius[c], &posvec[c * 3]);
        }
  }

  int setup_timedisc() {
    int method = cfg.method;
    butcher = true;
    switch (method) {
      case FGPU_MODIFIED_EULER:
        butcher = false; order = cfg.tdorder ? cfg.tdorder : 3;
        if (order < 1 || order > 3) { err = "time order must be one of 1,2,3"; return FGPU_EBADCFG; }
        if (order == 1) { tol_rel = 10.0; std::fill(tol_abs.begin(), tol_abs.end(), 1.0); }
        break;
      case FGPU_DORMAND_PRINCE: {
        order = cfg.tdorder ? cfg.tdorder : 5; if (order != 5) { err = "only order 5 supported"; return FGPU_EBADCFG; }
        m_stages = 7;
        double bh[7] = {35./384., 0., 500./1113., 125./192., -2187./6784., 11./84., 0.};
        double bl[7] = {5179./57600., 0., 7571./16695., 393./640., -92097./339200., 187./2100., 1./40.};
        double cc[7] = {0., .2, 3./10., 4./5., 8./9., 1., 1.};
        double a[49] = {0., 0., 0., 0., 0., 0., 0.,
                        .2, 0., 0., 0., 0., 0., 0.,
                        3./40., 9./40., 0., 0., 0., 0., 0.,
                        44./45., -56./15., 32./9., 0., 0., 0., 0.,
                        19372./6561., -25360./2187., 64448./6561., -212./729., 0., 0., 0.,
                        9017./3168., -355./33., 46732./5247., 49./176., -5103./18656., 0., 0.,
                        35./384., 0., 500./1113., 125./192., -2187./6784., 11./84., 0.};
        b_high.assign(bh, bh + 7); b_low.assign(bl, bl + 7); c_coef.assign(cc, cc + 7); A.assign(a, a + 49);
      } break;
      case FGPU_RK_FEHLBERG: {
        order = cfg.tdorder ? cfg.tdorder : 5;
        if (order == 3) {
          m_stages = 3;
          double bh[3] = {1.0/6.0, 2.0/3.0, 1.0/6.0}, bl[3] = {0.0, 1.0, 0.0}, cc[3] = {0.0, 0.5, 1.0};
          double a[9] = {0.0, 0.0, 0.0, 0.5, 0.0, 0.0, -1.0, 2.0, 0.0};
          b_high.assign(bh, bh + 3); b_low.assign(bl, bl + 3); c_coef.assign(cc, cc + 3); A.assign(a, a + 9);
        } else if (order == 5) {
          m_stages = 6;
          double bh[6] = {16.0/135.0, 0.0, 6656.0/12825.0, 28561.0/56430.0, -9.0/50.0, 2.0/55.0};
          double bl[6] = {25.0/216.0, 0.0, 1408.0/2565.0, 2197.0/4104.0, -0.2, 0.0};
          double cc[6] = {0.0, 0.25, 3.0/8.0, 12.0/13.0, 1.0, 0.5};
          double a[36] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
                          0.25, 0.0, 0.0, 0.0, 0.0, 0.0,
                          3.0/32.0, 9.0/32.0, 0.0, 0.0, 0.0, 0.0,
                          1932.0/2197.0, -7200.0/2197.0, 7296.0/2197.0, 0.0, 0.0, 0.0,
                          439.0/216.0, -8.0, 3680.0/513.0, -845.0/4104.0, 0.0, 0.0,
                          -8.0/27.0, 2.0, -3544.0/2565.0, 1859.0/4104.0, -11.0/40.0, 0.0};
          b_high.assign(bh, bh + 6); b_low.assign(bl, bl + 6); c_coef.assign(cc, cc + 6); A.assign(a, a + 36);
        } else { err = "time order must be 3 or 5"; return FGPU_EBADCFG; }
      } break;
      case FGPU_CASH_KARP: {
        order = cfg.tdorder ? cfg.tdorder : 5; if (order != 5) { err = "time order must be 5"; return FGPU_EBADCFG; }
        m_stages = 6;
        double bh[6] = {37.0/378.0, 0.0, 250.0/621.0, 125.0/594.0, 0.0, 512.0/1771.0};
        double bl[6] = {2825.0/27648.0, 0.0, 18575.0/48384.0, 13525.0/55296.0, 277.0/14336.0, 0.25};
        double cc[6] = {0.0, 0.2, 0.3, 0.6, 1.0, 7.0/8.0};
        double a[36] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
                        0.2, 0.0, 0.0, 0.0, 0.0, 0.0,
                        0.075, 0.225, 0.0, 0.0, 0.0, 0.0,
                        0.3, -0.9, 1.2, 0.0, 0.0, 0.0,
                        -11.0/54.0, 2.5, -70.0/27.0, 35.0/27.0, 0.0, 0.0,
                        1631.0/55296.0, 175.0/512.0, 575.0/13824.0, 44275.0/110592.0, 253.0/4096.0, 0.0};
        b_high.assign(bh, bh + 6); b_low.assign(bl, bl + 6); c_coef.assign(cc, cc + 6); A.assign(a, a + 36);
      } break;
      case FGPU_SSPRK: {
        order = cfg.tdorder ? cfg.tdorder : 5;
        if (order == 3) {
          m_stages = 3;
          double bh[3] = {1./6., 1./6., 2./3.}, bl[3] = {0.5, 0.5, 0.}, cc[3] = {0., 1., 0.5};
          double a[9] = {0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.25, 0.25, 0.0};
          b_high.assign(bh, bh + 3); b_low.assign(bl, bl + 3); c_coef.assign(cc, cc + 3); A.assign(a, a + 9);
        } else if (order == 5) {
          m_stages = 5;
          double bh[5] = {0.17279, 0.094505, 0.12947, 0.29899, 0.30424};
          double bl[5] = {0.12293, 0.31981, -0.15316, 0.31887, 0.39155};
          double cc[5] = {0., 0.36717, 0.58522, 0.44156, 0.8464};
          double a[25] = {0., 0., 0., 0., 0.,
                          0.36717, 0., 0., 0., 0.,
                          0.26802, 0.3172, 0., 0., 0.,
                          0.11606, 0.13735, 0.18816, 0., 0.,
                          0.11212, 0.13269, 0.18178, 0.4198, 0.};
          b_high.assign(bh, bh + 5); b_low.assign(bl, bl + 5); c_coef.assign(cc, cc + 5); A.assign(a, a + 25);
        } else { err = "time order must be 3 or 5"; return FGPU_EBADCFG; }
      } break;
      default: err = "unknown timedisc method"; return FGPU_EBADCFG;
    }
    if (butcher) { coeff.assign(m_stages, std::vector<double>(NC * VNUM, 0.0)); }
    return FGPU_OK;
  }

  int setup_pointmass() {
    // gravity_pointmass.f90:263-282 (NEWTON, no softening, point mass at the origin)
    accel.assign(NC * VDIM, 0.0);
    have_accel = true;
    double eps = 0.0, rs = 0.0;
    for (long c = 0; c < NC; ++c) {
      double r = radius[c];
      double om2 = 1. / fmax2(10 * TINY_, ((r * ((r - rs) * (r - rs))) + eps * eps * eps) / (cfg.gn * cfg.pm_mass));
      for (int l = 0; l < VDIM; ++l) accel[c + NC * l] = -om2 * posvec[c * 3 + dirs[l]];
    }
    return FGPU_OK;
  }

  // ---------------------------------------------------------------- physics elementals
  // physics_euler.f90:3033-3117 / physics_eulerisotherm.f90:2820-2892
  void cons2prim(const double* c, double* p) const {
    double inv_rho = 1. / c[0];
    p[0] = c[0];
    if (euler) {
      double s = 0.0;
      if (VDIM == 1) { p[1] = c[1] * inv_rho; p[2] = (cfg.gamma - 1.) * (c[2] - 0.5 * inv_rho * c[1] * c[1]); return; }
      for (int m = 0; m < VDIM; ++m) p[1 + m] = c[1 + m] * inv_rho;
      if (VDIM == 2) s = c[1] * c[1] + c[2] * c[2];
      else s = c[1] * c[1] + c[2] * c[2] + c[3] * c[3];
      p[VNUM - 1] = (cfg.gamma - 1.) * (c[VNUM - 1] - 0.5 * inv_rho * s);
    } else {
      if (VDIM == 1) { p[1] = c[1] / c[0]; return; }
      for (int m = 0; m < VDIM; ++m) p[1 + m] = c[1 + m] * inv_rho;
    }
  }
  void prim2cons(const double* p, double* c) const {
    c[0] = p[0];
    for (int m = 0; m < VDIM; ++m) c[1 + m] = p[0] * p[1 + m];
    if (euler) {
      double s;
      if (VDIM == 1) s = p[1] * p[1];
      else if (VDIM == 2) s = p[1] * p[1] + p[2] * p[2];
      else s = p[1] * p[1] + p[2] * p[2] + p[3] * p[3];
      c[VNUM - 1] = p[VNUM - 1] / (cfg.gamma - 1.) + 0.5 * p[0] * s;
    }
  }
  double soundspeed(double rho, double P) const {   // physics_euler.f90:2682-2689
    return std::sqrt(fmax2(2.0 * TINY_, cfg.gamma * P / rho));
  }
  void c2p_range(std::vector<double>& cv, std::vector<double>& pv, int i1, int i2, int j1, int j2, int k1, int k2) {
    PAR_FOR2
    for (int k = k1; k <= k2; ++k) for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) {
      double c[FGPU_MAXVAR], p[FGPU_MAXVAR];
      long id0 = id(i, j, k);
      for (int l = 0; l < VNUM; ++l) c[l] = cv[id0 + NC * l];
      cons2prim(c, p);
      for (int l = 0; l < VNUM; ++l) pv[id0 + NC * l] = p[l];
    }
  }
  void p2c_range(std::vector<double>& pv, std::vector<double>& cv, int i1, int i2, int j1, int j2, int k1, int k2) {
    PAR_FOR2
    for (int k = k1; k <= k2; ++k) for (int j = j1; j <= j2; ++j) for (int i = i1; i <= i2; ++i) {
      double c[FGPU_MAXVAR], p[FGPU_MAXVAR];
      long id0 = id(i, j, k);
      for (int l = 0; l < VNUM; ++l) p[l] = pv[id0 + NC * l];
      prim2cons(p, c);
      for (int l = 0; l < VNUM; ++l) cv[id0 + NC * l] = c[l];
    }
  }

  // ---------------------------------------------------------------- boundaries
  // boundary_generic.f90:287-418 CenterBoundary
  void center_boundary(std::vector<double>& pv, std::vector<double>& cv) {
    c2p_range(cv, pv, IMIN, IMAX, JMIN, JMAX, KMIN, KMAX);
    pflag(pv) = cflag(cv);
    if (INUM > 1) { set_bc(FGPU_WEST, pv); set_bc(FGPU_EAST, pv); }
    if (JNUM > 1) { set_bc(FGPU_SOUTH, pv); set_bc(FGPU_NORTH, pv); }
    if (KNUM > 1) { set_bc(FGPU_BOTTOM, pv); set_bc(FGPU_TOP, pv); }
    set_corner_edges(pv);
    if (INUM > 1) {
      p2c_range(pv, cv, IGMIN, IMIN - IP1, JGMIN, JGMAX, KGMIN, KGMAX);
      p2c_range(pv, cv, IMAX + IP1, IGMAX, JGMIN, JGMAX, KGMIN, KGMAX);
    }
    if (JNUM > 1) {
      p2c_range(pv, cv, IMIN, IMAX, JGMIN, JMIN - JP1, KGMIN, KGMAX);
      p2c_range(pv, cv, IMIN, IMAX, JMAX + JP1, JGMAX, KGMIN, KGMAX);
    }
    if (KNUM > 1) {
      p2c_range(pv, cv, IMIN, IMAX, JMIN, JMAX, KGMIN, KMIN - KP1);
      p2c_range(pv, cv, IMIN, IMAX, JMIN, JMAX, KMAX + KP1, KGMAX);
    }
  }

  // direction helpers: map (normal index a, transverse b, c) -> (i,j,k)
  void set_bc(int face, std::vector<double>& pv) {
    int type = cfg.bc[face];
    int d = face / 2;               // 0:x 1:y 2:z
    bool lo = (face % 2) == 0;
    int nmin = d == 0 ? IMIN : d == 1 ? JMIN : KMIN;
    int nmax = d == 0 ? IMAX : d == 1 ? JMAX : KMAX;
    int g = d == 0 ? GINUM : d == 1 ? GJNUM : GKNUM;
    // transverse ranges
    int t1lo, t1hi, t2lo, t2hi;
    bool full = (type == FGPU_PERIODIC);
    auto rng = [&](int dd, int& lo_, int& hi_) {
      if (dd == 0) { lo_ = full ? IGMIN : IMIN; hi_ = full ? IGMAX : IMAX; }
      else if (dd == 1) { lo_ = full ? JGMIN : JMIN; hi_ = full ? JGMAX : JMAX; }
      else { lo_ = full ? KGMIN : KMIN; hi_ = full ? KGMAX : KMAX; }
    };
    int da = (d + 1) % 3, db = (d + 2) % 3;
    rng(da, t1lo, t1hi); rng(db, t2lo, t2hi);
    auto at = [&](int n, int a, int b) -> long {
      int ijk[3]; ijk[d] = n; ijk[da] = a; ijk[db] = b; return id(ijk[0], ijk[1], ijk[2]);
    };
    int vn = -1;   // normal velocity slot for direction d
    for (int m = 0; m < NDIMS; ++m) if (dirs[m] == d) vn = vel(m);
    switch (type) {
      case FGPU_PERIODIC:   // boundary_periodic.f90:73-116
        for (int b = t2lo; b <= t2hi; ++b) for (int a = t1lo; a <= t1hi; ++a)
          for (int l = 0; l < VNUM; ++l) for (int s = 1; s <= g; ++s) {
            if (lo) pv[at(nmin - s, a, b) + NC * l] = pv[at(nmax - s + 1, a, b) + NC * l];
            else pv[at(nmax + s, a, b) + NC * l] = pv[at(nmin + s - 1, a, b) + NC * l];
          }
        break;
      case FGPU_REFLECTING:   // boundary_reflecting.f90:89-204
      case FGPU_AXIS:         // boundary_axis.f90: reflecting with AxisMasks (physics_eulerisotherm.f90:1701-1760)
        for (int l = 0; l < VNUM; ++l) {
          // the azimuthal velocity (second coordinate of the curvilinear meshes) is reflected too
          bool refl = (l == vn) || (type == FGPU_AXIS && d == 0 && cfg.geometry != FGPU_CARTESIAN && l == vel(1));
          for (int s = 1; s <= g; ++s)
            for (int b = t2lo; b <= t2hi; ++b) for (int a = t1lo; a <= t1hi; ++a) {
              double v = lo ? pv[at(nmin + s - 1, a, b) + NC * l] : pv[at(nmax - s + 1, a, b) + NC * l];
              pv[at(lo ? nmin - s : nmax + s, a, b) + NC * l] = refl ? -v : v;
            }
        }
        break;
      case FGPU_NO_GRADIENTS:   // boundary_nogradients.f90:75-125
        for (int s = 1; s <= g; ++s)
          for (int b = t2lo; b <= t2hi; ++b) for (int a = t1lo; a <= t1hi; ++a)
            for (int l = 0; l < VNUM; ++l)
              pv[at(lo ? nmin - s : nmax + s, a, b) + NC * l] = pv[at(lo ? nmin : nmax, a, b) + NC * l];
        break;
      case FGPU_ABSORBING:
        absorbing(face, d, lo, nmin, nmax, g, t1lo, t1hi, t2lo, t2hi, da, db, vn, pv);
        break;
      default: break;
    }
  }

  // boundary_absorbing.f90:114-211 with physics CalculateCharSystem*/CalculateBoundaryData*
  // (physics_eulerisotherm.f90:1764-2220, physics_euler.f90:743-1265, elementals :2799-2970)
  void absorbing(int face, int d, bool lo, int nmin, int nmax, int g, int t1lo, int t1hi, int t2lo, int t2hi,
                 int da, int db, int vn, std::vector<double>& pv) {
    (void)face;
    auto at = [&](int n, int a, int b) -> long {
      int ijk[3]; ijk[d] = n; ijk[da] = a; ijk[db] = b; return id(ijk[0], ijk[1], ijk[2]);
    };
    int i1 = lo ? nmin : nmax;           // boundary cell
    int i2 = lo ? nmin + 1 : nmax - 1;   // its interior neighbour
    int iL = std::min(i1, i2), iR = std::max(i1, i2);
    int ig = lo ? nmin - 1 : nmax + 1;   // first ghost cell
    int delta = ig - i1;
    // tangential velocity slots in the order fosite uses (vt ascending)
    int vt[2], nvt = 0;
    for (int m = 0; m < VDIM; ++m) if (vel(m) != vn) vt[nvt++] = vel(m);
    // face slots of direction d (recon/fcsound compressed numbering)
    int slot = 0; for (int m = 0; m < NDIMS; ++m) if (dirs[m] == d) slot = m;
    int fW = 2 * slot, fE = 2 * slot + 1;
    for (int b = t2lo; b <= t2hi; ++b) for (int a = t1lo; a <= t1hi; ++a) {
      long c1 = at(i1, a, b), cL = at(iL, a, b), cR = at(iR, a, b), cg = at(ig, a, b);
      double lam[FGPU_MAXVAR], xv[FGPU_MAXVAR];
      if (!euler) {
        // eigenvalues at i1: (v-cs, v[, v], v+cs)
        double cs = bccsound[c1], v = pv[c1 + NC * vn];
        lam[0] = v - cs; for (int t = 0; t < nvt; ++t) lam[1 + t] = v; lam[VNUM - 1] = v + cs;
        double csf = fcsound[cR + NC * fW];
        double dlnrho = std::log(pv[cR] / pv[cL]);
        double ducs = (pv[cR + NC * vn] - pv[cL + NC * vn]) / csf;
        xv[0] = dlnrho - ducs; xv[VNUM - 1] = dlnrho + ducs;
        for (int t = 0; t < nvt; ++t) xv[1 + t] = pv[cR + NC * vt[t]] - pv[cL + NC * vt[t]];
      } else {
        double gam = cfg.gamma;
        double cs = soundspeed(pv[c1], pv[c1 + NC * PRESSURE]);
        double v = pv[c1 + NC * vn];
        double l1 = v - cs, l3 = v + cs;
        lam[0] = l1; lam[1] = v; for (int t = 0; t < nvt; ++t) lam[2 + t] = v; lam[VNUM - 1] = l3;
        double dlnP = std::log(pv[cR + NC * PRESSURE] / pv[cL + NC * PRESSURE]);
        double gdu = 2 * gam * (pv[cR + NC * vn] - pv[cL + NC * vn]) / (l3 - l1);
        xv[0] = dlnP - gdu;
        xv[1] = dlnP - gam * std::log(pv[cR] / pv[cL]);
        for (int t = 0; t < nvt; ++t) xv[2 + t] = pv[cR + NC * vt[t]] - pv[cL + NC * vt[t]];
        xv[VNUM - 1] = dlnP + gdu;
      }
      for (int l = 0; l < VNUM; ++l) if (lo ? (lam[l] >= 0.0) : (lam[l] <= 0.0)) xv[l] = 0.0;
      if (!euler) {
        double csf = fcsound[c1 + NC * (lo ? fW : fE)];
        double rho1 = pv[c1], u1 = pv[c1 + NC * vn];
        pv[cg] = rho1 * std::exp(delta * 0.5 * (xv[VNUM - 1] + xv[0]));
        pv[cg + NC * vn] = u1 + delta * 0.5 * csf * (xv[VNUM - 1] - xv[0]);
        for (int t = 0; t < nvt; ++t) pv[cg + NC * vt[t]] = pv[c1 + NC * vt[t]] + delta * xv[1 + t];
      } else {
        double gam = cfg.gamma;
        double rho1 = pv[c1], u1 = pv[c1 + NC * vn], P1 = pv[c1 + NC * PRESSURE];
        double dlnP = 0.5 * (xv[VNUM - 1] + xv[0]);
        double rho2 = rho1 * std::exp(delta / gam * (dlnP - xv[1]));
        double P2 = P1 * std::exp(delta * dlnP);
        double cs = soundspeed(rho1 + rho2, P1 + P2);
        pv[cg] = rho2; pv[cg + NC * PRESSURE] = P2;
        pv[cg + NC * vn] = u1 + 0.5 * delta * cs / gam * (xv[VNUM - 1] - xv[0]);
        for (int t = 0; t < nvt; ++t) pv[cg + NC * vt[t]] = pv[c1 + NC * vt[t]] + delta * xv[2 + t];
      }
      for (int s = 2; s <= g; ++s) {
        long co = at(lo ? nmin - s : nmax + s, a, b);
        for (int l = 0; l < VNUM; ++l) pv[co + NC * l] = pv[cg + NC * l];
      }
    }
  }

  // boundary_generic.f90:434-763 SetCornerEdges (serial, GNUM = 2)
  void set_corner_edges(std::vector<double>& pv) {
    const int G = 2;
    auto cp = [&](int i, int j, int k, int i2, int j2, int k2) {
      for (int l = 0; l < VNUM; ++l) pv[id(i, j, k) + NC * l] = pv[id(i2, j2, k2) + NC * l];
    };
    auto avg2 = [&](int i, int j, int k, int ia, int ja, int ka, int ib, int jb, int kb) {
      for (int l = 0; l < VNUM; ++l)
        pv[id(i, j, k) + NC * l] = 0.5 * (pv[id(ia, ja, ka) + NC * l] + pv[id(ib, jb, kb) + NC * l]);
    };
    bool I = INUM != 1, J = JNUM != 1, K = KNUM != 1;
    if (I && J) {   // x-y corners/edges, all k
      for (int k = KGMIN; k <= KGMAX; ++k) {
        for (int j = 1; j <= G; ++j) {   // south-west
          for (int i = j + 1; i <= G; ++i) { cp(IMIN - i, JMIN - j, k, IMIN - i, JMIN - j + 1, k); cp(IMIN - j, JMIN - i, k, IMIN - j + 1, JMIN - i, k); }
          avg2(IMIN - j, JMIN - j, k, IMIN - j, JMIN, k, IMIN, JMIN - j, k);
        }
        for (int j = 1; j <= G; ++j) {   // south-east
          for (int i = j + 1; i <= G; ++i) { cp(IMAX + i, JMIN - j, k, IMAX + i, JMIN - j + 1, k); cp(IMAX + j, JMIN - i, k, IMAX + j - 1, JMIN - i, k); }
          avg2(IMAX + j, JMIN - j, k, IMAX + j, JMIN, k, IMAX, JMIN - j, k);
        }
        for (int j = 1; j <= G; ++j) {   // north-west
          for (int i = j + 1; i <= G; ++i) { cp(IMIN - i, JMAX + j, k, IMIN - i, JMAX + j - 1, k); cp(IMIN - j, JMAX + i, k, IMIN - j + 1, JMAX + i, k); }
          avg2(IMIN - j, JMAX + j, k, IMIN - j, JMAX, k, IMIN, JMAX + j, k);
        }
        for (int j = 1; j <= G; ++j) {   // north-east
          for (int i = j + 1; i <= G; ++i) { cp(IMAX + i, JMAX + j, k, IMAX + i, JMAX + j - 1, k); cp(IMAX + j, JMAX + i, k, IMAX + j - 1, JMAX + i, k); }
          avg2(IMAX + j, JMAX + j, k, IMAX + j, JMAX, k, IMAX, JMAX + j, k);
        }
      }
    }
    if (I && K) {   // x-z, all j
      for (int j = JGMIN; j <= JGMAX; ++j) {
        for (int i = 1; i <= G; ++i) {   // bottom-west
          for (int k = i + 1; k <= G; ++k) { cp(IMIN - i, j, KMIN - k, IMIN - i + 1, j, KMIN - k); cp(IMIN - k, j, KMIN - i, IMIN - k, j, KMIN - i + 1); }
          avg2(IMIN - i, j, KMIN - i, IMIN - i, j, KMIN, IMIN, j, KMIN - i);
        }
        for (int i = 1; i <= G; ++i) {   // bottom-east
          for (int k = i + 1; k <= G; ++k) { cp(IMAX + i, j, KMIN - k, IMAX + i - 1, j, KMIN - k); cp(IMAX + k, j, KMIN - i, IMAX + k, j, KMIN - i + 1); }
          avg2(IMAX + i, j, KMIN - i, IMAX, j, KMIN - i, IMAX + i, j, KMIN);
        }
        for (int i = 1; i <= G; ++i) {   // top-west
          for (int k = i + 1; k <= G; ++k) { cp(IMIN - i, j, KMAX + k, IMIN - i + 1, j, KMAX + k); cp(IMIN - k, j, KMAX + i, IMIN - k, j, KMAX + i - 1); }
          avg2(IMIN - i, j, KMAX + i, IMIN, j, KMAX + i, IMIN - i, j, KMAX);
        }
        for (int i = 1; i <= G; ++i) {   // top-east
          for (int k = i + 1; k <= G; ++k) { cp(IMAX + i, j, KMAX + k, IMAX + i - 1, j, KMAX + k); cp(IMAX + k, j, KMAX + i, IMAX + k, j, KMAX + i - 1); }
          avg2(IMAX + i, j, KMAX + i, IMAX, j, KMAX + i, IMAX + i, j, KMAX);
        }
      }
    }
    if (J && K) {   // y-z, all i
      for (int i = IGMIN; i <= IGMAX; ++i) {
        for (int j = 1; j <= G; ++j) {   // bottom-south
          for (int k = j + 1; k <= G; ++k) { cp(i, JMIN - j, KMIN - k, i, JMIN - j + 1, KMIN - k); cp(i, JMIN - k, KMIN - j, i, JMIN - k, KMIN - j + 1); }
          avg2(i, JMIN - j, KMIN - j, i, JMIN, KMIN - j, i, JMIN - j, KMIN);
        }
        for (int j = 1; j <= G; ++j) {   // bottom-north
          for (int k = j + 1; k <= G; ++k) { cp(i, JMAX + j, KMIN - k, i, JMAX + j - 1, KMIN - k); cp(i, JMAX + k, KMIN - j, i, JMAX + k, KMIN - j + 1); }
          avg2(i, JMAX + j, KMIN - j, i, JMAX, KMIN - j, i, JMAX + j, KMIN);
        }
        for (int j = 1; j <= G; ++j) {   // top-south
          for (int k = j + 1; k <= G; ++k) { cp(i, JMIN - j, KMAX + k, i, JMIN - j + 1, KMAX + k); cp(i, JMIN - k, KMAX + j, i, JMIN - k, KMAX + j - 1); }
          avg2(i, JMIN - j, KMAX + j, i, JMIN, KMAX + j, i, JMIN - j, KMAX);
        }
        for (int j = 1; j <= G; ++j) {   // top-north
          for (int k = j + 1; k <= G; ++k) { cp(i, JMAX + j, KMAX + k, i, JMAX + j - 1, KMAX + k); cp(i, JMAX + k, KMAX + j, i, JMAX + k, KMAX + j - 1); }
          avg2(i, JMAX + j, KMAX + j, i, JMAX, KMAX + j, i, JMAX + j, KMAX);
        }
      }
    }
    if (I && J && K) {   // 3D diagonal corner cells
      auto avg3 = [&](int i, int j, int k, int ia, int ja, int ka, int ib, int jb, int kb, int ic, int jc, int kc) {
        for (int l = 0; l < VNUM; ++l)
          pv[id(i, j, k) + NC * l] = (pv[id(ia, ja, ka) + NC * l] + pv[id(ib, jb, kb) + NC * l] + pv[id(ic, jc, kc) + NC * l]) / 3.0;
      };
      for (int s = 1; s <= G; ++s) {
        avg3(IMIN - s, JMIN - s, KMIN - s, IMIN - s, JMIN, KMIN, IMIN, JMIN - s, KMIN, IMIN, JMIN, KMIN - s);
        avg3(IMAX + s, JMIN - s, KMIN - s, IMAX + s, JMIN, KMIN, IMAX, JMIN - s, KMIN, IMAX, JMIN, KMIN - s);
        avg3(IMIN - s, JMAX + s, KMIN - s, IMIN - s, JMAX, KMIN, IMIN, JMAX + s, KMIN, IMIN, JMAX, KMIN - s);
        avg3(IMAX + s, JMAX + s, KMIN - s, IMAX + s, JMAX, KMIN, IMAX, JMAX + s, KMIN, IMAX, JMAX, KMIN - s);
        avg3(IMIN - s, JMIN - s, KMAX + s, IMIN - s, JMIN, KMAX, IMIN, JMIN - s, KMAX, IMIN, JMIN, KMAX + s);
        avg3(IMAX + s, JMIN - s, KMAX + s, IMAX + s, JMIN, KMAX, IMAX, JMIN - s, KMAX, IMAX, JMIN, KMAX + s);
        avg3(IMIN - s, JMAX + s, KMAX + s, IMIN - s, JMAX, KMAX, IMIN, JMAX + s, KMAX, IMIN, JMAX, KMAX + s);
        avg3(IMAX + s, JMAX + s, KMAX + s, IMAX + s, JMAX, KMAX, IMAX, JMAX + s, KMAX, IMAX, JMAX, KMAX + s);
      }
    }
  }

  // ---------------------------------------------------------------- fargo
  // Add/SubtractBackgroundVelocityX/Y: isothermal physics_eulerisotherm.f90:1229-1413,
  // Euler physics_euler.f90:1955-2047,2109-2203 (the energy first, with the old momentum)
  // w index of a (j,k) row (direction 1) or an (i,k) column (direction 2)
  long widx(int a, int k) const {
    return fdir == 1 ? (long)(a - JGMIN) + (long)NJ * (k - KGMIN) : (long)(a - IGMIN) + (long)NI * (k - KGMIN);
  }
  double wof(int i, int j, int k) const { return w[widx(fdir == 1 ? j : i, k)]; }
  void add_bg(std::vector<double>& pv, std::vector<double>& cv) {
    bool &c_tr = cflag(cv), &p_tr = pflag(pv);
    if (!c_tr) return;
    if (!p_tr) return;
    const int vi = fdir;   // the velocity component along the transport
    for (int k = KGMIN; k <= KGMAX; ++k) for (int j = JGMIN; j <= JGMAX; ++j) for (int i = IGMIN; i <= IGMAX; ++i) {
      long c = id(i, j, k); double wv = wof(i, j, k);
      if (euler) cv[c + NC * PRESSURE] = cv[c + NC * PRESSURE] + wv * (cv[c + NC * vi] + 0.5 * cv[c] * wv);
      pv[c + NC * vi] = pv[c + NC * vi] + wv;
      cv[c + NC * vi] = cv[c + NC * vi] + cv[c] * wv;
    }
    c_tr = false; p_tr = false;
  }
  void sub_bg(std::vector<double>& pv, std::vector<double>& cv) {
    bool &c_tr = cflag(cv), &p_tr = pflag(pv);
    if (c_tr) return;
    if (p_tr) return;
    const int vi = fdir;
    for (int k = KGMIN; k <= KGMAX; ++k) for (int j = JGMIN; j <= JGMAX; ++j) for (int i = IGMIN; i <= IGMAX; ++i) {
      long c = id(i, j, k); double wv = wof(i, j, k);
      if (euler) cv[c + NC * PRESSURE] = cv[c + NC * PRESSURE] - wv * (cv[c + NC * vi] - 0.5 * cv[c] * wv);
      pv[c + NC * vi] = pv[c + NC * vi] - wv;
      cv[c + NC * vi] = cv[c + NC * vi] - cv[c] * wv;
    }
    c_tr = true; p_tr = true;
  }
  // timedisc_base.f90:2243-2326 CalcBackgroundVelocity
  void calc_background_velocity(std::vector<double>& pv, std::vector<double>& cv) {
    add_bg(pv, cv);
    if (fdir == 1) {
      for (int k = KGMIN; k <= KGMAX; ++k) for (int j = JGMIN; j <= JGMAX; ++j) {
        double wf = wfactor[widx(j, k)];
        double wi = 0.0;
        for (int i = IMIN; i <= IMAX; ++i) wi = wi + pv[id(i, j, k) + NC * 1] * wf;
        w[widx(j, k)] = wi / INUM;
      }
      return;
    }
    for (int k = KGMIN; k <= KGMAX; ++k) for (int i = IGMIN; i <= IGMAX; ++i) {
      double wf = wfactor[widx(i, k)];
      double wi = 0.0;
      for (int j = JMIN; j <= JMAX; ++j) wi = wi + pv[id(i, j, k) + NC * 2] * wf;
      w[widx(i, k)] = wi / JNUM;
    }
  }
  // AddFargoSourcesX/Y (x-y momentum): isothermal physics_eulerisotherm.f90:1462-1518,1531-1586;
  // Euler physics_euler.f90:2267-2355,2368-2455 add the energy term -v*(tmp + GetGeometricalSource
  // with vz = P = mz = 0), physics_euler.f90:3128-3147
  void add_fargo_sources(std::vector<double>& pv, std::vector<double>& cv, std::vector<double>& sterm) {
    for (int k = KMIN; k <= KMAX; ++k) for (int j = JMIN; j <= JMAX; ++j) for (int i = IMIN; i <= IMAX; ++i) {
      long c = id(i, j, k);
      if (fdir == 1) {
        if (!euler) {
          sterm[c + NC * 1] = sterm[c + NC * 1] - cv[c + NC * 2] * 0.5 * (w[widx(j + 1, k)] - w[widx(j - 1, k)]) / dly[c];
        } else {
          double tmp = cv[c + NC * 2] * 0.5 * (w[widx(j + 1, k)] - w[widx(j - 1, k)]) / dly[c];
          sterm[c + NC * 1] = sterm[c + NC * 1] - tmp;
          double vx = pv[c + NC * 1], vy = pv[c + NC * 2], my = cv[c + NC * 2];
          double g = my * (cyxy[c] * vy - cxyx[c] * vx) + 0.0 * (czxz[c] * 0.0 - cxzx[c] * vx) + (cyxy[c] + czxz[c]) * 0.0;
          tmp = tmp + g;
          sterm[c + NC * PRESSURE] = sterm[c + NC * PRESSURE] - vx * tmp;
        }
      } else if (!euler) {
        sterm[c + NC * 2] = sterm[c + NC * 2] - cv[c + NC * 1] * 0.5 * (w[widx(i + 1, k)] - w[widx(i - 1, k)]) / dlx[c];
      } else {
        double tmp = cv[c + NC * 1] * 0.5 * (w[widx(i + 1, k)] - w[widx(i - 1, k)]) / dlx[c];
        sterm[c + NC * 2] = sterm[c + NC * 2] - tmp;
        double vx = pv[c + NC * 1], vy = pv[c + NC * 2], mx = cv[c + NC * 1];
        double g = 0.0 * (czyz[c] * 0.0 - cyzy[c] * vy) + mx * (cxyx[c] * vx - cyxy[c] * vy) + (cxyx[c] + czyz[c]) * 0.0;
        tmp = tmp + g;
        sterm[c + NC * PRESSURE] = sterm[c + NC * PRESSURE] - vy * tmp;
      }
    }
  }
  // timedisc_base.f90:1779-1914 FargoAdvectionX
  void fargo_advection_x() {
    for (int k = KGMIN; k <= KGMAX; ++k) for (int j = JGMIN; j <= JGMAX; ++j)
      delxy[widx(j, k)] = w[widx(j, k)] * dt / dlx[id(IMIN, j, k)];
    for (int k = KGMIN; k <= KGMAX; ++k) for (int j = JGMIN; j <= JGMAX; ++j) {
      double d = delxy[widx(j, k)];
      int s = (int)std::lround(d);   // NINT: round half away from zero
      shift[widx(j, k)] = s;
      delxy[widx(j, k)] = d - (double)s;
    }
    for (int l = 0; l < VNUM; ++l) {
      for (int k = KGMIN; k <= KGMAX; ++k) for (int j = JGMIN; j <= JGMAX; ++j)
        fdq[id(IGMIN, j, k)] = cvar[id(IGMIN + 1, j, k) + NC * l] - cvar[id(IGMIN, j, k) + NC * l];
      for (int i = IGMIN + 1; i <= IGMAX - 1; ++i)
        for (int k = KGMIN; k <= KGMAX; ++k) for (int j = JGMIN; j <= JGMAX; ++j) {
          fdq[id(i, j, k)] = cvar[id(i + 1, j, k) + NC * l] - cvar[id(i, j, k) + NC * l];
          double a = fdq[id(i - 1, j, k)], b = fdq[id(i, j, k)];
          if (fsign(1.0, a) * fsign(1.0, b) > 0.) fdql[id(i, j, k)] = fsign(fmin2(std::fabs(a), std::fabs(b)), a);
          else fdql[id(i, j, k)] = 0.;
        }
      for (int i = IMIN - 1; i <= IMAX; ++i)
        for (int k = KGMIN; k <= KGMAX; ++k) for (int j = JGMIN; j <= JGMAX; ++j) {
          double d = delxy[widx(j, k)];
          long c = id(i, j, k);
          if (d > 0.) fflux[c] = cvar[c + NC * l] + .5 * fdql[c] * (1. - d);
          else fflux[c] = cvar[id(i + 1, j, k) + NC * l] - .5 * fdql[id(i + 1, j, k)] * (1. + d);
          cvar[c + NC * l] = cvar[c + NC * l] - d * (fflux[c] - fflux[id(i - 1, j, k)]);
        }
    }
    std::vector<double> row(INUM);
    for (int l = 0; l < VNUM; ++l)
      for (int k = KGMIN; k <= KGMAX; ++k) for (int j = JGMIN; j <= JGMAX; ++j) {
        int s = shift[widx(j, k)];
        for (int i = 0; i < INUM; ++i) row[i] = cvar[id(IMIN + i, j, k) + NC * l];
        for (int i = 0; i < INUM; ++i) {
          // CSHIFT(a, -s): result(i) = a(i - s) (circular)
          int src = ((i - s) % INUM + INUM) % INUM;
          cvar[id(IMIN + i, j, k) + NC * l] = row[src];
        }
      }
  }
  // timedisc_base.f90:1935-2069 FargoAdvectionY
  void fargo_advection_y() {
    for (int k = KGMIN; k <= KGMAX; ++k) for (int i = IGMIN; i <= IGMAX; ++i)
      delxy[widx(i, k)] = w[widx(i, k)] * dt / dly[id(i, JMIN, k)];
    for (int k = KGMIN; k <= KGMAX; ++k) for (int i = IGMIN; i <= IGMAX; ++i) {
      double d = delxy[widx(i, k)];
      int s = (int)std::lround(d);   // NINT: round half away from zero
      shift[widx(i, k)] = s;
      delxy[widx(i, k)] = d - (double)s;
    }
    for (int l = 0; l < VNUM; ++l) {
      for (int k = KGMIN; k <= KGMAX; ++k) for (int i = IGMIN; i <= IGMAX; ++i)
        fdq[id(i, JGMIN, k)] = cvar[id(i, JGMIN + 1, k) + NC * l] - cvar[id(i, JGMIN, k) + NC * l];
      for (int j = JGMIN + 1; j <= JGMAX - 1; ++j)
        for (int k = KGMIN; k <= KGMAX; ++k) for (int i = IGMIN; i <= IGMAX; ++i) {
          fdq[id(i, j, k)] = cvar[id(i, j + 1, k) + NC * l] - cvar[id(i, j, k) + NC * l];
          double a = fdq[id(i, j - 1, k)], b = fdq[id(i, j, k)];
          if (fsign(1.0, a) * fsign(1.0, b) > 0.) fdql[id(i, j, k)] = fsign(fmin2(std::fabs(a), std::fabs(b)), a);
          else fdql[id(i, j, k)] = 0.;
        }
      for (int j = JMIN - 1; j <= JMAX; ++j)
        for (int k = KGMIN; k <= KGMAX; ++k) for (int i = IGMIN; i <= IGMAX; ++i) {
          double d = delxy[widx(i, k)];
          long c = id(i, j, k);
          if (d > 0.) fflux[c] = cvar[c + NC * l] + .5 * fdql[c] * (1. - d);
          else fflux[c] = cvar[id(i, j + 1, k) + NC * l] - .5 * fdql[id(i, j + 1, k)] * (1. + d);
          cvar[c + NC * l] = cvar[c + NC * l] - d * (fflux[c] - fflux[id(i, j - 1, k)]);
        }
    }
    std::vector<double> row(JNUM);
    for (int l = 0; l < VNUM; ++l)
      for (int k = KGMIN; k <= KGMAX; ++k) for (int i = IGMIN; i <= IGMAX; ++i) {
        int s = shift[widx(i, k)];
        for (int j = 0; j < JNUM; ++j) row[j] = cvar[id(i, JMIN + j, k) + NC * l];
        for (int j = 0; j < JNUM; ++j) {
          // CSHIFT(a, -s): result(j) = a(j - s) (circular)
          int src = ((j - s) % JNUM + JNUM) % JNUM;
          cvar[id(i, JMIN + j, k) + NC * l] = row[src];
        }
      }
  }

  // ---------------------------------------------------------------- spatial operator
  double limiter(double a1, double a2) const {   // reconstruction_linear.f90:645-733
    switch (cfg.limiter) {
      case FGPU_MINMOD:
        if (fsign(1.0, a1) * fsign(1.0, a2) > 0) return fsign(fmin2(std::fabs(a1), std::fabs(a2)), a1);
        return 0.;
      case FGPU_SWEBY: case FGPU_SUPERBEE: {
        double p = cfg.limiter == FGPU_SWEBY ? cfg.theta : 2.0;
        if (fsign(1.0, a1) * fsign(1.0, a2) > 0)
          return fsign(fmax2(fmin2(p * std::fabs(a1), std::fabs(a2)), fmin2(std::fabs(a1), p * std::fabs(a2))), a1);
        return 0.;
      }
      case FGPU_OSPRE:
        return 1.5 * a1 * a2 * (a1 + a2) / (a1 * (a1 + 0.5 * a2) + a2 * (a2 + 0.5 * a1) + TINY_);
      case FGPU_VANLEER: {
        double b1 = std::fabs(a1), b2 = std::fabs(a2);
        return (a1 * b2 + a2 * b1) / (b1 + b2 + TINY_);
      }
      case FGPU_NOLIMIT: return 0.5 * (a1 + a2);
      default: return 0.;
    }
  }
  double mc(double qm, double q0, double qp) const {
    double t = cfg.theta;
    double a1 = t * (q0 - qm), a2 = t * (qp - q0), a3 = 0.5 * (qp - qm);
    if (((fsign(1.0, a1) * fsign(1.0, a2)) > 0) && ((fsign(1.0, a2) * fsign(1.0, a3)) > 0))
      return fsign(fmin2(fmin2(std::fabs(a1), std::fabs(a2)), std::fabs(a3)), a1);
    return 0.;
  }

  // reconstruction_linear.f90:215-630
  void calculate_states(std::vector<double>& rv, std::vector<double>& rst) {
    if (cfg.order == FGPU_CONSTANT) {   // reconstruction_constant.f90:74-93
      PAR_FOR3
      for (int l = 0; l < VNUM; ++l) for (int n = 0; n < NFACES; ++n)
        for (long c = 0; c < NC; ++c) rst[c + NC * (n + (long)NFACES * l)] = rv[c + NC * l];
      return;
    }
    for (int m = 0; m < NDIMS; ++m) {
      int d = dirs[m];
      double inv = d == 0 ? invdx : d == 1 ? invdy : invdz;
      long str = d == 0 ? 1 : d == 1 ? NI : (long)NI * NJ;
      int lo_i = IGMIN, hi_i = IGMAX, lo_j = JGMIN, hi_j = JGMAX, lo_k = KGMIN, hi_k = KGMAX;
      if (d == 0) { lo_i = IGMIN + IP1; hi_i = IGMAX + IM1; }
      if (d == 1) { lo_j = JGMIN + 1; hi_j = JGMAX - 1; }
      if (d == 2) { lo_k = KGMIN + 1; hi_k = KGMAX - 1; }
      PAR_FOR2
      for (int l = 0; l < VNUM; ++l)
        for (int k = lo_k; k <= hi_k; ++k) for (int j = lo_j; j <= hi_j; ++j) for (int i = lo_i; i <= hi_i; ++i) {
          long c = id(i, j, k);
          double q0 = rv[c + NC * l], qm = rv[c - str + NC * l], qp = rv[c + str + NC * l];
          double s = (cfg.limiter == FGPU_MONOCENT) ? inv * mc(qm, q0, qp) : inv * limiter(q0 - qm, qp - q0);
          slopes[c + NC * ((long)m + (long)NDIMS * l)] = s;
        }
    }
    PAR_FOR3
    for (int l = 0; l < VNUM; ++l) for (int n = 0; n < NFACES; ++n)
      for (long c = 0; c < NC; ++c)
        rst[c + NC * (n + (long)NFACES * l)] = rv[c + NC * l] + slopes[c + NC * ((long)(n / 2) + (long)NDIMS * l)] * rdx[c + NC * n];
  }

  // fluxes_base.f90:368-397 CalculateFaceData + fluxes_kt.f90:109-208
  void calculate_fluxes(std::vector<double>& pv, std::vector<double>& cv) {
    bool prim_recon = (cfg.variables == FGPU_PRIMITIVE);
    if (prim_recon) {
      calculate_states(pv, fprim);
      PAR_FOR2
      for (int n = 0; n < NFACES; ++n) for (long x = 0; x < NC; ++x) {
        double c[FGPU_MAXVAR], p[FGPU_MAXVAR];
        for (int l = 0; l < VNUM; ++l) p[l] = fprim[x + NC * (n + (long)NFACES * l)];
        prim2cons(p, c);
        for (int l = 0; l < VNUM; ++l) fcons[x + NC * (n + (long)NFACES * l)] = c[l];
      }
    } else {
      calculate_states(cv, fcons);
      PAR_FOR2
      for (int n = 0; n < NFACES; ++n) for (long x = 0; x < NC; ++x) {
        double c[FGPU_MAXVAR], p[FGPU_MAXVAR];
        for (int l = 0; l < VNUM; ++l) c[l] = fcons[x + NC * (n + (long)NFACES * l)];
        cons2prim(c, p);
        for (int l = 0; l < VNUM; ++l) fprim[x + NC * (n + (long)NFACES * l)] = p[l];
      }
    }
    if (euler) {  // UpdateSoundSpeed on faces (physics_euler.f90:2555-2574)
      PAR_FOR2
      for (int n = 0; n < NFACES; ++n) for (long x = 0; x < NC; ++x)
        fcsound[x + NC * n] = soundspeed(fprim[x + NC * (n + (long)NFACES * 0)], fprim[x + NC * (n + (long)NFACES * PRESSURE)]);
    }
    // CalcWaveSpeeds_faces (physics_eulerisotherm.f90:555-686)
    for (int m = 0; m < NDIMS; ++m) {
      int d = dirs[m]; int vi = vel(m);
      long str = d == 0 ? 1 : d == 1 ? NI : (long)NI * NJ;
      int fw = 2 * m, fe = 2 * m + 1;
      PAR_FOR
      for (long x = 0; x < NC; ++x) {
        double cs = fcsound[x + NC * fw], v = fprim[x + NC * (fw + (long)NFACES * vi)];
        tmpw[x] = fmin2(0., v - cs); tmpw1[x] = fmax2(0., v + cs);
        cs = fcsound[x + NC * fe]; v = fprim[x + NC * (fe + (long)NFACES * vi)];
        minwav[x + NC * m] = fmin2(0., v - cs); maxwav[x + NC * m] = fmax2(0., v + cs);
      }
      int lo_i = IGMIN, hi_i = IGMAX, lo_j = JGMIN, hi_j = JGMAX, lo_k = KGMIN, hi_k = KGMAX;
      if (d == 0) { lo_i = IMIN + IM1; hi_i = IMAX; }
      if (d == 1) { lo_j = JMIN + JM1; hi_j = JMAX; }
      if (d == 2) { lo_k = KMIN + KM1; hi_k = KMAX; }
      PAR_FOR2
      for (int k = lo_k; k <= hi_k; ++k) for (int j = lo_j; j <= hi_j; ++j) for (int i = lo_i; i <= hi_i; ++i) {
        long x = id(i, j, k);
        minwav[x + NC * m] = fmin2(fmin2(0.0, tmpw[x + str]), minwav[x + NC * m]);
        maxwav[x + NC * m] = fmax2(fmax2(0.0, tmpw1[x + str]), maxwav[x + NC * m]);
      }
      // physical fluxes on both faces of direction m (CalcFluxes{X,Y,Z})
      PAR_FOR2
      for (int n = fw; n <= fe; ++n) for (long x = 0; x < NC; ++x) {
        auto P = [&](int l) { return fprim[x + NC * (n + (long)NFACES * l)]; };
        auto C = [&](int l) { return fcons[x + NC * (n + (long)NFACES * l)]; };
        double u = P(vi);
        double* f = &pfluxes[x + NC * (long)n];
        long fs = NC * (long)NFACES;
        f[0] = P(0) * u;
        if (euler) {
          double pr = P(PRESSURE);
          for (int t = 0; t < VDIM; ++t) f[fs * (1 + t)] = (1 + t == vi) ? C(vi) * u + pr : C(1 + t) * u;
          f[fs * PRESSURE] = (C(PRESSURE) + pr) * u;
        } else {
          double cs = fcsound[x + NC * n];
          for (int t = 0; t < VDIM; ++t) f[fs * (1 + t)] = (1 + t == vi) ? C(vi) * u + P(0) * cs * cs : C(1 + t) * u;
        }
      }
      // KT (fluxes_kt.f90:126-207)
      std::vector<double>& out = d == 0 ? xflux : d == 1 ? yflux : zflux;
      std::vector<double>& dA = d == 0 ? dAx : d == 1 ? dAy : dAz;
      PAR_FOR2
      for (int l = 0; l < VNUM; ++l)
        for (int k = lo_k; k <= hi_k; ++k) for (int j = lo_j; j <= hi_j; ++j) for (int i = lo_i; i <= hi_i; ++i) {
          long x = id(i, j, k);
          double ap = maxwav[x + NC * m], am = minwav[x + NC * m];
          out[x + NC * l] = dA[(x + str) * 2 + 0] / (ap - am) *
            (ap * pfluxes[x + NC * (fe + (long)NFACES * l)] - am * pfluxes[x + str + NC * (fw + (long)NFACES * l)] +
             am * ap * (fcons[x + str + NC * (fw + (long)NFACES * l)] - fcons[x + NC * (fe + (long)NFACES * l)]));
        }
    }
  }

  // physics GeometricalSources (physics_euler.f90:1706-1847, physics_eulerisotherm.f90:689-832)
  void geometrical_sources(std::vector<double>& pv, std::vector<double>& cv, std::vector<double>& s) {
    if (cfg.geometry == FGPU_CARTESIAN) return;
    if (!(NDIMS == 2 && dirs[0] == 0 && dirs[1] == 1) && NDIMS != 3) return;
    PAR_FOR
    for (long x = 0; x < NC; ++x) {
      double P = euler ? pv[x + NC * PRESSURE] : pv[x] * (bccsound[x] * bccsound[x]);
      double vx = pv[x + NC * 1], vy = pv[x + NC * 2];
      s[x] = 0.0;
      if (euler) s[x + NC * PRESSURE] = 0.0;
      if (NDIMS == 2) {
        double mx = cv[x + NC * 1], my = cv[x + NC * 2];
        s[x + NC * 1] = my * (cyxy[x] * vy - cxyx[x] * vx) + (cyxy[x] + czxz[x]) * P;
        s[x + NC * 2] = mx * (cxyx[x] * vx - cyxy[x] * vy) + (cxyx[x] + czyz[x]) * P;
      } else {
        double vz = pv[x + NC * 3];
        double mx = cv[x + NC * 1], my = cv[x + NC * 2], mz = cv[x + NC * 3];
        s[x + NC * 1] = my * (cyxy[x] * vy - cxyx[x] * vx) + mz * (czxz[x] * vz - cxzx[x] * vx) + (cyxy[x] + czxz[x]) * P;
        s[x + NC * 2] = mz * (czyz[x] * vz - cyzy[x] * vy) + mx * (cxyx[x] * vx - cyxy[x] * vy) + (cxyx[x] + czyz[x]) * P;
        s[x + NC * 3] = mx * (cxzx[x] * vx - czxz[x] * vz) + my * (cyzy[x] * vy - czyz[x] * vz) + (cxzx[x] + cyzy[x]) * P;
      }
    }
    zero_ghosts(s);
  }
  void zero_ghosts(std::vector<double>& s) {
    for (int l = 0; l < VNUM; ++l) for (int k = KGMIN; k <= KGMAX; ++k) for (int j = JGMIN; j <= JGMAX; ++j)
      for (int i = IGMIN; i <= IGMAX; ++i) {
        bool g = i < IMIN || i > IMAX || j < JMIN || j > JMAX || k < KMIN || k > KMAX;
        if (g) s[id(i, j, k) + NC * l] = 0.0;
      }
  }
  // ---------------------------------------------------------------- accretion
  double& BX(std::vector<double>& a, int j, int k, int face, int l) {
    return a[(((size_t)l * 2 + face) * KNUM + (k - KMIN)) * JNUM + (j - JMIN)];
  }
  // timedisc_modeuler.f90:223-236: boundary fluxes follow the stage update of the state,
  // fed by the boundary rows of rhs (ComputeRHS :1224-1231)
  void update_bflux(double e, double dtv) {
    for (int l = 0; l < VNUM; ++l)
      for (int k = KMIN; k <= KMAX; ++k) for (int j = JMIN; j <= JMAX; ++j) {
        BX(bxf, j, k, 0, l) = update_me(e, dtv, BX(bxo, j, k, 0, l), BX(bxf, j, k, 0, l), rhs[id(IMIN - IP1, j, k) + NC * l]);
        BX(bxf, j, k, 1, l) = update_me(e, dtv, BX(bxo, j, k, 1, l), BX(bxf, j, k, 1, l), rhs[id(IMAX + IP1, j, k) + NC * l]);
      }
  }
  // fluxes_base.f90:220-270 GetBoundaryFlux (serial): SUM(SUM(bxflux(J,K,face,:),1),1), density
  double boundary_mass_flux() {
    int face = outbound == 1 ? 0 : 1;
    double tot = 0.0;
    for (int k = KMIN; k <= KMAX; ++k) {
      double sj = 0.0;
      for (int j = JMIN; j <= JMAX; ++j) sj = sj + BX(bxf, j, k, face, 0);
      tot = tot + sj;
    }
    return tot;
  }
  // gravity_pointmass.f90:383-428 UpdateGravity_single (acclimit and switchon disabled)
  void update_gravity() {
    double bflux = boundary_mass_flux();
    double oldmass = pm_cur;
    double dmass = bflux - mdot;
    pm_cur = pm_cur + dmass;
    double massfac = pm_cur / oldmass;
    for (size_t x = 0; x < accel.size(); ++x) accel[x] = accel[x] * massfac;
    mdot = bflux;
  }

  // ---------------------------------------------------------------- viscosity
  // mesh_midpoint.f90:586-630 Divergence3D, arguments in the reference's order
  static double div3d(double aW, double aE, double aS, double aN, double aB, double aT,
                      double dydzdV_, double dxdzdV_, double dxdydV_,
                      double c_xyx, double c_xzx, double c_yxy, double c_zxz,
                      double TxxW, double TxxE, double TxyS, double TxyN, double TxzB, double TxzT,
                      double TyxC, double TzxC, double TyyC, double TzzC) {
    return dydzdV_ * (aE * TxxE - aW * TxxW) + dxdzdV_ * (aN * TxyN - aS * TxyS)
         + dxdydV_ * (aT * TxzT - aB * TxzB) + c_xyx * TyxC + c_xzx * TzxC - c_yxy * TyyC - c_zxz * TzzC;
  }
  // VectorDivergence2D_1 (x-y, mesh_midpoint.f90:156-183) / VectorDivergence3D (:474-502)
  // of the cell-centred vector (ax, ay[, az]) at cell x
  double vector_divergence(long x, const double* ax, const double* ay, const double* az) const {
    const long sy = NI, sz = (long)NI * NJ;
    if (NDIMS == 2)
      return div3d(dAx[x * 2], dAx[x * 2 + 1], dAy[x * 2], dAy[x * 2 + 1], 0.0, 0.0,
                   dydzdV[x], dzdxdV[x], 0.0, 0.0, 0.0, 0.0, 0.0,
                   0.5 * (ax[x - 1] + ax[x]), 0.5 * (ax[x + 1] + ax[x]),
                   0.5 * (ay[x - sy] + ay[x]), 0.5 * (ay[x + sy] + ay[x]),
                   0.0, 0.0, 0.0, 0.0, 0.0, 0.0);
    return div3d(dAx[x * 2], dAx[x * 2 + 1], dAy[x * 2], dAy[x * 2 + 1], dAz[x * 2], dAz[x * 2 + 1],
                 dydzdV[x], dzdxdV[x], dxdydV[x], 0.0, 0.0, 0.0, 0.0,
                 0.5 * (ax[x - 1] + ax[x]), 0.5 * (ax[x + 1] + ax[x]),
                 0.5 * (ay[x - sy] + ay[x]), 0.5 * (ay[x + sy] + ay[x]),
                 0.5 * (az[x - sz] + az[x]), 0.5 * (az[x + sz] + az[x]),
                 0.0, 0.0, 0.0, 0.0);
  }
  // sources_viscosity.f90:186-226: ephi/r (azimuthal unit vector over the distance to the
  // z-axis) from the Cartesian bary centres (Convert2Cartesian, geometry_cylindrical.f90:446-455,
  // geometry_logcylindrical.f90:344-356), converted to curvilinear components
  // (geometry_cylindrical.f90:485-494; identity for Cartesian meshes), the VDIM used ones
  void build_ephir() {
    ephir.assign(NC * VDIM, 0.0);
    for (int k = KGMIN; k <= KGMAX; ++k) for (int j = JGMIN; j <= JGMAX; ++j) for (int i = IGMIN; i <= IGMAX; ++i) {
      long c = id(i, j, k);
      const double x1 = cx[i - IGMIN], x2 = cy[j - JGMIN], x3 = cz[k - KGMIN];
      double X, Y;
      if (cfg.geometry == FGPU_CYLINDRICAL) { X = x1 * std::cos(x2); Y = x1 * std::sin(x2); }
      else if (cfg.geometry == FGPU_LOGCYLINDRICAL) { double r = cfg.gparam * std::exp(x1); X = r * std::cos(x2); Y = r * std::sin(x2); }
      else { X = x1; Y = x2; }
      (void)x3;
      const double r2 = radius[c] * radius[c];
      const double ex = -Y / r2, ey = X / r2, ez = 0.0;
      double e[3];
      if (cfg.geometry == FGPU_CARTESIAN) { e[0] = ex; e[1] = ey; e[2] = ez; }
      else {
        e[0] = ex * std::cos(x2) + ey * std::sin(x2);
        e[1] = -ex * std::sin(x2) + ey * std::cos(x2);
        e[2] = ez;
      }
      for (int l = 0; l < VDIM; ++l) ephir[c + NC * l] = e[dirs[l]];
    }
  }
  // sources_viscosity.f90:359-453 UpdateViscosity: recomputed only when the time differs from
  // the last update's (or is 0); the dynamic viscosity of ALPHA (alpha rho cs^2/|Omega|), BETA
  // (beta rho r^2 |Omega|) and POWERLAW (beta rho (r^2 |Omega|)^q) with Omega = ephi/r . v
  // (Mesh%Omega = 0), and the trace-free bulk viscosity -2/3 eta
  void update_viscosity(double t, std::vector<double>& pv) {
    if (!(t != vis_time || t == 0.0)) return;
    if (vismodel != FGPU_VIS_MOLECULAR) {
      for (long x = 0; x < NC; ++x) {
        double om = ephir[x] * pv[x + NC * 1];
        for (int l = 1; l < VDIM; ++l) om = om + ephir[x + NC * l] * pv[x + NC * (1 + l)];
        om = om + 0.0;
        const double rho = pv[x], r = radius[x];
        double eta;
        if (vismodel == FGPU_VIS_ALPHA) eta = dynconst * rho * (bccsound[x] * bccsound[x]) / std::fabs(om);
        else if (vismodel == FGPU_VIS_BETA) eta = dynconst * rho * (r * r) * std::fabs(om);
        else eta = dynconst * rho * std::pow(r * r * std::fabs(om), power);
        dynvis[x] = eta;
      }
      for (long x = 0; x < NC; ++x) bulkvis[x] = -2. / 3. * dynvis[x];
    }
    vis_time = t;
  }

  // physics_eulerisotherm.f90:1023-1198 CalcStresses (x-y and x-y-z velocities) with the
  // cell values of the dynamic and bulk viscosity
  void calc_stresses(std::vector<double>& pv) {
    const double* vx = &pv[NC * 1];
    const double* vy = &pv[NC * 2];
    const double* vz = NDIMS == 3 ? &pv[NC * 3] : nullptr;
    const long sy = NI, sz = (long)NI * NJ;
    for (int k = KGMIN + KP1; k <= KGMAX - KP1; ++k)
      for (int j = JGMIN + JP1; j <= JGMAX - JP1; ++j)
        for (int i = IGMIN + IP1; i <= IGMAX - IP1; ++i) {
          long x = id(i, j, k);
          vtmp[x] = bulkvis[x] * vector_divergence(x, vx, vy, vz);
        }
    for (int k = KMIN - KP1; k <= KMAX + KP1; ++k)
      for (int j = JMIN - JP1; j <= JMAX + JP1; ++j)
        for (int i = IMIN - IP1; i <= IMAX + IP1; ++i) {
          long x = id(i, j, k);
          const double dynvis = this->dynvis[x];
          if (NDIMS == 2) {
            btxx[x] = dynvis * ((vx[x + 1] - vx[x - 1]) / dlx[x] + 2.0 * cxyx[x] * vy[x]) + vtmp[x];
            btyy[x] = dynvis * ((vy[x + sy] - vy[x - sy]) / dly[x] + 2.0 * cyxy[x] * vx[x]) + vtmp[x];
            btxy[x] = dynvis * (0.5 * ((vy[x + 1] - vy[x - 1]) / dlx[x] + (vx[x + sy] - vx[x - sy]) / dly[x])
                                - cxyx[x] * vx[x] - cyxy[x] * vy[x]);
          } else {
            btxx[x] = dynvis * ((vx[x + 1] - vx[x - 1]) / dlx[x] + 2.0 * cxyx[x] * vy[x] + 2.0 * cxzx[x] * vz[x])
                      + vtmp[x];
            btyy[x] = dynvis * ((vy[x + sy] - vy[x - sy]) / dly[x] + 2.0 * cyxy[x] * vx[x] + 2.0 * cyzy[x] * vz[x])
                      + vtmp[x];
            btzz[x] = dynvis * ((vz[x + sz] - vz[x - sz]) / dlz[x] + 2.0 * czxz[x] * vx[x] + 2.0 * czyz[x] * vy[x])
                      + vtmp[x];
            btxy[x] = dynvis * (0.5 * ((vy[x + 1] - vy[x - 1]) / dlx[x] + (vx[x + sy] - vx[x - sy]) / dly[x])
                                - cxyx[x] * vx[x] - cyxy[x] * vy[x]);
            btxz[x] = dynvis * (0.5 * ((vz[x + 1] - vz[x - 1]) / dlx[x] + (vx[x + sz] - vx[x - sz]) / dlz[x])
                                - czxz[x] * vz[x] - cxzx[x] * vx[x]);
            btyz[x] = dynvis * (0.5 * ((vy[x + sz] - vy[x - sz]) / dlz[x] + (vz[x + sy] - vz[x - sy]) / dly[x])
                                - czyz[x] * vz[x] - cyzy[x] * vy[x]);
          }
        }
  }
  // sources_viscosity.f90:484-507 ExternalSources: CalcStresses, then ViscositySources
  // (physics_eulerisotherm.f90:982-1017 tensor divergence with btyx = btxy etc., mesh_midpoint.f90:
  // 283-323 / 508-580; physics_euler.f90:1887-1943 energy = div(v.T)), added to the list's sterm
  void viscosity_sources(double t, std::vector<double>& pv, std::vector<double>& s) {
    update_viscosity(t, pv);
    calc_stresses(pv);
    const double* vx = &pv[NC * 1];
    const double* vy = &pv[NC * 2];
    const double* vz = NDIMS == 3 ? &pv[NC * 3] : nullptr;
    const long sy = NI, sz = (long)NI * NJ;
    if (euler)   // v.T on the cells the divergence reads
      for (int k = KMIN - KP1; k <= KMAX + KP1; ++k)
        for (int j = JMIN - JP1; j <= JMAX + JP1; ++j)
          for (int i = IMIN - IP1; i <= IMAX + IP1; ++i) {
            long x = id(i, j, k);
            if (NDIMS == 2) {
              vtmp[x] = vx[x] * btxx[x] + vy[x] * btxy[x];
              vtmp1[x] = vx[x] * btxy[x] + vy[x] * btyy[x];
            } else {
              vtmp[x] = vx[x] * btxx[x] + vy[x] * btxy[x] + vz[x] * btxz[x];
              vtmp1[x] = vx[x] * btxy[x] + vy[x] * btyy[x] + vz[x] * btyz[x];
              vtmp2[x] = vx[x] * btxz[x] + vy[x] * btyz[x] + vz[x] * btzz[x];
            }
          }
    for (int k = KMIN; k <= KMAX; ++k) for (int j = JMIN; j <= JMAX; ++j) for (int i = IMIN; i <= IMAX; ++i) {
      long x = id(i, j, k);
      double sv[4];
      if (NDIMS == 2) {
        sv[0] = div3d(dAx[x * 2], dAx[x * 2 + 1], dAy[x * 2], dAy[x * 2 + 1], 0.0, 0.0,
                      dydzdV[x], dzdxdV[x], 0.0, cxyx[x], 0.0, cyxy[x], 0.0,
                      0.5 * (btxx[x - 1] + btxx[x]), 0.5 * (btxx[x + 1] + btxx[x]),
                      0.5 * (btxy[x - sy] + btxy[x]), 0.5 * (btxy[x + sy] + btxy[x]), 0.0, 0.0,
                      btxy[x], 0.0, btyy[x], 0.0);
        sv[1] = div3d(dAx[x * 2], dAx[x * 2 + 1], dAy[x * 2], dAy[x * 2 + 1], 0.0, 0.0,
                      dydzdV[x], dzdxdV[x], 0.0, -cxyx[x], 0.0, -cyxy[x], 0.0,
                      0.5 * (btxy[x - 1] + btxy[x]), 0.5 * (btxy[x + 1] + btxy[x]),
                      0.5 * (btyy[x - sy] + btyy[x]), 0.5 * (btyy[x + sy] + btyy[x]), 0.0, 0.0,
                      btxx[x], 0.0, btxy[x], 0.0);
        if (euler) sv[2] = vector_divergence(x, vtmp.data(), vtmp1.data(), nullptr);
      } else {
        const double aW = dAx[x * 2], aE = dAx[x * 2 + 1], aS = dAy[x * 2], aN = dAy[x * 2 + 1];
        const double aB = dAz[x * 2], aT = dAz[x * 2 + 1];
        sv[0] = div3d(aW, aE, aS, aN, aB, aT, dydzdV[x], dzdxdV[x], dxdydV[x], cxyx[x], cxzx[x], cyxy[x], czxz[x],
                      0.5 * (btxx[x - 1] + btxx[x]), 0.5 * (btxx[x + 1] + btxx[x]),
                      0.5 * (btxy[x - sy] + btxy[x]), 0.5 * (btxy[x + sy] + btxy[x]),
                      0.5 * (btxz[x - sz] + btxz[x]), 0.5 * (btxz[x + sz] + btxz[x]),
                      btxy[x], btxz[x], btyy[x], btzz[x]);
        sv[1] = div3d(aW, aE, aS, aN, aB, aT, dydzdV[x], dzdxdV[x], dxdydV[x], -cxyx[x], cyzy[x], -cyxy[x], czyz[x],
                      0.5 * (btxy[x - 1] + btxy[x]), 0.5 * (btxy[x + 1] + btxy[x]),
                      0.5 * (btyy[x - sy] + btyy[x]), 0.5 * (btyy[x + sy] + btyy[x]),
                      0.5 * (btyz[x - sz] + btyz[x]), 0.5 * (btyz[x + sz] + btyz[x]),
                      btxx[x], btyz[x], btxy[x], btzz[x]);
        sv[2] = div3d(aW, aE, aS, aN, aB, aT, dydzdV[x], dzdxdV[x], dxdydV[x], czyz[x], -cxzx[x], cyzy[x], -czxz[x],
                      0.5 * (btxz[x - 1] + btxz[x]), 0.5 * (btxz[x + 1] + btxz[x]),
                      0.5 * (btyz[x - sy] + btyz[x]), 0.5 * (btyz[x + sy] + btyz[x]),
                      0.5 * (btzz[x - sz] + btzz[x]), 0.5 * (btzz[x + sz] + btzz[x]),
                      btyz[x], btxx[x], btyy[x], btxz[x]);
        if (euler) sv[3] = vector_divergence(x, vtmp.data(), vtmp1.data(), vtmp2.data());
      }
      s[x] = s[x] + 0.0;
      for (int m = 0; m < VDIM; ++m) s[x + NC * (1 + m)] = s[x + NC * (1 + m)] + sv[m];
      if (euler) s[x + NC * PRESSURE] = s[x + NC * PRESSURE] + sv[VDIM];
    }
  }

  // sources_generic.f90:220-261 -> sources_gravity.f90:164-200 -> physics ExternalSources;
  // the list holds gravity first (prepended last, sources_generic.f90:190-199), then viscosity
  void external_sources(double t, std::vector<double>& pv, std::vector<double>& cv, std::vector<double>& s) {
    std::fill(s.begin(), s.end(), 0.0);
    external_gravity(cv, s);
    if (vismodel) viscosity_sources(t, pv, s);
    zero_ghosts(s);
  }
  void external_gravity(std::vector<double>& cv, std::vector<double>& s) {
    if (!have_accel) return;
    if (outbound) update_gravity();
    for (long x = 0; x < NC; ++x) {
      for (int n = 0; n < VDIM; ++n) s[x + NC * (1 + n)] = cv[x] * accel[x + NC * n];
      if (euler) {
        double e;
        if (VDIM == 1) e = cv[x + NC * 1] * accel[x];
        else if (VDIM == 2) e = cv[x + NC * 1] * accel[x] + cv[x + NC * 2] * accel[x + NC * 1];
        else e = cv[x + NC * 1] * accel[x] + cv[x + NC * 2] * accel[x + NC * 1] + cv[x + NC * 3] * accel[x + NC * 2];
        s[x + NC * PRESSURE] = e;
      }
    }
  }

  // timedisc_base.f90:1073-1271 ComputeRHS (rhstype 0) at time t
  void compute_rhs(double t, std::vector<double>& pv, std::vector<double>& cv, int checkbm, std::vector<double>& r) {
    if (fargo) add_bg(pv, cv);
    center_boundary(pv, cv);
    if ((checkbm & FGPU_CHECK_PMIN) && euler) {
      PAR_FOR
      for (long x = 0; x < NC; ++x) pv[x + NC * PRESSURE] = fmax2(pv[x + NC * PRESSURE], cfg.pmin);
      p2c_range(pv, cv, IGMIN, IGMAX, JGMIN, JGMAX, KGMIN, KGMAX);
    }
    if (euler) {  // UpdateSoundSpeed(this%pvar) (always_update_bccsound)
      PAR_FOR
      for (long x = 0; x < NC; ++x) bccsound[x] = soundspeed(pvar[x], pvar[x + NC * PRESSURE]);
    }
    if (checkbm != FGPU_CHECK_NOTHING) check_data(pv, cv, checkbm);
    geometrical_sources(pv, cv, geo_src);
    external_sources(t, pv, cv, src);
    if (fargo) {
      if (cfg.geometry == FGPU_CARTESIAN) std::fill(geo_src.begin(), geo_src.end(), 0.0);
      add_fargo_sources(pv, cv, geo_src);
      sub_bg(pv, cv);
    }
    calculate_fluxes(pv, cv);
    for (int l = 0; l < VNUM; ++l) {   // boundary flux rows
      for (int k = KMIN; k <= KMAX; ++k) for (int j = JMIN; j <= JMAX; ++j) {
        r[id(IMIN - IP1, j, k) + NC * l] = dy * dz * xflux[id(IMIN - IP1, j, k) + NC * l];
        r[id(IMAX + IP1, j, k) + NC * l] = -dy * dz * xflux[id(IMAX, j, k) + NC * l];
      }
      for (int k = KMIN; k <= KMAX; ++k) for (int i = IMIN; i <= IMAX; ++i) {
        r[id(i, JMIN - JP1, k) + NC * l] = dz * dx * yflux[id(i, JMIN - JP1, k) + NC * l];
        r[id(i, JMAX + JP1, k) + NC * l] = -dz * dx * yflux[id(i, JMAX, k) + NC * l];
      }
      for (int j = JMIN; j <= JMAX; ++j) for (int i = IMIN; i <= IMAX; ++i) {
        r[id(i, j, KMIN - KP1) + NC * l] = dx * dy * zflux[id(i, j, KMIN - KP1) + NC * l];
        r[id(i, j, KMAX + KP1) + NC * l] = -dx * dy * zflux[id(i, j, KMAX) + NC * l];
      }
    }
    PAR_FOR2
    for (int l = 0; l < VNUM; ++l)
      for (int k = KMIN; k <= KMAX; ++k) for (int j = JMIN; j <= JMAX; ++j) for (int i = IMIN; i <= IMAX; ++i) {
        long x = id(i, j, k), o = NC * l;
        r[x + o] = dydzdV[x] * (xflux[x + o] - xflux[id(i - IP1, j, k) + o])
                 + dzdxdV[x] * (yflux[x + o] - yflux[id(i, j - JP1, k) + o])
                 + dxdydV[x] * (zflux[x + o] - zflux[id(i, j, k - KP1) + o])
                 - geo_src[x + o] - src[x + o];
      }
  }

  // timedisc_base.f90:1666-1742 CheckData
  void check_data(std::vector<double>& pv, std::vector<double>& cv, int bm) {
    int f = 0;
    if ((bm & FGPU_CHECK_CSOUND)) {
      double mn = HUGE_; for (long x = 0; x < NC; ++x) mn = fmin2(mn, bccsound[x]);
      if (mn <= 0.) f |= FGPU_CHECK_CSOUND;
    }
    if ((bm & FGPU_CHECK_PMIN) && euler) {
      double mn = HUGE_;
      for (int k = KMIN; k <= KMAX; ++k) for (int j = JMIN; j <= JMAX; ++j) for (int i = IMIN; i <= IMAX; ++i)
        mn = fmin2(mn, pv[id(i, j, k) + NC * PRESSURE]);
      if (mn < cfg.pmin) f |= FGPU_CHECK_PMIN;
    }
    if ((bm & FGPU_CHECK_RHOMIN)) {
      double mn = HUGE_;
      for (int k = KMIN; k <= KMAX; ++k) for (int j = JMIN; j <= JMAX; ++j) for (int i = IMIN; i <= IMAX; ++i)
        mn = fmin2(mn, pv[id(i, j, k)]);
      if (mn < cfg.rhomin) f |= FGPU_CHECK_RHOMIN;
    }
    if ((bm & FGPU_CHECK_INVALID)) {
      for (long x = 0; x < NC * VNUM; ++x)
        // timedisc_base.f90:1716-1725: NaN (x /= x) or above HUGE; negative infinity passes
        if (cv[x] != cv[x] || pv[x] != pv[x] || cv[x] > HUGE_ || pv[x] > HUGE_) { f |= FGPU_CHECK_INVALID; break; }
    }
    if (f) { brk = true; checkflags |= f; }
  }

  // timedisc_base.f90:818-909 CalcTimestep
  double calc_timestep() {
    // CalcWaveSpeeds_center on this%pvar with bccsound
    double invdt = 0.0;
    std::vector<double> dls[3] = {dlx, dly, dlz};
    auto amax = [&](long x, int m) {
      double cs = bccsound[x], v = pvar[x + NC * vel(m)];
      double mn = fmin2(0., v - cs), mx = fmax2(0., v + cs);
      return fmax2(mx, -mn);
    };
    if (NDIMS == 1) {
      const std::vector<double>& dl = dls[dirs[0]];
      for (long x = 0; x < NC; ++x) invdt = x == 0 ? amax(x, 0) / dl[x] : fmax2(invdt, amax(x, 0) / dl[x]);
    } else if (NDIMS == 2) {
      const std::vector<double>& d1 = dls[dirs[0]]; const std::vector<double>& d2 = dls[dirs[1]];
      for (long x = 0; x < NC; ++x) {
        double v = amax(x, 0) / d1[x] + amax(x, 1) / d2[x];
        invdt = x == 0 ? v : fmax2(invdt, v);
      }
    } else {
      double ix = 0, iy = 0, iz = 0;
      for (long x = 0; x < NC; ++x) {
        double a = amax(x, 0) / dlx[x], b = amax(x, 1) / dly[x], c = amax(x, 2) / dlz[x];
        if (x == 0) { ix = a; iy = b; iz = c; } else { ix = fmax2(ix, a); iy = fmax2(iy, b); iz = fmax2(iz, c); }
      }
      invdt = fmax2(fmax2(iy, iz), ix);
    }
    double dt_cfl = cfl / invdt;
    dtcause = 0;
    // sources_generic.f90:264-293: the point mass returns HUGE (sources_c_accel.f90:113-126),
    // the viscosity its advection-diffusion limit (sources_viscosity.f90:511-581)
    double dt = dt_cfl;
    if (vismodel) {
      update_viscosity(time, pvar);
      for (long x = 0; x < NC; ++x) kinvis[x] = dynvis[x] / pvar[x];
      double ivis = 0.0;
      for (long x = 0; x < NC; ++x) {
        const double kinvis = this->kinvis[x];
        double v = 0.0;
        for (int m = 0; m < NDIMS; ++m) {
          const double dl = dls[dirs[m]][x];
          const double t = (amax(x, m) + 2.0 * kinvis / dl) / dl;
          v = m == 0 ? t : v + t;
        }
        ivis = x == 0 ? v : fmax2(ivis, v);
      }
      const double dt_new = ivis > TINY_ ? cvis / ivis : HUGE_;
      if (dt_new < dt) dtcause = FGPU_DTCAUSE_VISCOSITY;
      dt = fmin2(dt, dt_new);
    }
    return dt;
  }

  // timedisc_base.f90:1012-1053 ComputeError
  double compute_error(std::vector<double>& hi, std::vector<double>& lo) {
    double maxerr = 0.0;
    for (int l = 0; l < VNUM; ++l) {
      double rel = -HUGE_;
      PAR_FOR
      for (long x = 0; x < NC; ++x) {
        double v = hi[x + NC * l];
        cerr[x + NC * l] = std::fabs(v - lo[x + NC * l]) / (tol_rel * std::fabs(v) + tol_abs[l]);
      }
      for (int k = KMIN; k <= KMAX; ++k) for (int j = JMIN; j <= JMAX; ++j) for (int i = IMIN; i <= IMAX; ++i)
        rel = fmax2(rel, cerr[id(i, j, k) + NC * l]);
      maxerr = l == 0 ? rel : fmax2(maxerr, rel);
    }
    return maxerr;
  }

  // correctly rounded EXP and LOG: evaluated in binary128 and rounded once to double
  // (glibc before 2.28 rounded these correctly; later versions are within 0.52 ulp and
  // differ from the correct rounding for about 1 argument in 1000)
  static double exp_cr(double x) { return (double)expq((__float128)x); }
  static double log_cr(double x) { return (double)logq((__float128)x); }

  // timedisc_base.f90:759-814 AdjustTimestep
  double adjust_timestep(double maxerr, double dtold_) {
    double dtnew, dttmp;
    if (tol_rel >= 1.0) return HUGE_;
    if (maxerr > 0.) dttmp = 0.9 * dtold_ * exp_cr(-log_cr(maxerr) / order);
    else dttmp = 4. * dtold_;
    if (maxerrold > 0.) dtnew = dttmp * exp_cr(-beta * log_cr(maxerrold / maxerr));
    else dtnew = dttmp;
    if (maxerr < 1.0) {
      dtnew = fmin2(dtnew, 4. * dtold_);
      if (dtnew < dtold_) dtcause = FGPU_DTCAUSE_SMALLERR;
    } else {
      if (dtnew > dtold_) dtnew = dttmp;
      dtnew = fmax2(dtnew, 0.25 * dtold_);
    }
    maxerrold = maxerr;
    return dtnew;
  }

  static double update_me(double eta, double dtv, double y0, double yn, double r) {
    return yn - dtv * r + eta * (y0 - yn + dtv * r);   // timedisc_modeuler.f90:279-291
  }

  // timedisc_modeuler.f90:125-195 / timedisc_rkfehlberg.f90:170-268
  void solve_ode(double t0, double& dtv, double& errv) {
    static const double eta[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.5, 0.0}, {0.0, 0.75, 1.0 / 3.0}};  // eta(n,order) = eta[order-1][n-1]
    static const double zeta[3][3] = {{0.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 1.0, 0.5}};
    long NS = NC * VNUM;
    if (!butcher) {
      if (tol_rel >= 1.0) {
        for (int n = 1; n <= order; ++n) {
          double e = eta[order - 1][n - 1];
          PAR_FOR
          for (long x = 0; x < NS; ++x) cvar[x] = update_me(e, dtv, cold[x], cvar[x], rhs[x]);
          if (outbound) update_bflux(e, dtv);
          if (n < order) compute_rhs(t0 + zeta[order - 1][n - 1] * dtv, pvar, cvar, FGPU_CHECK_NOTHING, rhs);
        }
        errv = 0.0; dtv = HUGE_;
      } else {
        std::vector<double>* P[4] = {&pvar, &ptmp, &pvar, &pvar};
        std::vector<double>* C[4] = {&cvar, &ctmp, &cvar, &cvar};
        for (int n = 1; n <= order; ++n) {
          double e = eta[order - 1][n - 1];
          std::vector<double>& cin = *C[n - 1]; std::vector<double>& cout = *C[n];
          PAR_FOR
          for (long x = 0; x < NS; ++x) cout[x] = update_me(e, dtv, cold[x], cin[x], rhs[x]);
          if (n == 2 && order == 3)
            for (long x = 0; x < NS; ++x) ctmp[x] = update_me(eta[1][1], dtv, cold[x], ctmp[x], rhs[x]);
          if (n < order) compute_rhs(t0 + zeta[order - 1][n - 1] * dtv, *P[n], *C[n], FGPU_CHECK_NOTHING, rhs);
        }
        errv = compute_error(cvar, ctmp);
        dtv = adjust_timestep(errv, dtv);
      }
      (void)zeta;
      return;
    }
    // Butcher engine; coeff[0] is this%rhs
    std::vector<double>* K[8];
    K[0] = &rhs;
    for (int m = 1; m < m_stages; ++m) K[m] = &coeff[m];
    for (int m = 2; m <= m_stages; ++m) {
      double a1 = A[(m - 1) * m_stages + 0];
      PAR_FOR
      for (long x = 0; x < NS; ++x) ctmp[x] = cvar[x] - a1 * dtv * (*K[0])[x];
      for (int mm = 2; mm <= m - 1; ++mm) {
        double a = A[(m - 1) * m_stages + (mm - 1)];
        PAR_FOR
        for (long x = 0; x < NS; ++x) ctmp[x] = ctmp[x] - a * dtv * (*K[mm - 1])[x];
      }
      compute_rhs(t0 + c_coef[m - 1] * dtv, ptmp, ctmp, FGPU_CHECK_NOTHING, *K[m - 1]);
    }
    ctmp = cvar;
    for (int m = 1; m <= m_stages; ++m) {
      double bl = b_low[m - 1], bh = b_high[m - 1];
      std::vector<double>& k = *K[m - 1];
      PAR_FOR
      for (long x = 0; x < NS; ++x) {
        ctmp[x] = ctmp[x] - bl * dtv * k[x];
        cvar[x] = cvar[x] - bh * dtv * k[x];
      }
    }
    if (tol_rel <= 1.0) {
      errv = compute_error(cvar, ctmp);
      dtv = adjust_timestep(errv, dtv);
    }
  }

  // timedisc_base.f90:649-750 IntegrationStep
  void integration_step() {
    if (fargo == 1) calc_background_velocity(pvar, cvar);
    if (fargo) sub_bg(pvar, cvar);
    double t = time, d = dt;
    if (d < dtmin && dtcause != FGPU_DTCAUSE_FILEIO) { dtmin = d; dtmincause = dtcause; }
    double dtold_ = 0.0;
    while (!brk && t + d <= time + dt) {
      dtold_ = d;
      double e = 0.0;
      solve_ode(t, d, e);
      last_err = e;
      if (e != e) brk = true;
      else if (e > HUGE_) brk = true;
      else if (e >= 1.0) {   // RejectSolution
        cvar = cold;
        compute_rhs(t, pvar, cvar, FGPU_CHECK_NOTHING, rhs);
        if (outbound) bxf = bxo;   // RejectSolution (timedisc_base.f90:980-1000)
        n_adj++; dtcause = FGPU_DTCAUSE_ERRADJ;
        if (d < dtmin) { dtmin = d; dtmincause = dtcause; }
      } else {               // AcceptSolution
        t = t + dtold_;
        if (t < time + dt) { compute_rhs(t, pvar, cvar, checkdatabm, rhs); cold = cvar; }
        if (outbound) bxo = bxf;   // AcceptSolution (timedisc_base.f90:937-958)
        iter++;
      }
      if (d < dtlimit) brk = true;
    }
    if (!brk) {
      dt = t - time;
      time = t;
      dtold = d;
      if (fargo) {
        center_boundary(pvar, cvar);
        if (fdir == 1) fargo_advection_x();
        else fargo_advection_y();
        c2p_range(cvar, pvar, IGMIN, IGMAX, JGMIN, JGMAX, KGMIN, KGMAX);
        p_trans = c_trans;
        compute_rhs(time, pvar, cvar, checkdatabm, rhs);
      } else {
        compute_rhs(time, pvar, cvar, checkdatabm, rhs);
      }
      cold = cvar;
    }
  }

  // fosite.f90:258-348 FirstStep
  void first_step() {
    iter = 0;
    if (fargo == 1) { center_boundary(pvar, cvar); calc_background_velocity(pvar, cvar); }
    compute_rhs(time, pvar, cvar, FGPU_CHECK_ALL, rhs);
    dt = calc_timestep();
    cold = cvar;
  }

  // fosite.f90:367-464 Step (datafile time = tout)
  int step() {
    if (iter == -1) first_step();
    if (std::fabs(stoptime - time) <= 1.0E-05 * stoptime) return FGPU_STOPTIME;
    double tout = cfg.tout > 0 ? cfg.tout : stoptime;
    if ((time + dt) / tout > 1.0) { dt = tout - time; dtcause = FGPU_DTCAUSE_FILEIO; }
    else if ((time + 1.5 * dt) / tout > 1.0) { dt = 0.5 * (tout - time); dtcause = FGPU_DTCAUSE_FILEIO; }
    integration_step();
    if (brk) return FGPU_BREAK;
    dt = calc_timestep();
    return FGPU_OK;
  }
};

}  // namespace

extern "C" {

typedef struct orc_handle { Oracle o; } orc_handle;

int orc_create(const fgpu_config* cfg, orc_handle** out) {
  orc_handle* h = new orc_handle();
  int rc = h->o.init(cfg);
  if (rc) { delete h; *out = nullptr; return rc; }
  *out = h;
  return 0;
}
void orc_destroy(orc_handle* h) { delete h; }
// host threads of the data-parallel loops (1 = the serial restatement); returns the count in use
int orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}
int64_t orc_cell_count(orc_handle* h) { return h->o.NC; }
int orc_vnum(orc_handle* h) { return h->o.VNUM; }
int orc_nfaces(orc_handle* h) { return h->o.NFACES; }

int orc_get_mesh(orc_handle* h, int which, double* out) {
  Oracle& o = h->o;
  for (int k = o.KGMIN; k <= o.KGMAX; ++k) for (int j = o.JGMIN; j <= o.JGMAX; ++j) for (int i = o.IGMIN; i <= o.IGMAX; ++i) {
    long c = o.id(i, j, k);
    switch (which) {
      case FGPU_MESH_X: out[c] = o.cx[i - o.IGMIN]; break;
      case FGPU_MESH_Y: out[c] = o.cy[j - o.JGMIN]; break;
      case FGPU_MESH_Z: out[c] = o.cz[k - o.KGMIN]; break;
      case FGPU_MESH_RADIUS: out[c] = o.radius[c]; break;
      default: return FGPU_EARG;
    }
  }
  return 0;
}
int orc_set_sound_speeds(orc_handle* h, const double* bcc, const double* fcs) {
  Oracle& o = h->o;
  std::memcpy(o.bccsound.data(), bcc, sizeof(double) * o.NC);
  std::memcpy(o.fcsound.data(), fcs, sizeof(double) * o.NC * o.NFACES);
  return 0;
}
// Timedisc%w of FARGO type 2 (user supplied, timedisc_base.f90:421-424), by padded i
// (direction 2) or padded j (direction 1)
int orc_set_fargo_velocity(orc_handle* h, const double* w, int64_t n) {
  Oracle& o = h->o;
  if (o.fargo != 2 || n < (int64_t)o.w.size()) return FGPU_EARG;
  std::memcpy(o.w.data(), w, sizeof(double) * o.w.size());
  return 0;
}
int orc_set_state(orc_handle* h, int which, const double* data) {
  Oracle& o = h->o;
  long n = o.NC * o.VNUM;
  if (which == FGPU_CVAR) { std::memcpy(o.cvar.data(), data, sizeof(double) * n); o.c2p_range(o.cvar, o.pvar, o.IGMIN, o.IGMAX, o.JGMIN, o.JGMAX, o.KGMIN, o.KGMAX); }
  else if (which == FGPU_PVAR) { std::memcpy(o.pvar.data(), data, sizeof(double) * n); o.p2c_range(o.pvar, o.cvar, o.IGMIN, o.IGMAX, o.JGMIN, o.JGMAX, o.KGMIN, o.KGMAX); }
  else return FGPU_EARG;
  return 0;
}
int orc_get(orc_handle* h, int which, double* out) {
  Oracle& o = h->o;
  long n = o.NC * o.VNUM;
  switch (which) {
    case FGPU_CVAR: std::memcpy(out, o.cvar.data(), sizeof(double) * n); break;
    case FGPU_PVAR: std::memcpy(out, o.pvar.data(), sizeof(double) * n); break;
    case FGPU_RHS: std::memcpy(out, o.rhs.data(), sizeof(double) * n); break;
    case FGPU_BCCSOUND: std::memcpy(out, o.bccsound.data(), sizeof(double) * o.NC); break;
    case FGPU_XFLUX: std::memcpy(out, o.xflux.data(), sizeof(double) * n); break;
    case FGPU_YFLUX: std::memcpy(out, o.yflux.data(), sizeof(double) * n); break;
    case FGPU_ZFLUX: std::memcpy(out, o.zflux.data(), sizeof(double) * n); break;
    default: return FGPU_EARG;
  }
  return 0;
}
int orc_first_step(orc_handle* h) { h->o.first_step(); return h->o.brk ? FGPU_BREAK : 0; }
int orc_step(orc_handle* h) { return h->o.step(); }
int orc_compute_rhs(orc_handle* h) { h->o.compute_rhs(h->o.time, h->o.pvar, h->o.cvar, FGPU_CHECK_NOTHING, h->o.rhs); return 0; }
double orc_calc_timestep(orc_handle* h) { return h->o.calc_timestep(); }
int orc_get_status(orc_handle* h, fgpu_status* st) {
  Oracle& o = h->o;
  std::memset(st, 0, sizeof(*st));
  st->time = o.time; st->dt = o.dt; st->dtold = o.dtold; st->dtmin = o.dtmin; st->maxerr = o.last_err;
  st->iter = o.iter; st->n_adj = o.n_adj; st->dtcause = o.dtcause; st->brk = o.brk; st->checkflags = o.checkflags;
  return 0;
}
const char* orc_error(orc_handle* h) { return h ? h->o.err.c_str() : ""; }
int orc_get_pointmass(orc_handle* h, double* mass, double* mdot) {
  *mass = h->o.outbound ? h->o.pm_cur : h->o.cfg.pm_mass;
  *mdot = h->o.mdot;
  return 0;
}

}  // extern "C"
