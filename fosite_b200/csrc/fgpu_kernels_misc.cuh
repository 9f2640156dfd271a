// fgpu_kernels_misc.cuh -- boundary-cell CFL/CheckData reduction with the
// step finalisation, interior CFL pass, and the padded download kernel.
#pragma once
#include "fgpu_kernels.cuh"

namespace fgpu {

enum { FIN_NONE = 0, FIN_FIRST = 1, FIN_STEP = 2 };

struct BndArgs {
  Grid g;
  PhysP ph;
  MetricP mt;
  StateRef in;
  int roundtrip;
  int checkdata;
  Ctl* ctl;
  int finalize;
  long long nghost;
  double* out_p;   // optional: padded primitive output (ghost cells)
  double* out_c;   // optional: padded conservative output (ghost cells)
  long long npad;  // padded cell count (field stride of out_p/out_c)
  // FARGO: background velocity subtracted after the boundary fill (the co-moving
  // frame that CalcTimestep and the caller's cvar/pvar see); null = off
  const double* w_sub;
  int gate;        // device-clock attempt slots (ACT_* bits)
};

// FARGO frame of a checked cell (i, j): the real-frame p/c computed from the state go to
// the co-moving frame, SubtractBackgroundVelocityX/Y (physics_eulerisotherm.f90:1339-1413)
template <int ND, bool EU>
__device__ __forceinline__ void to_comoving(const double* w_sub, const Grid& g, int i, int j, double* p, double* c) {
  if (ND == 2 && w_sub) {
    double w = w_sub[fargo_ix(g, i, j)];
    sub_velocity(p, w, g.fdir);
    frame_change<Phys<ND, EU>::V>(c, -1.0, w, g.fdir);
  }
}

// ghost cell number t -> padded coordinates (x slabs, then y slabs, then z slabs)
template <int ND>
__device__ __forceinline__ void ghost_coords(const Grid& g, long long t, int& px, int& py, int& pz) {
  const int NXp = g.nx + 4, NYp = g.ny + 4, NZp = ND == 3 ? g.nz + 4 : 1;
  long long nxs = 4LL * NYp * NZp;
  if (t < nxs) {
    int q = (int)(t % 4); long long r = t / 4;
    px = q < 2 ? q : NXp - 4 + q;
    py = (int)(r % NYp); pz = (int)(r / NYp);
    return;
  }
  t -= nxs;
  long long nys = 4LL * g.nx * NZp;
  if (t < nys) {
    int q = (int)(t % 4); long long r = t / 4;
    py = q < 2 ? q : NYp - 4 + q;
    px = 2 + (int)(r % g.nx); pz = (int)(r / g.nx);
    return;
  }
  t -= nys;
  int q = (int)(t % 4); long long r = t / 4;
  pz = q < 2 ? q : NZp - 4 + q;
  px = 2 + (int)(r % g.nx); py = 2 + (int)(r / g.nx);
}

// The step's closing scalar work, run by the last block of the boundary pass:
// CalcTimestep (timedisc_base.f90:818-909), the time advance of IntegrationStep
// (timedisc_base.f90:714-720), the stop test of fosite%Step (fosite.f90:383-388)
// and the output-time clip of fileio%AdjustTimestep (io/fileio_base.f90:604-621).
template <int ND>
__device__ void finalize_step(Ctl* c, int mode) {
  if (mode == FIN_STEP) {
    c->time = c->time + c->dt;
    c->dtold = c->dt;
    c->iter += 1;
  }
  if (c->flags) c->brk = 1;
  double invdt;
  if (ND == 2) invdt = __longlong_as_double((long long)c->invdt[0]);
  else {
    double ix = __longlong_as_double((long long)c->invdt[0]);
    double iy = __longlong_as_double((long long)c->invdt[1]);
    double iz = __longlong_as_double((long long)c->invdt[2]);
    invdt = dmax(dmax(iy, iz), ix);
  }
  const double ivis = __longlong_as_double((long long)c->invdt[3]);
  c->invdt[0] = c->invdt[1] = c->invdt[2] = c->invdt[3] = 0ULL;
  if (c->brk) { c->stop = 1; return; }
  double dt = c->cfl / invdt;
  int cause = 0;
  if (c->vis) {
    // sources list (sources_generic.f90:264-293): the viscous limit (sources_viscosity.f90:
    // 576-580) replaces dt where smaller, with dtcause = VISCOSITY
    const double dtv = ivis > DBL_MIN ? c->cvis / ivis : DBL_MAX;
    if (dtv < dt) cause = 3;
    dt = dmin(dt, dtv);
  }
  if (fabs(c->stoptime - c->time) <= 1.0E-05 * c->stoptime) { c->stop = 1; c->dt = dt; c->dtcause = cause; return; }
  double tout = c->tout;
  if ((c->time + dt) / tout > 1.0) { dt = tout - c->time; cause = -4; }
  else if ((c->time + 1.5 * dt) / tout > 1.0) { dt = 0.5 * (tout - c->time); cause = -4; }
  if (dt < c->dtmin && cause != -4) c->dtmin = dt;
  c->dt = dt;
  c->dtcause = cause;
}

// Block blk of nblk (256 threads each) of the ghost-cell pass of one grid.
template <int ND, bool EU>
__device__ __forceinline__ void boundary_block(const BndArgs& A, const int blk, const int nblk) {
  using PH = Phys<ND, EU>;
  using CE = Cells<ND, EU>;
  constexpr int V = PH::V;
  __shared__ double sred[RED_STRIDE * 8];
  __shared__ bool is_last;
  if (A.ctl && A.finalize != FIN_FIRST && (A.ctl->stop | A.ctl->brk)) return;
  if (gated_out(A.ctl, A.gate)) return;
  const MetricP& M = A.mt;
  double cflv[4] = {0.0, 0.0, 0.0, 0.0};
  int flags = 0;
  for (long long t = blk * 256LL + threadIdx.x; t < A.nghost; t += nblk * 256LL) {
    int px, py, pz;
    ghost_coords<ND>(A.g, t, px, py, pz);
    double p[V], c[V];
    CE::cell_p(A.in, A.g, A.ph, M, px - 2, py - 2, ND == 3 ? pz - 2 : 0, p);
    if (EU && A.roundtrip) p[V - 1] = dmax(p[V - 1], A.ph.pmin);
    PH::p2c(p, c, A.ph);
    double cs = EU ? PH::cs_of(p, A.ph) : M.cs[px];
    if ((A.checkdata & 0x01) && !(cs > 0.)) flags |= 0x01;
    if (A.checkdata & 0x08)
      for (int v = 0; v < V; ++v) if (invalid_value(p[v]) || invalid_value(c[v])) flags |= 0x08;
    to_comoving<ND, EU>(A.w_sub, A.g, px - 2, py - 2, p, c);
    double v3[4];
    CE::cfl_cell(p, cs, M, px, v3);
#pragma unroll
    for (int q = 0; q < 4; ++q) cflv[q] = dmax(cflv[q], v3[q]);
    if (A.out_p) {
      long long pi = px + (long long)(A.g.nx + 4) * (py + (long long)(A.g.ny + 4) * pz);
      for (int v = 0; v < V; ++v) {
        A.out_p[v * A.npad + pi] = p[v];
        A.out_c[v * A.npad + pi] = c[v];
      }
    }
  }
  if (!A.ctl) return;
  block_reduce_emit<256>(cflv, M.vis ? 4 : (ND == 3 ? 3 : 1), flags, A.ctl->invdt, &A.ctl->flags, sred);
  if (A.finalize == FIN_NONE) return;
  __threadfence();
  if (threadIdx.x == 0) {
    unsigned int done = atomicAdd(&A.ctl->blocks_done, 1u);
    is_last = (done == (unsigned)nblk - 1);
  }
  __syncthreads();
  if (is_last && threadIdx.x == 0) {
    __threadfence();
    A.ctl->blocks_done = 0;
    finalize_step<ND>(A.ctl, A.finalize);
  }
}

template <int ND, bool EU>
__global__ void __launch_bounds__(256) boundary_kernel(const __grid_constant__ BndArgs A) {
  boundary_block<ND, EU>(A, blockIdx.x, gridDim.x);
}

// Batched ensemble: block b runs block (y) of (z) of grid (x) of entry b.
template <int ND, bool EU>
__global__ void __launch_bounds__(256) batched_boundary_kernel(const BndArgs* __restrict__ args,
                                                               const int4* __restrict__ blocks) {
  const int4 T = blocks[blockIdx.x];
  boundary_block<ND, EU>(args[T.x], T.y, T.z);
}

// CFL and CheckData of the interior cells of a stored state (FirstStep).
template <int ND, bool EU>
__global__ void __launch_bounds__(256) interior_cfl_kernel(const __grid_constant__ BndArgs A) {
  using PH = Phys<ND, EU>;
  using CE = Cells<ND, EU>;
  constexpr int V = PH::V;
  __shared__ double sred[RED_STRIDE * 8];
  const MetricP& M = A.mt;
  double cflv[4] = {0.0, 0.0, 0.0, 0.0};
  int flags = 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < A.g.n;
       t += (long long)gridDim.x * blockDim.x) {
    int i = (int)(t % A.g.nx);
    const int j = (int)((t / A.g.nx) % A.g.ny);
    double u[V], p[V], c[V];
    state_at<V>(A.in, A.g.n, t, u);
    if (ND == 2 && A.in.pre.n) apply_chain<V>(A.in.pre, u, A.g, i, j);
    PH::c2p(u, p, A.ph);
    if (EU && A.roundtrip) { p[V - 1] = dmax(p[V - 1], A.ph.pmin); PH::p2c(p, c, A.ph); }
    else { for (int v = 0; v < V; ++v) c[v] = u[v]; }
    double cs = EU ? PH::cs_of(p, A.ph) : M.cs[i + 2];
    if ((A.checkdata & 0x01) && !(cs > 0.)) flags |= 0x01;
    if (EU && (A.checkdata & 0x02) && p[V - 1] < A.ph.pmin) flags |= 0x02;
    if ((A.checkdata & 0x04) && p[0] < A.ph.rhomin) flags |= 0x04;
    if (A.checkdata & 0x08)
      for (int v = 0; v < V; ++v) if (invalid_value(p[v]) || invalid_value(c[v])) flags |= 0x08;
    to_comoving<ND, EU>(A.w_sub, A.g, i, j, p, c);
    double v3[4];
    CE::cfl_cell(p, cs, M, i + 2, v3);
#pragma unroll
    for (int q = 0; q < 4; ++q) cflv[q] = dmax(cflv[q], v3[q]);
  }
  block_reduce_emit<256>(cflv, M.vis ? 4 : (ND == 3 ? 3 : 1), flags, A.ctl->invdt, &A.ctl->flags, sred);
}

// Interior cells of a stored state into padded primitive/conservative arrays.
template <int ND, bool EU>
__global__ void __launch_bounds__(256) pack_interior_kernel(const __grid_constant__ BndArgs A) {
  using PH = Phys<ND, EU>;
  constexpr int V = PH::V;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < A.g.n;
       t += (long long)gridDim.x * blockDim.x) {
    int i = (int)(t % A.g.nx);
    long long r = t / A.g.nx;
    int j = (int)(r % A.g.ny), k = (int)(r / A.g.ny);
    double u[V], p[V], c[V];
    state_at<V>(A.in, A.g.n, t, u);
    if (ND == 2 && A.in.pre.n) apply_chain<V>(A.in.pre, u, A.g, i, j);
    PH::c2p(u, p, A.ph);
    if (EU && A.roundtrip) { p[V - 1] = dmax(p[V - 1], A.ph.pmin); PH::p2c(p, c, A.ph); }
    else { for (int v = 0; v < V; ++v) c[v] = u[v]; }
    to_comoving<ND, EU>(A.w_sub, A.g, i, j, p, c);
    int kk = ND == 3 ? k + 2 : 0;
    long long pi = (i + 2) + (long long)(A.g.nx + 4) * ((j + 2) + (long long)(A.g.ny + 4) * kk);
    for (int v = 0; v < V; ++v) {
      A.out_p[v * A.npad + pi] = p[v];
      A.out_c[v * A.npad + pi] = c[v];
    }
  }
}

// Interior cells of a ghost-padded caller array into the stored state
// (fgpu_upload_state); primitive input is converted with Prim2Cons.
template <int ND, bool EU>
__global__ void __launch_bounds__(256) unpack_kernel(const double* __restrict__ pad, double* __restrict__ out,
                                                     Grid g, long long npad, int prim, PhysP P) {
  using PH = Phys<ND, EU>;
  constexpr int V = PH::V;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < g.n; t += (long long)gridDim.x * blockDim.x) {
    int i = (int)(t % g.nx);
    long long r = t / g.nx;
    int j = (int)(r % g.ny), k = (int)(r / g.ny);
    int kk = ND == 3 ? k + 2 : 0;
    long long pi = (i + 2) + (long long)(g.nx + 4) * ((j + 2) + (long long)(g.ny + 4) * kk);
    double u[V], c[V];
    for (int v = 0; v < V; ++v) u[v] = pad[v * npad + pi];
    if (prim) PH::p2c(u, c, P);
    else for (int v = 0; v < V; ++v) c[v] = u[v];
    for (int v = 0; v < V; ++v) out[v * g.n + t] = c[v];
  }
}

// Point-mass accretion after a Shu-Osher stage of a 2D grid: the boundary fluxes
// follow the stage update of the state (timedisc_modeuler.f90:223-236, the same
// update formula), then the next ComputeRHS's UpdateGravity
// (gravity_pointmass.f90:383-428, acclimit and switch-on disabled): the face sum
// of the accumulated mass flux in j order (fluxes_base.f90:220-270), the mass
// change against the last sum, and the acceleration scaled in place by
// new/old mass.  One block; grav = [mass, mdot].
struct AccArgs {
  double* bx;          // accumulated boundary mass flux, by j
  double* bxold;       // value at the last accepted step
  const double* brow;  // boundary row of the stage's RHS, by j
  int ny;
  double eta;
  const double* dt;
  int last;            // last stage: AcceptSolution's bxfold = bxflux
  double* grav;
  double* accel;       // point-mass acceleration, naccel values
  int naccel;
  Ctl* ctl;
};
__global__ void __launch_bounds__(256) accrete_kernel(const __grid_constant__ AccArgs A) {
  __shared__ double s_fac;
  if (A.ctl && (A.ctl->stop | A.ctl->brk)) return;
  const double dt = *A.dt;
  for (int j = threadIdx.x; j < A.ny; j += blockDim.x) {
    const double y0 = A.bxold[j], yn = A.bx[j], r = A.brow[j];
    const double y = yn - dt * r + A.eta * (y0 - yn + dt * r);
    A.bx[j] = y;
    if (A.last) A.bxold[j] = y;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sj = 0.0;
    for (int j = 0; j < A.ny; ++j) sj = sj + A.bx[j];
    const double bflux = 0.0 + sj;
    const double oldmass = A.grav[0];
    const double dmass = bflux - A.grav[1];
    const double mass = oldmass + dmass;
    A.grav[0] = mass;
    A.grav[1] = bflux;
    s_fac = mass / oldmass;
  }
  __syncthreads();
  const double f = s_fac;
  for (int q = threadIdx.x; q < A.naccel; q += blockDim.x) A.accel[q] = A.accel[q] * f;
}

// The end of a Butcher attempt as a streaming pass (timedisc_rkfehlberg.f90:198-265 and
// ComputeError, timedisc_base.f90:1012-1053): high and low order solutions
// base - sum b_q dt k_q in the reference's order, the high one written as the new
// state, max |h-l|/(tol_rel|h| + tol_abs) reduced into ctl->err.  Same arithmetic as
// the fused last-stage epilogue of the stage kernel.
struct CombineArgs {
  const double* base;
  const double* K[FGPU_MAXK];
  double bh_dt[FGPU_MAXK], bl_dt[FGPU_MAXK];
  int nstage;
  double* out_high;
  double tol_rel;
  double tol_abs[FGPU_MAXV];
  long long n;
  Ctl* ctl;
  const double* dt_dev;   // device clock: bh_dt/bl_dt hold the weights, times *dt_dev
  int gate;
};
template <int V>
__global__ void __launch_bounds__(256) combine_kernel(const __grid_constant__ CombineArgs A) {
  __shared__ double sred[RED_STRIDE * 8];
  if (A.gate && (A.ctl->stop | A.ctl->brk)) return;
  if (gated_out(A.ctl, A.gate)) return;
  double bh[FGPU_MAXK], bl[FGPU_MAXK];
  for (int q = 0; q < A.nstage; ++q) {
    bh[q] = A.dt_dev ? A.bh_dt[q] * *A.dt_dev : A.bh_dt[q];
    bl[q] = A.dt_dev ? A.bl_dt[q] * *A.dt_dev : A.bl_dt[q];
  }
  double errv = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < A.n; t += (long long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const double b = __ldg(A.base + (long long)v * A.n + t);
      double h = b, l = b;
      for (int q = 0; q < A.nstage; ++q) {
        const double kq = __ldg(A.K[q] + (long long)v * A.n + t);
        l = l - bl[q] * kq;
        h = h - bh[q] * kq;
      }
      A.out_high[(long long)v * A.n + t] = h;
      const double e = fabs(h - l) / (A.tol_rel * fabs(h) + A.tol_abs[v]);
      errv = dmax(errv, e);
    }
  }
  double vals[3] = {errv, 0.0, 0.0};
  block_reduce_emit<256>(vals, 1, 0, &A.ctl->err, nullptr, sred);
}

// Pointwise Shu-Osher update with a stored RHS (the first stage of the adaptive
// modified Euler scheme, whose RHS is the step's k1): out = yn - dt*r + eta*(y0 - yn + dt*r)
// (timedisc_modeuler.f90:279-291), over n values.
__global__ void __launch_bounds__(256) shu_osher_update_kernel(const double* __restrict__ y0, const double* __restrict__ yn,
                                                               const double* __restrict__ r, double* __restrict__ out,
                                                               long long n, double eta, double dt_host,
                                                               const double* dt_dev, const Ctl* ctl, int gate) {
  if (gate && (ctl->stop | ctl->brk)) return;
  if (gated_out(ctl, gate)) return;
  const double dt = dt_dev ? *dt_dev : dt_host;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    out[t] = yn[t] - dt * r[t] + eta * (y0[t] - yn[t] + dt * r[t]);
}

// A gated copy of n doubles (AcceptSolution's state into cvar at the end of a device-clock step).
__global__ void __launch_bounds__(256) gated_copy_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                                         long long n, const Ctl* ctl, int gate) {
  if (ctl->stop | ctl->brk) return;
  if (gated_out(ctl, gate)) return;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    dst[t] = src[t];
}

// The reconstruction variables of a Butcher stage state, formed once per cell:
// out = base - sum coef*K (the reference's accumulation order), converted with
// Cons2Prim for primitive reconstruction.  Values are identical to what the
// stage kernel forms at every stencil point.
template <int ND, bool EU, bool PRIM>
__global__ void __launch_bounds__(256) form_kernel(const __grid_constant__ StateRef in, Grid g, PhysP P,
                                                   double* __restrict__ out, const Ctl* ctl, int gate) {
  using PH = Phys<ND, EU>;
  constexpr int V = PH::V;
  if (gate && (ctl->stop | ctl->brk)) return;
  if (gated_out(ctl, gate)) return;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < g.n; t += (long long)gridDim.x * blockDim.x) {
    double u[V], p[V];
    state_at<V>(in, g.n, t, u);
    if (PRIM) PH::c2p(u, p, P);
#pragma unroll
    for (int v = 0; v < V; ++v) out[(long long)v * g.n + t] = PRIM ? p[v] : u[v];
  }
}

// Apply the CHECK_PMIN round trip to a stored state: out = P2C(MAX(C2P(in),pmin)).
template <int ND, bool EU>
__global__ void __launch_bounds__(256) roundtrip_kernel(const double* __restrict__ in, double* __restrict__ out,
                                                        long long n, PhysP P) {
  using PH = Phys<ND, EU>;
  constexpr int V = PH::V;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    double u[V], p[V], c[V];
    for (int v = 0; v < V; ++v) u[v] = in[v * n + t];
    PH::c2p(u, p, P);
    if (EU) p[V - 1] = dmax(p[V - 1], P.pmin);
    PH::p2c(p, c, P);
    for (int v = 0; v < V; ++v) out[v * n + t] = c[v];
  }
}

}  // namespace fgpu
