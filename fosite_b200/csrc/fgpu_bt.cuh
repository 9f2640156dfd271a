// fgpu_bt.cuh -- the embedded Runge-Kutta step loop on the device clock.
//
// fosite's IntegrationStep (timedisc_base.f90:649-750) repeats attempts until
// the sub-steps cover dt: reject (cvar = cold, RHS again), accept (advance t,
// RHS at t while t < time + dt), then the closing RHS with CheckData and
// CalcTimestep; the step size comes from AdjustTimestep's PI controller
// (timedisc_base.f90:759-814).  Here that loop is a state machine in the
// control block: every captured "slot" runs one attempt -- bt_begin_kernel opens
// a fosite step when the previous one is done (stop test, output-time clip),
// the stage kernels run with dt read on the device, bt_decide_kernel evaluates
// the error norm, the controller and the accept/reject predicate, and the
// slot's remaining kernels (the RHS of the restored or advanced state, the
// closing RHS, the CFL reduction and bt_finish_kernel) run only when their
// action bit is set.  The host replays slots without reading anything back
// until it wants to know how far the run has come.
#pragma once
#include "fgpu_kernels_misc.cuh"
#include "fgpu_ddmath.h"

namespace fgpu {

struct BtParams {
  int order;        // the scheme's order (the controller's exponent)
  double beta;      // PI controller parameter
  double tol_rel;
};

// fosite%Step's opening (fosite.f90:367-388 stop test; io/fileio_base.f90:604-621
// output-time clip) and IntegrationStep's loop head (timedisc_base.f90:649-676)
// when the slot starts a step; then this slot's attempt.
__device__ void bt_begin_body(Ctl* c) {
  c->act = 0;
  if (c->stop | c->brk) return;
  int open = 0;
  if (c->phase == 0) {
    open = ACT_OPEN;
    if (c->steps_left <= 0) return;
    if (fabs(c->stoptime - c->time) <= 1.0E-05 * c->stoptime) { c->stop = 1; return; }
    if ((c->time + c->dt) / c->tout > 1.0) { c->dt = c->tout - c->time; c->dtcause = -4; }
    else if ((c->time + 1.5 * c->dt) / c->tout > 1.0) { c->dt = 0.5 * (c->tout - c->time); c->dtcause = -4; }
    c->t_loc = c->time;
    c->d_att = c->dt;
    if (c->d_att < c->dtmin && c->dtcause != -4) c->dtmin = c->d_att;
    c->rhs_done = 0;
    c->phase = 1;
  }
  c->dtold_att = c->d_att;
  c->act = ACT_ATTEMPT | open;
}
__global__ void bt_begin_kernel(Ctl* c) { bt_begin_body(c); }

// timedisc_base.f90:759-814 AdjustTimestep with correctly rounded exp/log
__device__ double bt_adjust(Ctl* c, const BtParams& P, double maxerr, double dtold_) {
  double dtnew, dttmp;
  if (P.tol_rel >= 1.0) return DBL_MAX;
  if (maxerr > 0.) dttmp = 0.9 * dtold_ * ddm::exp_cr(-ddm::log_cr(maxerr) / P.order);
  else dttmp = 4. * dtold_;
  if (c->maxerrold > 0.) dtnew = dttmp * ddm::exp_cr(-P.beta * ddm::log_cr(c->maxerrold / maxerr));
  else dtnew = dttmp;
  if (maxerr < 1.0) {
    const double cap = 4. * dtold_;
    dtnew = cap < dtnew ? cap : dtnew;
    if (dtnew < dtold_) c->dtcause = -2;
  } else {
    if (dtnew > dtold_) dtnew = dttmp;
    const double floor_ = 0.25 * dtold_;
    dtnew = dtnew < floor_ ? floor_ : dtnew;
  }
  c->maxerrold = maxerr;
  return dtnew;
}

// The body of IntegrationStep's loop after SolveODE (timedisc_base.f90:684-710): break on a
// NaN/Inf error, RejectSolution or AcceptSolution (timedisc_base.f90:911-1009), the dtlimit
// test, the loop condition, and the loop's closing (timedisc_base.f90:712-720).
__device__ void bt_decide_body(Ctl* c, const BtParams& P) {
  if (!(c->act & ACT_ATTEMPT) || (c->stop | c->brk)) { c->act = 0; return; }
  const double e = __longlong_as_double((long long)c->err);
  c->err = 0ULL;
  c->last_err = e;
  const double d = bt_adjust(c, P, e, c->dtold_att);
  int act = 0;
  c->rhs_done = 0;
  if (e != e) c->brk = 1;
  else if (e > DBL_MAX) c->brk = 1;
  else if (e >= 1.0) {
    act |= ACT_REJECT;
    c->n_adj += 1;
    c->dtcause = -1;
    if (d < c->dtmin) c->dtmin = d;
  } else {
    c->t_loc = c->t_loc + c->dtold_att;
    if (c->t_loc < c->time + c->dt) { act |= ACT_SUB; c->rhs_done = 1; }
    c->iter += 1;
  }
  if (d < c->dtlimit) c->brk = 1;
  c->d_att = d;
  if (!c->brk && !(c->t_loc + d <= c->time + c->dt)) {
    c->time_prev = c->time;
    c->dt_prev = c->dt;
    c->dtold_prev = c->dtold;
    c->dt = c->t_loc - c->time;
    c->time = c->t_loc;
    c->dtold = d;
    act |= ACT_END;
    act |= c->rhs_done ? ACT_COPY : ACT_ENDNC;
  }
  c->act = act;
}
__global__ void bt_decide_kernel(Ctl* c, BtParams P) { bt_decide_body(c, P); }

// CheckData of AcceptSolution's ComputeRHS inside the step (timedisc_base.f90:926-931): a
// failure breaks IntegrationStep's loop; the step then ends without its closing (time, dt and
// dtold stay those of the step's start).  The stored state keeps the accepted solution, whose
// CHECK_PMIN round trip gives cvar as that ComputeRHS left it; bt_finish breaks and the
// slot's closing kernels do nothing.
__device__ void bt_subcheck_body(Ctl* c) {
  if (!(c->act & ACT_SUB) || (c->stop | c->brk)) return;
  if (c->flags) {
    c->checkflags |= c->flags;
    c->flags = 0;
    if (c->act & ACT_END) {
      c->time = c->time_prev;
      c->dt = c->dt_prev;
      c->dtold = c->dtold_prev;
    }
    c->act = ACT_BRK;
  }
}
__global__ void bt_subcheck_kernel(Ctl* c) { bt_subcheck_body(c); }

// CalcTimestep's closing arithmetic after the step's closing RHS and ghost-cell pass
// (timedisc_base.f90:885-909, the sources list's viscous limit), CheckData's break, and the
// count of completed fosite steps.
__device__ void bt_finish_body(Ctl* c, int nd) {
  if (c->stop | c->brk) return;
  if (c->act & ACT_BRK) {
    c->brk = 1;
    return;
  }
  if (!(c->act & ACT_END)) return;
  auto D = [](unsigned long long b) { return __longlong_as_double((long long)b); };
  const double invdt = nd == 2 ? D(c->invdt[0]) : dmax(dmax(D(c->invdt[1]), D(c->invdt[2])), D(c->invdt[0]));
  const double ivis = D(c->invdt[3]);
  c->invdt[0] = c->invdt[1] = c->invdt[2] = c->invdt[3] = 0ULL;
  if (c->flags) {
    c->checkflags |= c->flags;
    c->flags = 0;
    c->brk = 1;
    return;
  }
  double dt = c->cfl / invdt;
  int cause = 0;
  if (c->vis) {
    const double dtv = ivis > DBL_MIN ? c->cvis / ivis : DBL_MAX;
    if (dtv < dt) cause = 3;
    dt = dtv < dt ? dtv : dt;
  }
  c->dt = dt;
  c->dtcause = cause;
  c->phase = 0;
  c->steps_left -= 1;
}
__global__ void bt_finish_kernel(Ctl* c, int nd) { bt_finish_body(c, nd); }

// ---- batches of grids with embedded schemes: one thread per member for the scalar work,
// block tables (member, block, blocks of the member) for the per-cell passes
__global__ void bt_subcheck_batch_kernel(Ctl* const* ctls, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) bt_subcheck_body(ctls[i]);
}
__global__ void bt_begin_batch_kernel(Ctl* const* ctls, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) bt_begin_body(ctls[i]);
}
__global__ void bt_decide_batch_kernel(Ctl* const* ctls, const BtParams* P, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) bt_decide_body(ctls[i], P[i]);
}
__global__ void bt_finish_batch_kernel(Ctl* const* ctls, int n, int nd) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) bt_finish_body(ctls[i], nd);
}

struct FormArgs {
  StateRef in;
  Grid g;
  PhysP ph;
  double* out;
  const Ctl* ctl;
  int gate;
};
template <int ND, bool EU, bool PRIM>
__global__ void __launch_bounds__(256) batched_form_kernel(const FormArgs* __restrict__ args,
                                                           const int4* __restrict__ blocks) {
  using PH = Phys<ND, EU>;
  constexpr int V = PH::V;
  const int4 T = blocks[blockIdx.x];
  const FormArgs& A = args[T.x];
  if (A.ctl->stop | A.ctl->brk) return;
  if (gated_out(A.ctl, A.gate)) return;
  for (long long t = T.y * 256LL + threadIdx.x; t < A.g.n; t += T.z * 256LL) {
    double u[V], p[V];
    state_at<V>(A.in, A.g.n, t, u);
    if (PRIM) PH::c2p(u, p, A.ph);
#pragma unroll
    for (int v = 0; v < V; ++v) A.out[(long long)v * A.g.n + t] = PRIM ? p[v] : u[v];
  }
}

template <int V>
__global__ void __launch_bounds__(256) batched_combine_kernel(const CombineArgs* __restrict__ args,
                                                              const int4* __restrict__ blocks) {
  __shared__ double sred[RED_STRIDE * 8];
  const int4 T = blocks[blockIdx.x];
  const CombineArgs& A = args[T.x];
  if (A.ctl->stop | A.ctl->brk) return;
  if (gated_out(A.ctl, A.gate)) return;
  double bh[FGPU_MAXK], bl[FGPU_MAXK];
  for (int q = 0; q < A.nstage; ++q) {
    bh[q] = A.dt_dev ? A.bh_dt[q] * *A.dt_dev : A.bh_dt[q];
    bl[q] = A.dt_dev ? A.bl_dt[q] * *A.dt_dev : A.bl_dt[q];
  }
  double errv = 0.0;
  for (long long t = T.y * 256LL + threadIdx.x; t < A.n; t += T.z * 256LL) {
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

struct CopyArgs {
  const double* src;
  double* dst;
  long long n;
  const Ctl* ctl;
  int gate;
};
// The first stage of the embedded modified Euler scheme for a batch: out = yn - dt*r +
// eta*(y0 - yn + dt*r) with the member's attempt dt (shu_osher_update_kernel per member)
struct UpdArgs {
  const double* y0;
  const double* yn;
  const double* r;
  double* out;
  long long n;
  double eta;
  const double* dt_dev;
  const Ctl* ctl;
  int gate;
};
__global__ void __launch_bounds__(256) batched_update_kernel(const UpdArgs* __restrict__ args,
                                                             const int4* __restrict__ blocks) {
  const int4 T = blocks[blockIdx.x];
  const UpdArgs& A = args[T.x];
  if (A.ctl->stop | A.ctl->brk) return;
  if (gated_out(A.ctl, A.gate)) return;
  const double dt = *A.dt_dev;
  for (long long t = T.y * 256LL + threadIdx.x; t < A.n; t += T.z * 256LL)
    A.out[t] = A.yn[t] - dt * A.r[t] + A.eta * (A.y0[t] - A.yn[t] + dt * A.r[t]);
}

__global__ void __launch_bounds__(256) batched_copy_kernel(const CopyArgs* __restrict__ args,
                                                           const int4* __restrict__ blocks) {
  const int4 T = blocks[blockIdx.x];
  const CopyArgs& A = args[T.x];
  if (A.ctl->stop | A.ctl->brk) return;
  if (gated_out(A.ctl, A.gate)) return;
  for (long long t = T.y * 256LL + threadIdx.x; t < A.n; t += T.z * 256LL) A.dst[t] = A.src[t];
}

}  // namespace fgpu
