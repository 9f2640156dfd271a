// fgpu_batch.cuh -- batched ensembles of independent grids and the launch
// autotuner (included at the end of fgpu_host.cu; uses its helpers).
//
// fosite integrates one grid per process.  An ensemble of many small grids
// (parameter studies of disks, a serving queue of mixed requests) leaves most
// of a B200 idle when each grid is stepped by its own launches: a 64x128 disk
// is 32 tiles, a fifth of one wave.  A batch advances all its grids with ONE
// persistent stage launch per Runge-Kutta stage over the flattened tile queue
// of every grid (grid, bx, by, bz), plus one ghost/CFL/finalize launch whose
// blocks are distributed over the grids.  Every grid keeps its own arguments
// (metric, limiter, boundaries, dt, time, stop flags) in a device table, so a
// grid's results are bitwise the same alone or in any batch.

struct fgpu_batch {
  std::vector<fgpu_handle*> m;
  int nd = 2, order = 3;
  bool euler = false, prim = false;
  cudaStream_t stream = nullptr;
  int variant = 0;               // stage layout: 0/2/3 shared-memory tiles, 6 TMA-staged tiles (2D)
  StageArgs* d_args = nullptr;   // [order][n] step stages, then [n] RHS probes of the tuner
  CUtensorMap* d_maps = nullptr; // [order + 1][n] tensor maps of the stage inputs of d_args (layout 6)
  int tma_lim = -1;              // compiled-in limiter of layout 6, -1 when the batch cannot use it
  int4* d_tcols = nullptr;       // layout 6: (member, bx, byb, 0), columns of kchunk tiles per block
  int ntcols = 0;
  std::vector<char> tma_red;     // layout 6: per row of d_args, whether some member's stage reduces
  BndArgs* d_bnd = nullptr;      // [n]
  int4* d_tiles = nullptr;
  int ntiles = 0;
  int4* d_bblocks = nullptr;
  int nbblocks = 0;
  Ctl* h_ctls = nullptr;         // pinned [n]
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
  int graph_variant = -1;
  int sms = 148;
  int64_t pending_steps = 0;     // enqueued since the last collect
  std::vector<long long> it0;    // member iteration counts at the first enqueue
  std::string err;
  // embedded Runge-Kutta members (fgpu_bt.cuh): one replayed attempt slot advances every
  // member by one attempt; every member keeps its own controller, dt and error norm
  bool embedded = false;
  int stages = 0;                // tableau stages m
  Ctl** d_ctlp = nullptr;        // [n] members' control blocks
  BtParams* d_btp = nullptr;     // [n]
  StageArgs* d_eargs = nullptr;  // [m-1] attempt stages, then reject, sub-step and closing RHS: [(m+2)][n]
  FormArgs* d_fargs = nullptr;   // [m-1][n]
  CombineArgs* d_cargs = nullptr;// [n]
  CopyArgs* d_copy = nullptr;    // [n]
  BndArgs* d_ebnd = nullptr;     // [n] closing ghost/CFL pass
  bool adaptive_me = false;      // embedded modified Euler members: stage 1 by d_upd, no forms
  int me_order = 0;
  UpdArgs* d_upd = nullptr;      // [n]
  int4* d_cblocks = nullptr;     // per-member cell blocks (member, block, blocks)
  int ncblocks = 0;
  cudaGraphExec_t slot_graph = nullptr;
  std::vector<long long> adj0;
  // FARGO members (fixed-step Shu-Osher): per-step background velocity (type 1), advection
  // and the copy of w_new into w, over per-member tables and block tables
  int fdir = 0;                  // the FARGO members' common transport direction, 0 = none
  FargoWArgs* d_fw = nullptr;    int4* d_fwb = nullptr;  int nfwb = 0;
  FargoAdvArgs* d_fa = nullptr;  int4* d_fab = nullptr;  int nfab = 0;
  CopyArgs* d_fwc = nullptr;     int4* d_fwcb = nullptr; int nfwcb = 0;
};

namespace {

int bset_err(fgpu_batch* b, int code, const std::string& msg) {
  if (b) b->err = msg; else g_create_error = msg;
  return code;
}
#define BCUDA_TRY(b, call)                                                                   \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return bset_err(b, e_ == cudaErrorMemoryAllocation ? FGPU_ENOMEM : FGPU_ECUDA,         \
                      std::string(#call) + ": " + cudaGetErrorString(e_));                   \
  } while (0)

int launch_batched_stage(fgpu_batch* b, const StageArgs* args, int variant) {
  if (variant == 6) {   // TMA-staged tiles: tensor maps parallel to the step and probe tables
    if (!b->d_maps || args < b->d_args || args >= b->d_args + (size_t)(b->order + 1) * b->m.size())
      return bset_err(b, FGPU_EUNSUPPORTED, "the TMA layout serves fixed-step 2D batches only");
    const size_t row = (size_t)(args - b->d_args) / b->m.size();
    BCUDA_TRY(b, tma_batched_launch_2d(b->euler, b->prim, b->tma_lim, b->tma_red[row] != 0, args,
                                       b->d_maps + (args - b->d_args), b->d_tcols, b->ntcols, b->stream));
    return FGPU_OK;
  }
  // the shared-memory base tile of the batch's tile queue: layouts 0, 2, 3
  if (b->nd == 2)
    BCUDA_TRY(b, legacy_batched_launch_2d(b->euler, b->prim, variant, args, b->d_tiles, b->ntiles, b->sms, b->stream));
  else
    BCUDA_TRY(b, legacy_batched_launch_3d(b->euler, b->prim, variant, args, b->d_tiles, b->ntiles, b->sms, b->stream));
  return FGPU_OK;
}

int launch_batched_boundary(fgpu_batch* b) {
  if (b->nd == 2) {
    if (b->euler) batched_boundary_kernel<2, true><<<b->nbblocks, 256, 0, b->stream>>>(b->d_bnd, b->d_bblocks);
    else batched_boundary_kernel<2, false><<<b->nbblocks, 256, 0, b->stream>>>(b->d_bnd, b->d_bblocks);
  } else {
    if (b->euler) batched_boundary_kernel<3, true><<<b->nbblocks, 256, 0, b->stream>>>(b->d_bnd, b->d_bblocks);
    else batched_boundary_kernel<3, false><<<b->nbblocks, 256, 0, b->stream>>>(b->d_bnd, b->d_bblocks);
  }
  BCUDA_TRY(b, cudaGetLastError());
  return FGPU_OK;
}

template <bool EU>
void launch_batched_fargo_t(fgpu_batch* b, bool w) {
  if (w) {
    if (b->fdir == 1) batched_fargo_w_kernel<EU, 1><<<b->nfwb, 256, 0, b->stream>>>(b->d_fw, b->d_fwb);
    else batched_fargo_w_kernel<EU, 2><<<b->nfwb, FW_NT, 0, b->stream>>>(b->d_fw, b->d_fwb);
  } else {
    if (b->fdir == 1) batched_fargo_advect_kernel<EU, 1><<<b->nfab, 256, 0, b->stream>>>(b->d_fa, b->d_fab);
    else batched_fargo_advect_kernel<EU, 2><<<b->nfab, FA_TX * FA_TY, 0, b->stream>>>(b->d_fa, b->d_fab);
  }
}

int enqueue_batch_step(fgpu_batch* b) {
  const int n = (int)b->m.size();
  // FARGO members: CalcBackgroundVelocity (type 1) before the stages, FargoAdvection and the
  // closing pass after them, then w = w_new (the single-grid FARGO step's order)
  if (b->nfwb) {
    b->euler ? launch_batched_fargo_t<true>(b, true) : launch_batched_fargo_t<false>(b, true);
    BCUDA_TRY(b, cudaGetLastError());
  }
  for (int s = 0; s < b->order; ++s)
    if (int rc = launch_batched_stage(b, b->d_args + (size_t)s * n, b->variant)) return rc;
  if (b->nfab) {
    b->euler ? launch_batched_fargo_t<true>(b, false) : launch_batched_fargo_t<false>(b, false);
    BCUDA_TRY(b, cudaGetLastError());
  }
  if (int rc = launch_batched_boundary(b)) return rc;
  if (b->nfwcb) {
    batched_copy_kernel<<<b->nfwcb, 256, 0, b->stream>>>(b->d_fwc, b->d_fwcb);
    BCUDA_TRY(b, cudaGetLastError());
  }
  return FGPU_OK;
}

int build_batch_graph(fgpu_batch* b, int steps) {
  if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
  cudaGraph_t gr;
  BCUDA_TRY(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  int rc = 0;
  for (int s = 0; s < steps && !rc; ++s) rc = enqueue_batch_step(b);
  cudaError_t e = cudaStreamEndCapture(b->stream, &gr);
  if (rc) return rc;
  if (e != cudaSuccess) return bset_err(b, FGPU_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&b->graph, gr, 0);
  cudaGraphDestroy(gr);
  if (e != cudaSuccess) return bset_err(b, FGPU_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  b->graph_steps = steps;
  b->graph_variant = b->variant;
  return FGPU_OK;
}

// time reps launches of fn on stream s (CUDA events), milliseconds per launch
template <class F>
double time_launches(cudaStream_t s, int reps, F&& fn) {
  cudaEvent_t a, z;
  cudaEventCreate(&a);
  cudaEventCreate(&z);
  fn();   // warm-up (first-touch, instruction cache)
  auto run = [&](int n) {
    cudaEventRecord(a, s);
    for (int r = 0; r < n; ++r) fn();
    cudaEventRecord(z, s);
    cudaEventSynchronize(z);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, z);
    return (double)ms;
  };
  double total = run(reps);
  // short launches (small grids): repeat until the timed run lasts about 2 ms, so that the
  // layouts' differences are not lost in event and launch jitter
  if (total > 0.0 && total < 2.0) {
    const int more = std::min(400, (int)std::ceil(2.0 / (total / reps)));
    if (more > reps) {
      reps = more;
      total = run(reps);
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(z);
  return total / reps;
}

// ---- embedded-scheme batches
template <class T>
int upload_table(fgpu_batch* b, T** dst, const std::vector<T>& v) {
  BCUDA_TRY(b, cudaMalloc(dst, sizeof(T) * std::max<size_t>(1, v.size())));
  BCUDA_TRY(b, cudaMemcpyAsync(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, b->stream));
  return FGPU_OK;
}

// The argument tables of the attempt slot: what enqueue_bt_slot launches for one grid,
// for every member (the same arguments, member by member)
int build_embedded_tables(fgpu_batch* b) {
  const int n = (int)b->m.size();
  const Tableau& T0 = b->m[0]->T;
  const int M = T0.m;
  b->stages = M;
  std::vector<Ctl*> ctlp(n);
  std::vector<BtParams> btp(n);
  std::vector<StageArgs> eargs((size_t)(M + 2) * n);
  std::vector<FormArgs> fargs((size_t)(M - 1) * n);
  std::vector<CombineArgs> cargs(n);
  std::vector<CopyArgs> copy(n);
  std::vector<BndArgs> ebnd(n);
  std::vector<UpdArgs> upd(b->adaptive_me ? n : 0);
  std::vector<int4> cblocks;
  for (int i = 0; i < n; ++i) {
    fgpu_handle* h = b->m[i];
    const Tableau& T = h->T;
    double* P = h->buf[0];
    double* base = h->buf[1];
    double* K1 = h->buf[2];
    Ctl* c = h->d_ctl;
    ctlp[i] = c;
    btp[i].order = T.order; btp[i].beta = h->beta; btp[i].tol_rel = h->tol_rel;
    if (b->adaptive_me) {
      // timedisc_modeuler.f90:163-192: stage 1 pointwise, stages 2..order with the embedded
      // solution and the error norm (modeuler_attempt's launches per member)
      const int ord = h->order;
      double* S1 = h->buf[3];
      double* S2 = h->buf[4];
      double* LO = h->buf[5];
      UpdArgs& U = upd[i];
      U.y0 = base; U.yn = base; U.r = K1; U.out = S1; U.n = (long long)h->V * h->g.n;
      U.eta = kEta[ord - 1][0]; U.dt_dev = &c->d_att; U.ctl = c; U.gate = ACT_ATTEMPT;
      for (int m = 2; m <= ord; ++m) {
        StageArgs A = base_args(h);
        A.in = plain_state(m == 2 ? S1 : S2, false);
        A.out_mode = OUT_SSPRK;
        A.eta = kEta[ord - 1][m - 1];
        A.y0 = base;
        A.dt_dev = &c->d_att;
        if (m == ord) {
          A.out = P;
          A.err_low = ord == 3 ? LO : S1;
        } else {
          A.out = S2;
          A.out2 = LO;
          A.eta2 = kEta[1][1];
        }
        A.gate = ACT_ATTEMPT;
        A.kchunk = h->kchunk;
        eargs[(size_t)(m - 2) * n + i] = A;
      }
    }
    for (int m = 2; m <= M && !b->adaptive_me; ++m) {
      StageArgs A = base_args(h);
      A.in.base = base;
      A.in.nk = m - 1;
      for (int q = 0; q < m - 1; ++q) { A.in.K[q] = h->buf[2 + q]; A.in.coef[q] = T.A[(m - 1) * T.m + q]; }
      A.in.dt_dev = &c->d_att;
      FormArgs F;
      std::memset(&F, 0, sizeof(F));
      F.in = A.in; F.g = h->g; F.ph = h->ph; F.out = stage_rbuf(h, m); F.ctl = c; F.gate = ACT_ATTEMPT;
      fargs[(size_t)(m - 2) * n + i] = F;
      A.rin = plain_state(stage_rbuf(h, m), false);
      A.rin.ready = h->prim ? 1 : 0;
      A.out_mode = OUT_RHS;
      A.out = h->buf[2 + m - 1];
      set_fnext(h, A, m, 0.0, &c->d_att);
      if (m == M && h->fuse_end) set_last_stage(h, A, P, 0.0);
      A.gate = ACT_ATTEMPT;
      A.kchunk = h->kchunk;
      eargs[(size_t)(m - 2) * n + i] = A;
    }
    CombineArgs& Cb = cargs[i];
    std::memset(&Cb, 0, sizeof(Cb));
    Cb.base = base;
    // (the embedded modified Euler scheme has no weights: its combination is the last stage's)
    if (!b->adaptive_me)
      for (int q = 0; q < T.m; ++q) { Cb.K[q] = h->buf[2 + q]; Cb.bh_dt[q] = T.bh[q]; Cb.bl_dt[q] = T.bl[q]; }
    Cb.nstage = T.m; Cb.out_high = P; Cb.tol_rel = h->tol_rel;
    for (int v = 0; v < FGPU_MAXV; ++v) Cb.tol_abs[v] = h->tol_abs[v];
    Cb.n = h->g.n; Cb.ctl = c; Cb.dt_dev = &c->d_att; Cb.gate = ACT_ATTEMPT;
    {   // RejectSolution's RHS of cold
      StageArgs A = base_args(h);
      A.out_mode = OUT_RHS; A.out = K1; A.in = plain_state(base, false); A.gate = ACT_REJECT; A.kchunk = h->kchunk;
      eargs[(size_t)(M - 1) * n + i] = A;
    }
    {   // AcceptSolution's RHS inside the step
      StageArgs A = base_args(h);
      A.out_mode = OUT_RHS; A.out = K1; A.in = plain_state(P, h->roundtrip_cfg); A.out_base = base;
      A.checkdata = h->cfg.checkdata; A.cfl_mode = h->cfg.checkdata ? 3 : 0; A.gate = ACT_SUB; A.kchunk = h->kchunk;
      eargs[(size_t)M * n + i] = A;
    }
    {   // the closing RHS with the CFL reduction
      StageArgs A = base_args(h);
      A.out_mode = OUT_RHS; A.out = K1; A.in = plain_state(P, h->roundtrip_cfg); A.out_base = base;
      A.checkdata = h->cfg.checkdata; A.cfl_mode = 2; A.gate = ACT_END; A.kchunk = h->kchunk;
      eargs[(size_t)(M + 1) * n + i] = A;
    }
    copy[i].src = base; copy[i].dst = P; copy[i].n = (long long)h->V * h->g.n; copy[i].ctl = c; copy[i].gate = ACT_COPY;
    ebnd[i] = bnd_args(h, P, h->roundtrip_cfg, FIN_NONE);
    ebnd[i].checkdata = h->cfg.checkdata;
    ebnd[i].gate = ACT_END;
    const long long nb = std::max<long long>(1, std::min<long long>((h->g.n + 255) / 256, 1024));
    for (int q = 0; q < (int)nb; ++q) cblocks.push_back(make_int4(i, q, (int)nb, 0));
  }
  b->ncblocks = (int)cblocks.size();
  if (int rc = upload_table(b, &b->d_ctlp, ctlp)) return rc;
  if (int rc = upload_table(b, &b->d_btp, btp)) return rc;
  if (int rc = upload_table(b, &b->d_eargs, eargs)) return rc;
  if (int rc = upload_table(b, &b->d_fargs, fargs)) return rc;
  if (int rc = upload_table(b, &b->d_cargs, cargs)) return rc;
  if (int rc = upload_table(b, &b->d_copy, copy)) return rc;
  if (int rc = upload_table(b, &b->d_ebnd, ebnd)) return rc;
  if (int rc = upload_table(b, &b->d_cblocks, cblocks)) return rc;
  if (b->adaptive_me)
    if (int rc = upload_table(b, &b->d_upd, upd)) return rc;
  BCUDA_TRY(b, cudaStreamSynchronize(b->stream));
  return FGPU_OK;
}

template <int ND, bool EU, bool PRIM>
void launch_batched_form_t(fgpu_batch* b, const FormArgs* a) {
  batched_form_kernel<ND, EU, PRIM><<<b->ncblocks, 256, 0, b->stream>>>(a, b->d_cblocks);
}
int launch_batched_form(fgpu_batch* b, const FormArgs* a) {
  if (b->nd == 2) {
    if (b->euler) b->prim ? launch_batched_form_t<2, true, true>(b, a) : launch_batched_form_t<2, true, false>(b, a);
    else b->prim ? launch_batched_form_t<2, false, true>(b, a) : launch_batched_form_t<2, false, false>(b, a);
  } else {
    if (b->euler) b->prim ? launch_batched_form_t<3, true, true>(b, a) : launch_batched_form_t<3, true, false>(b, a);
    else b->prim ? launch_batched_form_t<3, false, true>(b, a) : launch_batched_form_t<3, false, false>(b, a);
  }
  BCUDA_TRY(b, cudaGetLastError());
  return FGPU_OK;
}

// one attempt of every member (enqueue_bt_slot, batched)
int enqueue_batch_slot(fgpu_batch* b) {
  const int n = (int)b->m.size();
  const int M = b->stages;
  const unsigned mb = (unsigned)((n + 127) / 128);
  bt_begin_batch_kernel<<<mb, 128, 0, b->stream>>>(b->d_ctlp, n);
  BCUDA_TRY(b, cudaGetLastError());
  if (b->adaptive_me) {
    batched_update_kernel<<<b->ncblocks, 256, 0, b->stream>>>(b->d_upd, b->d_cblocks);
    BCUDA_TRY(b, cudaGetLastError());
    for (int m = 2; m <= b->me_order; ++m)
      if (int rc = launch_batched_stage(b, b->d_eargs + (size_t)(m - 2) * n, b->variant)) return rc;
  }
  for (int m = 2; m <= M && !b->adaptive_me; ++m) {
    if (m == 2 || !b->m[0]->fuse_form)
      if (int rc = launch_batched_form(b, b->d_fargs + (size_t)(m - 2) * n)) return rc;
    if (int rc = launch_batched_stage(b, b->d_eargs + (size_t)(m - 2) * n, b->variant)) return rc;
  }
  if (!b->m[0]->fuse_end && !b->adaptive_me) {
    switch (b->m[0]->V) {
      case 3: batched_combine_kernel<3><<<b->ncblocks, 256, 0, b->stream>>>(b->d_cargs, b->d_cblocks); break;
      case 4: batched_combine_kernel<4><<<b->ncblocks, 256, 0, b->stream>>>(b->d_cargs, b->d_cblocks); break;
      default: batched_combine_kernel<5><<<b->ncblocks, 256, 0, b->stream>>>(b->d_cargs, b->d_cblocks); break;
    }
    BCUDA_TRY(b, cudaGetLastError());
  }
  bt_decide_batch_kernel<<<mb, 128, 0, b->stream>>>(b->d_ctlp, b->d_btp, n);
  BCUDA_TRY(b, cudaGetLastError());
  if (int rc = launch_batched_stage(b, b->d_eargs + (size_t)(M - 1) * n, b->variant)) return rc;
  if (int rc = launch_batched_stage(b, b->d_eargs + (size_t)M * n, b->variant)) return rc;
  bt_subcheck_batch_kernel<<<mb, 128, 0, b->stream>>>(b->d_ctlp, n);
  BCUDA_TRY(b, cudaGetLastError());
  batched_copy_kernel<<<b->ncblocks, 256, 0, b->stream>>>(b->d_copy, b->d_cblocks);
  BCUDA_TRY(b, cudaGetLastError());
  if (int rc = launch_batched_stage(b, b->d_eargs + (size_t)(M + 1) * n, b->variant)) return rc;
  if (b->nd == 2) {
    if (b->euler) batched_boundary_kernel<2, true><<<b->nbblocks, 256, 0, b->stream>>>(b->d_ebnd, b->d_bblocks);
    else batched_boundary_kernel<2, false><<<b->nbblocks, 256, 0, b->stream>>>(b->d_ebnd, b->d_bblocks);
  } else {
    if (b->euler) batched_boundary_kernel<3, true><<<b->nbblocks, 256, 0, b->stream>>>(b->d_ebnd, b->d_bblocks);
    else batched_boundary_kernel<3, false><<<b->nbblocks, 256, 0, b->stream>>>(b->d_ebnd, b->d_bblocks);
  }
  BCUDA_TRY(b, cudaGetLastError());
  bt_finish_batch_kernel<<<mb, 128, 0, b->stream>>>(b->d_ctlp, n, b->nd);
  BCUDA_TRY(b, cudaGetLastError());
  return FGPU_OK;
}

__global__ void add_steps_kernel(Ctl* const* ctls, int n, long long k) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) ctls[i]->steps_left += k;
}

int build_slot_graph(fgpu_batch* b, int slots);

constexpr int kSlotGraph = 8;
int launch_slots(fgpu_batch* b, long long slots) {
  if (!b->slot_graph || b->graph_variant != b->variant) { if (int rc = build_slot_graph(b, kSlotGraph)) return rc; }
  for (long long k = 0; k < (slots + kSlotGraph - 1) / kSlotGraph; ++k)
    BCUDA_TRY(b, cudaGraphLaunch(b->slot_graph, b->stream));
  const int n = (int)b->m.size();
  for (int i = 0; i < n; ++i)
    BCUDA_TRY(b, cudaMemcpyAsync(b->h_ctls + i, b->m[i]->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, b->stream));
  return FGPU_OK;
}

// members' host state into their control blocks (as bt_run does), nsteps each, and a first
// round of attempt slots (most steps take one attempt); collect_embedded runs the rest
int enqueue_embedded(fgpu_batch* b, int64_t nsteps) {
  const int n = (int)b->m.size();
  if (b->pending_steps == 0) {
    b->it0.resize(n);
    b->adj0.resize(n);
    for (int i = 0; i < n; ++i) {
      fgpu_handle* h = b->m[i];
      b->it0[i] = h->iter;
      b->adj0[i] = h->n_adj;
      Ctl& c = b->h_ctls[i];
      std::memset(&c, 0, sizeof(Ctl));
      c.time = h->time; c.dt = h->dt; c.dtold = h->dtold; c.dtmin = h->dtmin;
      c.stoptime = h->stoptime; c.tout = h->tout; c.cfl = h->cfl; c.dtlimit = h->dtlimit;
      c.iter = h->iter; c.brk = h->brk ? 1 : 0; c.dtcause = h->dtcause;
      c.cvis = h->cvis; c.vis = h->vis ? 1 : 0;
      c.maxerrold = h->maxerrold; c.last_err = h->last_err; c.n_adj = h->n_adj;
      c.checkflags = h->checkflags;
      c.steps_left = nsteps;
      BCUDA_TRY(b, cudaMemcpyAsync(h->d_ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, b->stream));
    }
  } else {
    add_steps_kernel<<<(n + 127) / 128, 128, 0, b->stream>>>(b->d_ctlp, n, (long long)nsteps);
    BCUDA_TRY(b, cudaGetLastError());
  }
  b->pending_steps += nsteps;
  return launch_slots(b, nsteps + nsteps / 4 + 1);
}

int collect_embedded(fgpu_batch* b, int* active) {
  const int n = (int)b->m.size();
  const int64_t ns = b->pending_steps;
  long long extra = 0;
  const long long cap = slot_cap(64 * (long long)ns + 64);
  bool stalled = false;
  while (true) {
    BCUDA_TRY(b, cudaStreamSynchronize(b->stream));
    bool busy = false;
    for (int i = 0; i < n; ++i) {
      const Ctl& c = b->h_ctls[i];
      if (c.steps_left > 0 && !c.stop && !c.brk) busy = true;
    }
    if (!busy || ns == 0) break;
    if (extra > cap) { stalled = true; break; }
    if (int rc = launch_slots(b, kSlotGraph)) return rc;
    extra += kSlotGraph;
  }
  int act = 0;
  for (int i = 0; i < n; ++i) {
    fgpu_handle* h = b->m[i];
    const Ctl& c = b->h_ctls[i];
    if (ns > 0) {
      *h->h_ctl = c;
      h->time = c.time; h->dt = c.dt; h->dtold = c.dtold; h->dtmin = c.dtmin;
      h->iter = c.iter; h->brk = c.brk != 0; h->dtcause = c.dtcause;
      h->maxerrold = c.maxerrold; h->last_err = c.last_err; h->n_adj = c.n_adj;
      h->checkflags = c.checkflags;
      if (h->iter > b->it0[i]) h->pre_rt = h->roundtrip_cfg;
      h->stats.attempts += (h->iter - b->it0[i]) + (h->n_adj - b->adj0[i]);
      h->stats.cell_updates += (h->iter - b->it0[i]) * h->g.n;
    }
    if (!c.stop && !c.brk) ++act;
  }
  b->pending_steps = 0;
  if (active) *active = act;
  // no progress within the slot budget: the members' bookkeeping above is the device's
  if (stalled) return bset_err(b, FGPU_ETIMEOUT, "batched device-clock step loop: no progress");
  return FGPU_OK;
}

int build_slot_graph(fgpu_batch* b, int slots) {
  if (b->slot_graph) { cudaGraphExecDestroy(b->slot_graph); b->slot_graph = nullptr; }
  cudaGraph_t gr;
  BCUDA_TRY(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  int rc = 0;
  for (int k = 0; k < slots && !rc; ++k) rc = enqueue_batch_slot(b);
  cudaError_t e = cudaStreamEndCapture(b->stream, &gr);
  if (rc) return rc;
  if (e != cudaSuccess) return bset_err(b, FGPU_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&b->slot_graph, gr, 0);
  cudaGraphDestroy(gr);
  if (e != cudaSuccess) return bset_err(b, FGPU_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  b->graph_variant = b->variant;
  return FGPU_OK;
}

}  // namespace

extern "C" {

int fgpu_batch_create(fgpu_handle* const* members, int n, fgpu_batch** out) {
  if (!members || n < 1 || !out) return bset_err(nullptr, FGPU_EARG, "null argument or empty batch");
  *out = nullptr;
  fgpu_batch* b = new fgpu_batch();
  auto fail = [&](int code, const std::string& msg) { g_create_error = msg; fgpu_batch_destroy(b); return code; };
  const fgpu_handle* h0 = members[0];
  if (!h0) return fail(FGPU_EARG, "null member");
  b->nd = h0->nd; b->euler = h0->euler; b->prim = h0->prim; b->order = h0->order;
  b->embedded = h0->butcher;
  for (int i = 0; i < n; ++i) {
    fgpu_handle* h = members[i];
    if (!h) return fail(FGPU_EARG, "null member");
    if (h->butcher != b->embedded) return fail(FGPU_EBADCFG, "batch members mix fixed-step and embedded schemes");
    if (h->butcher) {
      if (h->adaptive_me != h0->adaptive_me || (h->adaptive_me && h->order != h0->order))
        return fail(FGPU_EBADCFG, "embedded batch members mix modified Euler and Butcher schemes or orders");
      b->adaptive_me = h->adaptive_me;
      b->me_order = h->order;
      if (!h->materialize) return fail(FGPU_EUNSUPPORTED, "embedded batch members need the formed stage states");
      if (h->fuse_form != h0->fuse_form || h->fuse_end != h0->fuse_end)
        return fail(FGPU_EBADCFG, "embedded batch members differ in stage-state formation");
      if (h->cfg.method != h0->cfg.method || h->T.m != h0->T.m || h->T.order != h0->T.order)
        return fail(FGPU_EBADCFG, "embedded batch members differ in method or order");
    }
    if (h->fargo) {
      if (h->butcher) return fail(FGPU_EUNSUPPORTED, "FARGO batch members with the fixed-step modified Euler scheme");
      if (h->fargo_phase != 2)
        return fail(FGPU_EBADCFG, "a FARGO member must take its first step alone (that step has its own frame changes)");
      if (b->fdir && h->fdir != b->fdir) return fail(FGPU_EBADCFG, "FARGO batch members differ in transport direction");
      b->fdir = h->fdir;
    }
    if (h->accrete) return fail(FGPU_EUNSUPPORTED, "batch members without point-mass accretion");
    if (h->vis) return fail(FGPU_EUNSUPPORTED, "batch members without the viscosity source");
    if (!h->butcher && h->order < 2) return fail(FGPU_EUNSUPPORTED, "batch members of time order 2 or 3");
    if (h->nd != b->nd || h->euler != b->euler || h->prim != b->prim || h->order != b->order)
      return fail(FGPU_EBADCFG, "batch members differ in dimensionality, physics, reconstruction variables or order");
    if (h->device != h0->device) return fail(FGPU_EBADCFG, "batch members live on different devices");
    if (!h->first_done) return fail(FGPU_EBADCFG, "call fgpu_first_step on every member before batching");
    if (h->pre_rt != h->roundtrip_cfg)
      return fail(FGPU_EBADCFG, "an ideal-gas member whose checkdata lacks CHECK_PMIN must take its first step "
                                "alone (FirstStep's CHECK_ALL round trip)");
    b->m.push_back(h);
  }
  cudaSetDevice(h0->device);
  cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, h0->device);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(FGPU_ECUDA, "stream");
  b->variant = (h0->variant == 1 || h0->variant >= 4) ? 0 : h0->variant;
  if (b->embedded) b->order = 0;   // no fixed stages: d_args holds the tuner's probes only
  // argument tables: step stages of every member, then the tuner's RHS probes
  std::vector<StageArgs> args((size_t)(b->order + 1) * n);
  std::vector<BndArgs> bnd(n);
  std::vector<int4> tiles, bblocks;
  std::vector<FargoWArgs> fw;
  std::vector<FargoAdvArgs> fa;
  std::vector<CopyArgs> fwc;
  std::vector<int4> fwb, fab, fwcb;
  for (int i = 0; i < n; ++i) {
    fgpu_handle* h = b->m[i];
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return fail(FGPU_ECUDA, "member stream");
    const FargoStep F = h->fargo ? fargo_step_of(h) : FargoStep{};
    for (int s = 1; s <= b->order; ++s) {
      StageArgs A = h->fargo ? fargo_stage_args(h, F, s) : shu_osher_stage(h, s);
      A.kchunk = h->kchunk;
      args[(size_t)(s - 1) * n + i] = A;
    }
    if (h->fargo) {
      const Grid& g = h->g;
      if (F.dyn) {
        const int k = (int)fw.size();
        fw.push_back(fargo_w_args(h, F));
        const int nb = h->fdir == 1 ? (g.ny + 4 + FX_WY - 1) / FX_WY : (g.nx + 4 + FW_WX - 1) / FW_WX;
        for (int q = 0; q < nb; ++q) fwb.push_back(make_int4(k, q, 0, 0));
        CopyArgs C;
        C.src = F.Wn; C.dst = h->d_w; C.n = h->nw; C.ctl = h->d_ctl; C.gate = 0;
        const int kc = (int)fwc.size();
        fwc.push_back(C);
        fwcb.push_back(make_int4(kc, 0, 1, 0));
      }
      const int ka = (int)fa.size();
      fa.push_back(fargo_adv_args(h, F));
      if (h->fdir == 1) {
        const int nb = (int)std::max<long long>(1, std::min<long long>((g.n + 255) / 256, 148 * 8));
        for (int q = 0; q < nb; ++q) fab.push_back(make_int4(ka, q, nb, 0));
      } else {
        const int chunk = fa.back().chunk;
        const int gx = (g.nx + FA_TX - 1) / FA_TX, gy = (g.ny + FA_TY * chunk - 1) / (FA_TY * chunk);
        for (int y = 0; y < gy; ++y)
          for (int x = 0; x < gx; ++x) fab.push_back(make_int4(ka, x, y, 0));
      }
    }
    StageArgs R = base_args(h);
    R.in = plain_state(h->buf[0], false);
    R.out_mode = OUT_RHS;
    R.out = b->embedded ? h->buf[2 + h->T.m - 1] : h->buf[2];   // scratch between steps
    R.ctl = nullptr;
    R.kchunk = h->kchunk;
    args[(size_t)b->order * n + i] = R;
    bnd[i] = h->fargo ? fargo_closing_bnd(h, F) : bnd_args(h, h->buf[0], h->roundtrip_cfg, FIN_STEP);
    const Grid& g = h->g;
    const int TY = b->nd == 2 ? kBaseTY2 : kBaseTY3;
    const int tx = (g.nx + 31) / 32, ty = (g.ny + TY - 1) / TY;
    const int tz = b->nd == 3 ? (g.nz + h->kchunk - 1) / h->kchunk : 1;
    for (int z = 0; z < tz; ++z)
      for (int y = 0; y < ty; ++y)
        for (int x = 0; x < tx; ++x) tiles.push_back(make_int4(i, x, y, z));
    long long nb = std::min<long long>((bnd[i].nghost + 255) / 256, 4096);
    if (nb < 1) nb = 1;
    for (int q = 0; q < (int)nb; ++q) bblocks.push_back(make_int4(i, q, (int)nb, 0));
  }
  b->ntiles = (int)tiles.size();
  b->nbblocks = (int)bblocks.size();
  if (cudaMalloc(&b->d_args, sizeof(StageArgs) * args.size()) != cudaSuccess ||
      cudaMalloc(&b->d_bnd, sizeof(BndArgs) * bnd.size()) != cudaSuccess ||
      cudaMalloc(&b->d_tiles, sizeof(int4) * tiles.size()) != cudaSuccess ||
      cudaMalloc(&b->d_bblocks, sizeof(int4) * bblocks.size()) != cudaSuccess ||
      cudaMallocHost(&b->h_ctls, sizeof(Ctl) * n) != cudaSuccess)
    return fail(FGPU_ENOMEM, "batch tables");
  cudaMemcpyAsync(b->d_args, args.data(), sizeof(StageArgs) * args.size(), cudaMemcpyHostToDevice, b->stream);
  cudaMemcpyAsync(b->d_bnd, bnd.data(), sizeof(BndArgs) * bnd.size(), cudaMemcpyHostToDevice, b->stream);
  cudaMemcpyAsync(b->d_tiles, tiles.data(), sizeof(int4) * tiles.size(), cudaMemcpyHostToDevice, b->stream);
  cudaMemcpyAsync(b->d_bblocks, bblocks.data(), sizeof(int4) * bblocks.size(), cudaMemcpyHostToDevice, b->stream);
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return fail(FGPU_ECUDA, "batch table upload");
  if (!fa.empty()) {
    auto up = [&](auto** dst, const auto& v) {
      using T = typename std::decay_t<decltype(v)>::value_type;
      if (v.empty()) return true;
      if (cudaMalloc(dst, sizeof(T) * v.size()) != cudaSuccess) return false;
      return cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice) == cudaSuccess;
    };
    if (!up(&b->d_fw, fw) || !up(&b->d_fwb, fwb) || !up(&b->d_fa, fa) || !up(&b->d_fab, fab) || !up(&b->d_fwc, fwc) ||
        !up(&b->d_fwcb, fwcb))
      return fail(FGPU_ENOMEM, "batch fargo tables");
    b->nfwb = (int)fwb.size();
    b->nfab = (int)fab.size();
    b->nfwcb = (int)fwcb.size();
  }
  // tensor maps of every stage input for the TMA layout: fixed-step 2D members whose stages
  // it serves (the same conditions as a lone grid's), the limiter compiled in when shared
  if (b->nd == 2 && !b->embedded) {
    std::vector<CUtensorMap> maps(args.size());
    bool ok = true;
    int lim = -2;
    for (size_t q = 0; q < args.size() && ok; ++q) {
      fgpu_handle* h = b->m[q % n];
      const StageArgs& A = args[q];
      ok = tma_eligible(h, A);
      if (!ok) break;
      const StateRef& SR = A.rin.base ? A.rin : A.in;
      const CUtensorMap* mp = stage_tmap(h, SR.base, kTmaTX, kTmaTY);
      ok = mp != nullptr;
      if (ok) maps[q] = *mp;
      const int l = compiled_limiter(A.limiter, A.constant_recon != 0, A.theta);
      lim = lim == -2 ? l : (lim == l ? lim : 0);
    }
    if (ok && !args.empty()) {
      // blocks of tpb tiles along y (the boxes double-buffered); the 2D stage arguments carry
      // tpb in kchunk, which the shared-memory tiles of 2D meshes do not read
      const int tpb = tma_tiles_per_block(b->ntiles, 3);
      std::vector<int4> cols;
      for (int i = 0; i < n; ++i) {
        const Grid& g = b->m[i]->g;
        const int tx = (g.nx + kTmaTX - 1) / kTmaTX, tyb = ((g.ny + kTmaTY - 1) / kTmaTY + tpb - 1) / tpb;
        for (int y = 0; y < tyb; ++y)
          for (int x = 0; x < tx; ++x) cols.push_back(make_int4(i, x, y, 0));
      }
      for (auto& A : args) A.kchunk = tpb;
      b->ntcols = (int)cols.size();
      // stages whose arguments reduce CFL / CheckData / error maxima for some member
      b->tma_red.assign(b->order + 1, 0);
      for (size_t q = 0; q < args.size(); ++q)
        if (args[q].cfl_mode || args[q].last_stage || args[q].err_low) b->tma_red[q / n] = 1;
      if (cudaMalloc(&b->d_maps, sizeof(CUtensorMap) * maps.size()) != cudaSuccess ||
          cudaMemcpy(b->d_maps, maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
          cudaMalloc(&b->d_tcols, sizeof(int4) * cols.size()) != cudaSuccess ||
          cudaMemcpy(b->d_tcols, cols.data(), sizeof(int4) * cols.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
          cudaMemcpy(b->d_args, args.data(), sizeof(StageArgs) * args.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(FGPU_ENOMEM, "batch tensor maps");
      b->tma_lim = lim;
      if (h0->variant >= 6) b->variant = 6;
    }
  }
  if (b->embedded) { if (int rc = build_embedded_tables(b)) return fail(rc, b->err); }
  *out = b;
  return FGPU_OK;
}

void fgpu_batch_destroy(fgpu_batch* b) {
  if (!b) return;
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->d_args) cudaFree(b->d_args);
  if (b->d_maps) cudaFree(b->d_maps);
  if (b->d_tcols) cudaFree(b->d_tcols);
  if (b->d_bnd) cudaFree(b->d_bnd);
  if (b->d_tiles) cudaFree(b->d_tiles);
  if (b->d_bblocks) cudaFree(b->d_bblocks);
  if (b->h_ctls) cudaFreeHost(b->h_ctls);
  if (b->slot_graph) cudaGraphExecDestroy(b->slot_graph);
  for (void* p : {(void*)b->d_ctlp, (void*)b->d_btp, (void*)b->d_eargs, (void*)b->d_fargs, (void*)b->d_cargs,
                  (void*)b->d_copy, (void*)b->d_ebnd, (void*)b->d_cblocks, (void*)b->d_fw, (void*)b->d_fwb,
                  (void*)b->d_fa, (void*)b->d_fab, (void*)b->d_fwc, (void*)b->d_fwcb, (void*)b->d_upd})
    if (p) cudaFree(p);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

int fgpu_batch_last_error(const fgpu_batch* b, char* buf, int len) {
  const std::string& s = b ? b->err : g_create_error;
  if (buf && len > 0) {
    int k = std::min<int>((int)s.size(), len - 1);
    std::memcpy(buf, s.data(), k);
    buf[k] = 0;
  }
  return (int)s.size();
}

int fgpu_batch_size(const fgpu_batch* b, int* members, int* tiles) {
  if (!b) return FGPU_EARG;
  if (members) *members = (int)b->m.size();
  if (tiles) *tiles = b->ntiles;
  return FGPU_OK;
}

int fgpu_batch_layout(const fgpu_batch* b, int* variant) {
  if (!b || !variant) return FGPU_EARG;
  *variant = b->variant;
  return FGPU_OK;
}

int fgpu_batch_enqueue(fgpu_batch* b, int64_t nsteps) {
  if (!b || nsteps < 0) return FGPU_EARG;
  if (b->embedded) return enqueue_embedded(b, nsteps);
  if (b->pending_steps == 0) {
    b->it0.resize(b->m.size());
    for (size_t i = 0; i < b->m.size(); ++i) b->it0[i] = b->m[i]->iter;
  }
  const int G = 16;
  int64_t full = nsteps / G, rest = nsteps % G;
  if (full > 0) {
    if (b->graph_steps != G || b->graph_variant != b->variant) { if (int rc = build_batch_graph(b, G)) return rc; }
    for (int64_t r = 0; r < full; ++r) BCUDA_TRY(b, cudaGraphLaunch(b->graph, b->stream));
  }
  for (int64_t r = 0; r < rest; ++r) { if (int rc = enqueue_batch_step(b)) return rc; }
  const int n = (int)b->m.size();
  for (int i = 0; i < n; ++i)
    BCUDA_TRY(b, cudaMemcpyAsync(b->h_ctls + i, b->m[i]->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, b->stream));
  b->pending_steps += nsteps;
  return FGPU_OK;
}

int fgpu_batch_collect(fgpu_batch* b, int* active) {
  if (!b) return FGPU_EARG;
  if (b->embedded) return collect_embedded(b, active);
  BCUDA_TRY(b, cudaStreamSynchronize(b->stream));
  const int n = (int)b->m.size();
  int act = 0;
  const int64_t ns = b->pending_steps;
  for (int i = 0; i < n; ++i) {
    fgpu_handle* h = b->m[i];
    if (ns > 0) {
      *h->h_ctl = b->h_ctls[i];
      sync_from_ctl(h);
      h->stats.attempts += h->iter - b->it0[i];
      h->stats.cell_updates += (h->iter - b->it0[i]) * h->g.n;
      h->stats.stage_launches += (int64_t)b->order * ns;
      h->stats.launches += (int64_t)(b->order + 1) * ns;
    }
    if (!h->h_ctl->stop && !h->h_ctl->brk) ++act;
  }
  b->pending_steps = 0;
  if (active) *active = act;
  return FGPU_OK;
}

int fgpu_batch_run(fgpu_batch* b, int64_t nsteps, int* active) {
  if (int rc = fgpu_batch_enqueue(b, nsteps)) return rc;
  return fgpu_batch_collect(b, active);
}

int fgpu_batch_autotune(fgpu_batch* b, int reps, int* variant) {
  if (!b) return FGPU_EARG;
  if (reps < 1) reps = 3;
  const StageArgs* probe = b->d_args + (size_t)b->order * b->m.size();
  std::vector<int> cand = {0, 2, 3};
  if (b->d_maps) cand.push_back(6);
  double best = 1e300;
  int bv = b->variant;
  for (int v : cand) {
    int rc = FGPU_OK;
    double ms = time_launches(b->stream, reps, [&] { if (!rc) rc = launch_batched_stage(b, probe, v); });
    if (rc) return rc;
    BCUDA_TRY(b, cudaGetLastError());
    if (ms < best) { best = ms; bv = v; }
  }
  b->variant = bv;
  if (variant) *variant = bv;
  return FGPU_OK;
}

}  // extern "C"

namespace {
// Tuning decisions of this process, by the key of what the stage kernel's cost depends on
// (device, dimensionality, physics, reconstruction variables and limiter, geometry, mesh
// size and the optional source/transport features): a grid with a known key reuses the
// measured layout without probing.
struct TuneKey {
  int device, nd, euler, prim, order, limiter, geometry, nx, ny, nz, features;
  bool operator<(const TuneKey& o) const {
    return std::memcmp(this, &o, sizeof(TuneKey)) < 0;
  }
};
struct TuneChoice { int variant, kchunk; };
std::mutex g_tune_mutex;
std::map<TuneKey, TuneChoice> g_tune_cache;
TuneKey tune_key(const fgpu_handle* h) {
  TuneKey k;
  std::memset(&k, 0, sizeof(k));
  k.device = h->device; k.nd = h->nd; k.euler = h->euler; k.prim = h->prim;
  k.order = h->cfg.order; k.limiter = h->cfg.limiter; k.geometry = h->cfg.geometry;
  k.nx = h->g.nx; k.ny = h->g.ny; k.nz = h->g.nz;
  k.features = (h->fargo ? 1 : 0) | (h->accrete ? 2 : 0) | (h->vis ? 4 : 0) | (h->has_accel ? 8 : 0) |
               (h->butcher ? 16 : 0) | (h->materialize ? 32 : 0);
  return k;
}
}  // namespace

extern "C" {

// Measures each stage-kernel layout on this grid (RHS evaluations into a
// scratch array, the state is not touched) and keeps the fastest; a grid whose
// tuning key was measured before in this process takes the cached choice
// (reps < 0 measures |reps| times regardless and refreshes the cache).
int fgpu_autotune(fgpu_handle* h, int reps, int* variant) {
  if (!h) return FGPU_EARG;
  const TuneKey key = tune_key(h);
  if (reps >= 0) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      if (h->variant != it->second.variant || h->kchunk != it->second.kchunk) {
        if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; h->graph_steps = 0; }
        if (h->bt_graph) { cudaGraphExecDestroy(h->bt_graph); h->bt_graph = nullptr; }
      }
      h->variant = it->second.variant;
      h->kchunk = it->second.kchunk;
      if (variant) *variant = it->second.variant;
      return FGPU_OK;
    }
  }
  reps = reps < 0 ? -reps : reps;
  if (reps < 1) reps = 3;
  double* scratch = h->butcher ? h->buf[2 + h->T.m - 1] : h->buf[2];
  StageArgs A = base_args(h);
  A.in = plain_state(h->buf[0], false);
  A.out_mode = OUT_RHS;
  A.out = scratch;
  A.ctl = nullptr;
  A.visc = h->vis ? h->d_visc : nullptr;   // the stencil's read of the viscous source
  if (!h->fargo && !h->vis && !h->accrete) {
    if (h->butcher && !h->adaptive_me && h->materialize && h->fuse_form && h->T.m >= 3) {
      // a late Butcher stage as the steps launch it: the formed input state, this stage's k and
      // the next stage's state formed from base and the earlier k (the heaviest epilogue
      // stream); only scratch buffers are written (k_{M-1}, a formed-state buffer)
      const int m = h->T.m - 1;
      A.rin = plain_state(stage_rbuf(h, m), false);
      A.rin.ready = h->prim ? 1 : 0;
      A.in.base = h->buf[1];
      A.in.nk = m - 1;
      for (int q = 0; q < m - 1; ++q) {
        A.in.K[q] = h->buf[2 + q];
        A.in.coef[q] = h->T.A[(m - 1) * h->T.m + q] * h->dt;
      }
      A.out = h->buf[2 + m - 1];
      set_fnext(h, A, m, h->dt, nullptr);
    } else if (!h->butcher && !h->adaptive_me && h->order >= 3) {
      // a middle Shu-Osher stage: scratch state in, scratch state out, the stored state as y0
      A = shu_osher_stage(h, 2);
      A.ctl = nullptr;
      A.cfl_mode = 0;
    }
  } else if (h->fargo && !h->vis && !h->accrete && !h->butcher && !h->adaptive_me && h->order >= 3) {
    // a middle FARGO Shu-Osher stage with its frame changes (scratch in, scratch out)
    A = fargo_stage_args(h, fargo_step_of(h), 2);
    A.ctl = nullptr;
    A.cfl_mode = 0;
  }
  const int cand[8] = {0, 2, 3, 4, 5, 1, 6, 7};
  // 3D: the z extent a block marches through (smaller chunks give small grids more blocks);
  // FGPU_KCHUNK fixes it
  std::vector<int> chunks;
  if (h->nd == 3 && !std::getenv("FGPU_KCHUNK")) {
    for (int kc : {4, 8, 16, 32})
      if (kc <= std::max(4, h->g.nz)) chunks.push_back(kc);
  } else {
    chunks.push_back(h->kchunk);
  }
  double best = 1e300;
  int bv = h->variant, bk = h->kchunk;
  const int keep = h->variant, keepk = h->kchunk;
  for (int v : cand) {
    // layout 1 lacks these features (Butcher steps gate their stages or form the next stage's state)
    if (v == 1 && (h->fargo || h->accrete || h->vis || h->butcher)) continue;
    // layouts 6, 7 (TMA-staged planes) serve grids without viscosity or accretion, even nx
    if (v >= 6 && (h->accrete || h->vis || h->g.nx % 2 != 0)) continue;
    if (v == 7 && h->nd == 3) continue;   // the 32 x 4 TMA tile is built for 2D meshes
    // the taller tiles (4, 5) differ from the oracle in the last bit on FARGO transport along x
    // with a user-supplied background velocity; such grids keep the 32 x 8 tiles
    if ((v == 4 || v == 5) && h->fargo && h->fdir == 1) continue;
    for (int kc : chunks) {
      h->variant = v;
      h->kchunk = kc;
      int rc = FGPU_OK;
      double ms = time_launches(h->stream, reps, [&] { if (!rc) rc = launch_stage_raw(h, A); });
      if (rc) { h->variant = keep; h->kchunk = keepk; return rc; }
      if (ms < best) { best = ms; bv = v; bk = kc; }
    }
  }
  h->variant = bv;
  h->kchunk = bk;
  if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; h->graph_steps = 0; }
  if (h->bt_graph) { cudaGraphExecDestroy(h->bt_graph); h->bt_graph = nullptr; }
  if (variant) *variant = bv;
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[key] = TuneChoice{bv, bk};
  }
  return FGPU_OK;
}

int fgpu_stage_layout(const fgpu_handle* h, int* variant, int* kchunk) {
  if (!h) return FGPU_EARG;
  if (variant) *variant = h->variant;
  if (kchunk) *kchunk = h->kchunk;
  return FGPU_OK;
}

}  // extern "C"
