// Continuous batching of mixed-precision solves on one batched operator.
//
// A lane owns the K members of a batched operator.  Each member runs the
// solve of vox_solve_refined for its own right-hand side: complex64 GMRES
// restart cycles inside FP64 iterative refinement.  All members' Arnoldi
// steps run as one captured graph (one launch per kernel for every member,
// the preconditioner's blocks read once for all of them); a member that is
// not in an inner solve is frozen and skipped.
//
// Step mode (restart + 1 <= kGsMaxCols, the default): the members' cycles
// are out of phase.  One vox_lane_step runs a fixed number of steps (one
// Arnoldi step of every member in a cycle, each at its own k); a member whose
// cycle ends restarts at the next step by itself, and a member whose inner
// solve ends waits only until the end of the current steps, not for the
// other members' cycles.  In-phase mode (longer restarts) runs whole cycles.
// Between launches the host advances each member on its own: a member whose
// inner solve ended gets its FP64 refinement step, a member whose solve ended
// is reported, and a free member can take a new right-hand side at once.
// Each member's arithmetic is exactly that of the single-right-hand-side
// solve on the same operator.  Included at the end of api.cu, after
// solver.cuh.
#pragma once

struct vox_lane_s {
  vox_op_s* op = nullptr;
  vox_precond_s* pc = nullptr;
  int side = 0;
  double tol = 1e-5;
  int restart = 50;
  int maxit_inner = 40;
  double inner_tol = 0.0;
  int max_refine = 10;
  int steps = 0;               // step mode: steps per vox_lane_step (0: in-phase cycles)
  double* hhist = nullptr;     // pinned: K residual histories (step mode)
  struct Member {
    int state = 0;             // 0 free, 1 solving, 2 finished (not yet collected)
    const double2* b = nullptr;
    double2* x = nullptr;
    double bn = 0.0;           // ||b||
    double rel = 1.0;          // ||b - A x|| / ||b|| (FP64)
    double rn = 0.0;           // ||r|| at the start of the inner solve
    double itol = 0.0;         // inner tolerance (relative)
    double ibn = 0.0;          // the inner solve's right-hand-side norm
    bool inner = false;        // in an inner solve (takes part in the cycles)
    int outit = 0;             // cycles of the current inner solve
    int p = 0;                 // iterations of its last cycle
    int outer_total = 0;
    vox_gmres_info info{};
    std::vector<double> rv;
  };
  std::vector<Member> m;
  std::vector<int> pending_done;  // finished at submission (zero right-hand side)
  ~vox_lane_s() {
    if (hhist) cudaFreeHost(hhist);
  }
};

namespace vox {

// Steps per vox_lane_step in step mode: VOX_LANE_STEPS (1..64; 0 runs whole
// in-phase cycles instead), default 2.
static int lane_steps_default() {
  const char* e = std::getenv("VOX_LANE_STEPS");
  if (e && *e) {
    const int v = std::atoi(e);
    if (v >= 0 && v <= 64) return v;
  }
  return 2;
}

// One member's header: zeroed solve state, restart length, tolerance, frozen.
// A member that begins an inner solve in step mode is flagged to start its
// first cycle at the next step, with the inner solve's stopping data (its
// right-hand side's norm, relative target and cycle limit).
static vox_status lane_header(vox_lane_s* L, int b, double tol_abs, int frozen, double ibn = 0.0,
                              double itol = 0.0) {
  GmresWork<float>& w = L->op->wf;
  std::vector<unsigned char> hdr(offsetof(GmresDev, resvec), 0);
  GmresDev* h = reinterpret_cast<GmresDev*>(hdr.data());
  h->m = w.m;
  h->tol_abs = tol_abs;
  h->frozen = frozen;
  h->ibn = ibn;
  h->itol = itol;
  h->maxit = L->maxit_inner;
  if (L->steps > 0) {
    h->start = frozen ? 0 : 1;
    h->done = 1;  // until its cycle starts (idle members never step)
  }
  VOX_CUDA(cudaMemcpyAsync(&w.st[b], hdr.data(), hdr.size(), cudaMemcpyHostToDevice,
                           L->op->stream));
  return VOX_OK;
}

static vox_status lane_freeze(vox_lane_s* L, int b) {
  const int one = 1;
  VOX_CUDA(cudaMemcpyAsync(&L->op->wf.st[b].frozen, &one, sizeof(int), cudaMemcpyHostToDevice,
                           L->op->stream));
  return VOX_OK;
}

static void lane_finish(vox_lane_s* L, int b) {
  vox_lane_s::Member& mb = L->m[b];
  mb.info.relres = mb.rel;
  mb.info.flag = mb.rel <= L->tol ? 0 : 1;
  mb.info.iter_inner = mb.p;
  mb.info.iter_outer = mb.outer_total;
  mb.inner = false;
  mb.state = 2;
}

// Start the next inner solve of every member in S: d solves (A/Gram) d = r/||r||.
static vox_status lane_start_inner(vox_lane_s* L, const std::vector<int>& S) {
  if (S.empty()) return VOX_OK;
  vox_op_s* op = L->op;
  GmresWork<float>& wf = op->wf;
  GmresWork<double>& wd = op->wd;
  const long long n = op->g.n;
  cudaStream_t st = op->stream;
  const int nb = nblk(n);
  const bool auto_tol = L->inner_tol <= 0;
  for (int b : S) {
    vox_lane_s::Member& mb = L->m[b];
    mb.rn = mb.rel * mb.bn;
    k_cast_scale<float><<<nb, 256, 0, st>>>(n, wd.mem(wd.r, b), 1.0 / mb.rn, wf.mem(wf.b, b));
    const double fac = inner_target_factor(L->pc, L->side, L->inner_tol);
    mb.itol = auto_tol ? std::min(0.5, fac * L->tol * mb.bn / mb.rn)
                       : std::min(0.5, std::max(L->inner_tol, 0.5 * L->tol * mb.bn / mb.rn));
    VOX_CUDA(cudaMemsetAsync(wf.mem(wf.x, b), 0, n * sizeof(float2), st));
    if (L->side == VOX_PREC_LEFT && L->pc) {
      Members one;
      one.m0 = b;
      VOX_TRY(pc_apply<float>(L->pc, wf.mem(wf.b, b), wf.mem(wf.r, b), st, nullptr, one));
      op->launches += 3;
    } else {
      VOX_CUDA(cudaMemcpyAsync(wf.mem(wf.r, b), wf.mem(wf.b, b), n * sizeof(float2),
                               cudaMemcpyDeviceToDevice, st));
    }
    k_norm2<float><<<kRedBlocks, kRedThreads, 0, st>>>(wf.st + b, wf.mem(wf.r, b), n, 1, 0, 0);
    op->launches += 2;
  }
  for (int b : S)
    VOX_CUDA(cudaMemcpyAsync(&wf.hscal[b], &wf.st[b].scal[1], sizeof(double),
                             cudaMemcpyDeviceToHost, st));
  VOX_TRY(wait_stream(st));
  for (int b : S) {
    vox_lane_s::Member& mb = L->m[b];
    mb.ibn = std::sqrt(wf.hscal[b]);
    mb.outit = 0;
    mb.p = 0;
    if (mb.ibn == 0.0) {
      // nothing to solve: d = 0 (the inner GMRES returns at once)
      mb.rv.push_back(0.0);
      mb.inner = false;
      VOX_TRY(lane_header(L, b, 0.0, 1));
      continue;
    }
    mb.rv.push_back(1.0);
    mb.inner = true;
    VOX_TRY(lane_header(L, b, mb.itol * mb.ibn, 0, mb.ibn, mb.itol));
  }
  return VOX_OK;
}

// FP64 refinement step of every member in R: x += ||r||/Gram d, r = b - A x.
// Finished members go to `done`, the others to `again`.
static vox_status lane_refine(vox_lane_s* L, const std::vector<int>& R, std::vector<int>* done,
                              std::vector<int>* again) {
  if (R.empty()) return VOX_OK;
  vox_op_s* op = L->op;
  GmresWork<float>& wf = op->wf;
  GmresWork<double>& wd = op->wd;
  const long long n = op->g.n;
  cudaStream_t st = op->stream;
  const int nb = nblk(n);
  for (int b : R) {
    vox_lane_s::Member& mb = L->m[b];
    k_axpy_d2_from<<<nb, 256, 0, st>>>(n, wf.mem(wf.x, b), mb.rn / op->gram, mb.x);
    Members one;
    one.m0 = b;
    VOX_TRY(matvec<double>(op, MV_AN, mb.x, wd.mem(wd.w, b), st, nullptr, one));
    k_sub<double><<<nb, 256, 0, st>>>(n, wd.mem(wd.b, b), wd.mem(wd.w, b), wd.mem(wd.r, b));
    k_norm2<double><<<kRedBlocks, kRedThreads, 0, st>>>(wd.st + b, wd.mem(wd.r, b), n, 2, 0, 0);
    op->launches += 7;
  }
  for (int b : R)
    VOX_CUDA(cudaMemcpyAsync(&wd.hscal[b], &wd.st[b].scal[2], sizeof(double),
                             cudaMemcpyDeviceToHost, st));
  VOX_TRY(wait_stream(st));
  for (int b : R) {
    vox_lane_s::Member& mb = L->m[b];
    mb.rel = std::sqrt(wd.hscal[b]) / mb.bn;
    mb.info.refinements += 1;
    if (mb.rel <= L->tol || mb.info.refinements >= L->max_refine) {
      lane_finish(L, b);
      done->push_back(b);
    } else {
      again->push_back(b);
    }
  }
  return VOX_OK;
}

static vox_status lane_check(vox_lane_s* L) {
  vox_op_s* op = L->op;
  if (L->pc && std::find(op->pcs.begin(), op->pcs.end(), L->pc) == op->pcs.end()) {
    set_error("lane: its preconditioner was destroyed");
    return VOX_ERR_BAD_ARG;
  }
  return VOX_OK;
}

static vox_status lane_submit(vox_lane_s* L, int b, const double2* bdev, double2* xdev) {
  VOX_TRY(lane_check(L));
  vox_op_s* op = L->op;
  if (b < 0 || b >= op->K || L->m[b].state != 0) {
    set_error("lane: member " + std::to_string(b) + " is not free");
    return VOX_ERR_BAD_ARG;
  }
  GmresWork<double>& wd = op->wd;
  const long long n = op->g.n;
  cudaStream_t st = op->stream;
  vox_lane_s::Member& mb = L->m[b];
  mb = vox_lane_s::Member();
  mb.b = bdev;
  mb.x = xdev;
  mb.state = 1;
  // FP64 state: x = 0, r = b
  VOX_CUDA(cudaMemsetAsync(xdev, 0, n * sizeof(double2), st));
  VOX_CUDA(cudaMemcpyAsync(wd.mem(wd.b, b), bdev, n * sizeof(double2), cudaMemcpyDeviceToDevice,
                           st));
  VOX_CUDA(cudaMemcpyAsync(wd.mem(wd.r, b), bdev, n * sizeof(double2), cudaMemcpyDeviceToDevice,
                           st));
  k_norm2<double><<<kRedBlocks, kRedThreads, 0, st>>>(wd.st + b, wd.mem(wd.b, b), n, 3, 0, 0);
  op->launches += 1;
  VOX_CUDA(cudaMemcpyAsync(&wd.hscal[b], &wd.st[b].scal[3], sizeof(double),
                           cudaMemcpyDeviceToHost, st));
  VOX_TRY(wait_stream(st));
  mb.bn = std::sqrt(wd.hscal[b]);
  mb.rel = 1.0;
  if (mb.bn == 0.0 || mb.rel <= L->tol) {
    if (mb.bn == 0.0) mb.rel = 0.0;
    lane_finish(L, b);
    L->pending_done.push_back(b);
    return VOX_OK;
  }
  return lane_start_inner(L, {b});
}

// One restart cycle for every member in an inner solve, then the members'
// transitions; the members that finished are written to done[0..*n_done).
static vox_status lane_step(vox_lane_s* L, int* done, int* n_done) {
  VOX_TRY(lane_check(L));
  vox_op_s* op = L->op;
  GmresWork<float>& wf = op->wf;
  cudaStream_t st = op->stream;
  const int K = op->K;
  std::vector<int> fin = L->pending_done;
  L->pending_done.clear();
  std::vector<int> R;
  bool any = false;
  for (int b = 0; b < K; b++) any = any || (L->m[b].state == 1 && L->m[b].inner);
  if (any && L->steps > 0) {
    // out-of-phase steps; the device restarts cycles and ends inner solves
    if (use_cycle_graphs()) {
      cudaGraphExec_t g = nullptr;
      VOX_TRY(get_step_graph<float>(op, L->pc, L->side, K, L->steps, &g));
      VOX_CUDA(cudaGraphLaunch(g, st));
      op->launches += op->graph_nodes[g];
    } else {
      int nk = 0;
      VOX_TRY(enqueue_steps<float>(op, L->pc, L->side, K, L->steps, st, &nk));
      op->launches += nk;
    }
    for (int b = 0; b < K; b++)
      if (L->m[b].state == 1 && L->m[b].inner)
        VOX_CUDA(cudaMemcpyAsync(wf.hdr(b), &wf.st[b], offsetof(GmresDev, resvec),
                                 cudaMemcpyDeviceToHost, st));
    VOX_TRY(wait_stream(st));
    std::vector<int> fin_inner;
    for (int b = 0; b < K; b++) {
      vox_lane_s::Member& mb = L->m[b];
      if (mb.state != 1 || !mb.inner || !wf.hdr(b)->ifin) continue;
      fin_inner.push_back(b);
      const int nh = std::min(wf.hdr(b)->nhist, kHist);
      if (nh > 0)
        VOX_CUDA(cudaMemcpyAsync(L->hhist + (size_t)b * kHist, wf.st[b].hist, nh * sizeof(double),
                                 cudaMemcpyDeviceToHost, st));
    }
    if (!fin_inner.empty()) VOX_TRY(wait_stream(st));
    for (int b : fin_inner) {
      vox_lane_s::Member& mb = L->m[b];
      const GmresDev* hb = wf.hdr(b);
      const int nh = std::min(hb->nhist, kHist);
      for (int i = 0; i < nh; i++) mb.rv.push_back(L->hhist[(size_t)b * kHist + i] / mb.ibn);
      mb.info.total_iters += hb->itot;
      mb.outit = hb->cycles;
      mb.outer_total += hb->cycles;
      mb.p = hb->kdone;
      mb.inner = false;
      R.push_back(b);
    }
  } else if (any) {
    if (use_cycle_graphs()) {
      cudaGraphExec_t cyc = nullptr;
      VOX_TRY(get_cycle_graph<float>(op, L->pc, L->side, K, &cyc));
      VOX_CUDA(cudaGraphLaunch(cyc, st));
      op->launches += op->graph_nodes[cyc];
    } else {
      int nk = 0;
      VOX_TRY(enqueue_cycle<float>(op, L->pc, L->side, K, st, &nk));
      op->launches += nk;
    }
    for (int b = 0; b < K; b++)
      if (L->m[b].state == 1 && L->m[b].inner)
        VOX_CUDA(cudaMemcpyAsync(wf.hdr(b), &wf.st[b], offsetof(GmresDev, sn),
                                 cudaMemcpyDeviceToHost, st));
    VOX_TRY(wait_stream(st));
    for (int b = 0; b < K; b++) {
      vox_lane_s::Member& mb = L->m[b];
      if (mb.state != 1 || !mb.inner) continue;
      const GmresDev* hb = wf.hdr(b);
      mb.outit++;
      mb.outer_total++;
      mb.p = hb->k;
      for (int i = 0; i < mb.p; i++) mb.rv.push_back(hb->resvec[i] / mb.ibn);
      mb.info.total_iters += mb.p;
      const double ri = (mb.p > 0) ? hb->resvec[mb.p - 1] / mb.ibn : 1.0;
      const bool stop = !(ri > mb.itol && mb.outit < L->maxit_inner) ||
                        (hb->breakdown && !hb->converged);
      if (stop) {
        mb.inner = false;
        VOX_TRY(lane_freeze(L, b));
        R.push_back(b);
      }
    }
  }
  // members whose inner solve ended without cycles (zero inner right-hand side)
  for (int b = 0; b < K; b++)
    if (L->m[b].state == 1 && !L->m[b].inner &&
        std::find(R.begin(), R.end(), b) == R.end())
      R.push_back(b);
  // right preconditioning: each ended inner solve's x holds u = sum of its
  // cycles' V y; one apply of M^{-1} for all of them (as the single solve does)
  if (L->side == VOX_PREC_RIGHT && L->pc && !R.empty()) {
    std::vector<char> sel(K, 0);
    for (int b : R) sel[b] = L->m[b].ibn != 0.0;
    VOX_TRY(right_finish<float>(op, L->pc, K, sel.data(), st));
  }
  std::vector<int> again;
  VOX_TRY(lane_refine(L, R, &fin, &again));
  VOX_TRY(lane_start_inner(L, again));
  *n_done = (int)fin.size();
  for (size_t i = 0; i < fin.size(); i++) done[i] = fin[i];
  return VOX_OK;
}

}  // namespace vox

extern "C" {

vox_status vox_lane_create(vox_op_t op, vox_precond_t pc, int side, double tol, int restart,
                           int maxit_inner, double inner_tol, int max_refine, vox_lane_t* out) {
  if (!op || !out) {
    set_error("vox_lane_create: NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  *out = nullptr;
  if (!op->has_d || !op->has_f) {
    set_error("vox_lane_create: the operator needs complex128 and complex64 copies");
    return VOX_ERR_BAD_ARG;
  }
  if (restart < 1 || restart > kMaxRestart || maxit_inner < 1) {
    set_error("vox_lane_create: restart must be 1.." + std::to_string(kMaxRestart) +
              " and maxit_inner positive");
    return VOX_ERR_BAD_ARG;
  }
  if (pc && pc->K < op->K) {
    set_error("vox_lane_create: the preconditioner handle holds work for fewer members than "
              "the operator (share it with this operator)");
    return VOX_ERR_BAD_ARG;
  }
  DeviceGuard dg(op->device);
  VOX_TRY(ensure_work<float>(op, restart));
  if (!op->wd.arena) VOX_TRY(ensure_work<double>(op, 1));
  std::unique_ptr<vox_lane_s> L(new vox_lane_s());
  L->op = op;
  L->pc = pc;
  L->side = pc ? side : VOX_PREC_NONE;
  L->tol = tol;
  L->restart = restart;
  L->maxit_inner = maxit_inner;
  L->inner_tol = inner_tol;
  L->max_refine = max_refine < 1 ? 10 : max_refine;
  L->steps = step_mode_ok(op->wf) ? lane_steps_default() : 0;
  if (L->steps > 0)
    VOX_CUDA(cudaMallocHost((void**)&L->hhist, (size_t)op->K * kHist * sizeof(double)));
  L->m.resize(op->K);
  // every member frozen until it takes a right-hand side
  for (int b = 0; b < op->K; b++) VOX_TRY(lane_header(L.get(), b, 0.0, 1));
  VOX_TRY(wait_stream(op->stream));
  if (use_cycle_graphs()) {
    cudaGraphExec_t cyc = nullptr;
    if (L->steps > 0)
      VOX_TRY(get_step_graph<float>(op, pc, L->side, op->K, L->steps, &cyc));
    else
      VOX_TRY(get_cycle_graph<float>(op, pc, L->side, op->K, &cyc));
  }
  op->lanes.push_back(L.get());
  *out = L.release();
  return VOX_OK;
}

void vox_lane_destroy(vox_lane_t lane) {
  if (!lane) return;
  vox_op_s* op = lane->op;
  op->lanes.erase(std::remove(op->lanes.begin(), op->lanes.end(), lane), op->lanes.end());
  delete lane;
}

vox_status vox_lane_submit_device(vox_lane_t lane, int member, const void* b, void* x) {
  if (!lane || !b || !x) {
    set_error("vox_lane_submit_device: NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  DeviceGuard dg(lane->op->device);
  return lane_submit(lane, member, (const double2*)b, (double2*)x);
}

vox_status vox_lane_submit(vox_lane_t lane, int member, const double* b_re, const double* b_im) {
  if (!lane || !b_re) {
    set_error("vox_lane_submit: NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  vox_op_s* op = lane->op;
  if (member < 0 || member >= op->K) {
    set_error("vox_lane_submit: member out of range");
    return VOX_ERR_BAD_ARG;
  }
  DeviceGuard dg(op->device);
  const long long n = op->g.n;
  double2* hb = op->h_in + member * n;
  split_to_d2(b_re, b_im, n, hb);
  VOX_CUDA(cudaMemcpyAsync(op->d_in + member * n, hb, n * sizeof(double2),
                           cudaMemcpyHostToDevice, op->stream));
  return lane_submit(lane, member, op->d_in + member * n, op->d_out + member * n);
}

vox_status vox_lane_step(vox_lane_t lane, int* done, int* n_done) {
  if (!lane || !done || !n_done) {
    set_error("vox_lane_step: NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  DeviceGuard dg(lane->op->device);
  return lane_step(lane, done, n_done);
}

vox_status vox_lane_collect(vox_lane_t lane, int member, double* x_re, double* x_im,
                            vox_gmres_info* info) {
  if (!lane || member < 0 || member >= lane->op->K) {
    set_error("vox_lane_collect: bad argument");
    return VOX_ERR_BAD_ARG;
  }
  vox_lane_s::Member& mb = lane->m[member];
  if (mb.state != 2) {
    set_error("vox_lane_collect: member " + std::to_string(member) + " has not finished");
    return VOX_ERR_BAD_ARG;
  }
  vox_op_s* op = lane->op;
  DeviceGuard dg(op->device);
  if (x_re) {
    const long long n = op->g.n;
    double2* hx = op->h_out + member * n;
    VOX_CUDA(cudaMemcpyAsync(hx, mb.x, n * sizeof(double2), cudaMemcpyDeviceToHost,
                             op->stream));
    VOX_TRY(wait_stream(op->stream));
    d2_to_split(hx, n, x_re, x_im);
  }
  if (info) {
    double* buf = info->resvec;
    const long long cap = info->resvec_cap;
    *info = mb.info;
    info->resvec = buf;
    info->resvec_cap = cap;
    fill_resvec(info, mb.rv);
  }
  mb = vox_lane_s::Member();
  return VOX_OK;
}

vox_status vox_lane_state(vox_lane_t lane, int* states) {
  if (!lane || !states) {
    set_error("vox_lane_state: NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  for (int b = 0; b < lane->op->K; b++) states[b] = lane->m[b].state;
  return VOX_OK;
}

}  // extern "C"
