// Preconditioner handles, device GMRES driver (pgmres semantics) and the
// complex64 + FP64-refinement solver.  Included at the end of api.cu.
#pragma once

namespace vox {
struct PcFactors;
}

struct vox_precond_s {
  vox_op_s* op = nullptr;
  int kind = 0;                // 0 per-x-mode blocks (level 1), 1 level 2, 2 sum of parts
  PcGeom g{};                  // the grid it acts on (the operator's, or a box of it)
  const int* vmap = nullptr;   // that grid's index map into the operator's vector
  FftPlan pl{};
  FftPlan ply{};               // level 2: FFT along y
  double2* twyd = nullptr;     // level 2: y twiddles
  float2* twyf = nullptr;
  std::vector<vox_precond_s*> parts;  // sum: the parts (owned)
  double2* Ad = nullptr;       // c128 inverse blocks, Lf blocks of ld x ld (column-major)
  float2* Af = nullptr;        // c64 copy (Gram * inverse, for the A/Gram operator)
  int ld = 0;                  // leading dimension of the blocks (3MN rounded up to 32)
  int* piv = nullptr;          // Lf * n3 getrf pivots
  int* perm = nullptr;         // Lf * n3 row permutation of the pivots
  int Lf = 0;                  // stored blocks (L, or L/2+1 with pairing)
  int paired = 0;              // mode L-f applied with the block of mode f
  double2* Dld = nullptr;      // inverted diagonal blocks of L and U (c128)
  double2* Dud = nullptr;
  float2* Dlf = nullptr;       // ... and of the c64 copy
  float2* Duf = nullptr;
  double2* tiles_d = nullptr;  // per-mode LU tile streams (c128, c64)
  float2* tiles_f = nullptr;
  double2* twd = nullptr;
  float2* twf = nullptr;
  double2* Td = nullptr;       // L * n3 work
  double2* Td2 = nullptr;
  float2* Tf = nullptr;
  float2* Tf2 = nullptr;
  double f_scale = 1.0;        // the c64 copy applies f_scale * M^{-1}
  int K = 0;                   // members whose work the T* buffers hold
  // Owner of the factor arrays above (Ad/Af/piv/perm/D*/tiles/tw): set once
  // construction succeeds; views made by vox_precond_share hold a copy, and the
  // arrays are freed with the last holder.  Work buffers T* are per handle.
  std::shared_ptr<vox::PcFactors> factors;
};

namespace vox {

static size_t pc_xsmem(const PcGeom& g, size_t cs) { return 2ull * g.ybx * g.sx * cs; }

template <typename R> Cx<R>* pc_A(vox_precond_s* p);
template <> double2* pc_A<double>(vox_precond_s* p) { return p->Ad; }
template <> float2* pc_A<float>(vox_precond_s* p) { return p->Af; }
template <typename R> Cx<R>* pc_T(vox_precond_s* p, int which);
template <> double2* pc_T<double>(vox_precond_s* p, int w) { return w ? p->Td2 : p->Td; }
template <> float2* pc_T<float>(vox_precond_s* p, int w) { return w ? p->Tf2 : p->Tf; }
template <typename R> Cx<R>* pc_Dl(vox_precond_s* p);
template <> double2* pc_Dl<double>(vox_precond_s* p) { return p->Dld; }
template <> float2* pc_Dl<float>(vox_precond_s* p) { return p->Dlf; }
template <typename R> Cx<R>* pc_Du(vox_precond_s* p);
template <> double2* pc_Du<double>(vox_precond_s* p) { return p->Dud; }
template <> float2* pc_Du<float>(vox_precond_s* p) { return p->Duf; }
template <typename R> Cx<R>* pc_tw(vox_precond_s* p);
template <> double2* pc_tw<double>(vox_precond_s* p) { return p->twd; }
template <> float2* pc_tw<float>(vox_precond_s* p) { return p->twf; }

// Right-hand-side columns of one inverse-block apply for km members: two per
// member slot, slots rounded up to a power of two (one instantiation each).
static int lu_cols(int km) {
  int ks = 1;
  while (ks < km) ks *= 2;
  return 2 * ks;
}
// Members per launch: every block is streamed once per launch, and the FMAs
// per streamed byte grow with the members; up to 4 members (8 columns, whose
// right-hand sides take 93 KiB (complex64) or 124 KiB (complex128) of shared
// memory at ld = 992) in either precision.  More members are applied in groups
// of this size.
template <typename R>
constexpr int apply_members() {
  return 4;
}

// Ring stages that fit beside the right-hand sides (at least 2 needed).
template <typename R>
static int str_stages(int ld, int P) {
  int s = 0;
  while (s < kStrMaxStages && str_smem<R>(ld, P, s + 1) <= (size_t)kSmemCap) s++;
  return s;
}

template <typename R, int P>
static void launch_inv_apply(vox_precond_s* p, const Cx<R>* T, Cx<R>* T2, cudaStream_t st,
                             const int* skip, int fs, int km) {
  const PcGeom& g = p->g;
  const int stages = str_stages<R>(p->ld, P);
  const dim3 grid(p->Lf);
  k_pc_inv_stream<R, P><<<grid, kStrThreads, str_smem<R>(p->ld, P, stages), st>>>(
      g, p->paired, p->ld, stages, pc_A<R>(p), T, T2, skip, fs, km);
}

// T2 = per-mode inverse blocks applied to T, for km members (in groups of
// apply_members, each group one launch).
template <typename R>
static vox_status inv_apply(vox_precond_s* p, const Cx<R>* T, Cx<R>* T2, cudaStream_t st,
                            const int* skip, int fs, int km) {
  const long long ws = pc_work_elems(p->g);
  for (int m0 = 0; m0 < km; m0 += apply_members<R>()) {
    const int kg = std::min(apply_members<R>(), km - m0);
    const int P = lu_cols(kg);
    if (p->ld > 2 * kStrConsumers || str_stages<R>(p->ld, P) < 2 ||
        str_smem<R>(p->ld, P, 2) > (size_t)kSmemCap) {
      set_error("preconditioner: blocks of " + std::to_string(p->ld) +
                " rows leave no room for the streaming ring at " + std::to_string(kg) +
                " members in this precision");
      return VOX_ERR_UNSUPPORTED;
    }
    const Cx<R>* Tg = T + m0 * ws;
    Cx<R>* T2g = T2 + m0 * ws;
    const int* sg = skip ? skip + (long long)m0 * fs : nullptr;
    switch (P) {
      case 2: launch_inv_apply<R, 2>(p, Tg, T2g, st, sg, fs, kg); break;
      case 4: launch_inv_apply<R, 4>(p, Tg, T2g, st, sg, fs, kg); break;
      default: launch_inv_apply<R, 8>(p, Tg, T2g, st, sg, fs, kg); break;
    }
  }
  return VOX_OK;
}

template <typename R> Cx<R>* pc_twy(vox_precond_s* p);
template <> double2* pc_twy<double>(vox_precond_s* p) { return p->twyd; }
template <> float2* pc_twy<float>(vox_precond_s* p) { return p->twyf; }

static int l2_cols(int km) {
  int c = 1;
  while (c < km) c *= 2;
  return c;
}

template <typename R, int P>
static void launch_l2_gemv(vox_precond_s* p, const Cx<R>* X, Cx<R>* Y, cudaStream_t st,
                           const int* skip, int fs, int km) {
  const PcGeom& g = p->g;
  const long long nb = ((long long)g.L * g.M + 7) / 8;
  k_l2_gemv<R, P><<<(unsigned)nb, 256, (size_t)8 * 3 * g.N * P * sizeof(Cx<R>), st>>>(
      g, pc_A<R>(p), X, Y, skip, fs, km);
}

// Level-2 per-(x, y)-mode products on the x-transformed work T of km members
// (T is overwritten; the result lands in T2).
template <typename R>
static vox_status l2_apply(vox_precond_s* p, Cx<R>* T, Cx<R>* T2, cudaStream_t st,
                           const int* skip, int fs, int km) {
  const PcGeom& g = p->g;
  const size_t ys = (size_t)2 * kL2Lines * pad_stride(g.M) * sizeof(Cx<R>);
  const dim3 gy((3 * g.N + kL2Lines - 1) / kL2Lines, g.L * km);
  k_l2_yfwd<R><<<gy, 256, ys, st>>>(g, p->ply, pc_twy<R>(p), T, T2, skip, fs);
  switch (l2_cols(km)) {
    case 1: launch_l2_gemv<R, 1>(p, T2, T, st, skip, fs, km); break;
    case 2: launch_l2_gemv<R, 2>(p, T2, T, st, skip, fs, km); break;
    case 4: launch_l2_gemv<R, 4>(p, T2, T, st, skip, fs, km); break;
    default: launch_l2_gemv<R, 8>(p, T2, T, st, skip, fs, km); break;
  }
  k_l2_yinv<R><<<gy, 256, ys, st>>>(g, p->ply, pc_twy<R>(p), T, T2, skip, fs);
  VOX_CUDA(cudaGetLastError());
  return VOX_OK;
}

// out = M^{-1} in (c128) or f_scale * M^{-1} in (c64 copy), for the members
// of mm (vectors mm.vs apart, skip flags mm.fs apart); mm.m0 selects the
// first member's work in this handle.
// x-FFT kernels of the preconditioner: the big-prime instantiation only for
// lengths L that need it.
static bool plan_has_big_prime(const FftPlan& pl) {
  for (int s = 0; s < pl.nst; s++)
    if (pl.radix[s] > 13) return true;
  return false;
}

template <typename R>
static void pc_xfwd_launch(vox_precond_s* p, const PcGeom& g, dim3 grid, cudaStream_t st,
                           const Cx<R>* in, const int* vmap, Cx<R>* T, const int* skip,
                           long long vs, int fs) {
  const size_t sm = pc_xsmem(g, sizeof(Cx<R>));
  if (plan_has_big_prime(p->pl))
    k_pc_xfwd<R, true><<<grid, 256, sm, st>>>(g, p->pl, pc_tw<R>(p), in, vmap, T, skip, vs, fs);
  else
    k_pc_xfwd<R, false><<<grid, 256, sm, st>>>(g, p->pl, pc_tw<R>(p), in, vmap, T, skip, vs, fs);
}

template <typename R>
static void pc_xinv_launch(vox_precond_s* p, const PcGeom& g, dim3 grid, cudaStream_t st,
                           const Cx<R>* T2, const int* vmap, Cx<R>* out, const int* skip,
                           long long vs, int fs) {
  const size_t sm = pc_xsmem(g, sizeof(Cx<R>));
  const R scale = (R)(1.0 / g.L);
  if (plan_has_big_prime(p->pl))
    k_pc_xinv<R, true><<<grid, 256, sm, st>>>(g, p->pl, pc_tw<R>(p), T2, vmap, scale, out, skip,
                                              vs, fs);
  else
    k_pc_xinv<R, false><<<grid, 256, sm, st>>>(g, p->pl, pc_tw<R>(p), T2, vmap, scale, out,
                                               skip, vs, fs);
}

template <typename R>
static vox_status pc_apply(vox_precond_s* p, const Cx<R>* in, Cx<R>* out, cudaStream_t st,
                           const int* skip, Members mm = Members()) {
  if (mm.m0 + mm.km > p->K) {
    set_error("preconditioner: this handle holds work for " + std::to_string(p->K) +
              " member(s); share it with the batched operator (vox_precond_share)");
    return VOX_ERR_BAD_ARG;
  }
  const PcGeom& g = p->g;
  const int nb = (g.n3 + g.ybx - 1) / g.ybx;
  const dim3 gx(nb, mm.km);
  Cx<R>* T = pc_T<R>(p, 0) + mm.m0 * pc_work_elems(g);
  Cx<R>* T2 = pc_T<R>(p, 1) + mm.m0 * pc_work_elems(g);
  if (p->kind == 2) {
    // sum: identity, then each part on its own box of the grid
    k_copy_members<R><<<dim3(nblk(p->op->g.n), mm.km), 256, 0, st>>>(p->op->g.n, in, out, skip,
                                                                     mm.vs, mm.fs);
    for (vox_precond_s* q : p->parts) VOX_TRY(pc_apply<R>(q, in, out, st, skip, mm));
    VOX_CUDA(cudaGetLastError());
    return VOX_OK;
  }
  pc_xfwd_launch<R>(p, g, gx, st, in, p->vmap, T, skip, mm.vs, mm.fs);
  if (p->kind == 1) {
    VOX_TRY(l2_apply<R>(p, T, T2, st, skip, mm.fs, mm.km));
  } else {
    VOX_TRY(inv_apply<R>(p, T, T2, st, skip, mm.fs, mm.km));
  }
  pc_xinv_launch<R>(p, g, gx, st, T2, p->vmap, out, skip, mm.vs, mm.fs);
  VOX_CUDA(cudaGetLastError());
  return VOX_OK;
}

template <typename R>
static vox_status pc_attrs() {
  VOX_TRY(smem_cap(k_pc_xfwd<R, false>));
  VOX_TRY(smem_cap(k_pc_xinv<R, false>));
  VOX_TRY(smem_cap(k_pc_xfwd<R, true>));
  VOX_TRY(smem_cap(k_pc_xinv<R, true>));
  VOX_TRY(smem_cap(k_pc_inv_stream<R, 2>));
  VOX_TRY(smem_cap(k_pc_inv_stream<R, 4>));
  VOX_TRY(smem_cap(k_pc_inv_stream<R, 8>));
  VOX_TRY(smem_cap(k_l2_yfwd<R>));
  VOX_TRY(smem_cap(k_l2_yinv<R>));
  VOX_TRY(smem_cap(k_l2_gemv<R, 1>));
  VOX_TRY(smem_cap(k_l2_gemv<R, 2>));
  VOX_TRY(smem_cap(k_l2_gemv<R, 4>));
  VOX_TRY(smem_cap(k_l2_gemv<R, 8>));
  VOX_TRY(smem_cap(k_lu_batched<R>));
  return VOX_OK;
}

// Per-handle work: the x-transformed vectors of every member of the operator.
static vox_status pc_alloc_work(vox_precond_s* p, int K) {
  const long long LT = pc_work_elems(p->g) * K;
  VOX_TRY(dalloc(&p->Td, LT));
  VOX_TRY(dalloc(&p->Td2, LT));
  VOX_TRY(dalloc(&p->Tf, LT));
  VOX_TRY(dalloc(&p->Tf2, LT));
  p->K = K;
  return VOX_OK;
}

// The factor arrays of a finished preconditioner; freed when the last handle
// (the original or a view made by vox_precond_share) lets go of them.
struct PcFactors {
  double2 *Ad = nullptr, *Dld = nullptr, *Dud = nullptr, *tiles_d = nullptr, *twd = nullptr;
  float2 *Af = nullptr, *Dlf = nullptr, *Duf = nullptr, *tiles_f = nullptr, *twf = nullptr;
  int *piv = nullptr, *perm = nullptr;
  double2* twyd = nullptr;
  float2* twyf = nullptr;
  int* vmap = nullptr;  // a box's own index map
  ~PcFactors() {
    dfree(twyd);
    dfree(twyf);
    dfree(vmap);
    dfree(Ad);
    dfree(Af);
    dfree(piv);
    dfree(perm);
    dfree(Dld);
    dfree(Dud);
    dfree(Dlf);
    dfree(Duf);
    dfree(tiles_d);
    dfree(tiles_f);
    dfree(twd);
    dfree(twf);
  }
};

// Hand the factor arrays to a shared owner (called once a handle is complete).
static void pc_seal(vox_precond_s* p) {
  auto f = std::make_shared<PcFactors>();
  f->Ad = p->Ad;
  f->Dld = p->Dld;
  f->Dud = p->Dud;
  f->tiles_d = p->tiles_d;
  f->twd = p->twd;
  f->Af = p->Af;
  f->Dlf = p->Dlf;
  f->Duf = p->Duf;
  f->tiles_f = p->tiles_f;
  f->twf = p->twf;
  f->piv = p->piv;
  f->perm = p->perm;
  f->twyd = p->twyd;
  f->twyf = p->twyf;
  if (p->op && p->vmap != p->op->vmap) f->vmap = const_cast<int*>(p->vmap);
  p->factors = std::move(f);
}

static void pc_free(vox_precond_s* p) {
  if (!p) return;
  for (vox_precond_s* q : p->parts) pc_free(q);  // a sum owns its parts
  p->parts.clear();
  if (p->factors) {
    p->factors.reset();  // frees the arrays only if no view still holds them
  } else {  // construction did not complete: the arrays are still this handle's
    PcFactors own;
    own.Ad = p->Ad;
    own.Dld = p->Dld;
    own.Dud = p->Dud;
    own.tiles_d = p->tiles_d;
    own.twd = p->twd;
    own.Af = p->Af;
    own.Dlf = p->Dlf;
    own.Duf = p->Duf;
    own.tiles_f = p->tiles_f;
    own.twf = p->twf;
    own.piv = p->piv;
    own.perm = p->perm;
    own.twyd = p->twyd;
    own.twyf = p->twyf;
    if (p->op && p->vmap && p->vmap != p->op->vmap) own.vmap = const_cast<int*>(p->vmap);
  }
  dfree(p->Td);
  dfree(p->Td2);
  dfree(p->Tf);
  dfree(p->Tf2);
  delete p;
}

// Grid, x-FFT plan, twiddles and work of a preconditioner acting on an
// L x M x N grid (the operator's, or a box of it with its own index map set
// by the caller); `lu` adds the checks of the per-x-mode LU build.
static vox_status pc_common(vox_op_s* op, vox_precond_s* p, int L, int M, int N, bool lu) {
  p->op = op;
  if (!p->vmap) p->vmap = op->vmap;
  PcGeom& g = p->g;
  g.L = L;
  g.M = M;
  g.N = N;
  g.n3 = 3 * g.M * g.N;
  g.V = (long long)L * M * N;
  if (!make_fft_plan(g.L, &p->pl)) {
    set_error("preconditioner: FFT length L has a prime factor above 64");
    return VOX_ERR_UNSUPPORTED;
  }
  g.sx = pad_stride(g.L);
  const size_t per = 2ull * g.sx * sizeof(double2);
  g.ybx = (int)std::max<size_t>(1, std::min<size_t>(8, kSmemBudget / per));
  if (per > (size_t)kSmemCap) {
    set_error("preconditioner: L too long for the shared-memory FFT");
    return VOX_ERR_UNSUPPORTED;
  }
  // the LU panel bound (n3 <= 1760) also keeps the streamed solve's
  // ring + right-hand sides (64 KiB + 32 B * n3) and the streamed apply's
  // (two 32 KiB stages + 32 B * ld) under the cap
  if (lu && ((size_t)g.n3 * kLuNb * sizeof(double2) > (size_t)kSmemCap ||
             lu_stream2_smem<double>(lu_npad(g.n3), kInvBuildCols) > (size_t)kSmemCap ||
             str_smem<double>((g.n3 + 31) / 32 * 32, 2, 2) > (size_t)kSmemCap ||
             (g.n3 + 31) / 32 * 32 > 2 * kStrConsumers)) {
    set_error("preconditioner: 3*M*N too large for the batched LU panel");
    return VOX_ERR_UNSUPPORTED;
  }
  std::vector<double2> tw = twiddles(g.L);
  std::vector<float2> twf(g.L);
  for (int i = 0; i < g.L; i++) twf[i] = make_float2((float)tw[i].x, (float)tw[i].y);
  VOX_TRY(dalloc(&p->twd, g.L));
  VOX_TRY(dalloc(&p->twf, g.L));
  VOX_CUDA(cudaMemcpyAsync(p->twd, tw.data(), g.L * sizeof(double2), cudaMemcpyHostToDevice,
                           op->stream));
  VOX_CUDA(cudaMemcpyAsync(p->twf, twf.data(), g.L * sizeof(float2), cudaMemcpyHostToDevice,
                           op->stream));
  VOX_TRY(pc_alloc_work(p, op->K));
  VOX_TRY(pc_attrs<double>());
  VOX_TRY(pc_attrs<float>());
  VOX_TRY(smem_cap(k_lu_inv_cols<kInvBuildCols>));
  p->ld = lu_npad(g.n3);
  return VOX_OK;
}

// Level-1 inverse blocks of the grid of p (pc_common done): per x-mode
// inv(gram_block*I - face3 .* circ_i(G)) times `scale`, G the L x M x N x 6
// Toeplitz-like tensor of that grid (level_1_parallel_func_N.m:1-281 +
// Bragg_MOR_script.m:61-72; with gram_block = 0, face3 = -1 and G = -Mc.*G +
// Gram*Mr(1) at the origin it is level_1_parallel_func.m:1-255).  Modes L-i
// reuse block i when the tensor allows it.
static vox_status build_level1(vox_op_s* op, vox_precond_s* p, const std::vector<double2>& G,
                               const std::vector<double>& face3, double gram_block,
                               double scale) {
  const PcGeom& g = p->g;
  cudaStream_t st = op->stream;
  const long long V = g.V;
  // Toeplitz -> Chan circulants -> FFT along x
  double2 *dG, *dC;
  VOX_TRY(dalloc(&dG, 6 * V));
  std::unique_ptr<double2, decltype(&dfree)> gG(dG, dfree);
  VOX_TRY(dalloc(&dC, 6 * V));
  std::unique_ptr<double2, decltype(&dfree)> gC(dC, dfree);
  VOX_CUDA(cudaMemcpyAsync(dG, G.data(), 6 * V * sizeof(double2), cudaMemcpyHostToDevice,
                           st));
  k_chan<<<nblk(6 * V), 256, 0, st>>>(g.L, V, dG, dC);
  VOX_CUDA(cudaGetLastError());
  VOX_TRY(fft_axis_d(dC, g.L, g.M, g.N, 1, g.L, (long long)g.L * g.M, V, 6, 0, -1, st));
  double* dface;
  VOX_TRY(dalloc(&dface, g.n3));
  std::unique_ptr<double, decltype(&dfree)> gF(dface, dfree);
  VOX_CUDA(cudaMemcpyAsync(dface, face3.data(), g.n3 * sizeof(double), cudaMemcpyHostToDevice,
                           st));
  // Pairing: the Chan circulants satisfy c[L-j] = s*c[j] (s = -1 for xy, xz),
  // so B_{L-i} = D B_i D exactly when G_xy and G_xz vanish on the x = 0 plane
  // (true of the physical tensor); then only modes 0..L/2 are factored.
  {
    double gmax = 0.0, g0 = 0.0;
    for (long long i = 0; i < 6 * V; i++) gmax = std::max(gmax, std::abs(G[i].x) + std::abs(G[i].y));
    for (int comp = 1; comp <= 2; comp++)
      for (long long c = 0; c < (long long)g.M * g.N; c++) {
        const double2 v = G[comp * V + c * g.L];
        g0 = std::max(g0, std::abs(v.x) + std::abs(v.y));
      }
    p->paired = (g0 <= 1e-13 * gmax) ? 1 : 0;
  }
  p->Lf = p->paired ? g.L / 2 + 1 : g.L;
  const int Lf = p->Lf;
  // factors kept column-major with leading dimension ld = 3MN rounded up to
  // whole 32-blocks (zero padding) for the streamed triangular solves
  const int ld = lu_npad(g.n3);
  const long long per = (long long)g.n3 * g.n3;
  const long long perp = (long long)ld * ld;
  const int nbd = (g.n3 + kTrsvNb - 1) / kTrsvNb;
  const long long dsz = (long long)Lf * nbd * kTrsvNb * kTrsvNb;
  VOX_TRY(dalloc(&p->Ad, Lf * perp));
  VOX_CUDA(cudaMemsetAsync(p->Ad, 0, Lf * perp * sizeof(double2), st));
  VOX_TRY(dalloc(&p->piv, (long long)Lf * g.n3));
  VOX_TRY(dalloc(&p->perm, (long long)Lf * g.n3));
  VOX_TRY(dalloc(&p->Dld, dsz));
  VOX_TRY(dalloc(&p->Dud, dsz));
  k_assemble_blocks<<<nblk(Lf * per), 256, 0, st>>>(g.L, g.M, g.N, V, 0, Lf, ld, dC, dface,
                                                     gram_block, p->Ad);
  VOX_CUDA(cudaGetLastError());
  int* dinfo;
  VOX_TRY(dalloc(&dinfo, Lf));
  std::unique_ptr<int, decltype(&dfree)> gI(dinfo, dfree);
  VOX_CUDA(cudaMemsetAsync(dinfo, 0, Lf * sizeof(int), st));
  k_lu_batched<double><<<Lf, 512, (size_t)g.n3 * kLuNb * sizeof(double2), st>>>(g.n3, ld, p->Ad,
                                                                                p->piv, dinfo);
  VOX_CUDA(cudaGetLastError());
  std::vector<int> info(Lf);
  VOX_CUDA(cudaMemcpyAsync(info.data(), dinfo, Lf * sizeof(int), cudaMemcpyDeviceToHost, st));
  VOX_TRY(wait_stream(st));
  for (int i = 0; i < Lf; i++)
    if (info[i]) {
      set_error("level-1 preconditioner: block " + std::to_string(i) + " is singular");
      return VOX_ERR_BAD_ARG;
    }
  k_lu_perm<<<Lf, 32, 0, st>>>(g.n3, p->piv, p->perm);
  k_tri_inv_blocks<<<dim3(nbd, Lf), 64, 0, st>>>(g.n3, ld, p->Ad, p->Dld, p->Dud);
  VOX_CUDA(cudaGetLastError());
  // repack the factors into per-mode tile streams in consumption order, then
  // solve for the explicit inverse blocks (the reference's circ_inv) column
  // group by column group into the factors' own buffer, which the tiles no
  // longer need
  const long long tsz = (long long)Lf * lu_tiles(nbd) * kTrsvNb * kTrsvNb;
  VOX_TRY(dalloc(&p->tiles_d, tsz));
  k_tile_pack<double><<<dim3(lu_tiles(nbd), Lf), 256, 0, st>>>(nbd, ld, p->Ad, p->Dld, p->Dud,
                                                               1.0, 1.0, p->tiles_d);
  VOX_CUDA(cudaMemsetAsync(p->Ad, 0, Lf * perp * sizeof(double2), st));
  k_lu_inv_cols<kInvBuildCols>
      <<<dim3((g.n3 + kInvBuildCols - 1) / kInvBuildCols, Lf), 32 * kRoundTiles,
         lu_stream2_smem<double>(ld, kInvBuildCols), st>>>(g, p->tiles_d, p->perm, ld, p->Ad);
  VOX_CUDA(cudaGetLastError());
  if (scale != 1.0) k_cast_scale<double><<<nblk(Lf * perp), 256, 0, st>>>(Lf * perp, p->Ad, scale,
                                                                         p->Ad);
  // c64 copy of Gram * inverse: it preconditions the c64 operator A/Gram
  p->f_scale = op->gram;
  if (op->has_f) {
    VOX_TRY(dalloc(&p->Af, Lf * perp));
    k_cast_scale<float><<<nblk(Lf * perp), 256, 0, st>>>(Lf * perp, p->Ad, op->gram, p->Af);
    VOX_CUDA(cudaGetLastError());
  }
  VOX_TRY(wait_stream(st));
  dfree(p->tiles_d);
  dfree(p->Dld);
  dfree(p->Dud);
  p->tiles_d = nullptr;
  p->Dld = p->Dud = nullptr;
  (void)dsz;
  p->kind = 0;
  p->ld = ld;
  return VOX_OK;
}

// Level-2 inverse blocks of the grid of p (pc_common done), from
// A = -Mc.*G + Gram*Mr(1) at the origin (level_2_parallel_func.m:1-193): per
// x-mode i and y-mode m the 3N x 3N block, inverted, times `scale`.
static vox_status build_level2(vox_op_s* op, vox_precond_s* p, const std::vector<double2>& A,
                               double scale) {
  const PcGeom& g = p->g;
  cudaStream_t st = op->stream;
  const long long V = g.V;
  const int n2 = 3 * g.N;
  if (n2 > 64) {
    set_error("level-2 preconditioner: 3N above 64");
    return VOX_ERR_UNSUPPORTED;
  }
  if (!make_fft_plan(g.M, &p->ply)) {
    set_error("level-2 preconditioner: FFT length M has a prime factor above 64");
    return VOX_ERR_UNSUPPORTED;
  }
  if ((size_t)2 * kL2Lines * pad_stride(g.M) * sizeof(double2) > (size_t)kSmemCap) {
    set_error("level-2 preconditioner: M too long for the shared-memory FFT");
    return VOX_ERR_UNSUPPORTED;
  }
  std::vector<double2> tw = twiddles(g.M);
  std::vector<float2> twf(g.M);
  for (int i = 0; i < g.M; i++) twf[i] = make_float2((float)tw[i].x, (float)tw[i].y);
  VOX_TRY(dalloc(&p->twyd, g.M));
  VOX_TRY(dalloc(&p->twyf, g.M));
  VOX_CUDA(cudaMemcpyAsync(p->twyd, tw.data(), g.M * sizeof(double2), cudaMemcpyHostToDevice,
                           st));
  VOX_CUDA(cudaMemcpyAsync(p->twyf, twf.data(), g.M * sizeof(float2), cudaMemcpyHostToDevice,
                           st));
  double2 *dA, *dC;
  VOX_TRY(dalloc(&dA, 6 * V));
  std::unique_ptr<double2, decltype(&dfree)> gA(dA, dfree);
  VOX_TRY(dalloc(&dC, 6 * V));
  std::unique_ptr<double2, decltype(&dfree)> gC(dC, dfree);
  VOX_CUDA(cudaMemcpyAsync(dA, A.data(), 6 * V * sizeof(double2), cudaMemcpyHostToDevice,
                           st));
  k_chan<<<nblk(6 * V), 256, 0, st>>>(g.L, V, dA, dC);
  VOX_CUDA(cudaGetLastError());
  VOX_TRY(fft_axis_d(dC, g.L, g.M, g.N, 1, g.L, (long long)g.L * g.M, V, 6, 0, -1, st));
  const long long nblocks = (long long)g.L * g.M;
  const long long tot = nblocks * n2 * n2;
  VOX_TRY(dalloc(&p->Ad, tot));
  VOX_TRY(smem_cap(k_level2_blocks));
  VOX_TRY(smem_cap(k_small_inv));
  k_level2_blocks<<<dim3(n2 * n2, g.L), 256, (size_t)2 * pad_stride(g.M) * sizeof(double2), st>>>(
      g.L, g.M, g.N, V, p->ply, p->twyd, dC, p->Ad);
  VOX_CUDA(cudaGetLastError());
  int* dinfo;
  VOX_TRY(dalloc(&dinfo, nblocks));
  std::unique_ptr<int, decltype(&dfree)> gI(dinfo, dfree);
  VOX_CUDA(cudaMemsetAsync(dinfo, 0, nblocks * sizeof(int), st));
  k_small_inv<<<(unsigned)nblocks, 128, (size_t)2 * n2 * n2 * sizeof(double2), st>>>(n2, p->Ad,
                                                                                     dinfo);
  VOX_CUDA(cudaGetLastError());
  std::vector<int> info(nblocks);
  VOX_CUDA(cudaMemcpyAsync(info.data(), dinfo, nblocks * sizeof(int), cudaMemcpyDeviceToHost, st));
  VOX_TRY(wait_stream(st));
  for (long long i = 0; i < nblocks; i++)
    if (info[i]) {
      set_error("level-2 preconditioner: block " + std::to_string(i) + " is singular");
      return VOX_ERR_BAD_ARG;
    }
  if (scale != 1.0) k_cast_scale<double><<<nblk(tot), 256, 0, st>>>(tot, p->Ad, scale, p->Ad);
  p->f_scale = op->gram;
  if (op->has_f) {
    VOX_TRY(dalloc(&p->Af, tot));
    k_cast_scale<float><<<nblk(tot), 256, 0, st>>>(tot, p->Ad, op->gram, p->Af);
  }
  VOX_CUDA(cudaGetLastError());
  VOX_TRY(wait_stream(st));
  p->kind = 1;
  p->Lf = g.L;
  p->paired = 0;
  p->ld = n2;
  return VOX_OK;
}

}  // namespace vox

extern "C" {

vox_status vox_precond_create_level1(vox_op_t op, const double* G_re, const double* G_im,
                                     const double* face3, vox_precond_t* out) {
  if (!op || !G_re || !face3 || !out) {
    set_error("vox_precond_create_level1: NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  *out = nullptr;
  DeviceGuard dg(op->device);
  std::unique_ptr<vox_precond_s, void (*)(vox_precond_s*)> p(new vox_precond_s(), pc_free);
  VOX_TRY(pc_common(op, p.get(), op->g.L, op->g.M, op->g.N, true));
  const long long V = p->g.V;
  std::vector<double2> G(6 * V);
  for (long long i = 0; i < 6 * V; i++) G[i] = make_double2(G_re[i], G_im ? G_im[i] : 0.0);
  std::vector<double> f3(face3, face3 + p->g.n3);
  VOX_TRY(build_level1(op, p.get(), G, f3, op->gram, 1.0));
  pc_seal(p.get());
  op->pcs.push_back(p.get());
  *out = p.release();
  return VOX_OK;
}

vox_status vox_precond_create_box(vox_op_t op, int level, int x0, int y0, int Ls, int Ms,
                                  const unsigned char* mask, const double* G_re,
                                  const double* G_im, const double* Mc_re, const double* Mc_im,
                                  double Mr1, double scale, vox_precond_t* out) {
  if (!op || !G_re || !Mc_re || !out) {
    set_error("vox_precond_create_box: NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  *out = nullptr;
  if (level != 1 && level != 2) {
    set_error("vox_precond_create_box: level must be 1 or 2");
    return VOX_ERR_BAD_ARG;
  }
  if (Ls < 1 || Ms < 1 || x0 < 0 || y0 < 0 || x0 + Ls > op->g.L || y0 + Ms > op->g.M) {
    set_error("vox_precond_create_box: the box leaves the operator's grid");
    return VOX_ERR_BAD_ARG;
  }
  DeviceGuard dg(op->device);
  const int Ns = op->g.N;
  const long long Vs = (long long)Ls * Ms * Ns;
  std::unique_ptr<vox_precond_s, void (*)(vox_precond_s*)> p(new vox_precond_s(), pc_free);
  // the box's own index map into the operator's vector
  int* vm;
  VOX_TRY(dalloc(&vm, 3 * Vs));
  p->vmap = vm;
  p->op = op;
  {
    unsigned char* dmask = nullptr;
    if (mask) {
      VOX_TRY(dalloc(&dmask, Vs));
      VOX_CUDA(cudaMemcpyAsync(dmask, mask, Vs, cudaMemcpyHostToDevice,
                               op->stream));
    }
    k_vmap_box<<<nblk(3 * Vs), 256, 0, op->stream>>>(op->g.L, op->g.M, Ns, x0, y0, Ls, Ms,
                                                     op->vmap, dmask, vm);
    VOX_CUDA(cudaGetLastError());
    VOX_TRY(wait_stream(op->stream));
    dfree(dmask);
  }
  VOX_TRY(pc_common(op, p.get(), Ls, Ms, Ns, level == 1));
  // A = -Mc .* G, Gram * Mr(1) added at the origin of the diagonal components
  std::vector<double2> A(6 * Vs);
  for (int c = 0; c < 6; c++)
    for (long long e = 0; e < Vs; e++) {
      const double gr = G_re[c * Vs + e], gi = G_im ? G_im[c * Vs + e] : 0.0;
      const double mr = Mc_re[e], mi = Mc_im ? Mc_im[e] : 0.0;
      A[c * Vs + e] = make_double2(-(mr * gr - mi * gi), -(mr * gi + mi * gr));
    }
  for (int c : {0, 3, 5}) A[c * Vs].x += op->gram * Mr1;
  if (level == 1) {
    std::vector<double> f3(p->g.n3, -1.0);
    VOX_TRY(build_level1(op, p.get(), A, f3, 0.0, scale));
  } else {
    VOX_TRY(build_level2(op, p.get(), A, scale));
  }
  pc_seal(p.get());
  op->pcs.push_back(p.get());
  *out = p.release();
  return VOX_OK;
}

vox_status vox_precond_create_sum(vox_op_t op, const vox_precond_t* parts, int n,
                                  vox_precond_t* out) {
  if (!op || !parts || n < 1 || !out) {
    set_error("vox_precond_create_sum: bad argument");
    return VOX_ERR_BAD_ARG;
  }
  *out = nullptr;
  for (int i = 0; i < n; i++)
    if (!parts[i] || parts[i]->op != op || parts[i]->kind == 2 ||
        std::find(op->pcs.begin(), op->pcs.end(), parts[i]) == op->pcs.end()) {
      set_error("vox_precond_create_sum: every part must be a box or level-1 handle of op");
      return VOX_ERR_BAD_ARG;
    }
  vox_precond_s* p = new vox_precond_s();
  p->op = op;
  p->kind = 2;
  p->K = op->K;
  p->f_scale = op->gram;
  p->g = parts[0]->g;
  for (int i = 0; i < n; i++) {
    p->parts.push_back(parts[i]);
    op->pcs.erase(std::remove(op->pcs.begin(), op->pcs.end(), parts[i]), op->pcs.end());
  }
  op->pcs.push_back(p);
  *out = p;
  return VOX_OK;
}

vox_status vox_precond_create_blocks(vox_op_t op, const double* blk_re, const double* blk_im,
                                     vox_precond_t* out) {
  if (!op || !blk_re || !out) {
    set_error("vox_precond_create_blocks: NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  *out = nullptr;
  DeviceGuard dg(op->device);
  std::unique_ptr<vox_precond_s, void (*)(vox_precond_s*)> p(new vox_precond_s(), pc_free);
  VOX_TRY(pc_common(op, p.get(), op->g.L, op->g.M, op->g.N, true));
  const PcGeom& g = p->g;
  // every mode's block, stored at the padded leading dimension (zeros beyond n3)
  const int ld = p->ld;
  const long long per = (long long)ld * ld;
  const long long tot = (long long)g.L * per;
  std::vector<double2> B(tot, make_double2(0.0, 0.0));
  for (long long i = 0; i < g.L; i++)
    for (long long c = 0; c < g.n3; c++)
      for (long long r = 0; r < g.n3; r++) {
        const long long s = (i * g.n3 + c) * g.n3 + r;
        B[i * per + c * ld + r] = make_double2(blk_re[s], blk_im ? blk_im[s] : 0.0);
      }
  VOX_TRY(dalloc(&p->Ad, tot));
  VOX_CUDA(cudaMemcpyAsync(p->Ad, B.data(), tot * sizeof(double2), cudaMemcpyHostToDevice,
                           op->stream));
  p->Lf = g.L;
  p->paired = 0;
  p->f_scale = op->gram;
  if (op->has_f) {
    VOX_TRY(dalloc(&p->Af, tot));
    k_cast_scale<float><<<nblk(tot), 256, 0, op->stream>>>(tot, p->Ad, op->gram, p->Af);
    VOX_CUDA(cudaGetLastError());
  }
  VOX_TRY(wait_stream(op->stream));
  pc_seal(p.get());
  op->pcs.push_back(p.get());
  *out = p.release();
  return VOX_OK;
}

void vox_precond_destroy(vox_precond_t p) {
  if (!p) return;
  pc_release(p);
}

}  // extern "C"

namespace vox {

// Unregister from the operator, drop cached GMRES graphs that captured this
// preconditioner and free it.
static void pc_release(vox_precond_s* p) {
  vox_op_s* op = p->op;
  DeviceGuard dg(op->device);
  // teardown waits without a limit (freeing under queued kernels would fault)
  cudaDeviceSynchronize();
  op->pcs.erase(std::remove(op->pcs.begin(), op->pcs.end(), p), op->pcs.end());
  // drop cached GMRES graphs that captured this preconditioner
  for (auto it = op->wd.graphs.begin(); it != op->wd.graphs.end();) {
    if (std::get<0>(it->first) == (void*)p) {
      cudaGraphExecDestroy(it->second);
      it = op->wd.graphs.erase(it);
    } else {
      ++it;
    }
  }
  for (auto it = op->wf.graphs.begin(); it != op->wf.graphs.end();) {
    if (std::get<0>(it->first) == (void*)p) {
      cudaGraphExecDestroy(it->second);
      it = op->wf.graphs.erase(it);
    } else {
      ++it;
    }
  }
  pc_free(p);
}

}  // namespace vox

extern "C" {

vox_status vox_precond_apply(vox_precond_t p, vox_prec prec, const double* in_re,
                             const double* in_im, double* out_re, double* out_im) {
  if (!p || !in_re || !out_re) {
    set_error("vox_precond_apply: NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  vox_op_s* op = p->op;
  VOX_TRY(check_prec(op, prec));
  DeviceGuard dg(op->device);
  const long long n = op->g.n;
  cudaStream_t st = op->stream;
  split_to_d2(in_re, in_im, n, op->h_in);
  VOX_CUDA(cudaMemcpyAsync(op->d_in, op->h_in, n * sizeof(double2), cudaMemcpyHostToDevice, st));
  if (prec == VOX_C128) {
    VOX_TRY(pc_apply<double>(p, op->d_in, op->d_out, st, nullptr));
  } else {
    k_from_d2<float><<<nblk(n), 256, 0, st>>>(n, op->d_in, op->f_in);
    VOX_TRY(pc_apply<float>(p, op->f_in, op->f_out, st, nullptr));
    k_to_d2<float><<<nblk(n), 256, 0, st>>>(n, op->f_out, 1.0 / p->f_scale, op->d_out);
  }
  VOX_CUDA(cudaMemcpyAsync(op->h_out, op->d_out, n * sizeof(double2), cudaMemcpyDeviceToHost, st));
  VOX_TRY(wait_stream(st));
  d2_to_split(op->h_out, n, out_re, out_im);
  return VOX_OK;
}

vox_status vox_precond_apply_device(vox_precond_t p, const void* in, void* out, void* stream) {
  if (!p || !in || !out) {
    set_error("vox_precond_apply_device: NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  vox_op_s* op = p->op;
  VOX_TRY(check_prec(op, VOX_C128));
  DeviceGuard dg(op->device);
  cudaStream_t st = stream ? (cudaStream_t)stream : op->stream;
  return pc_apply<double>(p, (const double2*)in, (double2*)out, st, nullptr);
}

}  // extern "C"

namespace vox {

// ------------------------------------------------------------ GMRES driver
template <typename R>
static vox_status ensure_work(vox_op_s* op, int m) {
  GmresWork<R>& w = work<R>(op);
  if (w.m == m && w.arena) return VOX_OK;
  VOX_TRY(wait_stream(op->stream));
  w.release();
  const long long n = op->g.n;
  const int K = op->K;
  w.K = K;
  w.ldv = (n + 31) / 32 * 32;
  w.vs = (long long)(m + 7) * w.ldv;
  VOX_TRY(dalloc(&w.arena, w.vs * K));
  w.V = w.arena;
  w.w = w.V + (long long)(m + 1) * w.ldv;
  w.t = w.w + w.ldv;
  w.r = w.t + w.ldv;
  w.x = w.r + w.ldv;
  w.b = w.x + w.ldv;
  w.c = w.b + w.ldv;
  VOX_TRY(dalloc(&w.st, K));
  VOX_CUDA(cudaMemsetAsync(w.st, 0, K * sizeof(GmresDev), op->stream));
  VOX_CUDA(cudaMallocHost((void**)&w.hst, K * kGmresHdr));
  VOX_CUDA(cudaMallocHost((void**)&w.hflag, K * sizeof(int)));
  VOX_CUDA(cudaMallocHost((void**)&w.hscal, K * sizeof(double)));
  VOX_CUDA(cudaMallocHost((void**)&w.hsel, K * sizeof(int)));
  VOX_TRY(dalloc(&w.dsel, K));
  w.m = m;
  return VOX_OK;
}

template <typename R>
static Members wmembers(const GmresWork<R>& w, int km) {
  Members mm;
  mm.km = km;
  mm.vs = w.vs;
  mm.fs = kFlagStride;
  return mm;
}

// Enqueue one restart cycle (pgmres_iter.m) for members 0..km-1 on stream st;
// *nk counts the kernels.
template <typename R>
static vox_status enqueue_cycle(vox_op_s* op, vox_precond_s* pc, int side, int km,
                                cudaStream_t st, int* nk) {
  GmresWork<R>& w = work<R>(op);
  const long long n = op->g.n;
  const long long ld = w.ldv;
  const int m = w.m;
  GmresDev* d = w.st;
  const int* skip = &d->done;
  const Members mm = wmembers(w, km);
  const dim3 gr(kRedBlocks, km), ge(nblk(n), km), g1(1, km);
  const bool right = side == VOX_PREC_RIGHT && pc, left = side == VOX_PREC_LEFT && pc;
  k_norm2<R><<<gr, kRedThreads, 0, st>>>(d, w.r, n, 0, w.vs, 1);
  k_cycle_init<<<g1, 32, 0, st>>>(d, 0);
  k_cycle_v0<R><<<ge, 256, 0, st>>>(d, w.V, w.r, n, w.vs, (Cx<R>*)nullptr, 0);
  *nk += 3;
  for (int k = 0; k < m; k++) {
    Cx<R>* vk = w.V + (long long)k * ld;
    const Cx<R>* src = vk;
    if (right) {
      VOX_TRY(pc_apply<R>(pc, vk, w.t, st, skip, mm));
      src = w.t;
    }
    VOX_TRY(matvec<R>(op, MV_AN, src, w.w, st, skip, mm));
    Cx<R>* wv = w.w;
    if (left) {
      VOX_TRY(pc_apply<R>(pc, w.w, w.t, st, skip, mm));
      wv = w.t;
    }
    if (m + 1 <= kGsMaxCols) {
      // CGS2 in two reads of the basis
      const dim3 gp(kGsBlocks, km);
      const size_t sm = gs_pass_smem<R>(k + 1);
      const int ns = gs_stages<R>(k + 1), rw = gs_rows<R>(k + 1);
      k_gs_pass<R, false><<<gp, kGsThreads, sm, st>>>(d, k, w.V, ld, wv, n, w.vs, ns, rw);
      k_gs_pass<R, true><<<gp, kGsThreads, sm, st>>>(d, k, w.V, ld, wv, n, w.vs, ns, rw);
      k_gs_finish<R><<<ge, kRedThreads, 0, st>>>(d, k, w.V, ld, wv,
                                                 w.V + (long long)(k + 1) * ld, n, w.vs,
                                                 (Cx<R>*)nullptr);
      *nk += 3 + ((right || left) ? 3 : 0) + 3;
    } else {
      k_gs_dots<R><<<gr, kRedThreads, 0, st>>>(d, k, w.V, ld, wv, n, w.vs);
      k_gs_update_dots<R><<<gr, kRedThreads, 0, st>>>(d, k, w.V, ld, wv, n, w.vs);
      k_gs_update_norm<R><<<gr, kRedThreads, 0, st>>>(d, k, w.V, ld, wv, n, w.vs);
      k_gs_scale<R><<<ge, 256, 0, st>>>(d, k, w.V + (long long)(k + 1) * ld, wv, n, w.vs);
      *nk += 3 + ((right || left) ? 3 : 0) + 4;
    }
  }
  // x += V y and r = V res (pgmres_iter.m:133-150).  With a right
  // preconditioner x accumulates u = sum over the cycles of V y, and the solve
  // applies M^{-1} to it once, after its last cycle (right_finish): x = M^{-1} u
  // by linearity, with one preconditioner apply per solve instead of one per
  // cycle (the restart residual r = V res needs no x)
  k_cycle_ls<<<g1, 32, 0, st>>>(d, 0);
  k_cycle_update<R><<<ge, 256, 0, st>>>(d, w.V, ld, w.x, w.r, n, w.vs, 0);
  *nk += 2;
  VOX_CUDA(cudaGetLastError());
  return VOX_OK;
}

// Right preconditioning: x = M^{-1} x for the members with sel[b] != 0, after
// their last cycle (x holds u = sum of the cycles' V y).  One launch sequence
// for all selected members.
template <typename R>
static vox_status right_finish(vox_op_s* op, vox_precond_s* pc, int km, const char* sel,
                               cudaStream_t st) {
  GmresWork<R>& w = work<R>(op);
  bool any = false;
  for (int b = 0; b < km; b++) {
    w.hsel[b] = sel[b] ? 0 : 1;  // skip flags
    any = any || sel[b];
  }
  if (!any) return VOX_OK;
  VOX_CUDA(cudaMemcpyAsync(w.dsel, w.hsel, km * sizeof(int), cudaMemcpyHostToDevice, st));
  Members mm = wmembers(w, km);
  mm.fs = 1;
  VOX_TRY(pc_apply<R>(pc, w.x, w.t, st, w.dsel, mm));
  const long long n = op->g.n;
  k_copy_members<R><<<dim3(nblk(n), km), 256, 0, st>>>(n, w.t, w.x, w.dsel, w.vs, 1);
  VOX_CUDA(cudaGetLastError());
  op->launches += 4;
  // the pinned skip flags are reused by the next call: wait for the copy
  return wait_stream(st);
}

// Step mode needs the two-read Gram-Schmidt (restart + 1 <= kGsMaxCols).
template <typename R>
static bool step_mode_ok(const GmresWork<R>& w) {
  return w.m >= 1 && w.m + 1 <= kGsMaxCols;
}

// Enqueue `steps` out-of-phase steps (step mode) for members 0..km-1: per
// step the cycle start of every member flagged to start (k_norm2, k_cycle_init,
// k_cycle_v0 into V(:,0) and vcur), one Arnoldi step of every member in a
// cycle at its own k (the matvec and preconditioner read vcur; the
// Gram-Schmidt passes take k from the member's record), the end-of-cycle
// update of every member whose cycle ended at this step, and k_step_end.
template <typename R>
static vox_status enqueue_steps(vox_op_s* op, vox_precond_s* pc, int side, int km, int steps,
                                cudaStream_t st, int* nk) {
  GmresWork<R>& w = work<R>(op);
  if (!step_mode_ok(w)) {
    set_error("step mode needs restart + 1 <= " + std::to_string(kGsMaxCols));
    return VOX_ERR_UNSUPPORTED;
  }
  const long long n = op->g.n;
  const long long ld = w.ldv;
  const int m = w.m;
  GmresDev* d = w.st;
  const int* skip = &d->done;
  const Members mm = wmembers(w, km);
  const dim3 gr(kRedBlocks, km), ge(nblk(n), km), g1(1, km);
  const bool right = side == VOX_PREC_RIGHT && pc, left = side == VOX_PREC_LEFT && pc;
  size_t sm = 0;
  for (int nj = 1; nj <= m; nj++) sm = std::max(sm, gs_pass_smem<R>(nj));
  const dim3 gp(kGsBlocks, km);
  for (int s = 0; s < steps; s++) {
    k_norm2<R><<<gr, kRedThreads, 0, st>>>(d, w.r, n, 0, w.vs, 2);
    k_cycle_init<<<g1, 32, 0, st>>>(d, 1);
    k_cycle_v0<R><<<ge, 256, 0, st>>>(d, w.V, w.r, n, w.vs, w.c, 1);
    k_step_begin<<<1, 32, 0, st>>>(d, km);
    const Cx<R>* src = w.c;
    if (right) {
      VOX_TRY(pc_apply<R>(pc, w.c, w.t, st, skip, mm));
      src = w.t;
    }
    VOX_TRY(matvec<R>(op, MV_AN, src, w.w, st, skip, mm));
    Cx<R>* wv = w.w;
    if (left) {
      VOX_TRY(pc_apply<R>(pc, w.w, w.t, st, skip, mm));
      wv = w.t;
    }
    k_gs_pass<R, false><<<gp, kGsThreads, sm, st>>>(d, -1, w.V, ld, wv, n, w.vs, 0, 0);
    k_gs_pass<R, true><<<gp, kGsThreads, sm, st>>>(d, -1, w.V, ld, wv, n, w.vs, 0, 0);
    k_gs_finish<R><<<ge, kRedThreads, 0, st>>>(d, -1, w.V, ld, wv, w.V, n, w.vs, w.c);
    // x += V y, r = V res (with a right preconditioner x accumulates u; the
    // lane applies M^{-1} when the inner solve ends: right_finish)
    k_cycle_ls<<<g1, 32, 0, st>>>(d, 1);
    k_cycle_update<R><<<ge, 256, 0, st>>>(d, w.V, ld, w.x, w.r, n, w.vs, 1);
    k_step_end<<<1, 32, 0, st>>>(d, km);
    *nk += 4 + 3 + ((right || left) ? 3 : 0) + 3 + 3;
  }
  VOX_CUDA(cudaGetLastError());
  return VOX_OK;
}

template <typename R>
static vox_status get_step_graph(vox_op_s* op, vox_precond_s* pc, int side, int km, int steps,
                                 cudaGraphExec_t* out) {
  GmresWork<R>& w = work<R>(op);
  auto key = std::make_tuple((void*)pc, side, km + 1000 * steps);
  auto it = w.graphs.find(key);
  if (it != w.graphs.end()) {
    *out = it->second;
    return VOX_OK;
  }
  cudaStream_t st = op->stream;
  cudaGraph_t graph;
  int nk = 0;
  VOX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  vox_status s = enqueue_steps<R>(op, pc, side, km, steps, st, &nk);
  cudaError_t e = cudaStreamEndCapture(st, &graph);
  if (s != VOX_OK) return s;
  if (e != cudaSuccess) {
    set_error(std::string("graph capture: ") + cudaGetErrorString(e));
    return VOX_ERR_CUDA;
  }
  size_t nnodes = 0;
  cudaGraphGetNodes(graph, nullptr, &nnodes);
  cudaGraphExec_t exec;
  e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    set_error(std::string("graph instantiate: ") + cudaGetErrorString(e));
    return VOX_ERR_CUDA;
  }
  op->graph_nodes[exec] = (int)nnodes;
  w.graphs[key] = exec;
  *out = exec;
  return VOX_OK;
}

template <typename R>
static vox_status get_cycle_graph(vox_op_s* op, vox_precond_s* pc, int side, int km,
                                  cudaGraphExec_t* out) {
  GmresWork<R>& w = work<R>(op);
  auto key = std::make_tuple((void*)pc, side, km);
  auto it = w.graphs.find(key);
  if (it != w.graphs.end()) {
    *out = it->second;
    return VOX_OK;
  }
  cudaStream_t st = op->stream;
  cudaGraph_t graph;
  int nk = 0;
  VOX_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  vox_status s = enqueue_cycle<R>(op, pc, side, km, st, &nk);
  cudaError_t e = cudaStreamEndCapture(st, &graph);
  if (s != VOX_OK) return s;
  if (e != cudaSuccess) {
    set_error(std::string("graph capture: ") + cudaGetErrorString(e));
    return VOX_ERR_CUDA;
  }
  size_t nnodes = 0;
  cudaGraphGetNodes(graph, nullptr, &nnodes);
  cudaGraphExec_t exec;
  e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    set_error(std::string("graph instantiate: ") + cudaGetErrorString(e));
    return VOX_ERR_CUDA;
  }
  op->graph_nodes[exec] = (int)nnodes;
  w.graphs[key] = exec;
  *out = exec;
  return VOX_OK;
}

template <typename R>
__global__ void k_sub(long long n, const Cx<R>* __restrict__ b, const Cx<R>* __restrict__ ax,
                      Cx<R>* r) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    r[i] = csub(b[i], ax[i]);
}

// VOX_GRAPHS=0 enqueues each cycle's kernels directly instead of replaying the
// captured graph (same kernels and order; for profilers that cannot follow
// stream capture)
static bool use_cycle_graphs() {
  static const bool on = [] {
    const char* e = std::getenv("VOX_GRAPHS");
    return !(e && e[0] == '0');
  }();
  return on;
}

// st[b].scal[slot] of the members with use[b] (all when use is null), one sync
template <typename R>
static vox_status read_scals(vox_op_s* op, int slot, int km, const char* use, double* v) {
  GmresWork<R>& w = work<R>(op);
  for (int b = 0; b < km; b++)
    if (!use || use[b])
      VOX_CUDA(cudaMemcpyAsync(&w.hscal[b], &w.st[b].scal[slot], sizeof(double),
                               cudaMemcpyDeviceToHost, op->stream));
  VOX_TRY(wait_stream(op->stream));
  for (int b = 0; b < km; b++)
    if (!use || use[b]) v[b] = w.hscal[b];
  return VOX_OK;
}

template <typename R>
static vox_status read_scal(vox_op_s* op, int slot, double* v) {
  return read_scals<R>(op, slot, 1, nullptr, v);
}

// pgmres.m:70-181 for members 0..km-1 in lockstep, on the right-hand sides
// already in each member's w.b; solutions in each member's w.x.  Members with
// take[b] == 0 are left untouched.  Every member runs exactly the cycles it
// would run alone (its own tolerance, restart count and stopping test); the
// preconditioned-residual history (relative) is appended to resvec[b].
template <typename R>
static vox_status pgmres_dev(vox_op_s* op, vox_precond_s* pc, int side, int km, const double* tol,
                             int maxit, vox_gmres_info* const* info,
                             std::vector<double>* resvec, const char* take) {
  GmresWork<R>& w = work<R>(op);
  const long long n = op->g.n;
  cudaStream_t st = op->stream;
  if (side != VOX_PREC_NONE && !pc) side = VOX_PREC_NONE;
  const Members mm = wmembers(w, km);
  // x0 = 0 -> r = b ; left preconditioning: r = M^{-1} b, bnorm = ||M^{-1} b||
  for (int b = 0; b < km; b++)
    if (take[b]) VOX_CUDA(cudaMemsetAsync(w.mem(w.x, b), 0, n * sizeof(Cx<R>), st));
  if (side == VOX_PREC_LEFT) {
    VOX_TRY(pc_apply<R>(pc, w.b, w.r, st, nullptr, mm));
    op->launches += 3;
  } else {
    for (int b = 0; b < km; b++)
      if (take[b])
        VOX_CUDA(cudaMemcpyAsync(w.mem(w.r, b), w.mem(w.b, b), n * sizeof(Cx<R>),
                                 cudaMemcpyDeviceToDevice, st));
  }
  k_norm2<R><<<dim3(kRedBlocks, km), kRedThreads, 0, st>>>(w.st, w.r, n, 1, w.vs, 0);
  op->launches += 1;
  std::vector<double> bn2(km, 0.0), bnorm(km, 0.0), rel(km, 1.0);
  VOX_TRY(read_scals<R>(op, 1, km, take, bn2.data()));
  std::vector<int> outit(km, 0), p(km, 0);
  std::vector<char> active(km, 0);
  std::vector<unsigned char> hdr(offsetof(GmresDev, resvec), 0);
  GmresDev* h = reinterpret_cast<GmresDev*>(hdr.data());
  for (int b = 0; b < km; b++) {
    std::fill(hdr.begin(), hdr.end(), 0);
    h->m = w.m;
    if (take[b]) {
      bnorm[b] = std::sqrt(bn2[b]);
      if (bnorm[b] == 0.0) {
        info[b]->flag = 0;
        info[b]->relres = 0.0;
        info[b]->iter_inner = info[b]->iter_outer = 0;
        if (resvec) resvec[b].push_back(0.0);
      } else {
        if (resvec) resvec[b].push_back(rel[b]);
        active[b] = rel[b] > tol[b] && maxit > 0;
      }
      h->tol_abs = tol[b] * bnorm[b];
    }
    h->frozen = active[b] ? 0 : 1;
    // reset the header fields (everything before resvec) of the member's state
    VOX_CUDA(cudaMemcpyAsync(&w.st[b], hdr.data(), hdr.size(), cudaMemcpyHostToDevice, st));
    VOX_TRY(wait_stream(st));
  }
  cudaGraphExec_t cyc = nullptr;
  if (use_cycle_graphs()) VOX_TRY(get_cycle_graph<R>(op, pc, side, km, &cyc));
  auto any = [&] {
    for (int b = 0; b < km; b++)
      if (active[b]) return true;
    return false;
  };
  while (any()) {
    if (cyc) {
      VOX_CUDA(cudaGraphLaunch(cyc, st));
      op->launches += op->graph_nodes[cyc];
    } else {
      int nk = 0;
      VOX_TRY(enqueue_cycle<R>(op, pc, side, km, st, &nk));
      op->launches += nk;
    }
    for (int b = 0; b < km; b++)
      if (active[b])
        VOX_CUDA(cudaMemcpyAsync(w.hdr(b), &w.st[b], offsetof(GmresDev, sn),
                                 cudaMemcpyDeviceToHost, st));
    VOX_TRY(wait_stream(st));
    for (int b = 0; b < km; b++) {
      if (!active[b]) continue;
      const GmresDev* hb = w.hdr(b);
      outit[b]++;
      p[b] = hb->k;
      for (int i = 0; i < p[b]; i++)
        if (resvec) resvec[b].push_back(hb->resvec[i] / bnorm[b]);
      info[b]->total_iters += p[b];
      if (p[b] > 0) rel[b] = hb->resvec[p[b] - 1] / bnorm[b];
      // exact breakdown: the Krylov space is invariant, the LS solution is exact
      const bool stop = !(rel[b] > tol[b] && outit[b] < maxit) || (hb->breakdown && !hb->converged);
      if (stop) {
        active[b] = 0;
        w.hflag[b] = 1;
        VOX_CUDA(cudaMemcpyAsync(&w.st[b].frozen, &w.hflag[b], sizeof(int),
                                 cudaMemcpyHostToDevice, st));
      }
    }
  }
  for (int b = 0; b < km; b++) {
    if (!take[b] || bnorm[b] == 0.0) continue;
    info[b]->iter_inner = p[b];
    info[b]->iter_outer = outit[b];
  }
  if (side == VOX_PREC_RIGHT) {
    std::vector<char> sel(km, 0);
    for (int b = 0; b < km; b++) sel[b] = take[b] && bnorm[b] != 0.0;
    VOX_TRY(right_finish<R>(op, pc, km, sel.data(), st));
  }
  return VOX_OK;
}

// relres = ||b - A x|| / ||b|| in the given precision's vectors (member 0)
template <typename R>
static vox_status true_relres(vox_op_s* op, double* relres) {
  GmresWork<R>& w = work<R>(op);
  const long long n = op->g.n;
  cudaStream_t st = op->stream;
  VOX_TRY(matvec<R>(op, MV_AN, w.x, w.w, st, nullptr));
  k_sub<R><<<nblk(n), 256, 0, st>>>(n, w.b, w.w, w.t);
  k_norm2<R><<<kRedBlocks, kRedThreads, 0, st>>>(w.st, w.t, n, 2, 0, 0);
  k_norm2<R><<<kRedBlocks, kRedThreads, 0, st>>>(w.st, w.b, n, 3, 0, 0);
  op->launches += 6;
  double a, b;
  VOX_TRY(read_scal<R>(op, 2, &a));
  VOX_TRY(read_scal<R>(op, 3, &b));
  *relres = b > 0 ? std::sqrt(a / b) : 0.0;
  return VOX_OK;
}

static void fill_resvec(vox_gmres_info* info, const std::vector<double>& rv) {
  if (!info) return;
  info->n_resvec = (long long)rv.size();
  if (info->resvec && info->resvec_cap > 0) {
    const long long c = std::min<long long>(info->resvec_cap, (long long)rv.size());
    std::memcpy(info->resvec, rv.data(), c * sizeof(double));
  }
}

template <typename R>
static vox_status pgmres_entry(vox_op_s* op, vox_precond_s* pc, int side, const double2* b_dev,
                               int restart, double tol, int maxit, double2* x_dev,
                               vox_gmres_info* info) {
  if (restart < 1 || restart > kMaxRestart) {
    set_error("restart must be in 1.." + std::to_string(kMaxRestart));
    return VOX_ERR_BAD_ARG;
  }
  VOX_TRY(ensure_work<R>(op, restart));
  GmresWork<R>& w = work<R>(op);
  const long long n = op->g.n;
  cudaStream_t st = op->stream;
  // b in the working precision (the c64 operator is A/Gram: scale b by 1/Gram)
  const double bscale = std::is_same<R, float>::value ? 1.0 / op->gram : 1.0;
  k_cast_scale<R><<<nblk(n), 256, 0, st>>>(n, b_dev, bscale, w.b);
  std::vector<double> rv;
  info->total_iters = 0;
  const char take = 1;
  VOX_TRY(pgmres_dev<R>(op, pc, side, 1, &tol, maxit, &info, &rv, &take));
  double relres;
  VOX_TRY(true_relres<R>(op, &relres));
  info->relres = relres;
  info->flag = relres <= tol ? 0 : 1;
  k_to_d2<R><<<nblk(n), 256, 0, st>>>(n, w.x, 1.0, x_dev);
  op->launches += 2;
  VOX_TRY(wait_stream(st));
  fill_resvec(info, rv);
  return VOX_OK;
}

__global__ void k_axpy_d2_from(long long n, const float2* __restrict__ d, double s, double2* x) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    x[i].x += s * (double)d[i].x;
    x[i].y += s * (double)d[i].y;
  }
}

// Fraction of the remaining relative target that an automatic inner solve aims
// at: its residual is the true one with a right preconditioner or none, the
// preconditioned one with a left preconditioner.
static double inner_target_factor(const vox_precond_s* pc, int side, double inner_tol) {
  if (inner_tol < 0) return std::min(1.0, -inner_tol);  // the caller's factor
  return (pc && side == VOX_PREC_LEFT) ? 0.3 : 0.9;
}

// complex64 GMRES inside FP64 iterative refinement, for `count` right-hand
// sides at once (members 0..count-1; b_dev and x_dev hold count vectors of n).
// Each member's result equals what the single-member solve gives for it.
static vox_status refined_run(vox_op_s* op, vox_precond_s* pc, int side, int count,
                              const double2* b_dev, double tol, int restart, int maxit_inner,
                              double inner_tol, int max_refine, double2* x_dev,
                              vox_gmres_info* const* info) {
  if (!op->has_d || !op->has_f) {
    set_error("refined solve needs both complex128 and complex64 operator copies");
    return VOX_ERR_BAD_ARG;
  }
  if (restart < 1 || restart > kMaxRestart) {
    set_error("restart must be in 1.." + std::to_string(kMaxRestart));
    return VOX_ERR_BAD_ARG;
  }
  if (count < 1 || count > op->K) {
    set_error("right-hand sides must number 1.." + std::to_string(op->K) +
              " (the operator's members)");
    return VOX_ERR_BAD_ARG;
  }
  // inner_tol <= 0: aim each inner solve at the remaining target directly,
  // f * tol * ||b|| / ||r||: f = 0.3 with a left preconditioner (room for the gap
  // between the preconditioned residual GMRES minimises and the true one),
  // f = 0.9 otherwise (GMRES minimises the true residual of the complex64 system)
  const bool auto_tol = inner_tol <= 0;
  const double fac = inner_target_factor(pc, side, inner_tol);
  if (max_refine < 1) max_refine = 10;
  VOX_TRY(ensure_work<float>(op, restart));
  if (!op->wd.arena) VOX_TRY(ensure_work<double>(op, 1));
  GmresWork<float>& wf = op->wf;
  GmresWork<double>& wd = op->wd;
  const long long n = op->g.n;
  cudaStream_t st = op->stream;
  const int nb = nblk(n);
  // FP64 state: x = 0, r = b
  for (int b = 0; b < count; b++) {
    VOX_CUDA(cudaMemsetAsync(x_dev + b * n, 0, n * sizeof(double2), st));
    VOX_CUDA(cudaMemcpyAsync(wd.mem(wd.b, b), b_dev + b * n, n * sizeof(double2),
                             cudaMemcpyDeviceToDevice, st));
    VOX_CUDA(cudaMemcpyAsync(wd.mem(wd.r, b), b_dev + b * n, n * sizeof(double2),
                             cudaMemcpyDeviceToDevice, st));
  }
  k_norm2<double><<<dim3(kRedBlocks, count), kRedThreads, 0, st>>>(wd.st, wd.b, n, 3, wd.vs, 0);
  op->launches += 1;
  std::vector<double> bn(count), rel(count, 1.0), rn(count), itol(count), r2(count);
  VOX_TRY(read_scals<double>(op, 3, count, nullptr, bn.data()));
  std::vector<char> active(count, 0);
  std::vector<std::vector<double>> rv(count);
  std::vector<int> outer_total(count, 0), last_inner(count, 0);
  for (int b = 0; b < count; b++) {
    bn[b] = std::sqrt(bn[b]);
    info[b]->total_iters = 0;
    info[b]->refinements = 0;
    if (bn[b] == 0.0) {
      rel[b] = 0.0;
    } else {
      active[b] = rel[b] > tol;
    }
  }
  // the inner solves run over every member of the operator (members beyond
  // count or already done are frozen), so one captured cycle serves every
  // batch size
  const int K = op->K;
  std::vector<vox_gmres_info> ii(K);
  std::vector<vox_gmres_info*> iip(K);
  std::vector<std::vector<double>> rvi(K);
  std::vector<char> take(K, 0);
  itol.resize(K, 0.0);
  for (int b = 0; b < K; b++) iip[b] = &ii[b];
  for (int it = 0; it < max_refine; it++) {
    bool anyact = false;
    for (int b = 0; b < count; b++) anyact = anyact || active[b];
    if (!anyact) break;
    for (int b = 0; b < count; b++) {
      ii[b] = vox_gmres_info{};
      if (!active[b]) continue;
      rn[b] = rel[b] * bn[b];
      // inner right-hand side: r / ||r|| in complex64 (operator copy is A/Gram)
      k_cast_scale<float><<<nb, 256, 0, st>>>(n, wd.mem(wd.r, b), 1.0 / rn[b], wf.mem(wf.b, b));
      // tolerance relative to ||r||; never ask for less than what reaches tol
      itol[b] = auto_tol ? std::min(0.5, fac * tol * bn[b] / rn[b])
                         : std::min(0.5, std::max(inner_tol, 0.5 * tol * bn[b] / rn[b]));
      op->launches += 1;
    }
    for (int b = 0; b < K; b++) take[b] = b < count && active[b];
    for (int b = 0; b < K; b++) rvi[b].clear();
    VOX_TRY(pgmres_dev<float>(op, pc, side, K, itol.data(), maxit_inner, iip.data(),
                              rvi.data(), take.data()));
    for (int b = 0; b < count; b++)
      if (active[b]) rv[b].insert(rv[b].end(), rvi[b].begin(), rvi[b].end());
    for (int b = 0; b < count; b++) {
      if (!active[b]) continue;
      info[b]->total_iters += ii[b].total_iters;
      outer_total[b] += ii[b].iter_outer;
      last_inner[b] = ii[b].iter_inner;
      double2* xb = x_dev + b * n;
      // x += (||r|| / Gram) * d   (d solves (A/Gram) d = r/||r||)
      k_axpy_d2_from<<<nb, 256, 0, st>>>(n, wf.mem(wf.x, b), rn[b] / op->gram, xb);
      // r = b - A x in FP64 (member b's operator)
      Members one;
      one.m0 = b;
      VOX_TRY(matvec<double>(op, MV_AN, xb, wd.mem(wd.w, b), st, nullptr, one));
      k_sub<double><<<nb, 256, 0, st>>>(n, wd.mem(wd.b, b), wd.mem(wd.w, b), wd.mem(wd.r, b));
      k_norm2<double><<<kRedBlocks, kRedThreads, 0, st>>>(wd.st + b, wd.mem(wd.r, b), n, 2, 0, 0);
      op->launches += 7;
    }
    VOX_TRY(read_scals<double>(op, 2, count, active.data(), r2.data()));
    for (int b = 0; b < count; b++) {
      if (!active[b]) continue;
      rel[b] = std::sqrt(r2[b]) / bn[b];
      info[b]->refinements = it + 1;
      active[b] = rel[b] > tol;
    }
  }
  for (int b = 0; b < count; b++) {
    info[b]->relres = rel[b];
    info[b]->flag = rel[b] <= tol ? 0 : 1;
    info[b]->iter_inner = last_inner[b];
    info[b]->iter_outer = outer_total[b];
    fill_resvec(info[b], rv[b]);
  }
  return VOX_OK;
}

static vox_status refined_entry(vox_op_s* op, vox_precond_s* pc, int side, const double2* b_dev,
                                double tol, int restart, int maxit_inner, double inner_tol,
                                int max_refine, double2* x_dev, vox_gmres_info* info) {
  return refined_run(op, pc, side, 1, b_dev, tol, restart, maxit_inner, inner_tol, max_refine,
                     x_dev, &info);
}

}  // namespace vox

// pgmres.m:176-180 reports non-convergence as flag = 1, not as an error, and so
// do the solver entry points when the caller passes an info record.  A caller
// that passes none cannot see the flag, so it gets VOX_ERR_NOT_CONVERGED.
static vox_status flag_status(vox_status s, bool caller_info, const vox_gmres_info& inf) {
  if (s == VOX_OK && !caller_info && inf.flag != 0) {
    set_error("the solve did not reach the tolerance (relres " + std::to_string(inf.relres) +
              "); pass a vox_gmres_info to receive flag = 1 instead of this status");
    return VOX_ERR_NOT_CONVERGED;
  }
  return s;
}

extern "C" {

vox_status vox_pgmres_device(vox_op_t op, vox_precond_t pc, int side, vox_prec prec,
                             const void* b, int restart, double tol, int maxit, void* x,
                             vox_gmres_info* info) {
  if (!op || !b || !x) {
    set_error("vox_pgmres_device: NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  VOX_TRY(check_prec(op, prec));
  DeviceGuard dg(op->device);
  vox_gmres_info local{};
  const bool given = info != nullptr;
  if (!info) info = &local;
  auto t0 = std::chrono::steady_clock::now();
  vox_status s = prec == VOX_C128
                     ? pgmres_entry<double>(op, pc, side, (const double2*)b, restart, tol, maxit,
                                            (double2*)x, info)
                     : pgmres_entry<float>(op, pc, side, (const double2*)b, restart, tol, maxit,
                                           (double2*)x, info);
  info->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return flag_status(s, given, *info);
}

vox_status vox_solve_refined_device(vox_op_t op, vox_precond_t pc, int side, const void* b,
                                    double tol, int restart, int maxit_inner, double inner_tol,
                                    int max_refine, void* x, vox_gmres_info* info) {
  if (!op || !b || !x) {
    set_error("vox_solve_refined_device: NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  DeviceGuard dg(op->device);
  vox_gmres_info local{};
  const bool given = info != nullptr;
  if (!info) info = &local;
  auto t0 = std::chrono::steady_clock::now();
  vox_status s = refined_entry(op, pc, side, (const double2*)b, tol, restart, maxit_inner,
                               inner_tol, max_refine, (double2*)x, info);
  info->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return flag_status(s, given, *info);
}

static vox_status host_solve(vox_op_t op, const double* b_re, const double* b_im, double* x_re,
                             double* x_im, vox_gmres_info* info,
                             const std::function<vox_status(const double2*, double2*)>& fn) {
  if (!op || !b_re || !x_re) {
    set_error("NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  DeviceGuard dg(op->device);
  const long long n = op->g.n;
  cudaStream_t st = op->stream;
  auto t0 = std::chrono::steady_clock::now();
  split_to_d2(b_re, b_im, n, op->h_in);
  VOX_CUDA(cudaMemcpyAsync(op->d_in, op->h_in, n * sizeof(double2), cudaMemcpyHostToDevice, st));
  VOX_TRY(fn(op->d_in, op->d_out));
  VOX_CUDA(cudaMemcpyAsync(op->h_out, op->d_out, n * sizeof(double2), cudaMemcpyDeviceToHost, st));
  VOX_TRY(wait_stream(st));
  d2_to_split(op->h_out, n, x_re, x_im);
  if (info)
    info->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return VOX_OK;
}

vox_status vox_pgmres(vox_op_t op, vox_precond_t pc, int side, vox_prec prec, const double* b_re,
                      const double* b_im, int restart, double tol, int maxit, double* x_re,
                      double* x_im, vox_gmres_info* info) {
  if (op) {
    vox_status s = check_prec(op, prec);
    if (s != VOX_OK) return s;
  }
  vox_gmres_info local{};
  vox_gmres_info* inf = info ? info : &local;
  return flag_status(
      host_solve(op, b_re, b_im, x_re, x_im, inf,
                 [&](const double2* b, double2* x) {
                   return prec == VOX_C128
                              ? pgmres_entry<double>(op, pc, side, b, restart, tol, maxit, x, inf)
                              : pgmres_entry<float>(op, pc, side, b, restart, tol, maxit, x, inf);
                 }),
      info != nullptr, *inf);
}

vox_status vox_solve_refined(vox_op_t op, vox_precond_t pc, int side, const double* b_re,
                             const double* b_im, double tol, int restart, int maxit_inner,
                             double inner_tol, int max_refine, double* x_re, double* x_im,
                             vox_gmres_info* info) {
  vox_gmres_info local{};
  vox_gmres_info* inf = info ? info : &local;
  return flag_status(host_solve(op, b_re, b_im, x_re, x_im, inf,
                                [&](const double2* b, double2* x) {
                                  return refined_entry(op, pc, side, b, tol, restart, maxit_inner,
                                                       inner_tol, max_refine, x, inf);
                                }),
                     info != nullptr, *inf);
}

vox_status vox_jvie_rhs(int L, int M, int N, const double* er_re, const double* er_im,
                        const double* Einc_re, const double* Einc_im, double gram, double freq,
                        const double* idx, long long n_idx, double* out_re, double* out_im) {
  if (!er_re || !Einc_re || !idx || !out_re || L < 1 || M < 1 || N < 1) {
    set_error("vox_jvie_rhs: bad argument");
    return VOX_ERR_BAD_ARG;
  }
  const double mu = 4e-7 * M_PI, co = 299792458.0;
  const double eo = 1.0 / (co * co) / mu;
  const double omega = 2.0 * M_PI * freq;
  const long long V = (long long)L * M * N;
  for (long long i = 0; i < n_idx; i++) {
    const long long p = (long long)idx[i] - 1;
    if (p < 0 || p >= 3 * V) {
      set_error("vox_jvie_rhs: idx out of range");
      return VOX_ERR_BAD_ARG;
    }
    const long long cell = p % V;
    const double er_r = er_re[cell], er_i = er_im ? er_im[cell] : 0.0;
    // tau = j omega eo (e_r - 1); Vrhs = Gram tau Einc / e_r
    const double tr = -omega * eo * er_i, ti = omega * eo * (er_r - 1.0);
    const double er = Einc_re[p], ei = Einc_im ? Einc_im[p] : 0.0;
    double vr = gram * (tr * er - ti * ei), vi = gram * (tr * ei + ti * er);
    const double dd = er_r * er_r + er_i * er_i;
    out_re[i] = (vr * er_r + vi * er_i) / dd;
    if (out_im) out_im[i] = (vi * er_r - vr * er_i) / dd;
  }
  return VOX_OK;
}

}  // extern "C"

namespace vox {

template <typename R>
__global__ void k_fill(long long n, R v, Cx<R>* x) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] = mkc<R>(v, (R)0.5 * v);
}

// Average device time (ms) of each kernel of one GMRES iteration, measured with
// CUDA events on the operator's stream: out[0..2] matvec (x-forward, plane,
// x-inverse), out[3..5] preconditioner (x-forward, per-mode solve, x-inverse),
// out[6..9] Gram-Schmidt (dots, update+dots, update+norm, scale) at basis size
// kgs+1.  Entries that do not apply are 0.
template <typename R>
static vox_status profile_stages(vox_op_s* op, vox_precond_s* pc, int restart, int kgs, int reps,
                                 double* out) {
  VOX_TRY(ensure_work<R>(op, restart));
  GmresWork<R>& w = work<R>(op);
  OpBuffers<R>& b = bufs<R>(op);
  const OpGeom& g = b.geo;
  const long long n = op->g.n;
  cudaStream_t st = op->stream;
  const size_t cs = sizeof(Cx<R>);
  // every member's whole arena (basis and vectors)
  k_fill<R><<<nblk(w.vs * op->K), 256, 0, st>>>(w.vs * op->K, (R)1e-3, w.arena);
  const int km = op->K;
  const long long ld = w.ldv;
  cudaEvent_t e0, e1;
  VOX_CUDA(cudaEventCreate(&e0));
  VOX_CUDA(cudaEventCreate(&e1));
  auto timeit = [&](auto&& launch) -> double {
    launch();  // warm-up
    VOX_CUDA(cudaEventRecord(e0, st));
    for (int r = 0; r < reps; r++) launch();
    VOX_CUDA(cudaEventRecord(e1, st));
    VOX_TRY(wait_event(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms / reps;
  };
  for (int i = 0; i < 10; i++) out[i] = 0;
  dim3 gx((g.M + g.ybx - 1) / g.ybx, g.N, 3 * km);
  const R scale = (R)(1.0 / ((double)g.Px * g.Py * g.Pz));
  out[0] = timeit([&] {
    k_xfwd<R><<<gx, g.xthr, xsmem(g, cs), st>>>(g, op->px, b.twX, w.V, op->vmap, b.Mc, MV_AN, b.T1,
                                              nullptr, w.vs, 0);
  });
  out[1] = timeit([&] { launch_plane<R>(op, b, b.T1, b.fN, b.T2, b.TY, km, nullptr, 0, st); });
  out[2] = timeit([&] {
    k_xinv<R><<<gx, g.xthr, xsmem(g, cs), st>>>(g, op->px, b.twX, b.T2, op->vmap, w.V, b.Mr, b.Mc,
                                              b.gram, scale, b.out_scale, MV_AN, w.w, nullptr,
                                              w.vs, 0);
  });
  if (pc && pc->kind != 0) {
    // level 2 or a sum: the whole apply as one stage
    out[4] = timeit([&] { pc_apply<R>(pc, w.V, w.t, st, nullptr, wmembers(w, km)); });
  } else if (pc) {
    const PcGeom& pg = pc->g;
    const int nb = (pg.n3 + pg.ybx - 1) / pg.ybx;
    Cx<R>* T = pc_T<R>(pc, 0);
    out[3] = timeit([&] {
      pc_xfwd_launch<R>(pc, pg, dim3(nb, km), st, w.V, pc->vmap, T, nullptr, w.vs, 0);
    });
    vox_status ps = VOX_OK;
    out[4] = timeit([&] {
      ps = inv_apply<R>(pc, T, pc_T<R>(pc, 1), st, nullptr, 0, km);
    });
    if (ps != VOX_OK) return ps;
    out[5] = timeit([&] {
      pc_xinv_launch<R>(pc, pg, dim3(nb, km), st, pc_T<R>(pc, 1), pc->vmap, w.t, nullptr, w.vs,
                        0);
    });
  }
  // Gram-Schmidt at basis size kgs+1 (done flag cleared before every launch)
  const int k = std::min(kgs, restart - 1);
  const int nb = nblk(n);
  const dim3 gr(kRedBlocks, km);
  int zero = 0;
  auto clear = [&] {
    for (int mb = 0; mb < km; mb++)
      cudaMemcpyAsync(&w.st[mb].done, &zero, sizeof(int), cudaMemcpyHostToDevice, st);
  };
  {
    // state header with m and a huge tolerance so no iteration "converges"
    std::vector<unsigned char> hdr(offsetof(GmresDev, resvec), 0);
    GmresDev* init = reinterpret_cast<GmresDev*>(hdr.data());
    init->m = restart;
    init->tol_abs = -1.0;
    for (int mb = 0; mb < km; mb++)
      VOX_CUDA(cudaMemcpyAsync(&w.st[mb], hdr.data(), hdr.size(), cudaMemcpyHostToDevice, st));
    VOX_TRY(wait_stream(st));
  }
  // the pass that forms the Hessenberg column sets done at the last column:
  // time it at k < m-1 with done cleared before every launch
  auto timed_clear = [&](auto&& launch) -> double {
    double tn = 0;
    for (int r = 0; r < reps + 1; r++) {
      clear();
      VOX_CUDA(cudaEventRecord(e0, st));
      launch();
      VOX_CUDA(cudaEventRecord(e1, st));
      VOX_TRY(wait_event(e1));
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (r > 0) tn += ms;
    }
    return tn / reps;
  };
  if (restart + 1 <= kGsMaxCols) {
    const dim3 gp(kGsBlocks, km);
    const size_t sm = gs_pass_smem<R>(k + 1);
    const int ns = gs_stages<R>(k + 1), rw = gs_rows<R>(k + 1);
    out[6] = timeit([&] {
      k_gs_pass<R, false><<<gp, kGsThreads, sm, st>>>(w.st, k, w.V, ld, w.w, n, w.vs, ns, rw);
    });
    out[7] = timed_clear([&] {
      k_gs_pass<R, true><<<gp, kGsThreads, sm, st>>>(w.st, k, w.V, ld, w.w, n, w.vs, ns, rw);
    });
    clear();
    out[8] = timeit([&] {
      k_gs_finish<R><<<dim3(nb, km), kRedThreads, 0, st>>>(
          w.st, k, w.V, ld, w.w, w.V + (long long)(k + 1) * ld, n, w.vs, (Cx<R>*)nullptr);
    });
  } else {
    out[6] = timeit([&] {
      k_gs_dots<R><<<gr, kRedThreads, 0, st>>>(w.st, k, w.V, ld, w.w, n, w.vs);
    });
    out[7] = timeit([&] {
      k_gs_update_dots<R><<<gr, kRedThreads, 0, st>>>(w.st, k, w.V, ld, w.w, n, w.vs);
    });
    out[8] = timed_clear([&] {
      k_gs_update_norm<R><<<gr, kRedThreads, 0, st>>>(w.st, k, w.V, ld, w.w, n, w.vs);
    });
    clear();
    out[9] = timeit([&] {
      k_gs_scale<R><<<dim3(nb, km), 256, 0, st>>>(w.st, k, w.V + (long long)(k + 1) * ld, w.w,
                                                   n, w.vs);
    });
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  VOX_CUDA(cudaGetLastError());
  VOX_TRY(wait_stream(st));
  return VOX_OK;
}

}  // namespace vox

extern "C" {

vox_status vox_op_set_stream(vox_op_t op, void* stream) {
  if (!op) {
    set_error("vox_op_set_stream: NULL operator");
    return VOX_ERR_BAD_ARG;
  }
  op->stream = stream ? (cudaStream_t)stream : op->own_stream;
  return VOX_OK;
}

}  // extern "C"

namespace vox {

// A second handle on src's factors bound to op, with its own work (a sum's
// parts are shared the same way).
static vox_status pc_share(vox_precond_s* src, vox_op_s* op, vox_precond_s** out) {
  *out = nullptr;
  std::unique_ptr<vox_precond_s, void (*)(vox_precond_s*)> p(new vox_precond_s(), pc_free);
  *p = *src;  // geometry, plans and factor pointers (shared owner copied)
  p->op = op;
  if (src->vmap == src->op->vmap) p->vmap = op->vmap;
  p->parts.clear();
  p->Td = p->Td2 = nullptr;
  p->Tf = p->Tf2 = nullptr;
  if (src->kind == 2) {
    p->K = op->K;
    for (vox_precond_s* q : src->parts) {
      vox_precond_s* qs;
      VOX_TRY(pc_share(q, op, &qs));
      p->parts.push_back(qs);
    }
  } else {
    VOX_TRY(pc_alloc_work(p.get(), op->K));
  }
  *out = p.release();
  return VOX_OK;
}

}  // namespace vox

extern "C" {

vox_status vox_precond_share(vox_precond_t src, vox_op_t op, vox_precond_t* out) {
  if (!src || !op || !out) {
    set_error("vox_precond_share: NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  *out = nullptr;
  const vox_op_s* so = src->op;
  if (op->g.L != so->g.L || op->g.M != so->g.M || op->g.N != so->g.N || op->g.n != so->g.n ||
      op->gram != so->gram || op->device != so->device || op->has_f != so->has_f) {
    set_error("vox_precond_share: the operator differs in grid, support size, Gram or device");
    return VOX_ERR_BAD_ARG;
  }
  DeviceGuard dg(op->device);
  vox_precond_s* p;
  VOX_TRY(pc_share(src, op, &p));
  op->pcs.push_back(p);
  *out = p;
  return VOX_OK;
}

vox_status vox_precond_info(vox_precond_t p, int* n_blocks, int* ld, int* paired) {
  if (!p) {
    set_error("vox_precond_info: NULL preconditioner");
    return VOX_ERR_BAD_ARG;
  }
  if (p->kind == 1) {
    if (n_blocks) *n_blocks = p->g.L * p->g.M;
    if (ld) *ld = p->ld;
    if (paired) *paired = 0;
    return VOX_OK;
  }
  if (p->kind == 2) {
    int nb = 0;
    for (vox_precond_s* q : p->parts) nb += q->kind == 1 ? q->g.L * q->g.M : q->Lf;
    if (n_blocks) *n_blocks = nb;
    if (ld) *ld = 0;
    if (paired) *paired = 0;
    return VOX_OK;
  }
  if (n_blocks) *n_blocks = p->Lf;
  if (ld) *ld = p->ld;
  if (paired) *paired = p->paired;
  return VOX_OK;
}

vox_status vox_op_flags(vox_op_t op, int* flags) {
  if (!op || !flags) {
    set_error("vox_op_flags: NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  *flags = op->g.sym ? 1 : 0;
  return VOX_OK;
}

}  // extern "C"

namespace vox {

template <typename R>
__global__ void k_lincomb_acc(long long n, const Cx<R>* __restrict__ src, double w, int first,
                              Cx<R>* dst) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const Cx<R> s = src[i];
    Cx<R> d = first ? czero<Cx<R>>() : dst[i];
    d.x += (R)w * s.x;
    d.y += (R)w * s.y;
    dst[i] = d;
  }
}

template <typename R>
static long long fN_count(const OpGeom& g) {
  return g.sym ? 6LL * (g.Px / 2 + 1) * (g.Py / 2 + 1) * (g.Pz / 2 + 1)
               : 6LL * g.Px * g.Py * g.Pz;
}

}  // namespace vox

extern "C" {

vox_status vox_op_interp_member(vox_op_t dst, int member, const vox_op_t* srcs, const double* w,
                                int n) {
  if (!dst || !srcs || !w || n < 1 || member < 0 || member >= dst->K) {
    set_error("vox_op_interp: bad argument");
    return VOX_ERR_BAD_ARG;
  }
  for (int i = 0; i < n; i++) {
    const vox_op_s* s = srcs[i];
    if (!s || s->g.L != dst->g.L || s->g.M != dst->g.M || s->g.N != dst->g.N ||
        s->g.Px != dst->g.Px || s->g.Py != dst->g.Py || s->g.Pz != dst->g.Pz ||
        s->g.sym != dst->g.sym || s->has_d != dst->has_d || s->has_f != dst->has_f ||
        s->gram != dst->gram || s->device != dst->device) {
      set_error("vox_op_interp: operators differ in grid, padding, storage or precisions");
      return VOX_ERR_BAD_ARG;
    }
  }
  DeviceGuard dg(dst->device);
  cudaStream_t st = dst->stream;
  const long long cnt = fN_count<double>(dst->g);
  for (int i = 0; i < n; i++) {
    // each source's member 0
    if (dst->has_d)
      k_lincomb_acc<double><<<nblk(cnt), 256, 0, st>>>(cnt, srcs[i]->d.fN, w[i], i == 0,
                                                        dst->d.fN + member * cnt);
    if (dst->has_f)
      k_lincomb_acc<float><<<nblk(cnt), 256, 0, st>>>(cnt, srcs[i]->f.fN, w[i], i == 0,
                                                       dst->f.fN + member * cnt);
  }
  VOX_CUDA(cudaGetLastError());
  return VOX_OK;
}

vox_status vox_op_interp(vox_op_t dst, const vox_op_t* srcs, const double* w, int n) {
  return vox_op_interp_member(dst, 0, srcs, w, n);
}

vox_status vox_op_members(vox_op_t op, int* members) {
  if (!op || !members) {
    set_error("vox_op_members: NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  *members = op->K;
  return VOX_OK;
}

vox_status vox_solve_refined_batch_device(vox_op_t op, vox_precond_t pc, int side, int count,
                                          const void* b, double tol, int restart,
                                          int maxit_inner, double inner_tol, int max_refine,
                                          void* x, vox_gmres_info* infos) {
  if (!op || !b || !x || !infos) {
    set_error("vox_solve_refined_batch_device: NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  if (count < 1 || count > op->K) {
    set_error("vox_solve_refined_batch_device: count must be 1.." + std::to_string(op->K));
    return VOX_ERR_BAD_ARG;
  }
  DeviceGuard dg(op->device);
  std::vector<vox_gmres_info*> ip(count);
  for (int i = 0; i < count; i++) ip[i] = &infos[i];
  auto t0 = std::chrono::steady_clock::now();
  VOX_TRY(refined_run(op, pc, side, count, (const double2*)b, tol, restart, maxit_inner,
                      inner_tol, max_refine, (double2*)x, ip.data()));
  VOX_TRY(wait_stream(op->stream));
  const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  for (int i = 0; i < count; i++) infos[i].seconds = sec;
  return VOX_OK;
}

vox_status vox_solve_refined_batch(vox_op_t op, vox_precond_t pc, int side, int count,
                                   const double* b_re, const double* b_im, double tol,
                                   int restart, int maxit_inner, double inner_tol,
                                   int max_refine, double* x_re, double* x_im,
                                   vox_gmres_info* infos) {
  if (!op || !b_re || !x_re || !infos) {
    set_error("vox_solve_refined_batch: NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  if (count < 1 || count > op->K) {
    set_error("vox_solve_refined_batch: count must be 1.." + std::to_string(op->K));
    return VOX_ERR_BAD_ARG;
  }
  DeviceGuard dg(op->device);
  const long long n = op->g.n;
  cudaStream_t st = op->stream;
  auto t0 = std::chrono::steady_clock::now();
  split_to_d2(b_re, b_im, count * n, op->h_in);
  VOX_CUDA(cudaMemcpyAsync(op->d_in, op->h_in, count * n * sizeof(double2),
                           cudaMemcpyHostToDevice, st));
  std::vector<vox_gmres_info*> ip(count);
  for (int i = 0; i < count; i++) ip[i] = &infos[i];
  VOX_TRY(refined_run(op, pc, side, count, op->d_in, tol, restart, maxit_inner, inner_tol,
                      max_refine, op->d_out, ip.data()));
  VOX_CUDA(cudaMemcpyAsync(op->h_out, op->d_out, count * n * sizeof(double2),
                           cudaMemcpyDeviceToHost, st));
  VOX_TRY(wait_stream(st));
  d2_to_split(op->h_out, count * n, x_re, x_im);
  const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  for (int i = 0; i < count; i++) infos[i].seconds = sec;
  return VOX_OK;
}

vox_status vox_op_stats(vox_op_t op, long long* launches) {
  if (!op || !launches) {
    set_error("vox_op_stats: NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  *launches = op->launches;
  return VOX_OK;
}

vox_status vox_profile_stages(vox_op_t op, vox_precond_t pc, vox_prec prec, int restart, int kgs,
                              int reps, double* ms_out) {
  if (!op || !ms_out || reps < 1 || restart < 1 || restart > kMaxRestart) {
    set_error("vox_profile_stages: bad argument");
    return VOX_ERR_BAD_ARG;
  }
  VOX_TRY(check_prec(op, prec));
  DeviceGuard dg(op->device);
  return prec == VOX_C128 ? profile_stages<double>(op, pc, restart, kgs, reps, ms_out)
                          : profile_stages<float>(op, pc, restart, kgs, reps, ms_out);
}

}  // extern "C"
