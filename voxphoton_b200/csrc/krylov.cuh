// Device-resident restarted GMRES (pgmres.m:70-181, pgmres_iter.m:22-150).
//
// Arnoldi uses classical Gram-Schmidt with one re-orthogonalisation pass
// (CGS2).  Inner products and norms accumulate in FP64 whatever the working
// precision R of the basis; the Hessenberg matrix, the Givens rotations and
// the least-squares solve live on the device in FP64.  Each kernel begins by
// reading the cycle's `done` flag, so a whole restart cycle (m iterations plus
// the solution update) is enqueued - and captured in one CUDA graph - without
// any host round trip; the host syncs once per cycle.
//
// Reductions are deterministic: every CTA writes its partial sums, and the
// last CTA to finish (atomic ticket) adds them in block order.
//
// Members: one launch serves every member of a batched operator (independent
// solves of the same shape).  The member is blockIdx.y; member b's vectors sit
// b * vs elements after member 0's (one workspace arena per member) and its
// state is st[b].  A member whose solve has finished is `frozen`: every kernel
// of the cycle leaves it untouched, so each member runs exactly the cycles it
// would run alone and its arithmetic does not depend on the other members.
#pragma once

#include "bulk.cuh"
#include "vox_common.cuh"

namespace vox {

constexpr int kMaxRestart = 128;
constexpr int kRedBlocks = 592;  // 4 CTAs per SM on 148 SMs
constexpr int kRedThreads = 256;
constexpr int kHist = 2048;       // residual history kept on the device per inner solve

struct GmresDev {
  int done;          // cycle finished (converged / breakdown / m reached)
  int k;             // iterations performed in this cycle
  int converged;     // LS residual below tol_abs
  int breakdown;     // H(k+1,k) == 0
  unsigned ticket;   // last-block counter
  int m;             // restart length
  int frozen;        // member takes no part in this cycle (batched launches)
  // step mode (lanes): members advance one Arnoldi step per launch sequence,
  // each at its own k, and restart on their own (k_step_begin / k_step_end)
  int start;         // begin a cycle at the next step (r holds its residual)
  int stepped;       // this member took the current step (set by gs_column)
  int endnow;        // its cycle ended in the current step
  int ifin;          // its inner solve ended (converged, breakdown or maxit cycles)
  int cycles;        // cycles of the current inner solve
  int maxit;         // cycle limit of the inner solve
  int nhist;         // entries of hist
  int itot;          // iterations of the current inner solve
  int kdone;         // iterations of its last cycle
  double ibn;        // the inner right-hand side's norm (relative residuals)
  double itol;       // relative target of the inner solve
  double tol_abs;    // tol * bnorm
  double beta;       // ||r|| at cycle start
  double inv_norm;   // 1/H(k+1,k) for the pending basis vector
  double resvec[kMaxRestart];
  double cs[kMaxRestart];
  double2 sn[kMaxRestart];
  double2 g[kMaxRestart + 1];
  double2 y[kMaxRestart];
  double2 res[kMaxRestart + 1];
  double2 h1[kMaxRestart + 1];
  double2 h2[kMaxRestart + 1];
  double2 H[(kMaxRestart + 1) * kMaxRestart];   // unrotated, column-major, ld m+1
  double2 Rm[(kMaxRestart + 1) * kMaxRestart];  // rotated (upper triangular part used)
  double2 partial[(kMaxRestart + 1) * kRedBlocks];
  double scal[4];    // misc reductions (norms)
  double hist[kHist];  // step mode: the LS residuals of every cycle of the inner solve
};

__device__ __forceinline__ double2 warp_sum(double2 v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, o);
    v.y += __shfl_down_sync(0xffffffffu, v.y, o);
  }
  return v;
}

// Block-wide sum of one double2 per thread; result valid in thread 0.
__device__ __forceinline__ double2 block_sum(double2 v, double2* sh) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    v = (lane < nw) ? sh[lane] : make_double2(0.0, 0.0);
    v = warp_sum(v);
  }
  return v;
}

// Returns true in exactly one CTA (the last to arrive), after all partials
// of all CTAs are visible.
__device__ __forceinline__ bool last_block(unsigned* ticket) {
  __shared__ bool amlast;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned t = atomicAdd(ticket, 1u);
    amlast = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (amlast) __threadfence();
  return amlast;
}

// partial[j*nb + b] for j < nj, reduced into out[j] (one warp per j, fixed
// order, so the result is deterministic).  Ends with __syncthreads().
__device__ __forceinline__ void reduce_partials(const double2* partial, int nj, int nb,
                                                double2* out, double2* sh) {
  (void)sh;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int j = warp; j < nj; j += nw) {
    double2 v = make_double2(0.0, 0.0);
    for (int b = lane; b < nb; b += 32) {
      const double2 p = __ldcg(&partial[j * nb + b]);
      v.x += p.x;
      v.y += p.y;
    }
    v = warp_sum(v);
    if (lane == 0) out[j] = v;
  }
  __syncthreads();
}

// Per-CTA dot products of nj basis vectors with w over the CTA's grid-stride
// elements, kDotBatch basis vectors per sweep (FP64 accumulation).
constexpr int kDotBatch = 8;

// acc += conj(v) * w in FP64
__device__ __forceinline__ void acc_cdot(double2& acc, double vx, double vy, double wx,
                                         double wy) {
  acc.x += vx * wx + vy * wy;
  acc.y += vx * wy - vy * wx;
}

// The rows of one batch: one row per thread and step (complex128: 16-byte loads).
template <typename R>
__device__ __forceinline__ void dots_rows(const Cx<R>* __restrict__ V, long long ldv, int j0,
                                          int nb, const Cx<R>* __restrict__ w, long long n,
                                          double2 (&acc)[kDotBatch]) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double2 wi = to_d2(w[i]);
#pragma unroll
    for (int q = 0; q < kDotBatch; q++) {
      if (q < nb) {
        const double2 v = to_d2(V[(j0 + q) * ldv + i]);
        acc_cdot(acc[q], v.x, v.y, wi.x, wi.y);
      }
    }
  }
}

// complex64: two rows per thread and step, 16-byte loads (the basis columns
// and w start on 256-byte boundaries of the Krylov arena); an odd last row
// goes to thread 0 of CTA 0.
template <>
__device__ __forceinline__ void dots_rows<float>(const float2* __restrict__ V, long long ldv,
                                                 int j0, int nb, const float2* __restrict__ w,
                                                 long long n, double2 (&acc)[kDotBatch]) {
  const long long n2 = n >> 1;
  const float4* __restrict__ w4 = reinterpret_cast<const float4*>(w);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n2;
       i += (long long)gridDim.x * blockDim.x) {
    const float4 wv = w4[i];
#pragma unroll
    for (int q = 0; q < kDotBatch; q++) {
      if (q < nb) {
        const float4 v = reinterpret_cast<const float4*>(V + (j0 + q) * ldv)[i];
        acc_cdot(acc[q], v.x, v.y, wv.x, wv.y);
        acc_cdot(acc[q], v.z, v.w, wv.z, wv.w);
      }
    }
  }
  if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
    const float2 wi = w[n - 1];
#pragma unroll
    for (int q = 0; q < kDotBatch; q++) {
      if (q < nb) {
        const float2 v = V[(j0 + q) * ldv + n - 1];
        acc_cdot(acc[q], v.x, v.y, wi.x, wi.y);
      }
    }
  }
}

// w <- w - V h over this thread's rows (the rows dots_rows<R> gives it, so a
// kernel may update and then take dots without a grid-wide barrier); returns
// the sum of |w_i|^2 over those rows in FP64.
template <typename R>
__device__ __forceinline__ double update_rows(const Cx<R>* __restrict__ V, long long ldv, int nj,
                                              const Cx<R>* hs, Cx<R>* w, long long n) {
  double nrm = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    Cx<R> wi = w[i];
#pragma unroll 4
    for (int j = 0; j < nj; j++) {
      const Cx<R> v = V[j * ldv + i];
      const Cx<R> h = hs[j];
      wi.x -= v.x * h.x - v.y * h.y;
      wi.y -= v.x * h.y + v.y * h.x;
    }
    w[i] = wi;
    nrm += (double)wi.x * wi.x + (double)wi.y * wi.y;
  }
  return nrm;
}

template <>
__device__ __forceinline__ double update_rows<float>(const float2* __restrict__ V, long long ldv,
                                                     int nj, const float2* hs, float2* w,
                                                     long long n) {
  double nrm = 0.0;
  const long long n2 = n >> 1;
  float4* w4 = reinterpret_cast<float4*>(w);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n2;
       i += (long long)gridDim.x * blockDim.x) {
    float4 wv = w4[i];
#pragma unroll 4
    for (int j = 0; j < nj; j++) {
      const float4 v = reinterpret_cast<const float4*>(V + j * ldv)[i];
      const float2 h = hs[j];
      wv.x -= v.x * h.x - v.y * h.y;
      wv.y -= v.x * h.y + v.y * h.x;
      wv.z -= v.z * h.x - v.w * h.y;
      wv.w -= v.z * h.y + v.w * h.x;
    }
    w4[i] = wv;
    nrm += (double)wv.x * wv.x + (double)wv.y * wv.y;
    nrm += (double)wv.z * wv.z + (double)wv.w * wv.w;
  }
  if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
    float2 wi = w[n - 1];
    for (int j = 0; j < nj; j++) {
      const float2 v = V[j * ldv + n - 1];
      const float2 h = hs[j];
      wi.x -= v.x * h.x - v.y * h.y;
      wi.y -= v.x * h.y + v.y * h.x;
    }
    w[n - 1] = wi;
    nrm += (double)wi.x * wi.x + (double)wi.y * wi.y;
  }
  return nrm;
}

template <typename R>
__device__ __forceinline__ void cta_dots(const Cx<R>* __restrict__ V, long long ldv, int nj,
                                         const Cx<R>* __restrict__ w, long long n,
                                         double2* partial, double2* sh) {
  (void)sh;
  __shared__ double2 red[kDotBatch][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int j0 = 0; j0 < nj; j0 += kDotBatch) {
    double2 acc[kDotBatch];
#pragma unroll
    for (int q = 0; q < kDotBatch; q++) acc[q] = make_double2(0.0, 0.0);
    const int nb = min(kDotBatch, nj - j0);
    dots_rows<R>(V, ldv, j0, nb, w, n, acc);
#pragma unroll
    for (int q = 0; q < kDotBatch; q++) {
      const double2 s = warp_sum(acc[q]);
      if (lane == 0) red[q][warp] = s;
    }
    __syncthreads();
    if (threadIdx.x < nb) {
      double2 s = make_double2(0.0, 0.0);
      for (int q = 0; q < nw; q++) {
        s.x += red[threadIdx.x][q].x;
        s.y += red[threadIdx.x][q].y;
      }
      partial[(j0 + threadIdx.x) * gridDim.x + blockIdx.x] = s;
    }
    __syncthreads();
  }
}

// h1 = V(:,0..k)^H w ; H(:,k) = h1
template <typename R>
__global__ void __launch_bounds__(kRedThreads) k_gs_dots(GmresDev* st, int k,
                                                         const Cx<R>* __restrict__ V,
                                                         long long ldv, const Cx<R>* __restrict__ w,
                                                         long long n, long long vs) {
  __shared__ double2 sh[32];
  st += blockIdx.y;
  V += blockIdx.y * vs;
  w += blockIdx.y * vs;
  if (st->done) return;
  cta_dots<R>(V, ldv, k + 1, w, n, st->partial, sh);
  if (last_block(&st->ticket)) {
    reduce_partials(st->partial, k + 1, gridDim.x, st->h1, sh);
    if (threadIdx.x == 0) st->ticket = 0;
  }
}

// w <- w - V h_in ; then partial dots of V^H w (second CGS pass)
template <typename R>
__global__ void __launch_bounds__(kRedThreads) k_gs_update_dots(GmresDev* st, int k,
                                                                const Cx<R>* __restrict__ V,
                                                                long long ldv, Cx<R>* w,
                                                                long long n, long long vs) {
  __shared__ double2 sh[32];
  __shared__ Cx<R> hs[kMaxRestart + 1];
  st += blockIdx.y;
  V += blockIdx.y * vs;
  w += blockIdx.y * vs;
  if (st->done) return;
  const int nj = k + 1;
  for (int j = threadIdx.x; j < nj; j += blockDim.x) hs[j] = from_d2<Cx<R>>(st->h1[j]);
  __syncthreads();
  update_rows<R>(V, ldv, nj, hs, w, n);
  __syncthreads();
  cta_dots<R>(V, ldv, nj, w, n, st->partial, sh);
  if (last_block(&st->ticket)) {
    reduce_partials(st->partial, nj, gridDim.x, st->h2, sh);
    if (threadIdx.x == 0) st->ticket = 0;
  }
}

// Complex Givens rotation zeroing b in (a, b).
__device__ __forceinline__ void givens(double2 a, double2 b, double* c, double2* s, double2* r) {
  const double ab = hypot(b.x, b.y);
  const double aa = hypot(a.x, a.y);
  if (ab == 0.0) {
    *c = 1.0;
    *s = make_double2(0.0, 0.0);
    *r = a;
    return;
  }
  if (aa == 0.0) {
    *c = 0.0;
    *s = make_double2(b.x / ab, -b.y / ab);  // conj(b)/|b|
    *r = make_double2(ab, 0.0);
    return;
  }
  const double nrm = hypot(aa, ab);
  const double2 ph = make_double2(a.x / aa, a.y / aa);
  *c = aa / nrm;
  // s = ph * conj(b) / nrm
  *s = make_double2((ph.x * b.x + ph.y * b.y) / nrm, (ph.y * b.x - ph.x * b.y) / nrm);
  *r = make_double2(ph.x * nrm, ph.y * nrm);
}

// Hessenberg column k from h1 + h2 and the norm of the orthogonalised w, the
// previous rotations, a new Givens rotation, the residual estimate and the
// cycle's stopping tests (one thread).
__device__ __forceinline__ void gs_column(GmresDev* st, int k, double nrm) {
  const int m = st->m;
  const int ld = m + 1;
  double2* Hc = st->H + (size_t)k * ld;
  double2* Rc = st->Rm + (size_t)k * ld;
  for (int j = 0; j <= k; j++) {
    Hc[j] = make_double2(st->h1[j].x + st->h2[j].x, st->h1[j].y + st->h2[j].y);
    Rc[j] = Hc[j];
  }
  Hc[k + 1] = make_double2(nrm, 0.0);
  Rc[k + 1] = Hc[k + 1];
  // apply previous rotations
  for (int i = 0; i < k; i++) {
    const double c = st->cs[i];
    const double2 sv = st->sn[i];
    const double2 a = Rc[i], b = Rc[i + 1];
    // a' = c a + s b ; b' = -conj(s) a + c b
    Rc[i] = make_double2(c * a.x + sv.x * b.x - sv.y * b.y, c * a.y + sv.x * b.y + sv.y * b.x);
    Rc[i + 1] = make_double2(-(sv.x * a.x + sv.y * a.y) + c * b.x,
                             -(sv.x * a.y - sv.y * a.x) + c * b.y);
  }
  double c;
  double2 sv, r;
  givens(Rc[k], Rc[k + 1], &c, &sv, &r);
  st->cs[k] = c;
  st->sn[k] = sv;
  Rc[k] = r;
  Rc[k + 1] = make_double2(0.0, 0.0);
  const double2 gk = st->g[k];
  st->g[k] = make_double2(c * gk.x, c * gk.y);
  // g(k+1) = -conj(s) g(k)
  st->g[k + 1] = make_double2(-(sv.x * gk.x + sv.y * gk.y), -(sv.x * gk.y - sv.y * gk.x));
  const double resid = hypot(st->g[k + 1].x, st->g[k + 1].y);
  st->resvec[k] = resid;
  st->k = k + 1;
  st->inv_norm = (nrm > 0.0) ? 1.0 / nrm : 0.0;
  if (resid < st->tol_abs) st->converged = 1;
  if (nrm == 0.0) st->breakdown = 1;
  st->stepped = 1;
  if (st->converged || st->breakdown || k + 1 >= m) {
    st->done = 1;
    st->endnow = 1;
  }
}

// w <- w - V h2 ; ||w||^2 ; last block: Hessenberg column, Givens, residual.
template <typename R>
__global__ void __launch_bounds__(kRedThreads) k_gs_update_norm(GmresDev* st, int k,
                                                                const Cx<R>* __restrict__ V,
                                                                long long ldv, Cx<R>* w,
                                                                long long n, long long vs) {
  __shared__ double2 sh[32];
  __shared__ Cx<R> hs[kMaxRestart + 1];
  st += blockIdx.y;
  V += blockIdx.y * vs;
  w += blockIdx.y * vs;
  if (st->done) return;
  const int nj = k + 1;
  for (int j = threadIdx.x; j < nj; j += blockDim.x) hs[j] = from_d2<Cx<R>>(st->h2[j]);
  __syncthreads();
  const double2 acc = make_double2(update_rows<R>(V, ldv, nj, hs, w, n), 0.0);
  const double2 s = block_sum(acc, sh);
  if (threadIdx.x == 0) st->partial[blockIdx.x] = s;
  if (last_block(&st->ticket)) {
    double2 tot[1];
    reduce_partials(st->partial, 1, gridDim.x, tot, sh);
    if (threadIdx.x == 0) {
      st->ticket = 0;
      gs_column(st, k, sqrt(tot[0].x));
    }
  }
}

// V(:,k+1) = w * inv_norm.  Runs for the step that just completed even when
// that step ended the cycle: the restart residual V(:,1:k+1)*res needs it.
template <typename R>
__global__ void k_gs_scale(GmresDev* st, int k, Cx<R>* __restrict__ Vnext,
                           const Cx<R>* __restrict__ w, long long n, long long vs) {
  st += blockIdx.y;
  Vnext += blockIdx.y * vs;
  w += blockIdx.y * vs;
  if (st->frozen || st->k != k + 1) return;
  const R s = (R)st->inv_norm;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    Vnext[i] = cscale(w[i], s);
  }
}

// ||x||^2 -> st->scal[slot] (deterministic, grid = (kRedBlocks, members));
// with in_cycle == 1 a frozen member is skipped, with in_cycle == 2 every
// member that does not start a cycle at this step (step mode).
template <typename R>
__global__ void __launch_bounds__(kRedThreads) k_norm2(GmresDev* st, const Cx<R>* __restrict__ x,
                                                       long long n, int slot, long long vs,
                                                       int in_cycle) {
  __shared__ double2 sh[32];
  st += blockIdx.y;
  x += blockIdx.y * vs;
  if (in_cycle == 1 && st->frozen) return;
  if (in_cycle == 2 && !st->start) return;  // step mode: members starting a cycle
  double2 acc = make_double2(0.0, 0.0);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double2 v = to_d2(x[i]);
    acc.x += v.x * v.x + v.y * v.y;
  }
  const double2 s = block_sum(acc, sh);
  if (threadIdx.x == 0) st->partial[blockIdx.x] = s;
  if (last_block(&st->ticket)) {
    double2 tot[1];
    reduce_partials(st->partial, 1, gridDim.x, tot, sh);
    if (threadIdx.x == 0) {
      st->ticket = 0;
      st->scal[slot] = tot[0].x;
    }
  }
}

// Start a cycle: beta = sqrt(scal[0]); V(:,0) = r / beta; g = beta e1.
// A frozen member ends its cycle before it starts (done, k = 0).  In step mode
// (step != 0) only the members flagged to start a cycle take part.
__global__ void k_cycle_init(GmresDev* st, int step) {
  st += blockIdx.y;
  if (step && !st->start) return;
  if (!step && st->frozen) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
      st->done = 1;
      st->k = 0;
    }
    return;
  }
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    st->beta = sqrt(st->scal[0]);
    st->inv_norm = st->beta > 0.0 ? 1.0 / st->beta : 0.0;
    st->done = 0;
    st->k = 0;
    st->converged = 0;
    st->breakdown = 0;
    for (int i = 0; i <= st->m; i++) st->g[i] = make_double2(0.0, 0.0);
    st->g[0] = make_double2(st->beta, 0.0);
  }
}

// V(:,0) = r / beta; in step mode also into vcur, the column the next step
// multiplies (the Arnoldi input of every member at its own k).
template <typename R>
__global__ void k_cycle_v0(const GmresDev* st, Cx<R>* __restrict__ V0, const Cx<R>* __restrict__ r,
                           long long n, long long vs, Cx<R>* vcur, int step) {
  st += blockIdx.y;
  V0 += blockIdx.y * vs;
  r += blockIdx.y * vs;
  if (step ? !st->start : st->frozen) return;
  if (vcur) vcur += blockIdx.y * vs;
  const R s = (R)st->inv_norm;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const Cx<R> v = cscale(r[i], s);
    V0[i] = v;
    if (vcur) vcur[i] = v;
  }
}

// Least squares after the cycle: y = Rm(0:kk-1,0:kk-1) \ g(0:kk-1) (back
// substitution), res = beta e1 - H(0:kk,0:kk-1) y  (pgmres_iter.m:117-119).
__global__ void k_cycle_ls(GmresDev* st, int step) {
  st += blockIdx.y;
  if (threadIdx.x != 0 || blockIdx.x != 0 || (step ? !st->endnow : st->frozen)) return;
  const int kk = st->k;
  const int ld = st->m + 1;
  for (int i = kk - 1; i >= 0; i--) {
    double2 s = st->g[i];
    for (int j = i + 1; j < kk; j++) {
      const double2 a = st->Rm[(size_t)j * ld + i];
      const double2 yj = st->y[j];
      s.x -= a.x * yj.x - a.y * yj.y;
      s.y -= a.x * yj.y + a.y * yj.x;
    }
    const double2 d = st->Rm[(size_t)i * ld + i];
    const double dd = d.x * d.x + d.y * d.y;
    st->y[i] = dd > 0.0 ? make_double2((s.x * d.x + s.y * d.y) / dd, (s.y * d.x - s.x * d.y) / dd)
                        : make_double2(0.0, 0.0);
  }
  for (int i = 0; i <= kk; i++) {
    double2 s = make_double2(i == 0 ? st->beta : 0.0, 0.0);
    for (int j = 0; j < kk; j++) {
      const double2 a = st->H[(size_t)j * ld + i];
      const double2 yj = st->y[j];
      s.x -= a.x * yj.x - a.y * yj.y;
      s.y -= a.x * yj.y + a.y * yj.x;
    }
    st->res[i] = s;
  }
}

// x += V(:,0:kk-1) y ; r = V(:,0:kk) res   (pgmres_iter.m:133-150).  With a right
// preconditioner x accumulates u = sum of the cycles' V y, to which the solve
// applies M^{-1} once after its last cycle.
template <typename R>
__global__ void k_cycle_update(const GmresDev* st, const Cx<R>* __restrict__ V, long long ldv,
                               Cx<R>* x, Cx<R>* r, long long n, long long vs, int step) {
  __shared__ Cx<R> ys[kMaxRestart];
  __shared__ Cx<R> rs[kMaxRestart + 1];
  st += blockIdx.y;
  V += blockIdx.y * vs;
  if (x) x += blockIdx.y * vs;
  r += blockIdx.y * vs;
  if (step ? !st->endnow : st->frozen) return;
  const int kk = st->k;
  for (int j = threadIdx.x; j <= kk; j += blockDim.x) {
    if (j < kk) ys[j] = from_d2<Cx<R>>(st->y[j]);
    rs[j] = from_d2<Cx<R>>(st->res[j]);
  }
  __syncthreads();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    Cx<R> xi = x ? x[i] : czero<Cx<R>>();
    Cx<R> ri = czero<Cx<R>>();
    for (int j = 0; j <= kk; j++) {
      const Cx<R> v = V[j * ldv + i];
      if (j < kk) cfma(xi, v, ys[j]);
      cfma(ri, v, rs[j]);
    }
    if (x) x[i] = xi;
    r[i] = ri;
  }
}

// ------------------------------------------- Gram-Schmidt in two basis reads
// For restart lengths up to kGsMaxCols - 1 an Arnoldi step reads the basis in
// two passes and a finishing sweep (CGS2; the kernels above read it four times):
//   k_gs_pass<false>: h1 = V^H w;
//   k_gs_pass<true>:  w' = w - V h1 (written back), h2 = V^H w' and ||w'||^2
//                     in the same read; its last CTA forms the Hessenberg
//                     column with ||w''||^2 = ||w'||^2 - ||h2||^2 (w'' = w' - V h2
//                     and h2 = V^H w' with V orthonormal);
//   k_gs_finish:      V(:,k+1) = (w' - V h2) / ||w''||.
// The two passes are producer/consumer pipelines: one producer warp streams
// chunks of gs_rows() rows of all k+1 basis columns and of w into a ring of
// shared-memory stages with bulk asynchronous copies (mbarrier completion,
// bounded waits), and sixteen consumer warps take the dot products out of
// shared memory, one warp per column, accumulating in FP64 in a fixed order
// (deterministic; in complex64 a lane sums its rows of one chunk with FP32
// FMAs first, so FP64 conversions are per chunk, not per element); the update
// of w' (pass<true>) runs one thread per row before the dots of the same stage.
constexpr int kGsMaxCols = 51;
constexpr int kGsConsumers = 512;
constexpr int kGsWarps = kGsConsumers / 32;  // consumer warps
constexpr int kGsThreads = kGsConsumers + 32;  // + one producer warp
constexpr int kGsColsPerWarp = (kGsMaxCols + kGsWarps - 1) / kGsWarps;
constexpr int kGsBlocks = 148;  // one CTA per SM
constexpr int kGsMaxStages = 6;
constexpr size_t kGsSmemBudget = 220 * 1024;

// Rows per chunk: each column segment of a chunk is one bulk copy, 4 KB when
// two stages of such chunks fit the budget, else 2 KB (long bases).
template <typename R>
__host__ __device__ inline int gs_rows(int nj) {
  const int r4 = 4096 / (int)sizeof(Cx<R>);
  return 2ull * (nj + 1) * r4 * sizeof(Cx<R>) <= kGsSmemBudget ? r4 : r4 / 2;
}
template <typename R>
__host__ __device__ inline int gs_stages(int nj) {
  const size_t st = ((size_t)nj + 1) * gs_rows<R>(nj) * sizeof(Cx<R>);
  const size_t s = kGsSmemBudget / st;
  return (int)(s < 2 ? 2 : (s > kGsMaxStages ? kGsMaxStages : s));
}
template <typename R>
__host__ __device__ inline size_t gs_pass_smem(int nj) {
  return (size_t)gs_stages<R>(nj) * ((size_t)nj + 1) * gs_rows<R>(nj) * sizeof(Cx<R>);
}

__device__ __forceinline__ void consumer_bar() {
  asm volatile("bar.sync 1, %0;" ::"n"(kGsConsumers) : "memory");
}

// k < 0 (step mode): each member's own basis size k = st->k, and the ring's
// stage count and chunk rows from it as the host computes them (the launch
// then carries the largest shared-memory size of its restart length).
template <typename R, bool kUpdate>
__global__ void __launch_bounds__(kGsThreads, 1) k_gs_pass(GmresDev* st, int k,
                                                           const Cx<R>* __restrict__ V,
                                                           long long ldv, Cx<R>* w, long long n,
                                                           long long vs, int stages, int RW) {
  using C = Cx<R>;
  __shared__ double2 sh[32];
  __shared__ C hs[kGsMaxCols];
  __shared__ __align__(8) uint64_t full[kGsMaxStages];
  __shared__ __align__(8) uint64_t empty[kGsMaxStages];
  __shared__ double2 tot[1];
  extern __shared__ __align__(128) unsigned char smem_raw[];
  st += blockIdx.y;
  V += blockIdx.y * vs;
  w += blockIdx.y * vs;
  if (st->done || kernel_err_set()) return;
  if (k < 0) {
    // read before any CTA of this launch can finish: the last CTA (which
    // advances st->k in gs_column) arrives only after every CTA has started
    k = st->k;
    stages = gs_stages<R>(k + 1);
    RW = gs_rows<R>(k + 1);
  }
  const int nj = k + 1;
  const size_t stage = ((size_t)nj + 1) * RW;  // elements of one stage
  C* buf = reinterpret_cast<C*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long nch = (n + RW - 1) / RW;
  const int mine = nch > blockIdx.x ? (int)((nch - 1 - blockIdx.x) / gridDim.x + 1) : 0;
  if (tid == 0) {
    for (int s = 0; s < stages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kGsWarps);
    }
    mbar_init_fence();
  }
  if (kUpdate)
    for (int j = tid; j < nj; j += blockDim.x) hs[j] = from_d2<C>(st->h1[j]);
  __syncthreads();
  if (warp == kGsWarps) {
    // producer: chunk i of this CTA into stage i % stages; lane j copies
    // column j (j = nj is w), sizes rounded up to 16 bytes inside the padding
    for (int i = 0; i < mine; i++) {
      const int s = i % stages;
      if (i >= stages && !mbar_wait(&empty[s], ((i / stages) - 1) & 1)) return;
      const long long r0 = (blockIdx.x + (long long)i * gridDim.x) * RW;
      const int rows = (int)min((long long)RW, n - r0);
      const unsigned bytes = (unsigned)(((size_t)rows * sizeof(C) + 15) / 16 * 16);
      if (lane == 0) mbar_arrive_expect_tx(&full[s], bytes * (nj + 1));
      __syncwarp();
      C* dst = buf + (size_t)s * stage;
      for (int j = lane; j <= nj; j += 32) {
        const C* src = (j < nj) ? V + (long long)j * ldv + r0 : w + r0;
        bulk_g2s(dst + (size_t)j * RW, src, bytes, &full[s]);
      }
    }
    return;
  }
  double2 acc[kGsColsPerWarp];
#pragma unroll
  for (int q = 0; q < kGsColsPerWarp; q++) acc[q] = make_double2(0.0, 0.0);
  double nrm = 0.0;
  // a consumer whose wait gave up keeps taking part in every consumer barrier
  // (its later waits return at once: the error word is set) and skips the work
  int failed = 0;
  for (int i = 0; i < mine; i++) {
    const int s = i % stages;
    const bool ok = mbar_wait(&full[s], (i / stages) & 1);
    failed |= !ok;
    const C* Vs = buf + (size_t)s * stage;
    C* ws = buf + (size_t)s * stage + (size_t)nj * RW;
    const long long r0 = (blockIdx.x + (long long)i * gridDim.x) * RW;
    const int rows = ok ? (int)min((long long)RW, n - r0) : 0;
    if (kUpdate) {
      if (tid < rows) {
        C wi = ws[tid];
        for (int j = 0; j < nj; j++) {
          const C v = Vs[(size_t)j * RW + tid];
          const C h = hs[j];
          wi.x -= v.x * h.x - v.y * h.y;
          wi.y -= v.x * h.y + v.y * h.x;
        }
        ws[tid] = wi;
        w[r0 + tid] = wi;
        if constexpr (sizeof(R) == 4)
          nrm += (double)fmaf(wi.x, wi.x, wi.y * wi.y);
        else
          nrm += (double)wi.x * wi.x + (double)wi.y * wi.y;
      }
      consumer_bar();
    }
#pragma unroll
    for (int q = 0; q < kGsColsPerWarp; q++) {
      const int j = warp + q * kGsWarps;
      if (j < nj) {
        if constexpr (sizeof(R) == 4) {
          // complex64: a lane's rows of the chunk (at most RW / 32 = 16) summed
          // with FP32 FMAs, the partial sum carried in FP64 across chunks (a
          // conversion per lane, column and chunk, not per element)
          float2 p = make_float2(0.f, 0.f);
          for (int r = lane; r < rows; r += 32) {
            const C v = Vs[(size_t)j * RW + r];
            const C x = ws[r];
            p.x = fmaf(v.x, x.x, p.x);
            p.x = fmaf(v.y, x.y, p.x);
            p.y = fmaf(v.x, x.y, p.y);
            p.y = fmaf(-v.y, x.x, p.y);
          }
          acc[q].x += (double)p.x;
          acc[q].y += (double)p.y;
        } else {
          for (int r = lane; r < rows; r += 32) {
            const double2 v = to_d2(Vs[(size_t)j * RW + r]);
            const double2 x = to_d2(ws[r]);
            acc_cdot(acc[q], v.x, v.y, x.x, x.y);
          }
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }
  if (named_bar_or<kGsConsumers>(1, failed)) return;  // nothing of this CTA is reduced
#pragma unroll
  for (int q = 0; q < kGsColsPerWarp; q++) {
    const int j = warp + q * kGsWarps;
    const double2 v = warp_sum(acc[q]);
    if (j < nj && lane == 0) st->partial[j * gridDim.x + blockIdx.x] = v;
  }
  if (kUpdate) {
    // consumer-only block sum of ||w'||^2
    double2 t = make_double2(nrm, 0.0);
    t = warp_sum(t);
    if (lane == 0) sh[warp] = t;
    consumer_bar();
    if (tid == 0) {
      double2 a = make_double2(0.0, 0.0);
      for (int q = 0; q < kGsWarps; q++) a.x += sh[q].x;
      st->partial[nj * gridDim.x + blockIdx.x] = a;
    }
  }
  // the last CTA (consumer threads only: the producer warp has left)
  __shared__ bool amlast;
  __threadfence();
  consumer_bar();
  if (tid == 0) amlast = atomicAdd(&st->ticket, 1u) == gridDim.x - 1;
  consumer_bar();
  if (!amlast) return;
  __threadfence();
  const int nr = kUpdate ? nj + 1 : nj;
  for (int j = warp; j < nr; j += kGsWarps) {
    double2 v = make_double2(0.0, 0.0);
    for (int b = lane; b < (int)gridDim.x; b += 32) {
      const double2 p = __ldcg(&st->partial[j * gridDim.x + b]);
      v.x += p.x;
      v.y += p.y;
    }
    v = warp_sum(v);
    if (lane == 0) {
      if (!kUpdate) st->h1[j] = v;
      else if (j < nj) st->h2[j] = v;
      else tot[0] = v;
    }
  }
  consumer_bar();
  if (tid == 0) {
    st->ticket = 0;
    if (kUpdate) {
      double hh = 0.0;
      for (int j = 0; j < nj; j++) hh += st->h2[j].x * st->h2[j].x + st->h2[j].y * st->h2[j].y;
      gs_column(st, k, sqrt(fmax(tot[0].x - hh, 0.0)));
    }
  }
}

// V(:,k+1) = (w' - V h2) * inv_norm, for the step that just completed (also
// when it ended the cycle: the restart residual needs that column).  k < 0
// (step mode): every member that took this step, at its own k, Vnext = V and
// the column also goes to vcur (the next step's input).
template <typename R>
__global__ void __launch_bounds__(kRedThreads) k_gs_finish(GmresDev* st, int k,
                                                           const Cx<R>* __restrict__ V,
                                                           long long ldv, const Cx<R>* w,
                                                           Cx<R>* __restrict__ Vnext,
                                                           long long n, long long vs,
                                                           Cx<R>* __restrict__ vcur) {
  using C = Cx<R>;
  __shared__ C hs[kGsMaxCols];
  st += blockIdx.y;
  V += blockIdx.y * vs;
  w += blockIdx.y * vs;
  Vnext += blockIdx.y * vs;
  if (k < 0) {
    if (!st->stepped) return;
    k = st->k - 1;
    Vnext += (long long)(k + 1) * ldv;
  } else if (st->frozen || st->k != k + 1) {
    return;
  }
  if (vcur) vcur += blockIdx.y * vs;
  const int nj = k + 1;
  for (int j = threadIdx.x; j < nj; j += blockDim.x) hs[j] = from_d2<C>(st->h2[j]);
  __syncthreads();
  const R s = (R)st->inv_norm;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    C wi = w[i];
#pragma unroll 8
    for (int j = 0; j < nj; j++) {
      const C v = V[(long long)j * ldv + i];
      const C h = hs[j];
      wi.x -= v.x * h.x - v.y * h.y;
      wi.y -= v.x * h.y + v.y * h.x;
    }
    const C o = cscale(wi, s);
    Vnext[i] = o;
    if (vcur) vcur[i] = o;
  }
}

// ------------------------------------------------------------ step mode
// A lane runs its members' restart cycles out of phase: a launch sequence
// takes one Arnoldi step of every member in a cycle, each at its own k, a
// member whose cycle ended runs its least-squares update in the same
// sequence, and a member restarts (or begins a new inner solve) at the next
// step without waiting for the others.  These two kernels (one thread per
// member) bracket a step; the arithmetic of every member is that of the
// in-phase cycle.

// After the cycle-start launches: clear the per-step flags.
__global__ void k_step_begin(GmresDev* st, int km) {
  const int b = threadIdx.x;
  if (b >= km) return;
  GmresDev* s = st + b;
  s->start = 0;
  s->stepped = 0;
  s->endnow = 0;
}

// After the end-of-cycle launches: a member whose cycle ended either stops
// its inner solve (converged, exact breakdown or its cycle limit: the stopping
// test of the in-phase driver, on the same numbers) or restarts at the next
// step.  The cycle's residuals are appended to hist.
__global__ void k_step_end(GmresDev* st, int km) {
  const int b = threadIdx.x;
  if (b >= km) return;
  GmresDev* s = st + b;
  if (!s->endnow) return;
  const int p = s->k;
  s->cycles += 1;
  s->itot += p;
  s->kdone = p;
  for (int i = 0; i < p && s->nhist < kHist; i++) s->hist[s->nhist++] = s->resvec[i];
  const double ri = p > 0 ? s->resvec[p - 1] / s->ibn : 1.0;
  const bool stop = !(ri > s->itol && s->cycles < s->maxit) || (s->breakdown && !s->converged);
  if (stop) {
    s->ifin = 1;
    s->frozen = 1;
  } else {
    s->start = 1;
  }
}

}  // namespace vox
