// Level-1 circulant preconditioner on the device.
//
// Build (level_1_parallel_func_N.m:1-281 + Bragg_MOR_script.m:61-72):
//   1. T. Chan optimal circulant of each Toeplitz component along x:
//      c(1) = A(1), c(i) = (L+1-i)/L A(i) +/- (i-1)/L A(L-i+2)  (- for xy, xz)
//   2. FFT along x (length L) of every (y, z, component) line
//   3. per x-mode i: the dense 3MN x 3MN block of Toeplitz-in-y / Toeplitz-in-z
//      sub-blocks (with the reference's sign pattern and triu symmetrisation
//      for the xz and yz blocks), B_i = Gram*I - diag(face3)*circ_i
//   4. batched LU with partial pivoting of all B_i (one CTA per block,
//      right-looking, 8-column panels staged in shared memory)
// Apply (chan_mvp_idx.m:4-16): scatter to the grid, FFT along x of every
// (y,z,c) line, per mode P*L*U solve (factor tiles streamed through shared
// memory, one CTA per factored mode; modes i and L-i share one factorisation),
// inverse FFT along x (1/L), gather.  The apply reads each factor once for two
// modes: (L/2+1)*(3MN)^2 complex values, about half the bytes of the
// reference's inverse-block GEMV.
// Caller-supplied inverse blocks (chan_mvp_idx's inv_blocks) are applied by a
// plain per-mode GEMV instead.
#pragma once

#include <type_traits>

#include "bulk.cuh"
#include "fft.cuh"
#include "krylov.cuh"

namespace vox {

constexpr int kLuNb = 8;        // panel width of the batched LU
constexpr int kTrsvNb = 32;     // diagonal block of the triangular solves
// right-hand-side length padded to whole diagonal blocks
inline int lu_npad(int n) { return (n + kTrsvNb - 1) / kTrsvNb * kTrsvNb; }

struct PcGeom {
  int L, M, N;
  int n3;          // 3*M*N
  long long V;
  int ybx;         // lines per CTA in the x-FFT kernels
  int sx;          // smem stride of a line
};

// Members of a batched apply (blockIdx.y, or one CTA for all members in the
// streamed solve): member b's x-transformed work follows member 0's at
// L*n3 elements, its input/output vectors at vs elements, its skip flag at fs
// ints.
__host__ __device__ inline long long pc_work_elems(const PcGeom& g) {
  return (long long)g.L * g.n3;
}

__device__ __forceinline__ float fmaR(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmaR(double a, double b, double c) { return __fma_rn(a, b, c); }

// acc += a * b and acc -= a * b, complex, as four fused multiply-adds each
template <typename C>
__device__ __forceinline__ void cmac(C& acc, C a, C b) {
  acc.x = fmaR(a.x, b.x, acc.x);
  acc.x = fmaR(-a.y, b.y, acc.x);
  acc.y = fmaR(a.x, b.y, acc.y);
  acc.y = fmaR(a.y, b.x, acc.y);
}
template <typename C>
__device__ __forceinline__ void cmsub(C& acc, C a, C b) {
  acc.x = fmaR(-a.x, b.x, acc.x);
  acc.x = fmaR(a.y, b.y, acc.x);
  acc.y = fmaR(-a.x, b.y, acc.y);
  acc.y = fmaR(-a.y, b.x, acc.y);
}

// two adjacent complex values in one access where possible (16-byte aligned)
__device__ __forceinline__ void ld_pair(const float2* p, float2& a, float2& b) {
  const float4 q = *reinterpret_cast<const float4*>(p);
  a = make_float2(q.x, q.y);
  b = make_float2(q.z, q.w);
}
__device__ __forceinline__ void ld_pair(const double2* p, double2& a, double2& b) {
  a = p[0];
  b = p[1];
}
__device__ __forceinline__ void st_pair(float2* p, float2 a, float2 b) {
  *reinterpret_cast<float4*>(p) = make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ void st_pair(double2* p, double2 a, double2 b) {
  p[0] = a;
  p[1] = b;
}

// --------------------------------------------------------------- apply: x-FFT
// kBig: the x length L has a prime factor above 13 (compiled big-prime
// butterflies; a separate instantiation keeps the others' register budget).
// Global loads are issued kPcBatch (gathers) or 2 kPcBatch (the transformed
// lines) per thread before their stores, so each thread keeps several reads in
// flight.
constexpr int kPcBatch = 6;

template <typename R, bool kBig>
__global__ void __launch_bounds__(256, kBig && sizeof(R) == 4 ? 2 : 1) k_pc_xfwd(PcGeom g, FftPlan pl, const Cx<R>* __restrict__ tw,
                                                 const Cx<R>* __restrict__ in,
                                                 const int* __restrict__ vmap,
                                                 Cx<R>* __restrict__ T, const int* skip,
                                                 long long vs, int fs) {
  using C = Cx<R>;
  const int mb = blockIdx.y;
  if (skip && skip[(long long)mb * fs]) return;
  in += mb * vs;
  T += mb * pc_work_elems(g);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + (size_t)g.ybx * g.sx;
  const int col0 = blockIdx.x * g.ybx;
  const int nl = min(g.ybx, g.n3 - col0);
  // gather in batches of kPcBatch per thread: the index-map loads, then the
  // vector loads, then the stores
  const int tot = g.ybx * g.L;
  for (int t0 = threadIdx.x; t0 < tot; t0 += kPcBatch * blockDim.x) {
    int m[kPcBatch];
#pragma unroll
    for (int u = 0; u < kPcBatch; u++) {
      const int t = t0 + u * blockDim.x;
      const int l = t / g.L;
      m[u] = (t < tot && l < nl) ? vmap[(long long)(col0 + l) * g.L + (t - l * g.L)] : -1;
    }
    C v[kPcBatch];
#pragma unroll
    for (int u = 0; u < kPcBatch; u++) v[u] = m[u] >= 0 ? in[m[u]] : czero<C>();
#pragma unroll
    for (int u = 0; u < kPcBatch; u++) {
      const int t = t0 + u * blockDim.x;
      const int l = t / g.L;
      if (t < tot) bufA[(size_t)l * g.sx + (t - l * g.L)] = v[u];
    }
  }
  __syncthreads();
  C* res = block_fft<C, kBig>(bufA, bufB, pl, g.ybx, g.sx, tw, -1);
  for (int t = threadIdx.x; t < nl * g.L; t += blockDim.x) {
    const int i = t / nl;
    const int l = t - i * nl;
    T[(long long)i * g.n3 + col0 + l] = res[(size_t)l * g.sx + i];
  }
}

template <typename R, bool kBig>
__global__ void __launch_bounds__(256, kBig && sizeof(R) == 4 ? 2 : 1) k_pc_xinv(PcGeom g, FftPlan pl, const Cx<R>* __restrict__ tw,
                                                 const Cx<R>* __restrict__ T,
                                                 const int* __restrict__ vmap, R scale,
                                                 Cx<R>* out, const int* skip, long long vs,
                                                 int fs) {
  using C = Cx<R>;
  const int mb = blockIdx.y;
  if (skip && skip[(long long)mb * fs]) return;
  T += mb * pc_work_elems(g);
  out += mb * vs;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + (size_t)g.ybx * g.sx;
  const int col0 = blockIdx.x * g.ybx;
  const int nl = min(g.ybx, g.n3 - col0);
  const int tot = g.ybx * g.L;
  for (int t0 = threadIdx.x; t0 < tot; t0 += 2 * kPcBatch * blockDim.x) {
    C v[2 * kPcBatch];
#pragma unroll
    for (int u = 0; u < 2 * kPcBatch; u++) {
      const int t = t0 + u * blockDim.x;
      const int i = t / g.ybx;
      const int l = t - i * g.ybx;
      v[u] = (t < tot && l < nl) ? T[(long long)i * g.n3 + col0 + l] : czero<C>();
    }
#pragma unroll
    for (int u = 0; u < 2 * kPcBatch; u++) {
      const int t = t0 + u * blockDim.x;
      const int i = t / g.ybx;
      if (t < tot) bufA[(size_t)(t - i * g.ybx) * g.sx + i] = v[u];
    }
  }
  __syncthreads();
  C* res = block_fft<C, kBig>(bufA, bufB, pl, g.ybx, g.sx, tw, +1);
  const int totw = nl * g.L;
  for (int t0 = threadIdx.x; t0 < totw; t0 += kPcBatch * blockDim.x) {
    int m[kPcBatch];
#pragma unroll
    for (int u = 0; u < kPcBatch; u++) {
      const int t = t0 + u * blockDim.x;
      const int l = t / g.L;
      m[u] = t < totw ? vmap[(long long)(col0 + l) * g.L + (t - l * g.L)] : -1;
    }
#pragma unroll
    for (int u = 0; u < kPcBatch; u++) {
      if (m[u] < 0) continue;
      const int t = t0 + u * blockDim.x;
      const int l = t / g.L;
      out[m[u]] = cscale(res[(size_t)l * g.sx + (t - l * g.L)], scale);
    }
  }
}

// ------------------------------------------------------------------- build
// Chan circulant along x of each component: src/dst [comp][z][y][x] (x fastest).
__global__ void k_chan(int L, long long V, const double2* __restrict__ G, double2* out) {
  const int sgn[6] = {1, -1, -1, 1, 1, 1};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 6 * V;
       t += (long long)gridDim.x * blockDim.x) {
    const int comp = (int)(t / V);
    const long long r = t - comp * V;
    const int x = (int)(r % L);
    const long long line = r - x;  // index of (0, y, z)
    const double2* A = G + comp * V + line;
    double2 v;
    if (x == 0) {
      v = A[0];
    } else {
      const double a = (double)(L - x) / L, b = sgn[comp] * (double)x / L;
      const double2 p = A[x], q = A[L - x];
      v = make_double2(a * p.x + b * q.x, a * p.y + b * q.y);
    }
    out[t] = v;
  }
}

// Entry (row, col) of the 3MN x 3MN block of x-mode i assembled from the
// x-transformed Chan circulants Cf [comp][z][y][x] with the reference's
// toeplitz / cell2mat / triu pattern (level_1_parallel_func_N.m:113-190, the
// same in level_1_parallel_func.m and level_2_parallel_func.m); row and col
// index (component, z, y) with y fastest.
__device__ __forceinline__ double2 circ_entry(const double2* __restrict__ Cf, int L, int M,
                                              int N, long long V, int i, int row, int col) {
  const int MN = M * N;
  const int bp = row / MN, bq = col / MN;
  const int p = row - bp * MN, q = col - bq * MN;
  const int yp = p % M, zp = p / M, yq = q % M, zq = q / M;
  const int dy = yp > yq ? yp - yq : yq - yp;
  const int dz = zp > zq ? zp - zq : zq - zp;
  auto C = [&](int comp, int y, int z) -> double2 {
    return Cf[comp * V + i + (long long)L * (y + (long long)M * z)];
  };
  const int b0 = bp < bq ? bp : bq, b1 = bp < bq ? bq : bp;
  if (b0 == 0 && b1 == 0) return C(0, dy, dz);
  if (b0 == 0 && b1 == 1) {
    // toeplitz([-CC(1) CC(2:M)], -CC(1:M)): y > y' -> CC, else -CC
    const double2 c = C(1, dy, dz);
    return (yp > yq) ? c : make_double2(-c.x, -c.y);
  }
  if (b0 == 0 && b1 == 2) {
    // -C3 symmetric, then triu antisymmetrised: p<q -> -C3, p>q -> +C3, p==q -> -C3
    const double2 c = C(2, dy, dz);
    return (p > q) ? c : make_double2(-c.x, -c.y);
  }
  if (b0 == 1 && b1 == 1) return C(3, dy, dz);
  if (b0 == 1 && b1 == 2) {
    // toeplitz([C5(1) -C5(2:M)], C5(1:M)) then triu symmetrised:
    // value of the upper entry (a<=b): y_a > y_b -> -C5, else C5
    const int a = p < q ? p : q, b = p < q ? q : p;
    const int ya = a % M, yb = b % M;
    const double2 c = C(4, dy, dz);
    return (ya > yb) ? make_double2(-c.x, -c.y) : c;
  }
  return C(5, dy, dz);
}

// Dense block of mode i (column-major, leading dimension ld) from the
// x-transformed Chan circulants Cf; B = gram*I - face3 .* circ.
__global__ void k_assemble_blocks(int L, int M, int N, long long V, int i0, int nmodes, int ld,
                                  const double2* __restrict__ Cf, const double* __restrict__ face3,
                                  double gram, double2* __restrict__ B) {
  const int n3 = 3 * M * N;
  const long long per = (long long)n3 * n3;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nmodes * per;
       t += (long long)gridDim.x * blockDim.x) {
    const int im = (int)(t / per);
    const long long e = t - im * per;
    const int col = (int)(e / n3);
    const int row = (int)(e - (long long)col * n3);
    const double2 v = circ_entry(Cf, L, M, N, V, i0 + im, row, col);
    const double f = face3[row];
    double2 o = make_double2(-f * v.x, -f * v.y);
    if (row == col) o.x += gram;
    B[(long long)im * ld * ld + (long long)col * ld + row] = o;
  }
}

// --------------------------------------------------------- level-2 (build)
// level_2_parallel_func.m:166-192: for x-mode i and the M x M sub-block (j, k)
// of its 3MN block (j, k = component * N + z), the T. Chan circulant along y
// of the sub-block's first column and row, c(y) = ((M-y) col(y) + y row(M-y))/M,
// diagonalised by an FFT along y: block m of x-mode i is the 3N x 3N matrix
// with entries fft(c_jk)(m).  One CTA per (j, k, i); output
// B2[((i*M + m)*n2 + k)*n2 + j] (column-major 3N x 3N blocks, n2 = 3N).
__global__ void __launch_bounds__(256) k_level2_blocks(int L, int M, int N, long long V,
                                                       FftPlan py,
                                                       const double2* __restrict__ tw,
                                                       const double2* __restrict__ Cf,
                                                       double2* __restrict__ B2) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int sy = pad_stride(M);
  double2* a = reinterpret_cast<double2*>(smem_raw);
  double2* b = a + sy;
  const int n2 = 3 * N;
  const int jk = blockIdx.x;
  const int j = jk % n2, k = jk / n2;
  const int i = blockIdx.y;
  for (int y = threadIdx.x; y < M; y += blockDim.x) {
    const double2 cv = circ_entry(Cf, L, M, N, V, i, j * M + y, k * M);
    double2 v = cv;
    if (y > 0) {
      const double2 rv = circ_entry(Cf, L, M, N, V, i, j * M, k * M + (M - y));
      const double wa = (double)(M - y) / M, wb = (double)y / M;
      v = make_double2(wa * cv.x + wb * rv.x, wa * cv.y + wb * rv.y);
    }
    a[y] = v;
  }
  __syncthreads();
  double2* res = block_fft(a, b, py, 1, sy, tw, -1);
  for (int m = threadIdx.x; m < M; m += blockDim.x)
    B2[(((long long)i * M + m) * n2 + k) * n2 + j] = res[m];
}

// In-place inverse of n x n column-major matrices (n <= 64), Gauss-Jordan with
// partial pivoting in shared memory, one CTA per matrix; info[mat] = 1 + the
// failing column when a pivot is zero.
__global__ void __launch_bounds__(128) k_small_inv(int n, double2* __restrict__ A,
                                                   int* __restrict__ info) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double2* a = reinterpret_cast<double2*>(smem_raw);  // n x 2n, column-major, ld n
  __shared__ int piv_row;
  __shared__ double2 pinv;
  const long long base = (long long)blockIdx.x * n * n;
  for (int t = threadIdx.x; t < 2 * n * n; t += blockDim.x) {
    const int c = t / n, r = t - c * n;
    a[t] = (c < n) ? A[base + t] : make_double2(c - n == r ? 1.0 : 0.0, 0.0);
  }
  __syncthreads();
  for (int k = 0; k < n; k++) {
    if (threadIdx.x == 0) {
      int best = k;
      double bv = -1.0;
      for (int r = k; r < n; r++) {
        const double2 v = a[k * n + r];
        const double m = fabs(v.x) + fabs(v.y);
        if (m > bv) {
          bv = m;
          best = r;
        }
      }
      piv_row = best;
      const double2 p = a[k * n + best];
      const double d = p.x * p.x + p.y * p.y;
      if (d == 0.0) {
        if (info) info[blockIdx.x] = k + 1;
        pinv = make_double2(0.0, 0.0);
      } else {
        pinv = make_double2(p.x / d, -p.y / d);
      }
    }
    __syncthreads();
    const int pr = piv_row;
    if (pr != k)
      for (int c = threadIdx.x; c < 2 * n; c += blockDim.x) {
        const double2 t = a[c * n + k];
        a[c * n + k] = a[c * n + pr];
        a[c * n + pr] = t;
      }
    __syncthreads();
    // scale the pivot row
    for (int c = threadIdx.x; c < 2 * n; c += blockDim.x) {
      const double2 v = a[c * n + k];
      a[c * n + k] = make_double2(v.x * pinv.x - v.y * pinv.y, v.x * pinv.y + v.y * pinv.x);
    }
    __syncthreads();
    // eliminate column k from the other rows
    for (int t = threadIdx.x; t < 2 * n * n; t += blockDim.x) {
      const int c = t / n, r = t - c * n;
      if (r == k || c == k) continue;
      const double2 f = a[k * n + r];
      const double2 pv = a[c * n + k];
      a[t] = make_double2(a[t].x - (f.x * pv.x - f.y * pv.y), a[t].y - (f.x * pv.y + f.y * pv.x));
    }
    __syncthreads();
    for (int r = threadIdx.x; r < n; r += blockDim.x)
      if (r != k) a[k * n + r] = make_double2(0.0, 0.0);
    __syncthreads();
  }
  for (int t = threadIdx.x; t < n * n; t += blockDim.x) A[base + t] = a[n * n + t];
}

// ---------------------------------------------------------- level-2 (apply)
// y-FFT of the lines of the x-transformed work T [member][i][j][y] (j = 3N
// lines of length M per x-mode), written transposed as U [member][i][m][j].
// grid (ceil(3N / kL2Lines), L * members).
constexpr int kL2Lines = 8;

template <typename R>
__global__ void __launch_bounds__(256) k_l2_yfwd(PcGeom g, FftPlan py, const Cx<R>* __restrict__ tw,
                                                 const Cx<R>* __restrict__ T, Cx<R>* __restrict__ U,
                                                 const int* skip, int fs) {
  using C = Cx<R>;
  const int n2 = 3 * g.N;
  const int mb = blockIdx.y / g.L;
  const int i = blockIdx.y - mb * g.L;
  if (skip && skip[(long long)mb * fs]) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int sy = pad_stride(g.M);
  C* a = reinterpret_cast<C*>(smem_raw);
  C* b = a + kL2Lines * sy;
  const int j0 = blockIdx.x * kL2Lines;
  const int nl = min(kL2Lines, n2 - j0);
  const long long plane = (long long)blockIdx.y * g.n3;
  for (int t = threadIdx.x; t < kL2Lines * g.M; t += blockDim.x) {
    const int l = t / g.M, y = t - l * g.M;
    a[l * sy + y] = (l < nl) ? T[plane + (long long)(j0 + l) * g.M + y] : czero<C>();
  }
  __syncthreads();
  C* res = block_fft(a, b, py, kL2Lines, sy, tw, -1);
  for (int t = threadIdx.x; t < nl * g.M; t += blockDim.x) {
    const int m = t / nl, l = t - m * nl;
    U[plane + (long long)m * n2 + j0 + l] = res[l * sy + m];
  }
  (void)i;
}

// Inverse of k_l2_yfwd: U [member][i][m][j] -> T [member][i][j][y], times 1/M.
template <typename R>
__global__ void __launch_bounds__(256) k_l2_yinv(PcGeom g, FftPlan py, const Cx<R>* __restrict__ tw,
                                                 const Cx<R>* __restrict__ U, Cx<R>* __restrict__ T,
                                                 const int* skip, int fs) {
  using C = Cx<R>;
  const int n2 = 3 * g.N;
  const int mb = blockIdx.y / g.L;
  if (skip && skip[(long long)mb * fs]) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int sy = pad_stride(g.M);
  C* a = reinterpret_cast<C*>(smem_raw);
  C* b = a + kL2Lines * sy;
  const int j0 = blockIdx.x * kL2Lines;
  const int nl = min(kL2Lines, n2 - j0);
  const long long plane = (long long)blockIdx.y * g.n3;
  for (int t = threadIdx.x; t < kL2Lines * g.M; t += blockDim.x) {
    const int m = t / kL2Lines, l = t - m * kL2Lines;
    a[l * sy + m] = (l < nl) ? U[plane + (long long)m * n2 + j0 + l] : czero<C>();
  }
  __syncthreads();
  C* res = block_fft(a, b, py, kL2Lines, sy, tw, +1);
  const R s = (R)(1.0 / g.M);
  for (int t = threadIdx.x; t < nl * g.M; t += blockDim.x) {
    const int l = t / g.M, y = t - l * g.M;
    T[plane + (long long)(j0 + l) * g.M + y] = cscale(res[l * sy + y], s);
  }
}

// Per (x-mode, y-mode) 3N x 3N products for km members (P >= km columns, the
// unused ones zero and not written): Y[mb][i][m] = B2[i][m] X[mb][i][m].
// One warp per (i, m); lanes take rows, each column summed in k order with
// fused multiply-adds, so a member's result does not depend on the others.
// grid (ceil(L*M / 8)), 256 threads, shared memory 8 * 3N * P values.
template <typename R, int P>
__global__ void __launch_bounds__(256) k_l2_gemv(PcGeom g, const Cx<R>* __restrict__ B2,
                                                 const Cx<R>* __restrict__ X, Cx<R>* __restrict__ Y,
                                                 const int* skip, int fs, int km) {
  using C = Cx<R>;
  if (skip) {
    bool all = true;
    for (int b = 0; b < km; b++) all = all && skip[(long long)b * fs] != 0;
    if (all) return;
  }
  const int n2 = 3 * g.N;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long im = (long long)blockIdx.x * 8 + warp;  // i * M + m
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* xw = reinterpret_cast<C*>(smem_raw) + (size_t)warp * n2 * P;  // this warp's columns
  if (im >= (long long)g.L * g.M) return;
  const long long ws = (long long)g.L * g.n3;  // member stride of the work
  for (int t = lane; t < n2 * P; t += 32) {
    const int k = t / P, q = t - k * P;
    xw[k * P + q] = (q < km) ? X[q * ws + im * n2 + k] : czero<C>();
  }
  __syncwarp();
  const C* Bb = B2 + im * n2 * n2;
  for (int r0 = 0; r0 < n2; r0 += 32) {
    const int r = r0 + lane;
    C acc[P];
#pragma unroll
    for (int q = 0; q < P; q++) acc[q] = czero<C>();
    if (r < n2) {
      for (int k = 0; k < n2; k++) {
        const C bv = Bb[(long long)k * n2 + r];
#pragma unroll
        for (int q = 0; q < P; q++) cmac(acc[q], bv, xw[k * P + q]);
      }
#pragma unroll
      for (int q = 0; q < P; q++)
        if (q < km) Y[q * ws + im * n2 + r] = acc[q];
    }
  }
}

// out = in for km members (the identity part of a sum of preconditioners)
template <typename R>
__global__ void k_copy_members(long long n, const Cx<R>* __restrict__ in, Cx<R>* __restrict__ out,
                               const int* skip, long long vs, int fs) {
  const int mb = blockIdx.y;
  if (skip && skip[(long long)mb * fs]) return;
  in += mb * vs;
  out += mb * vs;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = in[i];
}

// Index map of a box of the grid (all z): sub[c][z][y][x] = the operator's slot
// of voxel (x0+x, y0+y, z) when mask (Ls*Ms*N, or all) selects it, else -1.
__global__ void k_vmap_box(int L, int M, int N, int x0, int y0, int Ls, int Ms,
                           const int* __restrict__ vmap, const unsigned char* __restrict__ mask,
                           int* __restrict__ sub) {
  const long long Vs = (long long)Ls * Ms * N;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 3 * Vs;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t / Vs);
    const long long e = t - c * Vs;
    const int x = (int)(e % Ls);
    const int y = (int)((e / Ls) % Ms);
    const int z = (int)(e / ((long long)Ls * Ms));
    int v = -1;
    if (!mask || mask[e]) {
      const long long cell = (long long)(x0 + x) + (long long)L * ((y0 + y) + (long long)M * z);
      v = vmap[(long long)c * L * M * N + cell];
    }
    sub[t] = v;
  }
}

// Batched LU with partial pivoting, one CTA per matrix (column-major n x n).
// piv[k] = 0-based row swapped with row k at step k (LAPACK getrf order).
template <typename R>
__global__ void __launch_bounds__(512) k_lu_batched(int n, int ld, Cx<R>* A, int* piv, int* info) {
  using C = Cx<R>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* P = reinterpret_cast<C*>(smem_raw);  // panel: (n) x kLuNb, column-major, ld = n
  __shared__ int s_piv[kLuNb];
  __shared__ R s_best[32];
  __shared__ int s_bidx[32];
  C* Ai = A + (long long)blockIdx.x * ld * ld;  // column-major, leading dimension ld
  int* pv = piv + (long long)blockIdx.x * n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k0 = 0; k0 < n; k0 += kLuNb) {
    const int kb = min(kLuNb, n - k0);
    const int rows = n - k0;
    // load panel rows k0..n-1, columns k0..k0+kb-1
    for (int t = threadIdx.x; t < rows * kb; t += blockDim.x) {
      const int j = t / rows, r = t - j * rows;
      P[(size_t)j * n + r] = Ai[(long long)(k0 + j) * ld + k0 + r];
    }
    __syncthreads();
    for (int j = 0; j < kb; j++) {
      // pivot search over panel rows j..rows-1 of column j
      R best = -1;
      int bidx = j;
      for (int r = j + threadIdx.x; r < rows; r += blockDim.x) {
        const C a = P[(size_t)j * n + r];
        const R m = fabs(a.x) + fabs(a.y);
        if (m > best) {
          best = m;
          bidx = r;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const R ob = __shfl_down_sync(0xffffffffu, best, o);
        const int oi = __shfl_down_sync(0xffffffffu, bidx, o);
        if (ob > best || (ob == best && oi < bidx)) {
          best = ob;
          bidx = oi;
        }
      }
      if (lane == 0) {
        s_best[warp] = best;
        s_bidx[warp] = bidx;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        R b = s_best[0];
        int bi = s_bidx[0];
        for (int w = 1; w < nw; w++)
          if (s_best[w] > b || (s_best[w] == b && s_bidx[w] < bi)) {
            b = s_best[w];
            bi = s_bidx[w];
          }
        s_piv[j] = bi;
        pv[k0 + j] = k0 + bi;
        if (b <= 0 && info) atomicExch(info + blockIdx.x, k0 + j + 1);
      }
      __syncthreads();
      const int pr = s_piv[j];
      if (pr != j) {
        for (int c = threadIdx.x; c < kb; c += blockDim.x) {
          C a = P[(size_t)c * n + j];
          P[(size_t)c * n + j] = P[(size_t)c * n + pr];
          P[(size_t)c * n + pr] = a;
        }
      }
      __syncthreads();
      const C d = P[(size_t)j * n + j];
      const R dd = d.x * d.x + d.y * d.y;
      for (int r = j + 1 + threadIdx.x; r < rows; r += blockDim.x) {
        if (dd > 0) {
          const C a = P[(size_t)j * n + r];
          C l;
          l.x = (a.x * d.x + a.y * d.y) / dd;
          l.y = (a.y * d.x - a.x * d.y) / dd;
          P[(size_t)j * n + r] = l;
          for (int c = j + 1; c < kb; c++) {
            const C u = P[(size_t)c * n + j];
            C& e = P[(size_t)c * n + r];
            e.x -= l.x * u.x - l.y * u.y;
            e.y -= l.x * u.y + l.y * u.x;
          }
        }
      }
      __syncthreads();
    }
    // write the panel back
    for (int t = threadIdx.x; t < rows * kb; t += blockDim.x) {
      const int j = t / rows, r = t - j * rows;
      Ai[(long long)(k0 + j) * ld + k0 + r] = P[(size_t)j * n + r];
    }
    // row swaps on the columns outside the panel
    for (int c = threadIdx.x; c < n; c += blockDim.x) {
      if (c >= k0 && c < k0 + kb) continue;
      C* colp = Ai + (long long)c * ld;
      for (int j = 0; j < kb; j++) {
        const int pr = k0 + s_piv[j];
        if (pr != k0 + j) {
          C a = colp[k0 + j];
          colp[k0 + j] = colp[pr];
          colp[pr] = a;
        }
      }
    }
    __syncthreads();
    // U12 = L11^{-1} A12 and trailing update A22 -= L21 U12, one column per thread
    for (int c = k0 + kb + threadIdx.x; c < n; c += blockDim.x) {
      C* colp = Ai + (long long)c * ld;
      C u[kLuNb];
#pragma unroll
      for (int j = 0; j < kLuNb; j++) u[j] = (j < kb) ? colp[k0 + j] : czero<C>();
#pragma unroll
      for (int j = 0; j < kLuNb; j++) {
        if (j >= kb) break;
#pragma unroll
        for (int q = j + 1; q < kLuNb; q++) {
          if (q < kb) {
            const C l = P[(size_t)j * n + q];
            u[q].x -= l.x * u[j].x - l.y * u[j].y;
            u[q].y -= l.x * u[j].y + l.y * u[j].x;
          }
        }
      }
#pragma unroll
      for (int j = 0; j < kLuNb; j++)
        if (j < kb) colp[k0 + j] = u[j];
    }
    __syncthreads();
    // trailing update, threads over (row) inside column sweeps: coalesced rows
    const int r0 = k0 + kb;
    for (int c = r0 + warp; c < n; c += nw) {
      C* colp = Ai + (long long)c * ld;
      C u[kLuNb];
#pragma unroll
      for (int j = 0; j < kLuNb; j++) u[j] = (j < kb) ? colp[k0 + j] : czero<C>();
      for (int r = r0 + lane; r < n; r += 32) {
        C e = colp[r];
#pragma unroll
        for (int j = 0; j < kLuNb; j++) {
          if (j < kb) {
            const C l = P[(size_t)j * n + (r - k0)];
            e.x -= l.x * u[j].x - l.y * u[j].y;
            e.y -= l.x * u[j].y + l.y * u[j].x;
          }
        }
        colp[r] = e;
      }
    }
    __syncthreads();
  }
}

template <typename R>
__global__ void k_cast_scale(long long n, const double2* __restrict__ src, double s, Cx<R>* dst) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    dst[i] = from_d2<Cx<R>>(make_double2(src[i].x * s, src[i].y * s));
}

// ----------------------------------------- paired, blocked LU solves (apply)
// Row permutation of getrf's pivots: (P c)[k] = c[perm[k]] (one CTA per matrix).
__global__ void k_lu_perm(int n, const int* __restrict__ piv, int* __restrict__ perm) {
  if (threadIdx.x != 0) return;
  const int* pv = piv + (long long)blockIdx.x * n;
  int* pm = perm + (long long)blockIdx.x * n;
  for (int k = 0; k < n; k++) pm[k] = k;
  for (int k = 0; k < n; k++) {
    const int p = pv[k];
    if (p != k) {
      const int a = pm[k];
      pm[k] = pm[p];
      pm[p] = a;
    }
  }
}

// Inverses of the kTrsvNb x kTrsvNb diagonal blocks of the unit-lower L and of
// U, for every block of every matrix: grid (nblk, nmat).  Output column-major
// kTrsvNb^2 per block; a ragged last block is completed with the identity.
__global__ void k_tri_inv_blocks(int n, int ld, const double2* __restrict__ A,
                                 double2* __restrict__ Dl, double2* __restrict__ Du) {
  constexpr int B = kTrsvNb;
  __shared__ double2 Bk[B][B + 1];
  __shared__ double2 X[B][B + 1];
  const int nb = (n + B - 1) / B;
  const int bk = blockIdx.x, mat = blockIdx.y;
  const int k0 = bk * B, kb = min(B, n - k0);
  const double2* Am = A + (long long)mat * ld * ld;
  for (int t = threadIdx.x; t < B * B; t += blockDim.x) {
    const int r = t % B, c = t / B;
    double2 v = make_double2(r == c ? 1.0 : 0.0, 0.0);
    if (r < kb && c < kb) v = Am[(long long)(k0 + c) * ld + k0 + r];
    Bk[r][c] = v;
  }
  __syncthreads();
  const long long off = ((long long)mat * nb + bk) * B * B;
  if (threadIdx.x < B) {
    // column c of L^{-1}: X(r,c) = delta_rc - sum_{c<=q<r} L(r,q) X(q,c)
    const int c = threadIdx.x;
    for (int r = 0; r < B; r++) {
      double2 s = make_double2(r == c ? 1.0 : 0.0, 0.0);
      if (r > c) {
        for (int q = c; q < r; q++) {
          const double2 l = Bk[r][q], x = X[q][c];
          s.x -= l.x * x.x - l.y * x.y;
          s.y -= l.x * x.y + l.y * x.x;
        }
      } else if (r < c) {
        s = make_double2(0.0, 0.0);
      }
      X[r][c] = s;
    }
    for (int r = 0; r < B; r++) Dl[off + (long long)c * B + r] = X[r][c];
    // column c of U^{-1}: X(r,c) = (delta_rc - sum_{r<q<=c} U(r,q) X(q,c)) / U(r,r)
    for (int r = B - 1; r >= 0; r--) {
      double2 s = make_double2(r == c ? 1.0 : 0.0, 0.0);
      if (r < c) {
        for (int q = r + 1; q <= c; q++) {
          const double2 u = Bk[r][q], x = X[q][c];
          s.x -= u.x * x.x - u.y * x.y;
          s.y -= u.x * x.y + u.y * x.x;
        }
      } else if (r > c) {
        s = make_double2(0.0, 0.0);
      }
      if (r <= c) {
        const double2 d = Bk[r][r];
        const double dd = d.x * d.x + d.y * d.y;
        s = dd > 0 ? make_double2((s.x * d.x + s.y * d.y) / dd, (s.y * d.x - s.x * d.y) / dd)
                   : make_double2(0.0, 0.0);
      }
      X[r][c] = s;
    }
    for (int r = 0; r < B; r++) Du[off + (long long)c * B + r] = X[r][c];
  }
}

// ------------------------------------------ streamed LU solves (the apply)
// The factors are static, so their 32 x 32 tiles are streamed through a ring
// of shared-memory slots with cp.async, half the ring in flight, in exactly
// the order the substitution consumes them; only the arithmetic waits on the
// dependency chain.  Tile order: forward [Dl(k), L(c,k) for c > k] for
// k = 0..nb-1, then backward [Du(k), U(c,k) for c < k] for k = nb-1..0.
// Factor storage is padded to ld = nb*32 (zero rows/columns), so every tile
// column is 32 contiguous, 16-byte aligned values.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Position in the tile sequence: phase 0 forward / 1 backward, block column
// k, block row c (c = -1: the inverted diagonal block).
struct TileIt {
  int phase, k, c;
};
__device__ __forceinline__ void tile_next(TileIt& it, int nb) {
  if (it.phase == 0) {
    const int c = (it.c < 0) ? it.k + 1 : it.c + 1;
    if (c < nb) {
      it.c = c;
    } else if (it.k + 1 < nb) {
      it.k++;
      it.c = -1;
    } else {
      it.phase = 1;
      it.k = nb - 1;
      it.c = -1;
    }
  } else {
    const int c = it.c + 1;
    if (c < it.k) {
      it.c = c;
    } else {
      it.k--;
      it.c = -1;
    }
  }
}

// Number of tiles per mode in consumption order, and the (phase, k, c) of
// tile i (closed-form group search, O(nb)).
__host__ __device__ inline int lu_tiles(int nb) { return nb * (nb + 1); }
__device__ inline TileIt tile_at(int i, int nb) {
  TileIt it;
  const int half = nb * (nb + 1) / 2;
  if (i < half) {
    int k = 0, start = 0;
    while (i >= start + (nb - k)) {
      start += nb - k;
      k++;
    }
    it.phase = 0;
    it.k = k;
    it.c = (i == start) ? -1 : k + (i - start);
  } else {
    int i2 = i - half, k = nb - 1, start = 0;
    while (i2 >= start + (k + 1)) {
      start += k + 1;
      k--;
    }
    it.phase = 1;
    it.k = k;
    it.c = (i2 == start) ? -1 : (i2 - start - 1);
  }
  return it;
}

// Repack LU factors (ld-padded, column-major, c128) and the inverted diagonal
// blocks into per-mode tile streams in consumption order: tile i of mode f at
// out[(f * lu_tiles(nb) + i) * 1024], each 32 x 32 column-major.  U tiles and
// inverted U diagonal blocks are scaled by su (the c64 copy holds factors of
// B/Gram: U/Gram and Gram*inv(U_kk)).  grid (lu_tiles(nb), Lf).
template <typename R>
__global__ void k_tile_pack(int nb, int ld, const double2* __restrict__ A,
                            const double2* __restrict__ Dl, const double2* __restrict__ Du,
                            double su_panel, double su_diag, Cx<R>* __restrict__ out) {
  constexpr int B = kTrsvNb;
  const int i = blockIdx.x, f = blockIdx.y;
  const TileIt it = tile_at(i, nb);
  Cx<R>* o = out + ((long long)f * lu_tiles(nb) + i) * B * B;
  for (int e = threadIdx.x; e < B * B; e += blockDim.x) {
    const int j = e / B, q = e - j * B;
    double2 v;
    double s = 1.0;
    if (it.c < 0) {
      const double2* D = (it.phase == 0 ? Dl : Du) + ((long long)f * nb + it.k) * B * B;
      v = D[e];
      if (it.phase == 1) s = su_diag;
    } else {
      v = A[(long long)f * ld * ld + (long long)(it.k * B + j) * ld + it.c * B + q];
      if (it.phase == 1) s = su_panel;
    }
    o[e] = from_d2<Cx<R>>(make_double2(v.x * s, v.y * s));
  }
}

// The streamed triangular solve, used once per preconditioner to form the
// explicit inverse blocks: a tile is consumed by one warp (lane = tile row,
// 32 column steps, no cross-lane reduction), and up to kRoundTiles
// independent panel tiles of one block column are consumed per barrier round,
// one per warp.  The P right-hand sides are interleaved in shared memory, so
// each factor value is read once from shared memory for all of them.  Tiles
// keep their HBM layout in shared memory (32 x 32, column-major).
constexpr int kRoundTiles = 4;  // warps per CTA = panel tiles per round
template <typename R> struct Ring2;
template <> struct Ring2<float> { static constexpr int value = 8; };
template <> struct Ring2<double> { static constexpr int value = 4; };

template <typename R>
constexpr size_t lu_stream2_smem(int npad, int P) {
  return (size_t)Ring2<R>::value * kTrsvNb * kTrsvNb * sizeof(Cx<R>) +
         (size_t)npad * P * sizeof(Cx<R>) + (size_t)kTrsvNb * P * sizeof(Cx<R>);
}

__device__ __forceinline__ void cp_async_wait_n(int n) {
  switch (n) {
    case 0: cp_async_wait<0>(); break;
    case 1: cp_async_wait<1>(); break;
    case 2: cp_async_wait<2>(); break;
    case 3: cp_async_wait<3>(); break;
    case 4: cp_async_wait<4>(); break;
    case 5: cp_async_wait<5>(); break;
    case 6: cp_async_wait<6>(); break;
    default: cp_async_wait<7>(); break;
  }
}

// t (npad x P, interleaved) <- U^{-1} L^{-1} t for the mode whose tile stream
// starts at tf (tiles in consumption order).  ring / xb: shared-memory work.
template <typename R, int P>
__device__ void lu_stream_core(const Cx<R>* __restrict__ tf, int nb, Cx<R>* ring, Cx<R>* t,
                               Cx<R>* xb) {
  using C = Cx<R>;
  constexpr int B = kTrsvNb;
  constexpr int S = Ring2<R>::value;
  constexpr int TILE = B * B;
  constexpr int PER = 16 / (int)sizeof(C);  // values per 16-byte piece
  const int total = lu_tiles(nb);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nthr = blockDim.x;
  auto issue = [&](int i) {
    const C* src = tf + (long long)i * TILE;
    C* dst = ring + (i % S) * TILE;
    for (int p = tid; p < TILE / PER; p += nthr) cp_async16(dst + p * PER, src + p * PER);
    cp_async_commit();
  };
  int issued = 0;
  while (issued < total && issued < S) issue(issued++);
  __syncthreads();
  // at most half the ring is consumed per round, so the other half streams in
  constexpr int RMAX = (S / 2 < kRoundTiles) ? S / 2 : kRoundTiles;
  int ci = 0;
  TileIt it{0, 0, -1};
  while (ci < total) {
    int r = 1;
    if (it.c >= 0) {
      // panel tiles left in this block column: forward c = it.c..nb-1,
      // backward c = it.c..it.k-1
      const int left = (it.phase == 0) ? nb - it.c : it.k - it.c;
      r = min(RMAX, left);
    }
    cp_async_wait_n(issued - (ci + r));
    __syncthreads();
    const int k0 = it.k * B;
    if (it.c < 0) {
      if (warp == 0) {
        // x = inv(diag block) * t_blk, every column
        const C* D = ring + (ci % S) * TILE;
        C a[P];
#pragma unroll
        for (int q = 0; q < P; q++) a[q] = czero<C>();
#pragma unroll 4
        for (int c = 0; c < B; c++) {
          const C d = D[c * B + lane];
          const C* tc = t + P * (k0 + c);
#pragma unroll
          for (int q = 0; q < P; q += 2) {
            C u0, u1;
            ld_pair(tc + q, u0, u1);
            cmac(a[q], d, u0);
            cmac(a[q + 1], d, u1);
          }
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < P; q++) {
          xb[P * lane + q] = a[q];
          t[P * (k0 + lane) + q] = a[q];
        }
      }
    } else if (warp < r) {
      // t_rows(c) -= tile * x_blk, one tile per warp
      const int ti = ci + warp;
      const C* Pt = ring + (ti % S) * TILE;
      const int row = (it.c + warp) * B + lane;
      C a[P];
#pragma unroll
      for (int q = 0; q < P; q += 2) ld_pair(t + P * row + q, a[q], a[q + 1]);
#pragma unroll 4
      for (int j = 0; j < B; j++) {
        const C v = Pt[j * B + lane];
        const C* xj = xb + P * j;
#pragma unroll
        for (int q = 0; q < P; q += 2) {
          C x0, x1;
          ld_pair(xj + q, x0, x1);
          cmsub(a[q], v, x0);
          cmsub(a[q + 1], v, x1);
        }
      }
#pragma unroll
      for (int q = 0; q < P; q++) t[P * row + q] = a[q];
    }
    __syncthreads();
    ci += r;
    for (int q = 0; q < r; q++) tile_next(it, nb);
    while (issued < total && issued < ci + S) issue(issued++);
  }
  cp_async_wait<0>();
  __syncthreads();
}

// Columns c0 .. c0+P-1 of inv(B_f) = U^{-1} L^{-1} P for every factored mode
// f (grid (ceil(n3 / P), Lf)): the right-hand sides are the permuted unit
// vectors, (P e_j)[k] = [perm[k] == j].  Output column-major, leading
// dimension ld, one ld x ld block per mode (rows >= n3 left untouched).
constexpr int kInvBuildCols = 8;  // inverse columns per CTA in the build

template <int P>
__global__ void __launch_bounds__(32 * kRoundTiles) k_lu_inv_cols(
    PcGeom g, const double2* __restrict__ tiles, const int* __restrict__ perm, int ld,
    double2* __restrict__ Binv) {
  using C = double2;
  constexpr int B = kTrsvNb;
  constexpr int S = Ring2<double>::value;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* ring = reinterpret_cast<C*>(smem_raw);
  const int n = g.n3;
  const int nb = (n + B - 1) / B;
  const int npad = nb * B;
  C* t = ring + S * B * B;
  C* xb = t + P * npad;
  const int c0 = blockIdx.x * P;
  const int f = blockIdx.y;
  const int* pm = perm + (long long)f * n;
  for (int k = threadIdx.x; k < npad; k += blockDim.x) {
    const int p = (k < n) ? pm[k] : -1;
#pragma unroll
    for (int q = 0; q < P; q++) t[P * k + q] = make_double2(p == c0 + q ? 1.0 : 0.0, 0.0);
  }
  lu_stream_core<double, P>(tiles + (long long)f * lu_tiles(nb) * B * B, nb, ring, t, xb);
  double2* out = Binv + (long long)f * ld * ld;
  for (int q = 0; q < P; q++) {
    if (c0 + q >= n) break;
    for (int k = threadIdx.x; k < n; k += blockDim.x)
      out[(long long)(c0 + q) * ld + k] = t[P * k + q];
  }
}

// ------------------------------------------------ apply: streamed inverse blocks
// The product T2_f = inv(B_f) T_f for P columns (the modes f and L-f of every
// member) with one CTA per stored block: the block (column-major, ld rows) is
// streamed through a ring of shared-memory stages, each stage KC whole
// consecutive columns, which are contiguous in memory and so arrive as ONE bulk
// asynchronous copy of KC * ld values (32 KB at ld = 1024 in either
// precision); a producer warp issues the copies and 512 consumer threads, two
// rows each, multiply out of shared memory.  Up to kStrMaxStages stages are in
// flight per CTA, which is what keeps HBM busy; the producer starts while the
// consumers gather the right-hand sides.
//
// complex64 runs on the packed FP32 pipe (fma.rn.f32x2: one instruction, two
// FMAs) with three real multiplies per complex multiply-add (Gauss):
//   S1 += br xr,  S2 += bi xi,  S3 += (br + bi)(xr + xi);
//   re = S1 - S2,  im = (S3 - S1) - S2  (once, after the last column).
// The pair of a register is the two columns of one member (modes f and L-f),
// so the right-hand sides are held in shared memory as (xr_f, xr_L-f, xi_f,
// xi_L-f) and (xs_f, xs_L-f) with xs = xr + xi, and the block element's
// (br, br), (bi, bi), (br + bi, br + bi) are formed once per row for all
// members.  That is 3 FMAs per complex term instead of 4, on half the issue
// slots; the sums are the same terms in the same order for every P.
// complex128 uses the scalar FP64 pipe with the usual four multiplies.
//
// Columns n..ld-1 of every stored block are zero (both block builders clear
// the padding) and so are the gathered right-hand-side rows k >= n, so the
// last stage may run past n without a guard: the extra terms add exact zeros.
// Each row's sums run over the columns in increasing order, so a column's
// result does not depend on P or on the other members (batched and single
// solves agree bit for bit).  The ring slot and its phase advance by counting,
// with no division in the loop.  grid (blocks), kStrThreads threads, shared
// memory str_smem().
constexpr int kStrConsumers = 512;
constexpr int kStrThreads = kStrConsumers + 32;  // + one producer warp
constexpr int kStrMaxStages = 8;

// whole columns per stage: 32 KB at ld = 1024 in either precision
template <typename R>
constexpr int str_kc() {
  return sizeof(R) == 4 ? 4 : 2;
}
template <typename R>
inline size_t str_stage_bytes(int ld) {
  return (size_t)str_kc<R>() * ld * sizeof(Cx<R>);
}
// shared-memory bytes of one right-hand-side entry (one row of one column):
// complex128 16; complex64 12 (xr, xi and xr + xi)
template <typename R>
constexpr size_t str_x_bytes() {
  return sizeof(R) == 4 ? 12 : 16;
}
// right-hand sides [ld][P] + ring [stages][KC][ld]
template <typename R>
inline size_t str_smem(int ld, int P, int stages) {
  return (size_t)ld * P * str_x_bytes<R>() + (size_t)stages * str_stage_bytes<R>(ld);
}

// named barrier of the consumer threads (the producer warp may have left)
__device__ __forceinline__ int consumers_sync_or(int pred) {
  return named_bar_or<kStrConsumers>(1, pred);
}

// three packed sums of one row and one member's column pair
struct Sums3 {
  float2 s1, s2, s3;
};

template <typename R, int P>
__global__ void __launch_bounds__(kStrThreads, 1) k_pc_inv_stream(
    PcGeom g, int paired, int ld, int stages, const Cx<R>* __restrict__ Binv,
    const Cx<R>* __restrict__ Tin, Cx<R>* __restrict__ Tout, const int* skip, int fs, int km) {
  using C = Cx<R>;
  constexpr bool kPacked = sizeof(R) == 4;
  constexpr int KS = P / 2;
  constexpr int KC = str_kc<R>();
  static_assert(P % 2 == 0, "columns come in mode pairs");
  if (kernel_err_set()) return;
  if (skip) {
    bool all = true;
    for (int b = 0; b < km; b++) all = all && skip[(long long)b * fs] != 0;
    if (all) return;
  }
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full[kStrMaxStages];
  __shared__ __align__(8) uint64_t empty[kStrMaxStages];
  // right-hand sides: complex128 X[k * P + col]; complex64 XA[k * KS + b] =
  // (xr_f, xr_L-f, xi_f, xi_L-f) and XS[k * KS + b] = (xs_f, xs_L-f) of member b
  C* X = reinterpret_cast<C*>(smem_raw);
  float4* XA = reinterpret_cast<float4*>(smem_raw);
  float2* XS = reinterpret_cast<float2*>(smem_raw + (size_t)ld * KS * sizeof(float4));
  C* ring = reinterpret_cast<C*>(smem_raw + (size_t)ld * P * str_x_bytes<R>());  // [stages][KC][ld]
  const int n = g.n3;
  const int MN = n / 3;
  const int f = blockIdx.x;
  const int i2 = g.L - f;
  const bool two = paired && f != 0 && i2 != f;
  const long long wstride = pc_work_elems(g);
  // stages of KC columns up to n; KC divides 32 and ld is a multiple of 32,
  // so the last stage stays inside the block
  const int nkb = (n + KC - 1) / KC;
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < stages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kStrConsumers / 32);
    }
    mbar_init_fence();
  }
  __syncthreads();
  if (tid >= kStrConsumers) {
    // producer warp: stage kb = columns kb*KC .. kb*KC+KC-1, one contiguous copy
    const int lane = tid & 31;
    const C* src = Binv + (long long)f * ld * ld;
    const size_t step = (size_t)KC * ld;
    const unsigned bytes = (unsigned)(step * sizeof(C));
    int s = 0;
    unsigned ph = 0;  // phase of the slot's previous fill (waited on from the second lap)
    for (int kb = 0; kb < nkb; kb++) {
      if (kb >= stages && !mbar_wait(&empty[s], ph ^ 1u)) return;
      if (lane == 0) {
        mbar_arrive_expect_tx(&full[s], bytes);
        bulk_g2s(ring + (size_t)s * step, src, bytes, &full[s]);
      }
      __syncwarp();
      src += step;
      if (++s == stages) {
        s = 0;
        ph ^= 1u;
      }
    }
    return;
  }
  // right-hand sides (T_f, D T_{L-f}) of member b at row k, member fastest,
  // loads issued in batches; rows n..ld-1 zero
  {
    constexpr int kU = 4;
    const int tot = KS * ld;
    for (int t0 = tid; t0 < tot; t0 += kU * kStrConsumers) {
      C v1[kU], v2[kU];
#pragma unroll
      for (int u = 0; u < kU; u++) {
        const int t = t0 + u * kStrConsumers;
        const int b = t % KS, k = t / KS;
        v1[u] = v2[u] = czero<C>();
        if (t < tot && b < km && k < n) {
          v1[u] = Tin[b * wstride + (long long)f * n + k];
          if (two) {
            v2[u] = Tin[b * wstride + (long long)i2 * n + k];
            if (k < MN) v2[u] = cscale(v2[u], (R)-1);
          }
        }
      }
#pragma unroll
      for (int u = 0; u < kU; u++) {
        const int t = t0 + u * kStrConsumers;
        if (t >= tot) continue;
        if constexpr (kPacked) {
          XA[t] = make_float4(v1[u].x, v2[u].x, v1[u].y, v2[u].y);
          XS[t] = make_float2(v1[u].x + v1[u].y, v2[u].x + v2[u].y);
        } else {
          C* dst = X + (size_t)2 * t;  // X[k * P + 2b], t = k * KS + b
          dst[0] = v1[u];
          dst[1] = v2[u];
        }
      }
    }
  }
  consumers_sync_or(0);
  const int r = 2 * tid;  // this thread's rows r, r + 1 (both < ld)
  const bool active = r < n;
  // complex64: sums [row][member]; complex128: accumulators [row][column]
  Sums3 q3[2][kPacked ? KS : 1];
  C a0[kPacked ? 1 : P], a1[kPacked ? 1 : P];
  if constexpr (kPacked) {
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
      for (int b = 0; b < KS; b++) q3[h][b].s1 = q3[h][b].s2 = q3[h][b].s3 = make_float2(0.f, 0.f);
  } else {
#pragma unroll
    for (int q = 0; q < P; q++) a0[q] = a1[q] = czero<C>();
  }
  int failed = 0;
  int k0 = 0;  // first block column of the stage
  int s = 0;
  unsigned ph = 0;
  for (int kb = 0; kb < nkb; kb++) {
    const bool ok = mbar_wait(&full[s], ph);
    failed |= !ok;
    if (ok && active) {
      const C* st = ring + (size_t)s * KC * ld + r;
#pragma unroll 2
      for (int c = 0; c < KC; c++) {
        C b0, b1;
        ld_pair(st + (size_t)c * ld, b0, b1);
        const int k = k0 + c;
        if constexpr (kPacked) {
          const float2 br[2] = {make_float2(b0.x, b0.x), make_float2(b1.x, b1.x)};
          const float2 bi[2] = {make_float2(b0.y, b0.y), make_float2(b1.y, b1.y)};
          const float2 bs[2] = {__fadd2_rn(br[0], bi[0]), __fadd2_rn(br[1], bi[1])};
          const float4* xa = XA + (size_t)k * KS;
          const float2* xs = XS + (size_t)k * KS;
#pragma unroll
          for (int b = 0; b < KS; b++) {
            const float4 a = xa[b];
            const float2 xr = make_float2(a.x, a.y), xi = make_float2(a.z, a.w), xsb = xs[b];
#pragma unroll
            for (int h = 0; h < 2; h++) {
              q3[h][b].s1 = __ffma2_rn(br[h], xr, q3[h][b].s1);
              q3[h][b].s2 = __ffma2_rn(bi[h], xi, q3[h][b].s2);
              q3[h][b].s3 = __ffma2_rn(bs[h], xsb, q3[h][b].s3);
            }
          }
        } else {
          const C* xc = X + (size_t)P * k;
#pragma unroll
          for (int q = 0; q < P; q++) {
            const C x = xc[q];
            cmac(a0[q], b0, x);
            cmac(a1[q], b1, x);
          }
        }
      }
    }
    __syncwarp();
    if ((tid & 31) == 0) mbar_arrive(&empty[s]);
    k0 += KC;
    if (++s == stages) {
      s = 0;
      ph ^= 1u;
    }
  }
  if (consumers_sync_or(failed) || !active) return;
#pragma unroll
  for (int q = 0; q < P; q++) {
    const int b = q >> 1;
    if (b >= km) continue;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int row = r + h;
      if (row >= n) continue;
      C v;
      if constexpr (kPacked) {
        const Sums3& t = q3[h][b];
        const float s1 = (q & 1) ? t.s1.y : t.s1.x, s2 = (q & 1) ? t.s2.y : t.s2.x,
                    s3 = (q & 1) ? t.s3.y : t.s3.x;
        v = make_float2(s1 - s2, (s3 - s1) - s2);
      } else {
        v = h ? a1[q] : a0[q];
      }
      if ((q & 1) == 0) {
        Tout[b * wstride + (long long)f * n + row] = v;
      } else if (two) {
        Tout[b * wstride + (long long)i2 * n + row] = (row < MN) ? cscale(v, (R)-1) : v;
      }
    }
  }
}

}  // namespace vox
