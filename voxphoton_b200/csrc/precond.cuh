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
// (y,z,c) line, per mode P*L*U solve (blocked triangular solves, one CTA per
// mode), inverse FFT along x (1/L), gather.  The apply reads each factor once:
// L*(3MN)^2 complex values, the same bytes as the reference's inverse-block GEMV.
// Caller-supplied inverse blocks (chan_mvp_idx's inv_blocks) are applied by a
// plain per-mode GEMV instead.
#pragma once

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

// --------------------------------------------------------------- apply: x-FFT
template <typename R>
__global__ void __launch_bounds__(256) k_pc_xfwd(PcGeom g, FftPlan pl, const Cx<R>* __restrict__ tw,
                                                 const Cx<R>* __restrict__ in,
                                                 const int* __restrict__ vmap,
                                                 Cx<R>* __restrict__ T, const int* skip) {
  using C = Cx<R>;
  if (skip && *skip) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + (size_t)g.ybx * g.sx;
  const int col0 = blockIdx.x * g.ybx;
  const int nl = min(g.ybx, g.n3 - col0);
  for (int t = threadIdx.x; t < g.ybx * g.L; t += blockDim.x) {
    const int l = t / g.L;
    const int x = t - l * g.L;
    C v = czero<C>();
    if (l < nl) {
      const int m = vmap[(long long)(col0 + l) * g.L + x];
      if (m >= 0) v = in[m];
    }
    bufA[(size_t)l * g.sx + x] = v;
  }
  __syncthreads();
  C* res = block_fft(bufA, bufB, pl, g.ybx, g.sx, tw, -1);
  for (int t = threadIdx.x; t < nl * g.L; t += blockDim.x) {
    const int i = t / nl;
    const int l = t - i * nl;
    T[(long long)i * g.n3 + col0 + l] = res[(size_t)l * g.sx + i];
  }
}

template <typename R>
__global__ void __launch_bounds__(256) k_pc_xinv(PcGeom g, FftPlan pl, const Cx<R>* __restrict__ tw,
                                                 const Cx<R>* __restrict__ T,
                                                 const int* __restrict__ vmap, R scale,
                                                 Cx<R>* out, const int* skip) {
  using C = Cx<R>;
  if (skip && *skip) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + (size_t)g.ybx * g.sx;
  const int col0 = blockIdx.x * g.ybx;
  const int nl = min(g.ybx, g.n3 - col0);
  for (int t = threadIdx.x; t < g.ybx * g.L; t += blockDim.x) {
    const int i = t / g.ybx;
    const int l = t - i * g.ybx;
    bufA[(size_t)l * g.sx + i] = (l < nl) ? T[(long long)i * g.n3 + col0 + l] : czero<C>();
  }
  __syncthreads();
  C* res = block_fft(bufA, bufB, pl, g.ybx, g.sx, tw, +1);
  for (int t = threadIdx.x; t < nl * g.L; t += blockDim.x) {
    const int l = t / g.L;
    const int x = t - l * g.L;
    const int m = vmap[(long long)(col0 + l) * g.L + x];
    if (m >= 0) out[m] = cscale(res[(size_t)l * g.sx + x], scale);
  }
}

// --------------------------------------------------------- apply: block GEMV
// T_i <- B_i T_i with B_i column-major n3 x n3 (explicit inverse blocks).
template <typename R>
__global__ void __launch_bounds__(256) k_pc_gemv(PcGeom g, const Cx<R>* __restrict__ B,
                                                 const Cx<R>* __restrict__ Tin,
                                                 Cx<R>* __restrict__ Tout, const int* skip) {
  using C = Cx<R>;
  if (skip && *skip) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* xs = reinterpret_cast<C*>(smem_raw);
  const int n3 = g.n3;
  const int tilesR = (n3 + blockDim.x - 1) / blockDim.x;
  const int i = blockIdx.x / tilesR;
  const int r = (blockIdx.x % tilesR) * blockDim.x + threadIdx.x;
  for (int c = threadIdx.x; c < n3; c += blockDim.x) xs[c] = Tin[(long long)i * n3 + c];
  __syncthreads();
  if (r >= n3) return;
  const C* Bi = B + (long long)i * n3 * n3;
  C acc0 = czero<C>(), acc1 = czero<C>();
  int c = 0;
  for (; c + 1 < n3; c += 2) {
    cfma(acc0, Bi[(long long)c * n3 + r], xs[c]);
    cfma(acc1, Bi[(long long)(c + 1) * n3 + r], xs[c + 1]);
  }
  if (c < n3) cfma(acc0, Bi[(long long)c * n3 + r], xs[c]);
  Tout[(long long)i * n3 + r] = cadd(acc0, acc1);
}

// ------------------------------------------------ apply: LU triangular solves
// One CTA per mode: t = P t; t = L^{-1} t (unit lower); t = U^{-1} t.
// Factors column-major in A (n3 x n3 per mode), pivots 0-based rows in piv.
template <typename R>
__global__ void __launch_bounds__(512) k_pc_lu_solve(PcGeom g, const Cx<R>* __restrict__ A,
                                                     const int* __restrict__ piv, Cx<R>* T,
                                                     const int* skip) {
  using C = Cx<R>;
  if (skip && *skip) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* t = reinterpret_cast<C*>(smem_raw);  // n3
  const int n = g.n3;
  const int i = blockIdx.x;
  const C* Ai = A + (long long)i * n * n;
  const int* pv = piv + (long long)i * n;
  C* Ti = T + (long long)i * n;
  for (int c = threadIdx.x; c < n; c += blockDim.x) t[c] = Ti[c];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < n; k++) {
      const int p = pv[k];
      if (p != k) {
        C a = t[k];
        t[k] = t[p];
        t[p] = a;
      }
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // forward substitution with unit lower L, blocks of kTrsvNb columns
  for (int k0 = 0; k0 < n; k0 += kTrsvNb) {
    const int kb = min(kTrsvNb, n - k0);
    if (warp == 0) {
      // solve the diagonal block: lane r holds t[k0+r]
      C v = (lane < kb) ? t[k0 + lane] : czero<C>();
      for (int j = 0; j < kb; j++) {
        C tj;
        tj.x = __shfl_sync(0xffffffffu, v.x, j);
        tj.y = __shfl_sync(0xffffffffu, v.y, j);
        if (lane > j && lane < kb) {
          const C l = Ai[(long long)(k0 + j) * n + k0 + lane];
          v.x -= l.x * tj.x - l.y * tj.y;
          v.y -= l.x * tj.y + l.y * tj.x;
        }
      }
      if (lane < kb) t[k0 + lane] = v;
    }
    __syncthreads();
    // update the rows below with the panel columns
    for (int r = k0 + kb + threadIdx.x; r < n; r += blockDim.x) {
      C acc = t[r];
      for (int j = 0; j < kb; j++) {
        const C l = Ai[(long long)(k0 + j) * n + r];
        const C tj = t[k0 + j];
        acc.x -= l.x * tj.x - l.y * tj.y;
        acc.y -= l.x * tj.y + l.y * tj.x;
      }
      t[r] = acc;
    }
    __syncthreads();
  }
  // back substitution with U, blocks from the bottom
  const int nblk = (n + kTrsvNb - 1) / kTrsvNb;
  for (int bk = nblk - 1; bk >= 0; bk--) {
    const int k0 = bk * kTrsvNb;
    const int kb = min(kTrsvNb, n - k0);
    if (warp == 0) {
      C v = (lane < kb) ? t[k0 + lane] : czero<C>();
      for (int j = kb - 1; j >= 0; j--) {
        // v_j /= U(j,j)
        if (lane == j) {
          const C d = Ai[(long long)(k0 + j) * n + k0 + j];
          const R dd = d.x * d.x + d.y * d.y;
          C q;
          q.x = (v.x * d.x + v.y * d.y) / dd;
          q.y = (v.y * d.x - v.x * d.y) / dd;
          v = q;
        }
        C tj;
        tj.x = __shfl_sync(0xffffffffu, v.x, j);
        tj.y = __shfl_sync(0xffffffffu, v.y, j);
        if (lane < j) {
          const C u = Ai[(long long)(k0 + j) * n + k0 + lane];
          v.x -= u.x * tj.x - u.y * tj.y;
          v.y -= u.x * tj.y + u.y * tj.x;
        }
      }
      if (lane < kb) t[k0 + lane] = v;
    }
    __syncthreads();
    for (int r = threadIdx.x; r < k0; r += blockDim.x) {
      C acc = t[r];
      for (int j = 0; j < kb; j++) {
        const C u = Ai[(long long)(k0 + j) * n + r];
        const C tj = t[k0 + j];
        acc.x -= u.x * tj.x - u.y * tj.y;
        acc.y -= u.x * tj.y + u.y * tj.x;
      }
      t[r] = acc;
    }
    __syncthreads();
  }
  for (int c = threadIdx.x; c < n; c += blockDim.x) Ti[c] = t[c];
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

// Dense block of mode i (column-major n3 x n3) from the x-transformed Chan
// circulants Cf [comp][z][y][x]; B = gram*I - face3 .* circ.
__global__ void k_assemble_blocks(int L, int M, int N, long long V, int i0, int nmodes, int ld,
                                  const double2* __restrict__ Cf, const double* __restrict__ face3,
                                  double gram, double2* __restrict__ B) {
  const int MN = M * N, n3 = 3 * MN;
  const long long per = (long long)n3 * n3;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nmodes * per;
       t += (long long)gridDim.x * blockDim.x) {
    const int im = (int)(t / per);
    const long long e = t - im * per;
    const int col = (int)(e / n3);
    const int row = (int)(e - (long long)col * n3);
    const int i = i0 + im;
    const int bp = row / MN, bq = col / MN;
    const int p = row - bp * MN, q = col - bq * MN;
    const int yp = p % M, zp = p / M, yq = q % M, zq = q / M;
    const int dy = yp > yq ? yp - yq : yq - yp;
    const int dz = zp > zq ? zp - zq : zq - zp;
    auto C = [&](int comp, int y, int z) -> double2 {
      return Cf[comp * V + i + (long long)L * (y + (long long)M * z)];
    };
    double2 v;
    const int b0 = bp < bq ? bp : bq, b1 = bp < bq ? bq : bp;
    if (b0 == 0 && b1 == 0) {
      v = C(0, dy, dz);
    } else if (b0 == 0 && b1 == 1) {
      // toeplitz([-CC(1) CC(2:M)], -CC(1:M)): y > y' -> CC, else -CC
      const double2 c = C(1, dy, dz);
      v = (yp > yq) ? c : make_double2(-c.x, -c.y);
    } else if (b0 == 0 && b1 == 2) {
      // -C3 symmetric, then triu antisymmetrised: p<q -> -C3, p>q -> +C3, p==q -> -C3
      const double2 c = C(2, dy, dz);
      v = (p > q) ? c : make_double2(-c.x, -c.y);
    } else if (b0 == 1 && b1 == 1) {
      v = C(3, dy, dz);
    } else if (b0 == 1 && b1 == 2) {
      // toeplitz([C5(1) -C5(2:M)], C5(1:M)) then triu symmetrised:
      // value of the upper entry (a<=b): y_a > y_b -> -C5, else C5
      const int a = p < q ? p : q, b = p < q ? q : p;
      const int ya = a % M, yb = b % M;
      const double2 c = C(4, dy, dz);
      v = (ya > yb) ? make_double2(-c.x, -c.y) : c;
    } else {
      v = C(5, dy, dz);
    }
    const double f = face3[row];
    double2 o = make_double2(-f * v.x, -f * v.y);
    if (row == col) o.x += gram;
    B[(long long)im * ld * ld + (long long)col * ld + row] = o;
  }
}

// Batched LU with partial pivoting, one CTA per matrix (column-major n x n).
// piv[k] = 0-based row swapped with row k at step k (LAPACK getrf order).
template <typename R>
__global__ void __launch_bounds__(512) k_lu_batched(int n, int ld, Cx<R>* A, int* piv, int* info) {
  using C = Cx<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
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

// One CTA per factored mode f.  With pairing, the CTA also solves mode L-f:
// B_{L-f} = D B_f D (D negates the x-component rows), so
// x_{L-f} = D (B_f^{-1} (D b_{L-f})) reuses the same factors - each factor
// element is read once for two right-hand sides.  Blocked forward/back
// substitution: x_blk = inv(diag block) * t_blk, then a rank-kTrsvNb update of
// the remaining rows (column-major factor panels, coalesced).
template <typename R>
__global__ void __launch_bounds__(512) k_pc_lu_solve2(PcGeom g, int paired,
                                                      const Cx<R>* __restrict__ A,
                                                      const Cx<R>* __restrict__ Dl,
                                                      const Cx<R>* __restrict__ Du,
                                                      const int* __restrict__ perm, Cx<R>* T,
                                                      const int* skip) {
  using C = Cx<R>;
  constexpr int B = kTrsvNb;
  if (skip && *skip) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = g.n3;
  const int MN = n / 3;
  const int nb = (n + B - 1) / B;
  const int npad = nb * B;  // right-hand sides padded with zeros to whole blocks
  C* t1 = reinterpret_cast<C*>(smem_raw);
  C* t2 = t1 + npad;
  __shared__ C xb1[B], xb2[B];
  const int f = blockIdx.x;
  const int i2 = g.L - f;
  const bool two = paired && f != 0 && i2 != f;
  const C* Af = A + (long long)f * n * n;
  const int* pm = perm + (long long)f * n;
  C* T1 = T + (long long)f * n;
  C* T2 = T + (long long)(two ? i2 : f) * n;
  const int tid = threadIdx.x;
  for (int k = tid; k < npad; k += blockDim.x) {
    C v1 = czero<C>(), v2 = czero<C>();
    if (k < n) {
      const int p = pm[k];
      v1 = T1[p];
      if (two) {
        v2 = T2[p];
        if (p < MN) v2 = cscale(v2, (R)-1);
      }
    }
    t1[k] = v1;
    t2[k] = v2;
  }
  __syncthreads();
  const C* DL = Dl + (long long)f * nb * B * B;
  const C* DU = Du + (long long)f * nb * B * B;
  // x_blk = inv(diag block) * t_blk (padded blocks are identity on zeros):
  // 32 independent loads per thread, fully unrolled.
  auto diag = [&](const C* Dblk, int k0) {
    if (tid < 2 * B) {
      const int q = tid & (B - 1), which = tid / B;
      if (which == 0 || two) {
        const C* tv = (which ? t2 : t1) + k0;
        const C* D = Dblk + q;
        C acc = czero<C>();
#pragma unroll
        for (int c = 0; c < B; c++) cfma(acc, __ldg(D + c * B), tv[c]);
        (which ? xb2 : xb1)[q] = acc;
      }
    }
    __syncthreads();
    if (tid < B) {
      t1[k0 + tid] = xb1[tid];
      if (two) t2[k0 + tid] = xb2[tid];
    }
  };
  // t[r] -= sum_j F[r, k0+j] x_j for rows r in [r0, r1): column-major panel,
  // coalesced across threads, 16 loads in flight per thread
  auto update = [&](int k0, int kb, int r0, int r1) {
    const C* col = Af + (long long)k0 * n;
    for (int r = r0 + tid; r < r1; r += blockDim.x) {
      C a1 = t1[r], a2 = t2[r];
      if (kb == B) {
#pragma unroll 16
        for (int j = 0; j < B; j++) {
          const C l = __ldg(col + (long long)j * n + r);
          const C x1 = xb1[j];
          a1.x -= l.x * x1.x - l.y * x1.y;
          a1.y -= l.x * x1.y + l.y * x1.x;
          if (two) {
            const C x2 = xb2[j];
            a2.x -= l.x * x2.x - l.y * x2.y;
            a2.y -= l.x * x2.y + l.y * x2.x;
          }
        }
      } else {
        for (int j = 0; j < kb; j++) {
          const C l = __ldg(col + (long long)j * n + r);
          const C x1 = xb1[j];
          a1.x -= l.x * x1.x - l.y * x1.y;
          a1.y -= l.x * x1.y + l.y * x1.x;
          if (two) {
            const C x2 = xb2[j];
            a2.x -= l.x * x2.x - l.y * x2.y;
            a2.y -= l.x * x2.y + l.y * x2.x;
          }
        }
      }
      t1[r] = a1;
      if (two) t2[r] = a2;
    }
    __syncthreads();
  };
  // forward substitution with the unit-lower L, then back substitution with U
  for (int bk = 0; bk < nb; bk++) {
    const int k0 = bk * B;
    diag(DL + (long long)bk * B * B, k0);
    update(k0, min(B, n - k0), k0 + B, n);
  }
  for (int bk = nb - 1; bk >= 0; bk--) {
    const int k0 = bk * B;
    diag(DU + (long long)bk * B * B, k0);
    update(k0, min(B, n - k0), 0, k0);
  }
  for (int k = tid; k < n; k += blockDim.x) {
    T1[k] = t1[k];
    if (two) T2[k] = (k < MN) ? cscale(t2[k], (R)-1) : t2[k];
  }
}

// ------------------------------------------ streamed LU solves (the apply)
// The factors are static, so their 32 x 32 tiles are streamed through a ring
// of shared-memory slots with cp.async, kRing-1 tiles in flight, in exactly
// the order the substitution consumes them; only the arithmetic waits on the
// dependency chain.  Tile order: forward [Dl(k), L(c,k) for c > k] for
// k = 0..nb-1, then backward [Du(k), U(c,k) for c < k] for k = nb-1..0.
// Factor storage is padded to ld = nb*32 (zero rows/columns), so every tile
// column is 32 contiguous, 16-byte aligned values.
constexpr int kTileLd = 36;  // smem column stride of a tile (bank-conflict free)

template <typename R> struct RingDepth;
// ring depth: 4 slots keep 3 tiles in flight and fit 4 CTAs (c64) per SM, so
// up to 592 factored modes run in a single wave on 148 SMs
template <> struct RingDepth<float> { static constexpr int value = 4; };
template <> struct RingDepth<double> { static constexpr int value = 3; };

template <typename R>
constexpr size_t lu_stream_smem(int npad) {
  return (size_t)RingDepth<R>::value * kTrsvNb * kTileLd * sizeof(Cx<R>) +
         2 * (size_t)npad * sizeof(Cx<R>);
}

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

template <typename R>
__global__ void __launch_bounds__(256) k_pc_lu_stream(PcGeom g, int paired,
                                                      const Cx<R>* __restrict__ tiles,
                                                      const int* __restrict__ perm, Cx<R>* T,
                                                      const int* skip) {
  using C = Cx<R>;
  constexpr int B = kTrsvNb;
  constexpr int S = RingDepth<R>::value;
  constexpr int SLOT = B * kTileLd;
  constexpr int PPC = B * (int)sizeof(C) / 16;  // 16-byte pieces per tile column
  if (skip && *skip) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* ring = reinterpret_cast<C*>(smem_raw);
  const int n = g.n3;
  const int MN = n / 3;
  const int nb = (n + B - 1) / B;
  const int npad = nb * B;
  C* t1 = ring + S * SLOT;
  C* t2 = t1 + npad;
  __shared__ C xb[2][B];
  const int f = blockIdx.x;
  const int i2 = g.L - f;
  const bool two = paired && f != 0 && i2 != f;
  const int total = lu_tiles(nb);
  const C* tf = tiles + (long long)f * total * B * B;  // this mode's tile stream
  const int* pm = perm + (long long)f * n;
  C* T1 = T + (long long)f * n;
  C* T2 = T + (long long)(two ? i2 : f) * n;
  const int tid = threadIdx.x;

  // tile i is 32*32 contiguous values: coalesced 16-byte pieces
  auto issue = [&](int i, C* slot) {
    const C* src = tf + (long long)i * B * B;
    constexpr int per = 16 / (int)sizeof(C);
    for (int p = tid; p < B * PPC; p += blockDim.x) {
      const int j = p / PPC, q = p - j * PPC;
      cp_async16(slot + j * kTileLd + q * per, src + j * B + q * per);
    }
  };

  // right-hand sides: t = P (D b) for the paired mode
  for (int k = tid; k < npad; k += blockDim.x) {
    C v1 = czero<C>(), v2 = czero<C>();
    if (k < n) {
      const int p = pm[k];
      v1 = T1[p];
      if (two) {
        v2 = T2[p];
        if (p < MN) v2 = cscale(v2, (R)-1);
      }
    }
    t1[k] = v1;
    t2[k] = v2;
  }

  TileIt cons{0, 0, -1};
  for (int s = 0; s < S - 1; s++) {
    if (s < total) issue(s, ring + s * SLOT);
    cp_async_commit();
  }
  // thread mapping for a tile: warp w -> right-hand side w>>2 and rows
  // (w&3)*8 + (lane&7); lane>>3 picks 8 of the 32 tile columns
  const int lane = tid & 31, w = tid >> 5;
  const int which = w >> 2;
  const int q = (w & 3) * 8 + (lane & 7);
  const int jp = lane >> 3;
  const bool active = which == 0 || two;
  C* tv = which ? t2 : t1;
  __syncthreads();
  for (int ci = 0; ci < total; ci++) {
    const int pi = ci + S - 1;
    if (pi < total) issue(pi, ring + (pi % S) * SLOT);
    cp_async_commit();
    cp_async_wait<S - 1>();
    __syncthreads();
    const C* tile = ring + (ci % S) * SLOT;
    const int k0 = cons.k * B;
    if (cons.c < 0) {
      // x_blk = inv(diag block) * t_blk
      C acc = czero<C>();
      if (active) {
#pragma unroll
        for (int jj = 0; jj < 8; jj++) {
          const int j = jj * 4 + jp;
          cfma(acc, tile[j * kTileLd + q], tv[k0 + j]);
        }
      }
      acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 8);
      acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 8);
      acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 16);
      acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 16);
      if (active && jp == 0) xb[which][q] = acc;
      __syncthreads();
      if (active && jp == 0) tv[k0 + q] = acc;
    } else {
      // t_rows(c) -= tile * x_blk
      C acc = czero<C>();
      if (active) {
#pragma unroll
        for (int jj = 0; jj < 8; jj++) {
          const int j = jj * 4 + jp;
          cfma(acc, tile[j * kTileLd + q], xb[which][j]);
        }
      }
      acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 8);
      acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 8);
      acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 16);
      acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 16);
      if (active && jp == 0) {
        const int r = cons.c * B + q;
        tv[r] = csub(tv[r], acc);
      }
    }
    tile_next(cons, nb);
    __syncthreads();
  }
  cp_async_wait<0>();
  for (int k = tid; k < n; k += blockDim.x) {
    T1[k] = t1[k];
    if (two) T2[k] = (k < MN) ? cscale(t2[k], (R)-1) : t2[k];
  }
}

// Cast LU factors to precision R, scaling the upper triangle (U, with the
// diagonal) of every n x n column-major block by s.
template <typename R>
__global__ void k_cast_scale_upper(long long tot, int n, const double2* __restrict__ src, double s,
                                   Cx<R>* dst) {
  const long long per = (long long)n * n;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot;
       i += (long long)gridDim.x * blockDim.x) {
    const long long e = i % per;
    const int col = (int)(e / n), row = (int)(e - (long long)col * n);
    const double f = row <= col ? s : 1.0;
    dst[i] = from_d2<Cx<R>>(make_double2(src[i].x * f, src[i].y * f));
  }
}

}  // namespace vox
