// Tall-skinny block products of the reduced-order model of a wavelength sweep
// (Bragg_MOR_script.m:113-142, example_Bragg_1500nm_to_1600nm.m:97-100):
//
//   C = X^H Y        Vtemp(:,j)'*v, P'*Qtemp{iG}, P'*Vrhs
//   Y = beta Y + X W v - h(j,n)*Vtemp(:,j), P*x_temp, the orthonormal basis
//
// X is n x a and Y n x b, interleaved complex128, column-major with column
// strides ldx / ldy; a, b <= kBlkCols.  Both are HBM-bound streams over the
// blocks: per row, a + b complex loads (and b stores for the update) against
// a * b complex FP64 multiply-adds.
#pragma once

#include "vox_common.cuh"

namespace vox {

constexpr int kBlkCols = 32;     // widest block (columns of X or Y)
constexpr int kBlkRows = 64;     // rows staged per tile
constexpr int kBlkThreads = 256;
constexpr int kBlkCtas = 296;    // two CTAs per SM on 148 SMs
constexpr int kBlkAcc = kBlkCols * kBlkCols / kBlkThreads;  // entries per thread

__host__ __device__ inline int blk_stride(int c) { return c | 1; }  // odd: no bank conflicts

__host__ inline size_t block_dot_smem(int a, int b) {
  return (size_t)kBlkRows * (blk_stride(a) + blk_stride(b)) * sizeof(double2);
}

// Per CTA: partial[cta][i * b + j] = sum over its row tiles of conj(X[r,i]) Y[r,j].
// Tile t of kBlkRows rows goes to CTA t % gridDim.x, and every CTA adds its
// tiles in increasing order, so the partial sums do not depend on timing.
__global__ void __launch_bounds__(kBlkThreads)
k_block_dot_partial(long long n, int a, int b, const double2* __restrict__ X, long long ldx,
                    const double2* __restrict__ Y, long long ldy, double2* __restrict__ partial) {
  extern __shared__ double2 bsm[];
  const int sa = blk_stride(a), sb = blk_stride(b);
  double2* xs = bsm;                    // [row][sa]
  double2* ys = bsm + kBlkRows * sa;    // [row][sb]
  const int tid = threadIdx.x;
  const int ab = a * b;
  double2 acc[kBlkAcc];
#pragma unroll
  for (int q = 0; q < kBlkAcc; q++) acc[q] = make_double2(0.0, 0.0);
  const long long tiles = (n + kBlkRows - 1) / kBlkRows;
  for (long long t = blockIdx.x; t < tiles; t += gridDim.x) {
    const long long r0 = t * kBlkRows;
    __syncthreads();
    for (int e = tid; e < kBlkRows * a; e += kBlkThreads) {
      const int r = e % kBlkRows, i = e / kBlkRows;
      xs[r * sa + i] = (r0 + r < n) ? X[r0 + r + i * ldx] : make_double2(0.0, 0.0);
    }
    for (int e = tid; e < kBlkRows * b; e += kBlkThreads) {
      const int r = e % kBlkRows, j = e / kBlkRows;
      ys[r * sb + j] = (r0 + r < n) ? Y[r0 + r + j * ldy] : make_double2(0.0, 0.0);
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kBlkAcc; q++) {
      const int e = tid + q * kBlkThreads;
      if (e < ab) {
        const int i = e / b, j = e % b;
        double2 s = acc[q];
        for (int r = 0; r < kBlkRows; r++) {
          const double2 x = xs[r * sa + i], y = ys[r * sb + j];
          s.x = fma(x.x, y.x, fma(x.y, y.y, s.x));
          s.y = fma(x.x, y.y, fma(-x.y, y.x, s.y));
        }
        acc[q] = s;
      }
    }
  }
#pragma unroll
  for (int q = 0; q < kBlkAcc; q++) {
    const int e = tid + q * kBlkThreads;
    if (e < ab) partial[(long long)blockIdx.x * ab + e] = acc[q];
  }
}

// C[i + a j] = sum over CTAs, in CTA order, of partial[cta][i * b + j].
__global__ void k_block_dot_reduce(int a, int b, int ctas, const double2* __restrict__ partial,
                                   double2* __restrict__ C) {
  const int ab = a * b;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ab; e += gridDim.x * blockDim.x) {
    double2 s = make_double2(0.0, 0.0);
    for (int c = 0; c < ctas; c++) {
      const double2 v = partial[(long long)c * ab + e];
      s.x += v.x;
      s.y += v.y;
    }
    const int i = e / b, j = e % b;
    C[i + a * j] = s;
  }
}

// Y[r, j] = beta Y[r, j] + sum_i X[r, i] W[i + a j]; one thread per row, W
// staged in shared memory.  beta == 0 does not read Y.
__global__ void __launch_bounds__(kBlkThreads)
k_block_update(long long n, int a, int b, const double2* __restrict__ X, long long ldx,
               const double2* __restrict__ W, double beta, double2* __restrict__ Y,
               long long ldy) {
  __shared__ double2 ws[kBlkCols * kBlkCols];
  for (int e = threadIdx.x; e < a * b; e += blockDim.x) ws[e] = W[e];
  __syncthreads();
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x) {
    double2 acc[kBlkCols];
#pragma unroll
    for (int j = 0; j < kBlkCols; j++) acc[j] = make_double2(0.0, 0.0);
    for (int i = 0; i < a; i++) {
      const double2 x = X[r + i * ldx];
#pragma unroll
      for (int j = 0; j < kBlkCols; j++) {
        if (j < b) {
          const double2 w = ws[i + a * j];
          acc[j].x = fma(x.x, w.x, fma(-x.y, w.y, acc[j].x));
          acc[j].y = fma(x.x, w.y, fma(x.y, w.x, acc[j].y));
        }
      }
    }
#pragma unroll
    for (int j = 0; j < kBlkCols; j++) {
      if (j < b) {
        double2 y = acc[j];
        if (beta != 0.0) {
          const double2 o = Y[r + j * ldy];
          y.x = fma(beta, o.x, y.x);
          y.y = fma(beta, o.y, y.y);
        }
        Y[r + j * ldy] = y;
      }
    }
  }
}

}  // namespace vox
