// Kernel 2 of the matvec for planes of Py = 64 and Pz = 24 (the Bragg
// gratings of the benchmark: M <= 32, N <= 12), without the block-wide
// Stockham sweeps of k_plane:
//
//   A  forward y-FFT of the 3N rows, one warp per row: lane l holds x[l] and
//      x[l+32]; one in-lane radix-2 step and five shuffle (radix-2 DIF) steps
//      across the warp leave X[2 br(l)] and X[2 br(l)+1] in lane l (br: 5-bit
//      reversal), which are kept in that order (bit-reversed, for 64 points);
//   B  per ky column and component: the z-FFT of 24 points (N nonzero) in
//      registers (8 x 3 Cooley-Tukey), written to shared memory; then per
//      (column, component) the 3x3 symmetric tensor product over the three
//      components' spectra and the inverse z-FFT in registers, cropped to N;
//   C  inverse y-FFT of the rows, one warp per row, five shuffle (radix-2 DIT)
//      steps on the bit-reversed input and one in-lane step, natural order
//      out, cropped to M.
// One CTA per (kx, member); three barriers per plane; the plane's octant of fN
// is staged in shared memory while the rows are transformed.  Arithmetic as
// k_plane (no scaling here: 1/P is applied by k_xinv).
#pragma once

#include "bulk.cuh"
#include "mvp.cuh"

namespace vox {

constexpr int kPlPy = 64;
constexpr int kPlPz = 24;
constexpr int kPlThreads = 256;
constexpr int kPlSy = kPlPy + 1;  // row stride of the y-transformed plane

__device__ __forceinline__ int brev5(int v) { return (int)(__brev((unsigned)v) >> 27); }

// the plane's octant of fN: (Py/2 + 1) x (Pz/2 + 1) x 6
constexpr int kPlFn = (kPlPy / 2 + 1) * (kPlPz / 2 + 1) * 6;
// rows one warp preloads in phases A and C (3N <= 36 rows over 8 warps)
constexpr int kPlRowsPerWarp = 5;

// shared memory: y-transformed rows [3N][65] + z spectra [3][64][24 + 1] + the
// plane's octant of fN (from a 16-byte boundary: it arrives by a bulk copy)
template <typename R>
constexpr size_t plane64_fn_offset(int N) {
  return (((size_t)3 * N * kPlSy + (size_t)3 * kPlPy * (kPlPz + 1)) * sizeof(Cx<R>) + 15) /
         16 * 16;
}
template <typename R>
constexpr size_t plane64_smem(int N) {
  return plane64_fn_offset<R>(N) + (size_t)kPlFn * sizeof(Cx<R>);
}

template <typename C>
__device__ __forceinline__ C shfl_x(C v, int m) {
  v.x = __shfl_xor_sync(0xffffffffu, v.x, m);
  v.y = __shfl_xor_sync(0xffffffffu, v.y, m);
  return v;
}

// 32-point DIF across the warp (natural in, bit-reversed out), forward or
// inverse by the twiddles tw[s] = W_{2h}^{l & (h-1)} of stage s (h = 16 >> s).
template <typename C>
__device__ __forceinline__ C warp_dif32(C x, const C (&tw)[5], int lane) {
#pragma unroll
  for (int s = 0; s < 5; s++) {
    const int h = 16 >> s;
    const C p = shfl_x(x, h);
    const bool top = (lane & h) == 0;
    // top: x + p ; bottom: (p - x) * w
    C t;
    t.x = top ? x.x + p.x : p.x - x.x;
    t.y = top ? x.y + p.y : p.y - x.y;
    x = top ? t : cmul(t, tw[s]);
  }
  return x;
}

// 32-point DIT across the warp (bit-reversed in, natural out), tw[s] =
// W_{2h}^{l & (h-1)} of stage s (h = 1 << s).
template <typename C>
__device__ __forceinline__ C warp_dit32(C x, const C (&tw)[5], int lane) {
#pragma unroll
  for (int s = 0; s < 5; s++) {
    const int h = 1 << s;
    const C p = shfl_x(x, h);
    const bool top = (lane & h) == 0;
    // top: x + w p ; bottom: p - w x
    const C wb = cmul(tw[s], top ? p : x);
    const C a = top ? x : p;
    C y;
    y.x = top ? a.x + wb.x : a.x - wb.x;
    y.y = top ? a.y + wb.y : a.y - wb.y;
    x = y;
  }
  return x;
}

// 24-point DFT in registers (24 = 8 x 3): out[k1 + 8 k2] from in[3 n1 + n2];
// inputs at n >= nin are zero, outputs at k >= nout are not formed.
template <typename C>
__device__ __forceinline__ void fft24_regs(const C (&in)[kPlPz], C (&out)[kPlPz], int nin,
                                           int nout, const C* __restrict__ tz, int sign) {
  C A[3][8];
#pragma unroll
  for (int n2 = 0; n2 < 3; n2++) {
    C v[8];
#pragma unroll
    for (int n1 = 0; n1 < 8; n1++) v[n1] = (3 * n1 + n2 < nin) ? in[3 * n1 + n2] : czero<C>();
    dft8(v, sign);
#pragma unroll
    for (int k1 = 0; k1 < 8; k1++) {
      // W24^{n2 k1}
      A[n2][k1] = (n2 == 0 || k1 == 0) ? v[k1] : cmul(v[k1], tw_get(tz, n2 * k1, sign));
    }
  }
#pragma unroll
  for (int k1 = 0; k1 < 8; k1++) {
    C u[3] = {A[0][k1], A[1][k1], A[2][k1]};
    dft3(u, sign);
#pragma unroll
    for (int k2 = 0; k2 < 3; k2++)
      if (k1 + 8 * k2 < nout) out[k1 + 8 * k2] = u[k2];
  }
}

template <typename R, int kMinBlocks>
__global__ void __launch_bounds__(kPlThreads, kMinBlocks)
    k_plane64(OpGeom g, const Cx<R>* __restrict__ twY, const Cx<R>* __restrict__ twZ,
              const Cx<R>* __restrict__ T1, const Cx<R>* __restrict__ fN, Cx<R>* __restrict__ T2,
              const int* skip, int fs) {
  using C = Cx<R>;
  const int mb = blockIdx.y;
  if (skip && skip[(long long)mb * fs]) return;
  T1 += mb * plane_elems(g);
  T2 += mb * plane_elems(g);
  fN += mb * fN_elems(g);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t fbar;
  const int N = g.N, M = g.M;
  const int rows = 3 * N;
  C* yb = reinterpret_cast<C*>(smem_raw);  // [3N][kPlSy], columns bit-reversed
  C* zb = yb + (size_t)rows * kPlSy;        // [3][64][25] z spectra
  C* fsm = reinterpret_cast<C*>(smem_raw + plane64_fn_offset<R>(N));  // the plane's fN octant
  const int kx = blockIdx.x;
  const C* tin = T1 + (long long)kx * rows * M;
  C* tout = T2 + (long long)kx * rows * M;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // fN is stored as one octant (the operator's parity holds: plane64_ok); the
  // plane's octant is contiguous (kPlFn values from a 16-byte boundary) and
  // arrives by one bulk copy while the rows are transformed
  const int fx = 2 * kx > g.Px;
  const int hy = g.Py / 2 + 1, hz = g.Pz / 2 + 1;
  if (tid == 0) {
    const C* fplane = fN + (long long)(fx ? g.Px - kx : kx) * hy * hz * 6;
    mbar_init(&fbar, 1);
    mbar_init_fence();
    mbar_arrive_expect_tx(&fbar, (unsigned)(kPlFn * sizeof(C)));
    bulk_g2s(fsm, fplane, (unsigned)(kPlFn * sizeof(C)), &fbar);
  }

  // ---- A: forward y-FFT, one warp per row (the warp's rows loaded first)
  {
    C tw[5];
#pragma unroll
    for (int s = 0; s < 5; s++) {
      const int h = 16 >> s;
      tw[s] = tw_get(twY, (lane & (h - 1)) * (32 / h), -1);  // W_{2h}^{j} = W64^{j*32/h}
    }
    const C w64 = tw_get(twY, lane, -1);
    C x0[kPlRowsPerWarp], x1[kPlRowsPerWarp];
#pragma unroll
    for (int i = 0; i < kPlRowsPerWarp; i++) {
      const int r = warp + i * (kPlThreads / 32);
      x0[i] = (r < rows && lane < M) ? tin[(long long)r * M + lane] : czero<C>();
      x1[i] = (r < rows && lane + 32 < M) ? tin[(long long)r * M + 32 + lane] : czero<C>();
    }
#pragma unroll
    for (int i = 0; i < kPlRowsPerWarp; i++) {
      const int r = warp + i * (kPlThreads / 32);
      if (r >= rows) break;
      C a = cadd(x0[i], x1[i]);
      C b = cmul(csub(x0[i], x1[i]), w64);
      a = warp_dif32(a, tw, lane);
      b = warp_dif32(b, tw, lane);
      // lane l: X[2 br(l)] (a) and X[2 br(l) + 1] (b): bit-reversed order of 64
      yb[(size_t)r * kPlSy + lane] = a;
      yb[(size_t)r * kPlSy + 32 + lane] = b;
    }
  }
  __syncthreads();

  // ---- B: z-FFT per (column, component), product, inverse z-FFT
  const int j = tid % kPlPy;  // physical column
  const int c = tid / kPlPy;  // component (threads 192..255 idle in B)
  const int ky = j < 32 ? 2 * brev5(j) : 2 * brev5(j - 32) + 1;
  if (c < 3) {
    C v[kPlPz], Z[kPlPz];
#pragma unroll
    for (int z = 0; z < kPlPz; z++)
      v[z] = z < N ? yb[(size_t)(c * N + z) * kPlSy + j] : czero<C>();
    fft24_regs(v, Z, N, kPlPz, twZ, -1);
    C* zr = zb + ((size_t)c * kPlPy + j) * (kPlPz + 1);
#pragma unroll
    for (int kz = 0; kz < kPlPz; kz++) zr[kz] = Z[kz];
  }
  // the fN octant has landed (bounded wait; every thread leaves if any gave up)
  if (__syncthreads_or(!mbar_wait(&fbar, 0))) return;
  if (c < 3) {
    const int fy = 2 * ky > g.Py;
    const int yo = fy ? g.Py - ky : ky;
    // row c of the symmetric tensor: components (c,0), (c,1), (c,2) of
    // [xx, xy, xz, yy, yz, zz]
    const int i0 = c == 0 ? 0 : (c == 1 ? 1 : 2);
    const int i1 = c == 0 ? 1 : (c == 1 ? 3 : 4);
    const int i2 = c == 0 ? 2 : (c == 1 ? 4 : 5);
    const C* z0 = zb + ((size_t)0 * kPlPy + j) * (kPlPz + 1);
    const C* z1 = zb + ((size_t)1 * kPlPy + j) * (kPlPz + 1);
    const C* z2 = zb + ((size_t)2 * kPlPy + j) * (kPlPz + 1);
    C P[kPlPz], y[kPlPz];
#pragma unroll
    for (int kz = 0; kz < kPlPz; kz++) {
      const int fz = 2 * kz > g.Pz;
      const C* f = fsm + (yo * hz + (fz ? g.Pz - kz : kz)) * 6;
      // octant parity: xy flips with fx^fy, xz with fx^fz, yz with fy^fz
      C f0 = f[i0], f1 = f[i1], f2 = f[i2];
      const R sxy = (fx ^ fy) ? (R)-1 : (R)1, sxz = (fx ^ fz) ? (R)-1 : (R)1,
              syz = (fy ^ fz) ? (R)-1 : (R)1;
      if (i0 == 1) f0 = cscale(f0, sxy);
      if (i0 == 2) f0 = cscale(f0, sxz);
      if (i1 == 1) f1 = cscale(f1, sxy);
      if (i1 == 4) f1 = cscale(f1, syz);
      if (i2 == 2) f2 = cscale(f2, sxz);
      if (i2 == 4) f2 = cscale(f2, syz);
      C o = cmul(f0, z0[kz]);
      cfma(o, f1, z1[kz]);
      cfma(o, f2, z2[kz]);
      P[kz] = o;
    }
    fft24_regs(P, y, kPlPz, N, twZ, +1);
#pragma unroll
    for (int z = 0; z < kPlPz; z++)
      if (z < N) yb[(size_t)(c * N + z) * kPlSy + j] = y[z];
  }
  __syncthreads();

  // ---- C: inverse y-FFT, one warp per row (bit-reversed in, natural out)
  {
    C tw[5];
#pragma unroll
    for (int s = 0; s < 5; s++) {
      const int h = 1 << s;
      tw[s] = tw_get(twY, (lane & (h - 1)) * (32 / h), +1);
    }
    const C w64 = tw_get(twY, lane, +1);
    for (int r = warp; r < rows; r += kPlThreads / 32) {
      // E = IDFT32 of the even-index spectrum, O of the odd-index one
      const C e = warp_dit32(yb[(size_t)r * kPlSy + lane], tw, lane);
      C o = warp_dit32(yb[(size_t)r * kPlSy + 32 + lane], tw, lane);
      o = cmul(o, w64);
      if (lane < M) tout[(long long)r * M + lane] = cadd(e, o);
      if (lane + 32 < M) tout[(long long)r * M + 32 + lane] = csub(e, o);
    }
  }
}

}  // namespace vox
