// FFT-circulant matvec of the JVIE-II operator, fused into three kernels.
//
//   y = Gram*Mr.*J - Mc.*crop(ifftn(sum_k fN_ck .* fftn(pad(J_k))))      (mv_AN_const.m:102-134)
//
// Layouts in HBM (all interleaved complex, R = float or double):
//   vector  : the unknowns at the support positions idx (length n), as in MATLAB JIn0
//   vmap    : int32 [3][N][M][L] (column-major grid, x fastest) -> vector slot or -1
//   T1, T2  : [Px][3][N][M]  one contiguous "plane" of 3*M*N values per x-frequency
//   fN      : [Px][Py][Pz][6] the six unique tensor components of each padded cell
// Px, Py, Pz are the padded lengths (>= 2L-1, 2M-1, 2N-1, 7-smooth), chosen at
// operator creation; the circulant embedding is exact for any such length.
// Every FFT of the matvec is 7-smooth, so its kernels compile only the
// radices 2, 3, 4, 5, 7 and 8 (block_fft<C, false, true>).
//
// Kernel 1 (k_xfwd):  per (z,c) and a tile of y: gather J pencils along x,
//                     zero-pad to Px, forward FFT along x, write T1 planes.
// Kernel 2 (k_plane): per kx plane: y-FFT (padded to Py) of the 3N rows, then for
//                     chunks of ky: z-FFT (padded to Pz), 3x3 symmetric tensor
//                     product with fN, inverse z-FFT cropped to N, then inverse
//                     y-FFT cropped to M; write T2.
// Kernel 3 (k_xinv):  per (z,c) and a tile of y: inverse x-FFT cropped to L,
//                     1/P scaling, contrast Gram*Mr*J - Mc*(.), scatter to the
//                     output vector.
#pragma once

#include "fft.cuh"

namespace vox {

struct OpGeom {
  int L, M, N;
  int Px, Py, Pz;
  long long V;    // L*M*N
  long long n;    // vector length
  // launch shapes (chosen on the host)
  int ybx;        // pencils per CTA in kernels 1/3
  int xthr;       // threads per CTA in kernels 1/3 (256 or 512)
  int pl3;        // complex64 k_plane64 at three CTAs per SM (80 registers)
  int sx;         // smem stride of an x pencil
  int sy, sz;     // smem strides of y rows / z columns in kernel 2
  int rc, kc;     // rows per chunk / ky columns per chunk in kernel 2
  int sym;        // fN stored as one octant (exact per-axis parity), else full
  int split;      // kernel 2 split in three (a plane does not fit in shared memory)
  int ry;         // split: rows per CTA of the y-FFT kernels
  int kcs;        // split: ky columns per CTA of the z kernel
};

enum MvMode { MV_AN = 0, MV_AN_T = 1, MV_L = 2 };

template <typename R>
struct OpBuffers {
  Cx<R>* fN = nullptr;   // [Px][Py][Pz][6]
  Cx<R>* Mr = nullptr;   // V, nullptr when Mr == 1 everywhere
  Cx<R>* Mc = nullptr;   // V
  Cx<R>* twX = nullptr;  // Px
  Cx<R>* twY = nullptr;  // Py
  Cx<R>* twZ = nullptr;  // Pz
  Cx<R>* T1 = nullptr;
  Cx<R>* T2 = nullptr;
  Cx<R>* TY = nullptr;   // split kernel 2: [Px][3N][Py] y-transformed planes
  OpGeom geo{};          // sizes and launch shapes for this precision
  R gram = 0;            // Gram in this precision's units
  R out_scale = 1;       // multiplies the matvec output (1 or Gram for the scaled c64 copy)
};

__host__ __device__ inline int pad_stride(int n) { return (n % 2 == 0) ? n + 1 : n; }

// Members of a batched operator (independent solves of one shape, launched
// together): member b's plane scratch and fN follow member 0's at the strides
// below; its input/output vectors are vs elements apart and its skip flag fs
// ints apart.  A single-member launch has b = 0 throughout.
__host__ __device__ inline long long plane_elems(const OpGeom& g) {
  return (long long)g.Px * 3 * g.N * g.M;
}
__host__ __device__ inline long long planey_elems(const OpGeom& g) {
  return (long long)g.Px * 3 * g.N * g.Py;
}
__host__ __device__ inline long long fN_elems(const OpGeom& g) {
  if (g.sym) return 6LL * (g.Px / 2 + 1) * (g.Py / 2 + 1) * (g.Pz / 2 + 1);
  return 6LL * g.Px * g.Py * g.Pz;
}

// ---------------------------------------------------------------- kernel 1
template <typename R>
__global__ void __launch_bounds__(512) k_xfwd(OpGeom g, FftPlan px, const Cx<R>* __restrict__ tw,
                                              const Cx<R>* __restrict__ in,
                                              const int* __restrict__ vmap,
                                              const Cx<R>* __restrict__ Mc, int mode,
                                              Cx<R>* __restrict__ T1, const int* skip,
                                              long long vs, int fs) {
  using C = Cx<R>;
  const int mb = blockIdx.z / 3;
  if (skip && skip[(long long)mb * fs]) return;
  in += mb * vs;
  T1 += mb * plane_elems(g);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + (size_t)g.ybx * g.sx;
  const int y0 = blockIdx.x * g.ybx;
  const int z = blockIdx.y;
  const int c = blockIdx.z - 3 * mb;
  const int YB = g.ybx;
  const long long cellbase = (long long)g.L * ((long long)g.M * z);
  // zero padding x in [L, Px) of the YB pencils
  const int npad = g.Px - g.L;
  for (int t = threadIdx.x; t < YB * npad; t += blockDim.x) {
    const int yb = t / npad;
    bufA[(size_t)yb * g.sx + g.L + (t - yb * npad)] = czero<C>();
  }
  // gather J along x (x < L) for YB pencils in batches of kGather elements per
  // thread: the index-map loads, then the vector loads, then the stores, so a
  // thread keeps its dependent global reads in flight together
  constexpr int kGather = sizeof(R) == 4 ? 12 : 6;
  const int tot = YB * g.L;
  const int* vm = vmap + (long long)c * g.V + cellbase;
  for (int t0 = threadIdx.x; t0 < tot; t0 += kGather * blockDim.x) {
    int mm[kGather];
#pragma unroll
    for (int u = 0; u < kGather; u++) {
      const int t = t0 + u * blockDim.x;
      const int yb = t / g.L;
      const int y = y0 + yb;
      mm[u] = (t < tot && y < g.M) ? vm[g.L * y + (t - yb * g.L)] : -1;
    }
    C v[kGather];
#pragma unroll
    for (int u = 0; u < kGather; u++) v[u] = mm[u] >= 0 ? in[mm[u]] : czero<C>();
#pragma unroll
    for (int u = 0; u < kGather; u++) {
      const int t = t0 + u * blockDim.x;
      if (t >= tot) break;
      const int yb = t / g.L;
      const int x = t - yb * g.L;
      C w = v[u];
      if (mode == MV_AN_T && mm[u] >= 0)
        w = cmul(Mc[cellbase + (long long)g.L * (y0 + yb) + x], cconj(w));  // conj(conj(Mc) .* J)
      bufA[(size_t)yb * g.sx + x] = w;
    }
  }
  __syncthreads();
  C* res = block_fft<C, false, true>(bufA, bufB, px, YB, g.sx, tw, -1);
  // write planes: T1[kx][c][z][y]
  const int ny = min(YB, g.M - y0);
  for (int t = threadIdx.x; t < YB * g.Px; t += blockDim.x) {
    const int kx = t / YB;
    const int yb = t - kx * YB;
    if (yb < ny) {
      T1[(((long long)kx * 3 + c) * g.N + z) * g.M + y0 + yb] = res[(size_t)yb * g.sx + kx];
    }
  }
}

// ---------------------------------------------------------------- kernel 2
// complex64: three CTAs per SM (80 registers); complex128: its own register need
template <typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 3 : 1)
    k_plane(OpGeom g, FftPlan py, FftPlan pz, const Cx<R>* __restrict__ twY,
            const Cx<R>* __restrict__ twZ, const Cx<R>* __restrict__ T1,
            const Cx<R>* __restrict__ fN, Cx<R>* __restrict__ T2, const int* skip, int fs) {
  using C = Cx<R>;
  const int mb = blockIdx.y;
  if (skip && skip[(long long)mb * fs]) return;
  T1 += mb * plane_elems(g);
  T2 += mb * plane_elems(g);
  fN += mb * fN_elems(g);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int rows = 3 * g.N;
  C* ybuf = reinterpret_cast<C*>(smem_raw);          // [3N][sy]
  C* wA = ybuf + (size_t)rows * g.sy;
  const int wsize = max(g.rc * g.sy, 3 * g.kc * g.sz);
  C* wB = wA + wsize;
  // the y and z twiddle tables, read by every butterfly, from shared memory
  C* tys = wB + wsize;
  C* tzs = tys + g.Py;
  for (int t = threadIdx.x; t < g.Py; t += blockDim.x) tys[t] = twY[t];
  for (int t = threadIdx.x; t < g.Pz; t += blockDim.x) tzs[t] = twZ[t];
  const int kx = blockIdx.x;
  const C* tin = T1 + (long long)kx * rows * g.M;
  C* tout = T2 + (long long)kx * rows * g.M;

  // Phase A: forward y-FFT of all 3N rows
  for (int r0 = 0; r0 < rows; r0 += g.rc) {
    const int nr = min(g.rc, rows - r0);
    for (int t = threadIdx.x; t < nr * g.Py; t += blockDim.x) {
      const int r = t / g.Py;
      const int y = t - r * g.Py;
      wA[(size_t)r * g.sy + y] = (y < g.M) ? tin[(long long)(r0 + r) * g.M + y] : czero<C>();
    }
    __syncthreads();
    C* res = block_fft<C, false, true>(wA, wB, py, nr, g.sy, tys, -1);
    for (int t = threadIdx.x; t < nr * g.Py; t += blockDim.x) {
      const int r = t / g.Py;
      const int y = t - r * g.Py;
      ybuf[(size_t)(r0 + r) * g.sy + y] = res[(size_t)r * g.sy + y];
    }
    __syncthreads();
  }

  // Phase B: per ky chunk, z-FFT, tensor product, inverse z-FFT (crop to N)
  // octant storage: fN(-k) = s fN(k) per axis, with s = -1 for xy (x, y),
  // xz (x, z) and yz (y, z); index the octant and flip those signs
  const int fx = g.sym && (2 * kx > g.Px);
  const int hy = g.sym ? g.Py / 2 + 1 : g.Py, hz = g.sym ? g.Pz / 2 + 1 : g.Pz;
  const C* fplane = fN + (long long)(fx ? g.Px - kx : kx) * hy * hz * 6;
  for (int k0 = 0; k0 < g.Py; k0 += g.kc) {
    const int nk = min(g.kc, g.Py - k0);
    // gather columns: seq (c*nk + j), element z
    for (int t = threadIdx.x; t < 3 * nk * g.Pz; t += blockDim.x) {
      const int s = t / g.Pz;
      const int zz = t - s * g.Pz;
      const int c = s / nk;
      const int j = s - c * nk;
      wA[(size_t)s * g.sz + zz] =
          (zz < g.N) ? ybuf[(size_t)(c * g.N + zz) * g.sy + k0 + j] : czero<C>();
    }
    __syncthreads();
    C* res = block_fft<C, false, true>(wA, wB, pz, 3 * nk, g.sz, tzs, -1);
    // tensor product (in place in res)
    for (int t = threadIdx.x; t < nk * g.Pz; t += blockDim.x) {
      const int j = t / g.Pz;
      const int kz = t - j * g.Pz;
      const int ky = k0 + j;
      const int fy = g.sym && (2 * ky > g.Py);
      const int fz = g.sym && (2 * kz > g.Pz);
      const C* f = fplane + ((long long)(fy ? g.Py - ky : ky) * hz + (fz ? g.Pz - kz : kz)) * 6;
      C f1 = f[1], f2 = f[2], f4 = f[4];
      const C f0 = f[0], f3 = f[3], f5 = f[5];
      if (fx ^ fy) f1 = cscale(f1, (R)-1);
      if (fx ^ fz) f2 = cscale(f2, (R)-1);
      if (fy ^ fz) f4 = cscale(f4, (R)-1);
      C* p0 = res + (size_t)(0 * nk + j) * g.sz + kz;
      C* p1 = res + (size_t)(1 * nk + j) * g.sz + kz;
      C* p2 = res + (size_t)(2 * nk + j) * g.sz + kz;
      const C a = *p0, b = *p1, cc = *p2;
      C o0 = cmul(f0, a), o1 = cmul(f1, a), o2 = cmul(f2, a);
      cfma(o0, f1, b);
      cfma(o1, f3, b);
      cfma(o2, f4, b);
      cfma(o0, f2, cc);
      cfma(o1, f4, cc);
      cfma(o2, f5, cc);
      *p0 = o0;
      *p1 = o1;
      *p2 = o2;
    }
    __syncthreads();
    C* other = (res == wA) ? wB : wA;
    C* res2 = block_fft<C, false, true>(res, other, pz, 3 * nk, g.sz, tzs, +1);
    for (int t = threadIdx.x; t < 3 * nk * g.N; t += blockDim.x) {
      const int s = t / g.N;
      const int zz = t - s * g.N;
      const int c = s / nk;
      const int j = s - c * nk;
      ybuf[(size_t)(c * g.N + zz) * g.sy + k0 + j] = res2[(size_t)s * g.sz + zz];
    }
    __syncthreads();
  }

  // Phase C: inverse y-FFT of the 3N rows, crop to M, write T2
  for (int r0 = 0; r0 < rows; r0 += g.rc) {
    const int nr = min(g.rc, rows - r0);
    for (int t = threadIdx.x; t < nr * g.Py; t += blockDim.x) {
      const int r = t / g.Py;
      const int y = t - r * g.Py;
      wA[(size_t)r * g.sy + y] = ybuf[(size_t)(r0 + r) * g.sy + y];
    }
    __syncthreads();
    C* res = block_fft<C, false, true>(wA, wB, py, nr, g.sy, tys, +1);
    for (int t = threadIdx.x; t < nr * g.M; t += blockDim.x) {
      const int r = t / g.M;
      const int y = t - r * g.M;
      tout[(long long)(r0 + r) * g.M + y] = res[(size_t)r * g.sy + y];
    }
    __syncthreads();
  }
}

// ------------------------------------------------- kernel 2, split form
// For planes of 3N rows x Py that do not fit in shared memory, kernel 2's
// three phases run as three kernels through TY [kx][row][ky] (per member):
// forward y-FFT of row chunks; per ky chunk the z-FFT, tensor product and
// inverse z-FFT (in place in TY); inverse y-FFT of row chunks cropped to M.
template <typename R>
__global__ void __launch_bounds__(256) k_ysplit_fwd(OpGeom g, FftPlan py,
                                                    const Cx<R>* __restrict__ twY,
                                                    const Cx<R>* __restrict__ T1,
                                                    Cx<R>* __restrict__ TY, const int* skip,
                                                    int fs) {
  using C = Cx<R>;
  const int mb = blockIdx.z;
  if (skip && skip[(long long)mb * fs]) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* wA = reinterpret_cast<C*>(smem_raw);
  C* wB = wA + (size_t)g.ry * g.sy;
  C* tys = wB + (size_t)g.ry * g.sy;
  for (int t = threadIdx.x; t < g.Py; t += blockDim.x) tys[t] = twY[t];
  const int rows = 3 * g.N;
  const int kx = blockIdx.x;
  const int r0 = blockIdx.y * g.ry;
  const int nr = min(g.ry, rows - r0);
  const C* tin = T1 + mb * plane_elems(g) + (long long)kx * rows * g.M;
  C* ty = TY + mb * planey_elems(g) + (long long)kx * rows * g.Py;
  for (int t = threadIdx.x; t < nr * g.Py; t += blockDim.x) {
    const int r = t / g.Py;
    const int y = t - r * g.Py;
    wA[(size_t)r * g.sy + y] = (y < g.M) ? tin[(long long)(r0 + r) * g.M + y] : czero<C>();
  }
  __syncthreads();
  C* res = block_fft<C, false, true>(wA, wB, py, nr, g.sy, tys, -1);
  for (int t = threadIdx.x; t < nr * g.Py; t += blockDim.x) {
    const int r = t / g.Py;
    const int y = t - r * g.Py;
    ty[(long long)(r0 + r) * g.Py + y] = res[(size_t)r * g.sy + y];
  }
}

template <typename R>
__global__ void __launch_bounds__(256) k_zsplit(OpGeom g, FftPlan pz,
                                                const Cx<R>* __restrict__ twZ,
                                                const Cx<R>* __restrict__ fN,
                                                Cx<R>* __restrict__ TY, const int* skip, int fs) {
  using C = Cx<R>;
  const int mb = blockIdx.z;
  if (skip && skip[(long long)mb * fs]) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* wA = reinterpret_cast<C*>(smem_raw);
  C* wB = wA + (size_t)3 * g.kcs * g.sz;
  C* tzs = wB + (size_t)3 * g.kcs * g.sz;
  for (int t = threadIdx.x; t < g.Pz; t += blockDim.x) tzs[t] = twZ[t];
  const int kx = blockIdx.x;
  const int k0 = blockIdx.y * g.kcs;
  const int nk = min(g.kcs, g.Py - k0);
  C* ty = TY + mb * planey_elems(g) + (long long)kx * 3 * g.N * g.Py;
  fN += mb * fN_elems(g);
  for (int t = threadIdx.x; t < 3 * nk * g.Pz; t += blockDim.x) {
    const int s = t / g.Pz;
    const int zz = t - s * g.Pz;
    const int c = s / nk;
    const int j = s - c * nk;
    wA[(size_t)s * g.sz + zz] =
        (zz < g.N) ? ty[(long long)(c * g.N + zz) * g.Py + k0 + j] : czero<C>();
  }
  __syncthreads();
  C* res = block_fft<C, false, true>(wA, wB, pz, 3 * nk, g.sz, tzs, -1);
  // tensor product (octant storage: see k_plane)
  const int fx = g.sym && (2 * kx > g.Px);
  const int hy = g.sym ? g.Py / 2 + 1 : g.Py, hz = g.sym ? g.Pz / 2 + 1 : g.Pz;
  const C* fplane = fN + (long long)(fx ? g.Px - kx : kx) * hy * hz * 6;
  for (int t = threadIdx.x; t < nk * g.Pz; t += blockDim.x) {
    const int j = t / g.Pz;
    const int kz = t - j * g.Pz;
    const int ky = k0 + j;
    const int fy = g.sym && (2 * ky > g.Py);
    const int fz = g.sym && (2 * kz > g.Pz);
    const C* f = fplane + ((long long)(fy ? g.Py - ky : ky) * hz + (fz ? g.Pz - kz : kz)) * 6;
    C f1 = f[1], f2 = f[2], f4 = f[4];
    const C f0 = f[0], f3 = f[3], f5 = f[5];
    if (fx ^ fy) f1 = cscale(f1, (R)-1);
    if (fx ^ fz) f2 = cscale(f2, (R)-1);
    if (fy ^ fz) f4 = cscale(f4, (R)-1);
    C* p0 = res + (size_t)(0 * nk + j) * g.sz + kz;
    C* p1 = res + (size_t)(1 * nk + j) * g.sz + kz;
    C* p2 = res + (size_t)(2 * nk + j) * g.sz + kz;
    const C a = *p0, b = *p1, cc = *p2;
    C o0 = cmul(f0, a), o1 = cmul(f1, a), o2 = cmul(f2, a);
    cfma(o0, f1, b);
    cfma(o1, f3, b);
    cfma(o2, f4, b);
    cfma(o0, f2, cc);
    cfma(o1, f4, cc);
    cfma(o2, f5, cc);
    *p0 = o0;
    *p1 = o1;
    *p2 = o2;
  }
  __syncthreads();
  C* other = (res == wA) ? wB : wA;
  C* res2 = block_fft<C, false, true>(res, other, pz, 3 * nk, g.sz, tzs, +1);
  for (int t = threadIdx.x; t < 3 * nk * g.N; t += blockDim.x) {
    const int s = t / g.N;
    const int zz = t - s * g.N;
    const int c = s / nk;
    const int j = s - c * nk;
    ty[(long long)(c * g.N + zz) * g.Py + k0 + j] = res2[(size_t)s * g.sz + zz];
  }
}

template <typename R>
__global__ void __launch_bounds__(256) k_ysplit_inv(OpGeom g, FftPlan py,
                                                    const Cx<R>* __restrict__ twY,
                                                    const Cx<R>* __restrict__ TY,
                                                    Cx<R>* __restrict__ T2, const int* skip,
                                                    int fs) {
  using C = Cx<R>;
  const int mb = blockIdx.z;
  if (skip && skip[(long long)mb * fs]) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* wA = reinterpret_cast<C*>(smem_raw);
  C* wB = wA + (size_t)g.ry * g.sy;
  C* tys = wB + (size_t)g.ry * g.sy;
  for (int t = threadIdx.x; t < g.Py; t += blockDim.x) tys[t] = twY[t];
  const int rows = 3 * g.N;
  const int kx = blockIdx.x;
  const int r0 = blockIdx.y * g.ry;
  const int nr = min(g.ry, rows - r0);
  const C* ty = TY + mb * planey_elems(g) + (long long)kx * rows * g.Py;
  C* tout = T2 + mb * plane_elems(g) + (long long)kx * rows * g.M;
  for (int t = threadIdx.x; t < nr * g.Py; t += blockDim.x) {
    const int r = t / g.Py;
    const int y = t - r * g.Py;
    wA[(size_t)r * g.sy + y] = ty[(long long)(r0 + r) * g.Py + y];
  }
  __syncthreads();
  C* res = block_fft<C, false, true>(wA, wB, py, nr, g.sy, tys, +1);
  for (int t = threadIdx.x; t < nr * g.M; t += blockDim.x) {
    const int r = t / g.M;
    const int y = t - r * g.M;
    tout[(long long)(r0 + r) * g.M + y] = res[(size_t)r * g.sy + y];
  }
}

// ---------------------------------------------------------------- kernel 3
template <typename R>
__global__ void __launch_bounds__(512) k_xinv(OpGeom g, FftPlan px, const Cx<R>* __restrict__ tw,
                                              const Cx<R>* __restrict__ T2,
                                              const int* __restrict__ vmap,
                                              const Cx<R>* in, const Cx<R>* __restrict__ Mr,
                                              const Cx<R>* __restrict__ Mc, R gram, R scale,
                                              R out_scale, int mode, Cx<R>* out,
                                              const int* skip, long long vs, int fs) {
  using C = Cx<R>;
  const int mb = blockIdx.z / 3;
  if (skip && skip[(long long)mb * fs]) return;
  T2 += mb * plane_elems(g);
  in += mb * vs;
  out += mb * vs;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + (size_t)g.ybx * g.sx;
  const int y0 = blockIdx.x * g.ybx;
  const int z = blockIdx.y;
  const int c = blockIdx.z - 3 * mb;
  const int YB = g.ybx;
  const int ny = min(YB, g.M - y0);
  // the pencils' values of every plane, kLoad loads in flight per thread
  // before their stores
  constexpr int kLoad = sizeof(R) == 4 ? 16 : 8;
  const int tot = YB * g.Px;
  for (int t0 = threadIdx.x; t0 < tot; t0 += kLoad * blockDim.x) {
    C v[kLoad];
#pragma unroll
    for (int u = 0; u < kLoad; u++) {
      const int t = t0 + u * blockDim.x;
      const int kx = t / YB;
      const int yb = t - kx * YB;
      v[u] = (t < tot && yb < ny) ? T2[(((long long)kx * 3 + c) * g.N + z) * g.M + y0 + yb]
                                  : czero<C>();
    }
#pragma unroll
    for (int u = 0; u < kLoad; u++) {
      const int t = t0 + u * blockDim.x;
      const int kx = t / YB;
      if (t < tot) bufA[(size_t)(t - kx * YB) * g.sx + kx] = v[u];
    }
  }
  __syncthreads();
  C* res = block_fft<C, false, true>(bufA, bufB, px, YB, g.sx, tw, +1);
  const long long cellbase = (long long)g.L * ((long long)g.M * z);
  // batches of kScatter elements per thread: index-map loads, then the
  // vector and contrast loads, then the combination and the stores
  constexpr int kScatter = sizeof(R) == 4 ? 8 : 4;
  for (int t0 = threadIdx.x; t0 < YB * g.L; t0 += kScatter * blockDim.x) {
    int mm[kScatter];
    long long cl[kScatter];
#pragma unroll
    for (int u = 0; u < kScatter; u++) {
      const int t = t0 + u * blockDim.x;
      const int yb = t / g.L;
      const int x = t - yb * g.L;
      mm[u] = -1;
      cl[u] = cellbase + (long long)g.L * (y0 + yb) + x;
      if (t < YB * g.L && yb < ny) mm[u] = vmap[(long long)c * g.V + cl[u]];
    }
    C J[kScatter], mc[kScatter];
#pragma unroll
    for (int u = 0; u < kScatter; u++) {
      J[u] = mm[u] >= 0 ? in[mm[u]] : czero<C>();
      mc[u] = (mm[u] >= 0 && mode == MV_AN) ? Mc[cl[u]] : czero<C>();
    }
#pragma unroll
    for (int u = 0; u < kScatter; u++) {
      if (mm[u] < 0) continue;
      const int t = t0 + u * blockDim.x;
      const int yb = t / g.L;
      const int x = t - yb * g.L;
      const long long cell = cl[u];
      const C nj = cscale(res[(size_t)yb * g.sx + x], scale);
      C o;
      if (mode == MV_AN) {
        C a = cscale(J[u], gram);
        if (Mr) a = cmul(Mr[cell], a);
        o = csub(a, cmul(mc[u], nj));
      } else if (mode == MV_AN_T) {
        C a = cscale(J[u], gram);
        if (Mr) a = cmul(cconj(Mr[cell]), a);
        o = csub(a, cconj(nj));
      } else {
        o = csub(nj, cscale(J[u], gram));
      }
      out[mm[u]] = cscale(o, out_scale);
    }
  }
}

// ------------------------------------------------------------ setup kernels
// Batched 1-D FFT of lines of a 3-D array (element (i0,i1,i2) at
// i0*s0 + i1*s1 + i2*s2 + comp*scomp) along `axis`; `lb` adjacent lines (in the
// other axis with the smaller stride, `axA`) per CTA for coalescing.
struct AxisDesc {
  int d[3];
  long long s[3];
  long long scomp;
  int axis, axA, axB;
  int lb;
  int sstride;
};

template <typename R>
__global__ void k_fft_axis(AxisDesc a, FftPlan p, const Cx<R>* __restrict__ tw, int sign,
                           Cx<R>* data) {
  using C = Cx<R>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  C* bufA = reinterpret_cast<C*>(smem_raw);
  C* bufB = bufA + (size_t)a.lb * a.sstride;
  const int nA = a.d[a.axA];
  const int tilesA = (nA + a.lb - 1) / a.lb;
  const int ia0 = (blockIdx.x % tilesA) * a.lb;
  const int ib = blockIdx.x / tilesA;
  const int comp = blockIdx.y;
  const int n = a.d[a.axis];
  const int nl = min(a.lb, nA - ia0);
  C* base = data + comp * a.scomp + (long long)ib * a.s[a.axB] + (long long)ia0 * a.s[a.axA];
  for (int t = threadIdx.x; t < nl * n; t += blockDim.x) {
    const int i = t / nl;
    const int l = t - i * nl;
    bufA[(size_t)l * a.sstride + i] = base[(long long)l * a.s[a.axA] + (long long)i * a.s[a.axis]];
  }
  __syncthreads();
  C* res = block_fft(bufA, bufB, p, nl, a.sstride, tw, sign);
  for (int t = threadIdx.x; t < nl * n; t += blockDim.x) {
    const int i = t / nl;
    const int l = t - i * nl;
    base[(long long)l * a.s[a.axA] + (long long)i * a.s[a.axis]] = res[(size_t)l * a.sstride + i];
  }
}

// Map a padded coordinate x' of the new grid (length P) to the offset d in
// (-n, n) it represents and from there to the coordinate of the source grid of
// length Q (Q = 2n for the MATLAB embedding, or n for a Toeplitz source with
// sign flips).  Returns -1 for the zero band.
__device__ __forceinline__ int embed_offset(int xp, int P, int n) {
  if (xp < n) return xp;
  if (xp > P - n) return xp - P;  // negative offset
  return INT_MIN;
}

// Build the padded circulant from the MATLAB-layout circulant Gp(2L,2M,2N,6)
// (column-major, already inverse-transformed): fill [comp][x'][y'][z'] (z fastest).
__global__ void k_embed_from_circ(OpGeom g, const double2* __restrict__ Gp, double2* out) {
  const long long P = (long long)g.Px * g.Py * g.Pz;
  const int L2 = 2 * g.L, M2 = 2 * g.M, N2 = 2 * g.N;
  const long long Q = (long long)L2 * M2 * N2;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 6 * P;
       t += (long long)gridDim.x * blockDim.x) {
    const int comp = (int)(t / P);
    long long r = t - comp * P;
    const int zp = (int)(r % g.Pz);
    r /= g.Pz;
    const int yp = (int)(r % g.Py);
    const int xp = (int)(r / g.Py);
    const int dx = embed_offset(xp, g.Px, g.L);
    const int dy = embed_offset(yp, g.Py, g.M);
    const int dz = embed_offset(zp, g.Pz, g.N);
    double2 v = make_double2(0.0, 0.0);
    if (dx != INT_MIN && dy != INT_MIN && dz != INT_MIN) {
      const int sx = (dx + L2) % L2, sy = (dy + M2) % M2, sz = (dz + N2) % N2;
      v = Gp[comp * Q + sx + (long long)L2 * (sy + (long long)M2 * sz)];
    }
    out[t] = v;
  }
}

// Build the padded circulant directly from the Toeplitz G_mn(L,M,N,6)
// (column-major), mirroring with the per-axis parity of each component
// (gperiodic_coeff_nop.m:4-31: 'L' [+ - - + + +], 'M' [+ - + + - +], 'N' [+ + - + - +];
// the two- and three-axis octants take the products of these signs).
__global__ void k_embed_from_toeplitz(OpGeom g, const double2* __restrict__ G, double2* out) {
  const long long P = (long long)g.Px * g.Py * g.Pz;
  const long long V = g.V;
  const int sL[6] = {1, -1, -1, 1, 1, 1};
  const int sM[6] = {1, -1, 1, 1, -1, 1};
  const int sN[6] = {1, 1, -1, 1, -1, 1};
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 6 * P;
       t += (long long)gridDim.x * blockDim.x) {
    const int comp = (int)(t / P);
    long long r = t - comp * P;
    const int zp = (int)(r % g.Pz);
    r /= g.Pz;
    const int yp = (int)(r % g.Py);
    const int xp = (int)(r / g.Py);
    const int dx = embed_offset(xp, g.Px, g.L);
    const int dy = embed_offset(yp, g.Py, g.M);
    const int dz = embed_offset(zp, g.Pz, g.N);
    double2 v = make_double2(0.0, 0.0);
    if (dx != INT_MIN && dy != INT_MIN && dz != INT_MIN) {
      int s = 1;
      if (dx < 0) s *= sL[comp];
      if (dy < 0) s *= sM[comp];
      if (dz < 0) s *= sN[comp];
      const int ax = dx < 0 ? -dx : dx, ay = dy < 0 ? -dy : dy, az = dz < 0 ? -dz : dz;
      v = G[comp * V + ax + (long long)g.L * (ay + (long long)g.M * az)];
      v.x *= s;
      v.y *= s;
    }
    out[t] = v;
  }
}

// Largest parity defect |F(k) - s F(-k)| and largest |F(k)| of the
// transformed circulant [comp][x][y][z] (as float bit patterns, atomicMax).
__global__ void k_sym_defect(OpGeom g, const double2* __restrict__ F, unsigned* out) {
  const long long P = (long long)g.Px * g.Py * g.Pz;
  const int sx[6] = {1, -1, -1, 1, 1, 1}, sy[6] = {1, -1, 1, 1, -1, 1}, sz[6] = {1, 1, -1, 1, -1, 1};
  float dmax = 0.f, fmax = 0.f;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 6 * P;
       t += (long long)gridDim.x * blockDim.x) {
    const int comp = (int)(t / P);
    long long r = t - comp * P;
    const int z = (int)(r % g.Pz);
    r /= g.Pz;
    const int y = (int)(r % g.Py), x = (int)(r / g.Py);
    const int mx = (g.Px - x) % g.Px, my = (g.Py - y) % g.Py, mz = (g.Pz - z) % g.Pz;
    const double s = (double)(sx[comp] * sy[comp] * sz[comp]);
    const double2 a = F[t];
    const double2 b = F[comp * P + ((long long)mx * g.Py + my) * g.Pz + mz];
    dmax = fmaxf(dmax, (float)(fabs(a.x - s * b.x) + fabs(a.y - s * b.y)));
    fmax = fmaxf(fmax, (float)(fabs(a.x) + fabs(a.y)));
  }
  atomicMax(out, __float_as_uint(dmax));
  atomicMax(out + 1, __float_as_uint(fmax));
}

// Octant pack: [comp][x][y][z] -> [x'][y'][z'][comp] for x' <= Px/2, y' <= Py/2,
// z' <= Pz/2, converting precision and scaling.
template <typename R>
__global__ void k_pack_fN_sym(OpGeom g, const double2* __restrict__ src, double scale,
                              Cx<R>* dst) {
  const long long P = (long long)g.Px * g.Py * g.Pz;
  const int hx = g.Px / 2 + 1, hy = g.Py / 2 + 1, hz = g.Pz / 2 + 1;
  const long long H = (long long)hx * hy * hz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 6 * H;
       t += (long long)gridDim.x * blockDim.x) {
    const long long pt = t / 6;
    const int comp = (int)(t - pt * 6);
    const int z = (int)(pt % hz);
    const long long r = pt / hz;
    const int y = (int)(r % hy), x = (int)(r / hy);
    double2 v = src[comp * P + ((long long)x * g.Py + y) * g.Pz + z];
    v.x *= scale;
    v.y *= scale;
    dst[t] = from_d2<Cx<R>>(v);
  }
}

// [comp][x][y][z] -> [x][y][z][comp], converting precision and scaling.
template <typename R>
__global__ void k_pack_fN(long long P, const double2* __restrict__ src, double scale,
                          Cx<R>* dst) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 6 * P;
       t += (long long)gridDim.x * blockDim.x) {
    const long long pt = t / 6;
    const int comp = (int)(t - pt * 6);
    double2 v = src[comp * P + pt];
    v.x *= scale;
    v.y *= scale;
    dst[t] = from_d2<Cx<R>>(v);
  }
}

}  // namespace vox
