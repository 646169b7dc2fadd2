// Hand-written mixed-radix FFT for B200: batches of short sequences held in
// shared memory, transformed by a Stockham autosort sweep (natural order in and
// out, ping-pong between two shared buffers, one __syncthreads per stage).
//
// Stage s with radix R and Ns = product of the earlier radices: butterfly j
// (0 <= j < n/R) reads src[j + r*n/R], multiplies input r by W_{Ns*R}^{r*(j%Ns)},
// runs a length-R DFT and writes dst[(j/Ns)*Ns*R + j%Ns + r*Ns].
// Radices 2, 3, 4, 5, 8 are hand-coded; 7, 11, 13 (and, where a kernel asks,
// the primes 17..37) use the paired cos/sin form with compile-time R; any other
// prime factor up to 64 runs a runtime-R butterfly.
//
// Twiddles come from one table per length n, W_n^m = exp(-2*pi*i*m/n), built on
// the host in double precision (the float path uses the rounded copy).
#pragma once

#include "vox_common.cuh"

namespace vox {

constexpr int kMaxStages = 24;
constexpr int kMaxGenericRadix = 64;

struct FftPlan {
  int n;
  int nst;
  int radix[kMaxStages];
};

// Host: factor n into supported radices.  Returns false if a prime factor
// exceeds kMaxGenericRadix.
inline bool make_fft_plan(int n, FftPlan* p) {
  p->n = n;
  p->nst = 0;
  if (n < 1) return false;
  int m = n;
  while (m % 8 == 0) { p->radix[p->nst++] = 8; m /= 8; }
  if (m % 4 == 0) { p->radix[p->nst++] = 4; m /= 4; }
  if (m % 2 == 0) { p->radix[p->nst++] = 2; m /= 2; }
  for (int r = 3; m > 1 && r <= kMaxGenericRadix; r += 2) {
    while (m % r == 0) {
      if (p->nst >= kMaxStages) return false;
      p->radix[p->nst++] = r;
      m /= r;
    }
  }
  return m == 1;
}

// Twiddle for exponent m (0 <= m < n) of the forward table, in direction sign.
template <typename C>
__device__ __forceinline__ C tw_get(const C* __restrict__ tw, int m, int sign) {
  C w = tw[m];
  if (sign > 0) w.y = -w.y;
  return w;
}

// multiply by sign*i
template <typename C> __device__ __forceinline__ C mul_si(C a, int sign) {
  C r;
  r.x = -sign * a.y;
  r.y = sign * a.x;
  return r;
}

template <typename C> __device__ __forceinline__ void dft2(C* v) {
  C a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <typename C> __device__ __forceinline__ void dft4(C* v, int sign) {
  C s0 = cadd(v[0], v[2]), d0 = csub(v[0], v[2]);
  C s1 = cadd(v[1], v[3]), d1 = mul_si(csub(v[1], v[3]), sign);
  v[0] = cadd(s0, s1);
  v[2] = csub(s0, s1);
  v[1] = cadd(d0, d1);
  v[3] = csub(d0, d1);
}

template <typename C> __device__ __forceinline__ void dft8(C* v, int sign) {
  using RT = decltype(v[0].x);
  const RT h = (RT)0.70710678118654752440084436210484903928;  // 1/sqrt(2)
  C e[4] = {v[0], v[2], v[4], v[6]};
  C o[4] = {v[1], v[3], v[5], v[7]};
  dft4(e, sign);
  dft4(o, sign);
  // W8^1 = (1 + s i)/sqrt2, W8^2 = s i, W8^3 = (-1 + s i)/sqrt2
  C t1, t3;
  t1.x = h * (o[1].x - sign * o[1].y);
  t1.y = h * (o[1].y + sign * o[1].x);
  C t2 = mul_si(o[2], sign);
  t3.x = h * (-o[3].x - sign * o[3].y);
  t3.y = h * (-o[3].y + sign * o[3].x);
  v[0] = cadd(e[0], o[0]);
  v[4] = csub(e[0], o[0]);
  v[1] = cadd(e[1], t1);
  v[5] = csub(e[1], t1);
  v[2] = cadd(e[2], t2);
  v[6] = csub(e[2], t2);
  v[3] = cadd(e[3], t3);
  v[7] = csub(e[3], t3);
}

template <typename C> __device__ __forceinline__ void dft3(C* v, int sign) {
  using RT = decltype(v[0].x);
  const RT c = (RT)0.86602540378443864676372317075293618347;  // sqrt(3)/2
  C a = v[0];
  C t = cadd(v[1], v[2]);
  C d = mul_si(csub(v[1], v[2]), sign);
  C m;
  m.x = a.x - (RT)0.5 * t.x;
  m.y = a.y - (RT)0.5 * t.y;
  v[0] = cadd(a, t);
  v[1] = cadd(m, cscale(d, c));
  v[2] = csub(m, cscale(d, c));
}

template <typename C> __device__ __forceinline__ void dft5(C* v, int sign) {
  using RT = decltype(v[0].x);
  const RT c1 = (RT)0.30901699437494742410229341718281905886;   // cos(2pi/5)
  const RT c2 = (RT)-0.80901699437494742410229341718281905886;  // cos(4pi/5)
  const RT s1 = (RT)0.95105651629515357211643933337938214340;   // sin(2pi/5)
  const RT s2 = (RT)0.58778525229247312916870595463907276860;   // sin(4pi/5)
  C a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
  C a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
  C x0 = v[0];
  C p1, p2, q1, q2;
  p1.x = x0.x + c1 * a1.x + c2 * a2.x;
  p1.y = x0.y + c1 * a1.y + c2 * a2.y;
  p2.x = x0.x + c2 * a1.x + c1 * a2.x;
  p2.y = x0.y + c2 * a1.y + c1 * a2.y;
  C u1, u2;
  u1.x = s1 * b1.x + s2 * b2.x;
  u1.y = s1 * b1.y + s2 * b2.y;
  u2.x = s2 * b1.x - s1 * b2.x;
  u2.y = s2 * b1.y - s1 * b2.y;
  q1 = mul_si(u1, sign);
  q2 = mul_si(u2, sign);
  v[0] = cadd(x0, cadd(a1, a2));
  v[1] = cadd(p1, q1);
  v[4] = csub(p1, q1);
  v[2] = cadd(p2, q2);
  v[3] = csub(p2, q2);
}

// Odd prime R, paired form: y_k = v0 + sum_j a_j cos(2pi jk/R) + s i sum_j b_j sin(2pi jk/R),
// a_j = v_j + v_{R-j}, b_j = v_j - v_{R-j}; y_{R-k} flips the sine part.
// cos/sin read from the length-n forward table: W_R^q = tw[q*(n/R)] = (cos, -sin).
template <int R, typename C>
__device__ __forceinline__ void dft_odd(C* v, int sign, const C* __restrict__ tw, int nOverR) {
  constexpr int H = (R - 1) / 2;
  C a[H], b[H];
#pragma unroll
  for (int j = 1; j <= H; j++) {
    a[j - 1] = cadd(v[j], v[R - j]);
    b[j - 1] = csub(v[j], v[R - j]);
  }
  C x0 = v[0];
  C y0 = x0;
#pragma unroll
  for (int j = 0; j < H; j++) y0 = cadd(y0, a[j]);
#pragma unroll
  for (int k = 1; k <= H; k++) {
    C p = x0, u = czero<C>();
#pragma unroll
    for (int j = 1; j <= H; j++) {
      C w = tw[((j * k) % R) * nOverR];
      // cos = w.x, sin = -w.y
      p.x += a[j - 1].x * w.x;
      p.y += a[j - 1].y * w.x;
      u.x -= b[j - 1].x * w.y;
      u.y -= b[j - 1].y * w.y;
    }
    C q = mul_si(u, sign);
    v[k] = cadd(p, q);
    v[R - k] = csub(p, q);
  }
  v[0] = y0;
}

// The same butterfly for the large primes (17..37), written straight to its
// destination out[q * os]: the sums a_j, b_j replace v_j, v_{R-j} in place, the
// H distinct cosines and sines are loaded once, and each output pair is formed
// and stored at once, so the stage holds about R complex values in registers.
template <int R, typename C>
__device__ __forceinline__ void dft_odd_store(C* v, int sign, const C* __restrict__ tw,
                                              int nOverR, C* out, int os) {
  constexpr int H = (R - 1) / 2;
  using RT = decltype(v[0].x);
  // cos and sin of 2 pi q / R (q = 1..H); the angle of pair (j, k) is
  // q = jk mod R, with cos(R - q) = cos q and sin(R - q) = -sin q
  RT cs[H], sn[H];
#pragma unroll
  for (int q = 1; q <= H; q++) {
    const C w = tw[q * nOverR];  // (cos, -sin)
    cs[q - 1] = w.x;
    sn[q - 1] = -w.y;
  }
  C y0 = v[0];
#pragma unroll
  for (int j = 1; j <= H; j++) {
    const C t = v[j];
    v[j] = cadd(t, v[R - j]);      // a_j
    v[R - j] = csub(t, v[R - j]);  // b_j
    y0 = cadd(y0, v[j]);
  }
#pragma unroll
  for (int k = 1; k <= H; k++) {
    C p = v[0], u = czero<C>();
#pragma unroll
    for (int j = 1; j <= H; j++) {
      const int q = (j * k) % R;
      const RT c = q <= H ? cs[q - 1] : cs[R - q - 1];
      const RT sq = q <= H ? sn[q - 1] : -sn[R - q - 1];
      p.x += v[j].x * c;
      p.y += v[j].y * c;
      u.x += v[R - j].x * sq;
      u.y += v[R - j].y * sq;
    }
    const C q = mul_si(u, sign);
    out[k * os] = cadd(p, q);
    out[(R - k) * os] = csub(p, q);
  }
  out[0] = y0;
}

template <int R, typename C>
__device__ __forceinline__ void dft_small(C* v, int sign, const C* __restrict__ tw, int nOverR) {
  if constexpr (R == 2) dft2(v);
  else if constexpr (R == 3) dft3(v, sign);
  else if constexpr (R == 4) dft4(v, sign);
  else if constexpr (R == 5) dft5(v, sign);
  else if constexpr (R == 8) dft8(v, sign);
  else dft_odd<R>(v, sign, tw, nOverR);
}

// One Stockham stage over nseq sequences (sequence b starts at b*sstride).
template <int R, typename C>
__device__ __forceinline__ void fft_stage(const C* __restrict__ src, C* __restrict__ dst, int n,
                                          int Ns, int nseq, int sstride, const C* __restrict__ tw,
                                          int sign, int tid, int nthr) {
  const int nR = n / R;
  const int total = nseq * nR;
  const int twstep = n / (Ns * R);
  // butterfly t = b*nR + j, j = jq*Ns + k: start from t = tid and advance by
  // nthr with carries, so the loop body has no integer division
  const int nq = nR / Ns;
  int b = tid / nR;
  const int j0 = tid - b * nR;
  int jq = j0 / Ns;
  int k = j0 - jq * Ns;
  const int db = nthr / nR;
  const int dj = nthr - db * nR;
  const int dq = dj / Ns;
  const int dk = dj - dq * Ns;
  for (int t = tid; t < total; t += nthr) {
    const int j = jq * Ns + k;
    const C* s = src + (size_t)b * sstride;
    C* d = dst + (size_t)b * sstride;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = s[j + r * nR];
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; r++) v[r] = cmul(v[r], tw_get(tw, r * k * twstep, sign));
    }
    const int idxD = jq * Ns * R + k;
    if constexpr (R > 13) {
      dft_odd_store<R>(v, sign, tw, nR, d + idxD, Ns);
    } else {
      dft_small<R>(v, sign, tw, nR);
#pragma unroll
      for (int r = 0; r < R; r++) d[idxD + r * Ns] = v[r];
    }
    k += dk;
    jq += dq;
    b += db;
    if (k >= Ns) {
      k -= Ns;
      jq++;
    }
    if (jq >= nq) {
      jq -= nq;
      b++;
    }
  }
}

// Runtime-radix stage for prime factors without a compiled butterfly (setup only).
template <typename C>
__device__ void fft_stage_generic(const C* __restrict__ src, C* __restrict__ dst, int n, int R,
                                  int Ns, int nseq, int sstride, const C* __restrict__ tw, int sign,
                                  int tid, int nthr) {
  const int nR = n / R;
  const int total = nseq * nR;
  const int twstep = n / (Ns * R);
  for (int t = tid; t < total; t += nthr) {
    const int b = t / nR;
    const int j = t - b * nR;
    const int k = j % Ns;
    const C* s = src + (size_t)b * sstride;
    C* d = dst + (size_t)b * sstride;
    C v[kMaxGenericRadix];
    for (int r = 0; r < R; r++) {
      v[r] = s[j + r * nR];
      if (Ns > 1 && r > 0) v[r] = cmul(v[r], tw_get(tw, r * k * twstep, sign));
    }
    const int idxD = (j / Ns) * Ns * R + k;
    for (int q = 0; q < R; q++) {
      C acc = czero<C>();
      for (int r = 0; r < R; r++) cfma(acc, v[r], tw_get(tw, ((r * q) % R) * nR, sign));
      d[idxD + q * Ns] = acc;
    }
  }
}

// Compiled butterflies for the primes 17..37 (paired cos/sin form, dft_odd_store).
template <typename C>
__device__ __forceinline__ bool big_prime_stage(int R, const C* __restrict__ src,
                                                C* __restrict__ dst, int n, int Ns, int nseq,
                                                int sstride, const C* __restrict__ tw, int sign,
                                                int tid, int nthr) {
  switch (R) {
    case 17: fft_stage<17>(src, dst, n, Ns, nseq, sstride, tw, sign, tid, nthr); return true;
    case 19: fft_stage<19>(src, dst, n, Ns, nseq, sstride, tw, sign, tid, nthr); return true;
    case 23: fft_stage<23>(src, dst, n, Ns, nseq, sstride, tw, sign, tid, nthr); return true;
    case 29: fft_stage<29>(src, dst, n, Ns, nseq, sstride, tw, sign, tid, nthr); return true;
    case 31: fft_stage<31>(src, dst, n, Ns, nseq, sstride, tw, sign, tid, nthr); return true;
    case 37: fft_stage<37>(src, dst, n, Ns, nseq, sstride, tw, sign, tid, nthr); return true;
    default: return false;
  }
}

// Transform nseq sequences of length p.n held in bufA (stride sstride) in
// place of ping-pong buffers bufA/bufB.  Returns the buffer holding the result.
// All threads of the block must call it; it ends with __syncthreads().
// kBigPrimes compiles butterflies for the primes 17..37 as well: lengths with
// such a factor (the preconditioner's x-FFT of length L, e.g. 1160 = 8*5*29 or
// 1480 = 8*5*37) then avoid the runtime-radix stage.  Kernels whose lengths
// are 7-smooth leave it off and keep their register budget; kSmooth7 compiles
// only the radices 2, 3, 4, 5, 7 and 8 (for lengths known to be 7-smooth, such
// as the matvec's padded lengths), which lowers the kernel's register need.
template <typename C, bool kBigPrimes = false, bool kSmooth7 = false>
__device__ C* block_fft(C* bufA, C* bufB, const FftPlan& p, int nseq, int sstride,
                        const C* __restrict__ tw, int sign) {
  C* src = bufA;
  C* dst = bufB;
  int Ns = 1;
  const int tid = threadIdx.x, nthr = blockDim.x;
  for (int s = 0; s < p.nst; s++) {
    const int R = p.radix[s];
    switch (R) {
      case 2: fft_stage<2>(src, dst, p.n, Ns, nseq, sstride, tw, sign, tid, nthr); break;
      case 3: fft_stage<3>(src, dst, p.n, Ns, nseq, sstride, tw, sign, tid, nthr); break;
      case 4: fft_stage<4>(src, dst, p.n, Ns, nseq, sstride, tw, sign, tid, nthr); break;
      case 5: fft_stage<5>(src, dst, p.n, Ns, nseq, sstride, tw, sign, tid, nthr); break;
      case 7: fft_stage<7>(src, dst, p.n, Ns, nseq, sstride, tw, sign, tid, nthr); break;
      case 8: fft_stage<8>(src, dst, p.n, Ns, nseq, sstride, tw, sign, tid, nthr); break;
      default:
        if constexpr (!kSmooth7) {
          if (R == 11) {
            fft_stage<11>(src, dst, p.n, Ns, nseq, sstride, tw, sign, tid, nthr);
            break;
          }
          if (R == 13) {
            fft_stage<13>(src, dst, p.n, Ns, nseq, sstride, tw, sign, tid, nthr);
            break;
          }
          if constexpr (kBigPrimes) {
            if (big_prime_stage(R, src, dst, p.n, Ns, nseq, sstride, tw, sign, tid, nthr)) break;
          }
          fft_stage_generic(src, dst, p.n, R, Ns, nseq, sstride, tw, sign, tid, nthr);
        }
        break;
    }
    __syncthreads();
    C* t = src;
    src = dst;
    dst = t;
    Ns *= R;
  }
  return src;
}

}  // namespace vox
