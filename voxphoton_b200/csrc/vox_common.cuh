// Common device/host helpers for libvox (B200, sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

namespace vox {

// Interleaved complex in the working precision: float2 (c64) or double2 (c128).
template <typename R> struct CplxOf;
template <> struct CplxOf<float> { using type = float2; };
template <> struct CplxOf<double> { using type = double2; };
template <typename R> using Cx = typename CplxOf<R>::type;

template <typename R> __host__ __device__ __forceinline__ Cx<R> mkc(R re, R im) {
  Cx<R> c;
  c.x = re;
  c.y = im;
  return c;
}
template <typename C> __host__ __device__ __forceinline__ C cadd(C a, C b) {
  C c;
  c.x = a.x + b.x;
  c.y = a.y + b.y;
  return c;
}
template <typename C> __host__ __device__ __forceinline__ C csub(C a, C b) {
  C c;
  c.x = a.x - b.x;
  c.y = a.y - b.y;
  return c;
}
template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
  C c;
  c.x = a.x * b.x - a.y * b.y;
  c.y = a.x * b.y + a.y * b.x;
  return c;
}
// conj(a) * b
template <typename C> __host__ __device__ __forceinline__ C cmulc(C a, C b) {
  C c;
  c.x = a.x * b.x + a.y * b.y;
  c.y = a.x * b.y - a.y * b.x;
  return c;
}
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) {
  a.y = -a.y;
  return a;
}
template <typename C, typename S> __host__ __device__ __forceinline__ C cscale(C a, S s) {
  a.x *= s;
  a.y *= s;
  return a;
}
// acc += a * b
template <typename C> __host__ __device__ __forceinline__ void cfma(C& acc, C a, C b) {
  acc.x += a.x * b.x - a.y * b.y;
  acc.y += a.x * b.y + a.y * b.x;
}
template <typename C> __host__ __device__ __forceinline__ C czero() {
  C c;
  c.x = 0;
  c.y = 0;
  return c;
}

__host__ __device__ __forceinline__ double2 to_d2(float2 a) { return make_double2(a.x, a.y); }
__host__ __device__ __forceinline__ double2 to_d2(double2 a) { return a; }
template <typename C> __host__ __device__ __forceinline__ C from_d2(double2 a);
template <> __host__ __device__ __forceinline__ float2 from_d2<float2>(double2 a) {
  return make_float2((float)a.x, (float)a.y);
}
template <> __host__ __device__ __forceinline__ double2 from_d2<double2>(double2 a) { return a; }

// Last CUDA/argument error text, per thread (vox_last_error()).
void set_error(const std::string& msg);
const char* last_error();

}  // namespace vox

#define VOX_CUDA(call)                                                              \
  do {                                                                              \
    cudaError_t e__ = (call);                                                       \
    if (e__ != cudaSuccess) {                                                       \
      vox::set_error(std::string(#call) + ": " + cudaGetErrorString(e__) + " at " + \
                     __FILE__ + ":" + std::to_string(__LINE__));                    \
      return VOX_CUDA_ERROR;                                                        \
    }                                                                               \
  } while (0)
