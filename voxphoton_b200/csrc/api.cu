// libvox C-ABI: operator handles, matvec entry points, device GMRES driver and
// the FP32 + FP64-refinement solver.  One translation unit holds all device
// code so constant tables and templates are instantiated once.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <type_traits>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/vox.h"
#include "bulk.cuh"
#include "krylov.cuh"
#include "mvp.cuh"
#include "plane.cuh"
#include "precond.cuh"
#include "block.cuh"
#include "cubature.cuh"

namespace vox {

static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }
const char* last_error() { return g_err.c_str(); }

// ------------------------------------------------------------ size choice
// Cost (in complex-add units per point) of one Stockham stage of radix r.
static double stage_cost(int r) {
  switch (r) {
    case 2: return 2.0;
    case 3: return 2.7;
    case 4: return 2.5;
    case 5: return 3.2;
    case 7: return 4.5;
    case 8: return 3.0;
    default: return 1.0 + 0.5 * r;
  }
}

static bool smooth7(int n) {
  for (int p : {2, 3, 5, 7})
    while (n % p == 0) n /= p;
  return n == 1;
}

static double fft_cost(int n) {
  FftPlan p;
  if (!make_fft_plan(n, &p)) return 1e300;
  double c = 0;
  for (int s = 0; s < p.nst; s++) c += stage_cost(p.radix[s]);
  return c * n;
}

// Padded length for a Toeplitz axis of length n: the cheapest 7-smooth size
// in [2n-1, 1.15*(2n-1)+8].
static int choose_pad(int n) {
  const int lo = std::max(1, 2 * n - 1);
  const int hi = (int)(lo * 1.15) + 8;
  int best = -1;
  double bc = 1e300;
  for (int p = lo; p <= hi; p++) {
    if (!smooth7(p)) continue;
    const double c = fft_cost(p);
    if (c < bc) {
      bc = c;
      best = p;
    }
  }
  return best;
}

// Forward twiddle table W_n^m = exp(-2 pi i m / n), m in [0, n).
static std::vector<double2> twiddles(int n) {
  std::vector<double2> w(n);
  for (int m = 0; m < n; m++) {
    // reduce the angle to the first octant for accuracy
    const long long num = (long long)m;
    const double a = 2.0 * M_PI * (double)num / (double)n;
    w[m] = make_double2(std::cos(a), -std::sin(a));
  }
  // exact values at the quarter points
  for (int m = 0; m < n; m++) {
    if ((4LL * m) % n == 0) {
      const int q = (int)((4LL * m) / n);
      const double c[4] = {1, 0, -1, 0}, s[4] = {0, 1, 0, -1};
      w[m] = make_double2(c[q], -s[q]);
    }
  }
  return w;
}

// Device bytes held by the library, per device: every device allocation goes
// through dalloc and every release through dfree, so a caller can measure what
// an object (an operator, a lane) holds apart from the CUDA context, the loaded
// modules and other libraries' pools (vox_mem_in_use).
constexpr int kMemDevices = 64;
static std::mutex g_mem_mu;
static std::map<void*, std::pair<int, size_t>> g_mem_blocks;
static long long g_mem_bytes[kMemDevices];

static cudaError_t dfree(void* p) {
  if (!p) return cudaSuccess;
  {
    std::lock_guard<std::mutex> lk(g_mem_mu);
    auto it = g_mem_blocks.find(p);
    if (it != g_mem_blocks.end()) {
      g_mem_bytes[it->second.first] -= (long long)it->second.second;
      g_mem_blocks.erase(it);
    }
  }
  return cudaFree(p);
}

template <typename T>
static vox_status dalloc(T** p, size_t count) {
  *p = nullptr;
  if (count == 0) return VOX_OK;
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error(std::string("cudaMalloc of ") + std::to_string(count * sizeof(T)) +
              " bytes failed: " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? VOX_ERR_OOM : VOX_ERR_CUDA;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= kMemDevices) dev = 0;
  std::lock_guard<std::mutex> lk(g_mem_mu);
  g_mem_blocks[(void*)*p] = {dev, count * sizeof(T)};
  g_mem_bytes[dev] += (long long)(count * sizeof(T));
  return VOX_OK;
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

#define VOX_TRY(x)                  \
  do {                              \
    vox_status s__ = (x);           \
    if (s__ != VOX_OK) return s__;  \
  } while (0)

// ------------------------------------------------------------ bounded waits
// Every host wait on the device polls the stream against a deadline instead of
// blocking in cudaStreamSynchronize: a wait that outlasts the limit returns
// VOX_ERR_TIMEOUT (the work stays queued and the context stays usable; the
// caller decides whether to wait again or tear down).  The limit is
// process-wide: VOX_WAIT_TIMEOUT_S in the environment, or vox_set_wait_timeout.
static std::atomic<double> g_wait_limit_s{-1.0};

static double wait_limit_s() {
  double v = g_wait_limit_s.load();
  if (v > 0) return v;
  const char* e = std::getenv("VOX_WAIT_TIMEOUT_S");
  v = (e && std::atof(e) > 0) ? std::atof(e) : 600.0;
  g_wait_limit_s.store(v);
  return v;
}

// The module's kernel error word (a bounded in-kernel wait gave up), read
// after the stream it was left on has drained; cleared once reported.
static vox_status kernel_err_status(cudaStream_t st) {
  // a device-to-pageable copy returns once it has landed (the stream is idle)
  int h = 0;
  VOX_CUDA(cudaMemcpyFromSymbolAsync(&h, g_kernel_err, sizeof(int), 0, cudaMemcpyDeviceToHost,
                                     st));
  if (h != 0) {
    const int zero = 0;
    VOX_CUDA(cudaMemcpyToSymbolAsync(g_kernel_err, &zero, sizeof(int), 0,
                                     cudaMemcpyHostToDevice, st));
    set_error("a kernel's bounded pipeline wait gave up (error word " + std::to_string(h) +
              "); its results are invalid");
    return VOX_ERR_TIMEOUT;
  }
  return VOX_OK;
}

static vox_status wait_stream(cudaStream_t st) {
  const double lim = wait_limit_s();
  const auto t0 = std::chrono::steady_clock::now();
  for (int spin = 0;; spin++) {
    const cudaError_t e = cudaStreamQuery(st);
    if (e == cudaSuccess) return kernel_err_status(st);
    if (e != cudaErrorNotReady) {
      cudaGetLastError();
      set_error(std::string("stream wait: ") + cudaGetErrorString(e));
      return VOX_ERR_CUDA;
    }
    const double dt =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (dt > lim) {
      set_error("device work did not finish within the wait limit of " + std::to_string(lim) +
                " s (VOX_WAIT_TIMEOUT_S / vox_set_wait_timeout); it is still queued");
      return VOX_ERR_TIMEOUT;
    }
    // spin briefly (short restart cycles), then back off to a light poll
    if (spin > 64) std::this_thread::sleep_for(std::chrono::microseconds(spin < 2000 ? 20 : 200));
  }
}

// The same for one recorded event.
static vox_status wait_event(cudaEvent_t ev) {
  const double lim = wait_limit_s();
  const auto t0 = std::chrono::steady_clock::now();
  for (int spin = 0;; spin++) {
    const cudaError_t e = cudaEventQuery(ev);
    if (e == cudaSuccess) return VOX_OK;
    if (e != cudaErrorNotReady) {
      cudaGetLastError();
      set_error(std::string("event wait: ") + cudaGetErrorString(e));
      return VOX_ERR_CUDA;
    }
    const double dt =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (dt > lim) {
      set_error("device work did not finish within the wait limit of " + std::to_string(lim) +
                " s; it is still queued");
      return VOX_ERR_TIMEOUT;
    }
    if (spin > 64) std::this_thread::sleep_for(std::chrono::microseconds(spin < 2000 ? 20 : 200));
  }
}

// Bytes of a GmresDev record read back per cycle (everything before sn).
constexpr size_t kGmresHdr = (offsetof(GmresDev, sn) + 15) / 16 * 16;

// GMRES workspace for one precision and restart length, for every member of
// the operator.  Member b's vectors form one arena, vs elements after member
// 0's: [V (m+1 columns) | w | t | r | x | b | c], each column ldv elements long
// (c: the column the next out-of-phase step multiplies, step mode).
template <typename R>
struct GmresWork {
  int m = 0;
  int K = 0;
  long long ldv = 0;        // column length (n rounded up to 32)
  long long vs = 0;         // member stride = (m + 7) * ldv
  Cx<R>* arena = nullptr;
  Cx<R>* V = nullptr;       // member 0's pointers into the arena
  Cx<R>* w = nullptr;
  Cx<R>* t = nullptr;       // preconditioner output / right-precond temp
  Cx<R>* r = nullptr;
  Cx<R>* x = nullptr;
  Cx<R>* b = nullptr;
  Cx<R>* c = nullptr;       // step mode: each member's current basis column
  GmresDev* st = nullptr;   // K records
  unsigned char* hst = nullptr;  // pinned: K headers of kGmresHdr bytes
  int* hflag = nullptr;          // pinned: K frozen flags
  double* hscal = nullptr;       // pinned: K scalars
  int* hsel = nullptr;           // pinned: K skip flags (right_finish)
  int* dsel = nullptr;           // device copy of hsel
  // (precond, side, members launched [+ 1000 x steps in step mode]) -> captured
  // cycle or step sequence
  std::map<std::tuple<void*, int, int>, cudaGraphExec_t> graphs;
  GmresDev* hdr(int mb) { return reinterpret_cast<GmresDev*>(hst + (size_t)mb * kGmresHdr); }
  template <typename T> T* mem(T* p, int mb) const { return p + mb * vs; }
  void release() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    graphs.clear();
    dfree(arena);
    dfree(st);
    if (hst) cudaFreeHost(hst);
    if (hflag) cudaFreeHost(hflag);
    if (hscal) cudaFreeHost(hscal);
    if (hsel) cudaFreeHost(hsel);
    dfree(dsel);
    arena = V = w = t = r = x = b = c = nullptr;
    st = nullptr;
    hst = nullptr;
    hflag = nullptr;
    hscal = nullptr;
    hsel = nullptr;
    dsel = nullptr;
    m = 0;
  }
};

// members of one operator: the streamed LU solve takes up to 16 columns
constexpr int kMaxMembers = 8;

// int stride between the skip flags of consecutive members (GmresDev::done)
constexpr int kFlagStride = (int)(sizeof(GmresDev) / sizeof(int));
static_assert(sizeof(GmresDev) % sizeof(int) == 0, "GmresDev size");

}  // namespace vox

using namespace vox;

struct vox_lane_s;

struct vox_op_s {
  int device = 0;
  int K = 1;                          // members (independent solves of this shape)
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;  // created here; `stream` may be the caller's
  long long launches = 0;             // kernels launched by solver entry points
  std::map<cudaGraphExec_t, int> graph_nodes;
  OpGeom g{};
  FftPlan px{}, py{}, pz{};
  int* vmap = nullptr;
  bool has_d = false, has_f = false;
  OpBuffers<double> d;
  OpBuffers<float> f;
  double gram = 0;
  // host staging (pinned) and device vectors for host-buffer entry points
  // (K vectors of n for d_in/d_out and the host buffers)
  double2* h_in = nullptr;
  double2* h_out = nullptr;
  double2* d_in = nullptr;
  double2* d_out = nullptr;
  float2* f_in = nullptr;
  float2* f_out = nullptr;
  GmresWork<double> wd;
  GmresWork<float> wf;
  std::vector<vox_precond_s*> pcs;
  std::vector<vox_lane_s*> lanes;  // continuous-batching lanes on this operator
};

namespace vox {

template <typename R> OpBuffers<R>& bufs(vox_op_s* op);
template <> OpBuffers<double>& bufs<double>(vox_op_s* op) { return op->d; }
template <> OpBuffers<float>& bufs<float>(vox_op_s* op) { return op->f; }
template <typename R> GmresWork<R>& work(vox_op_s* op);
template <> GmresWork<double>& work<double>(vox_op_s* op) { return op->wd; }
template <> GmresWork<float>& work<float>(vox_op_s* op) { return op->wf; }

static size_t xsmem(const OpGeom& g, size_t csz) { return 2ull * g.ybx * g.sx * csz; }
// k_plane: the plane's y-transformed rows, two work buffers, the y and z twiddles
static size_t psmem(const OpGeom& g, size_t csz) {
  const size_t wsize = std::max((size_t)g.rc * g.sy, (size_t)3 * g.kc * g.sz);
  return ((size_t)3 * g.N * g.sy + 2 * wsize + g.Py + g.Pz) * csz;
}
// split form: ry rows (k_ysplit_*) or 3 kcs columns (k_zsplit), ping-pong, twiddles
static size_t ysmem(const OpGeom& g, size_t csz) {
  return (2ull * g.ry * g.sy + g.Py) * csz;
}
static size_t zsmem(const OpGeom& g, size_t csz) {
  return (2ull * 3 * g.kcs * g.sz + g.Pz) * csz;
}

// Members taking part in one launch: km members starting at m0 (their fN
// and plane scratch), vectors vs elements apart, skip flags fs ints apart.
struct Members {
  int km = 1;
  int m0 = 0;
  long long vs = 0;
  int fs = 0;
};

// Every launch shape is checked against kSmemCap before use.  The attribute
// below is a property of the kernel (per device), not of one operator, so it
// is always raised to this one fixed cap: operators and preconditioners of
// different sizes then coexist, and setting it from several host threads is
// idempotent.
static const int kSmemCap = 220 * 1024;

// Kernel 2 of the matvec for km members: the register/shuffle plane kernel
// when the padded plane is 64 x 24 (the Bragg gratings), the split kernels
// when a plane does not fit in shared memory, else the general k_plane.
template <typename R>
static bool plane64_ok(const OpGeom& g) {
  return !g.split && g.sym && g.Py == kPlPy && g.Pz == kPlPz && g.M <= kPlPy &&
         3 * g.N <= kPlRowsPerWarp * (kPlThreads / 32) && plane64_smem<R>(g.N) <= (size_t)kSmemCap;
}

template <typename R>
static void launch_plane(vox_op_s* op, const OpBuffers<R>& b, const Cx<R>* T1, const Cx<R>* fN,
                         Cx<R>* T2, Cx<R>* TY, int km, const int* skip, int fs, cudaStream_t st) {
  const OpGeom& g = b.geo;
  const size_t cs = sizeof(Cx<R>);
  if (g.split) {
    const int rows = 3 * g.N;
    const dim3 gy(g.Px, (rows + g.ry - 1) / g.ry, km);
    const dim3 gz(g.Px, (g.Py + g.kcs - 1) / g.kcs, km);
    const size_t ysm = ysmem(g, cs), zsm = zsmem(g, cs);
    k_ysplit_fwd<R><<<gy, 256, ysm, st>>>(g, op->py, b.twY, T1, TY, skip, fs);
    k_zsplit<R><<<gz, 256, zsm, st>>>(g, op->pz, b.twZ, fN, TY, skip, fs);
    k_ysplit_inv<R><<<gy, 256, ysm, st>>>(g, op->py, b.twY, TY, T2, skip, fs);
  } else if (plane64_ok<R>(g)) {
    if (sizeof(R) == 4 && g.pl3)
      k_plane64<R, 3><<<dim3(g.Px, km), kPlThreads, plane64_smem<R>(g.N), st>>>(
          g, b.twY, b.twZ, T1, fN, T2, skip, fs);
    else
      k_plane64<R, 2><<<dim3(g.Px, km), kPlThreads, plane64_smem<R>(g.N), st>>>(
          g, b.twY, b.twZ, T1, fN, T2, skip, fs);
  } else {
    k_plane<R><<<dim3(g.Px, km), 256, psmem(g, cs), st>>>(g, op->py, op->pz, b.twY, b.twZ, T1,
                                                           fN, T2, skip, fs);
  }
}

// Plane intermediates supplied by the caller instead of the operator's own
// (one member, unsplit kernel 2 only: vox_mv_AN_noalloc).
template <typename R>
struct PlaneScratch {
  Cx<R>* T1 = nullptr;
  Cx<R>* T2 = nullptr;
};

// Launch the three matvec kernels.
template <typename R>
static vox_status matvec(vox_op_s* op, int mode, const Cx<R>* in, Cx<R>* out, cudaStream_t st,
                         const int* skip, Members mm = Members(),
                         PlaneScratch<R> scratch = PlaneScratch<R>()) {
  OpBuffers<R>& b = bufs<R>(op);
  const OpGeom& g = b.geo;
  const size_t cs = sizeof(Cx<R>);
  dim3 gx((g.M + g.ybx - 1) / g.ybx, g.N, 3 * mm.km);
  const R scale = (R)(1.0 / ((double)g.Px * g.Py * g.Pz));
  if (scratch.T1 && (mm.km != 1 || g.split)) {
    set_error("matvec: caller scratch serves one member of an unsplit operator");
    return VOX_ERR_BAD_ARG;
  }
  Cx<R>* T1 = scratch.T1 ? scratch.T1 : b.T1 + mm.m0 * plane_elems(g);
  Cx<R>* T2 = scratch.T2 ? scratch.T2 : b.T2 + mm.m0 * plane_elems(g);
  const Cx<R>* fN = b.fN + mm.m0 * fN_elems(g);
  k_xfwd<R><<<gx, g.xthr, xsmem(g, cs), st>>>(g, op->px, b.twX, in, op->vmap, b.Mc, mode, T1, skip,
                                            mm.vs, mm.fs);
  launch_plane<R>(op, b, T1, fN, T2, g.split ? b.TY + mm.m0 * planey_elems(g) : nullptr, mm.km,
                  skip, mm.fs, st);
  k_xinv<R><<<gx, g.xthr, xsmem(g, cs), st>>>(g, op->px, b.twX, T2, op->vmap, in, b.Mr, b.Mc,
                                            b.gram, scale, b.out_scale, mode, out, skip, mm.vs,
                                            mm.fs);
  VOX_CUDA(cudaGetLastError());
  return VOX_OK;
}


template <typename K>
static vox_status smem_cap(K* kernel) {
  VOX_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemCap));
  return VOX_OK;
}

template <typename R>
static vox_status set_smem_attrs() {
  VOX_TRY(smem_cap(k_xfwd<R>));
  VOX_TRY(smem_cap(k_xinv<R>));
  VOX_TRY(smem_cap(k_plane<R>));
  VOX_TRY(smem_cap(k_ysplit_fwd<R>));
  VOX_TRY(smem_cap(k_zsplit<R>));
  VOX_TRY(smem_cap(k_ysplit_inv<R>));
  VOX_TRY(smem_cap(k_plane64<R, 2>));
  VOX_TRY(smem_cap(k_plane64<R, 3>));
  VOX_TRY(smem_cap(k_gs_pass<R, false>));
  VOX_TRY(smem_cap(k_gs_pass<R, true>));
  return VOX_OK;
}

static const size_t kSmemBudget = 110 * 1024;  // two CTAs per SM
// k_plane in complex64: three CTAs per SM (at most 80 registers a thread, its
// launch bounds), which measured faster than two CTAs of 110 KB
static const size_t kPlaneBudget = 72 * 1024;

// Pick launch shapes for precision of size csz; returns false if a plane
// cannot be staged in shared memory.
static bool pick_shapes(OpGeom& g, size_t csz) {
  g.sx = pad_stride(g.Px);
  g.sy = pad_stride(g.Py);
  g.sz = pad_stride(g.Pz);
  int yb = (int)(kSmemBudget / (2ull * g.sx * csz));
  if (yb < 1) {
    if (2ull * g.sx * csz > (size_t)kSmemCap) return false;
    yb = 1;
  }
  g.ybx = std::max(1, std::min({yb, 8, g.M}));
  g.xthr = 256;
  // complex64 k_plane64 at three CTAs per SM (80 registers, measured 12% faster
  // than two CTAs of 113 registers on the 1160 x 30 x 11 grating)
  g.pl3 = csz == sizeof(float2) ? 1 : 0;
  if (csz == sizeof(float2)) {
    // tuning overrides (complex64): pencils per x-kernel CTA, its threads, and
    // the plane kernel's CTAs per SM
    if (const char* e = std::getenv("VOX_XK_YB")) {
      const int v = std::atoi(e);
      if (v >= 1 && v <= 8 && 2ull * v * g.sx * csz <= (size_t)kSmemCap) g.ybx = std::min(v, g.M);
    }
    if (const char* e = std::getenv("VOX_XK_THREADS")) {
      const int v = std::atoi(e);
      if (v == 256 || v == 512) g.xthr = v;
    }
    if (const char* e = std::getenv("VOX_PL_MINB")) g.pl3 = std::atoi(e) != 2;
  }
  // kernel 2: try all rows and all ky columns, then shrink the chunks
  const int rows = 3 * g.N;
  g.rc = rows;
  g.kc = g.Py;
  auto fits = [&](size_t budget) { return psmem(g, csz) <= budget; };
  const size_t pbudget = csz == sizeof(float2) ? kPlaneBudget : kSmemBudget;
  while (!fits(pbudget) && (g.kc > 1 || g.rc > 1)) {
    if ((size_t)3 * g.kc * g.sz >= (size_t)g.rc * g.sy && g.kc > 1)
      g.kc = (g.kc + 1) / 2;
    else if (g.rc > 1)
      g.rc = (g.rc + 1) / 2;
    else
      g.kc = (g.kc + 1) / 2;
  }
  g.split = 0;
  if (fits(kSmemCap)) return true;
  // the 3N y-transformed rows of a plane do not fit: split kernel 2 in three
  g.split = 1;
  const size_t rowb = 2ull * g.sy * csz, colb = 2ull * 3 * g.sz * csz;
  const size_t twy = (size_t)g.Py * csz, twz = (size_t)g.Pz * csz;
  if (rowb + twy > (size_t)kSmemCap || colb + twz > (size_t)kSmemCap) return false;
  g.ry = (int)std::max<size_t>(
      1, std::min<size_t>(rows, (kSmemBudget - std::min(kSmemBudget, twy)) / rowb));
  g.kcs = (int)std::max<size_t>(
      1, std::min<size_t>(g.Py, (kSmemBudget - std::min(kSmemBudget, twz)) / colb));
  return true;
}

// In-place batched FFT of a 3-D array along one axis (setup path).
static vox_status fft_axis_d(double2* data, int d0, int d1, int d2, long long s0, long long s1,
                             long long s2, long long scomp, int ncomp, int axis, int sign,
                             cudaStream_t st) {
  AxisDesc a;
  a.d[0] = d0;
  a.d[1] = d1;
  a.d[2] = d2;
  a.s[0] = s0;
  a.s[1] = s1;
  a.s[2] = s2;
  a.scomp = scomp;
  a.axis = axis;
  int o1 = (axis + 1) % 3, o2 = (axis + 2) % 3;
  if (a.s[o1] <= a.s[o2]) {
    a.axA = o1;
    a.axB = o2;
  } else {
    a.axA = o2;
    a.axB = o1;
  }
  const int n = a.d[axis];
  FftPlan p;
  if (!make_fft_plan(n, &p)) {
    set_error("FFT length " + std::to_string(n) + " has a prime factor above 64");
    return VOX_ERR_UNSUPPORTED;
  }
  a.sstride = pad_stride(n);
  const size_t per = 2ull * a.sstride * sizeof(double2);
  int lb = (a.s[axis] == 1) ? 1 : (int)std::min<size_t>(8, std::max<size_t>(1, 96 * 1024 / per));
  lb = std::min(lb, a.d[a.axA]);
  a.lb = lb;
  const size_t smem = (size_t)lb * per;
  if (smem > (size_t)kSmemCap) {
    set_error("FFT length " + std::to_string(n) + " too long for the setup kernel");
    return VOX_ERR_UNSUPPORTED;
  }
  std::vector<double2> tw = twiddles(n);
  double2* dtw;
  VOX_TRY(dalloc(&dtw, n));
  VOX_CUDA(cudaMemcpyAsync(dtw, tw.data(), n * sizeof(double2), cudaMemcpyHostToDevice, st));
  VOX_TRY(smem_cap(k_fft_axis<double>));
  const int tilesA = (a.d[a.axA] + lb - 1) / lb;
  dim3 grid(tilesA * a.d[a.axB], ncomp);
  k_fft_axis<double><<<grid, 256, smem, st>>>(a, p, dtw, sign, data);
  VOX_CUDA(cudaGetLastError());
  VOX_TRY(wait_stream(st));
  dfree(dtw);
  return VOX_OK;
}

template <typename R>
__global__ void k_to_prec(long long n, const double2* __restrict__ src, double s, Cx<R>* dst) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    dst[i] = from_d2<Cx<R>>(make_double2(src[i].x * s, src[i].y * s));
}

static int nblk(long long n, int t = 256) {
  long long b = (n + t - 1) / t;
  return (int)std::min<long long>(std::max<long long>(b, 1), 148LL * 16);
}

template <typename R>
static vox_status upload_precision(vox_op_s* op, const double2* fN_packed_src /*[comp][P]*/,
                                   const std::vector<double2>& Mr, bool has_Mr,
                                   const std::vector<double2>& Mc, double scale) {
  OpBuffers<R>& b = bufs<R>(op);
  const OpGeom& g = b.geo;
  const long long P = (long long)g.Px * g.Py * g.Pz;
  cudaStream_t st = op->stream;
  const long long fe = fN_elems(g);
  VOX_TRY(dalloc(&b.fN, fe * op->K));
  if (g.sym) {
    k_pack_fN_sym<R><<<nblk(fe), 256, 0, st>>>(g, fN_packed_src, scale, b.fN);
  } else {
    k_pack_fN<R><<<nblk(fe), 256, 0, st>>>(P, fN_packed_src, scale, b.fN);
  }
  VOX_CUDA(cudaGetLastError());
  // every member starts as a copy of member 0
  for (int mb = 1; mb < op->K; mb++)
    VOX_CUDA(cudaMemcpyAsync(b.fN + mb * fe, b.fN, fe * sizeof(Cx<R>), cudaMemcpyDeviceToDevice,
                             st));
  double2* tmp;
  VOX_TRY(dalloc(&tmp, g.V));
  if (has_Mr) {
    VOX_TRY(dalloc(&b.Mr, g.V));
    VOX_CUDA(cudaMemcpyAsync(tmp, Mr.data(), g.V * sizeof(double2), cudaMemcpyHostToDevice, st));
    k_to_prec<R><<<nblk(g.V), 256, 0, st>>>(g.V, tmp, 1.0, b.Mr);
  }
  VOX_TRY(dalloc(&b.Mc, g.V));
  VOX_CUDA(cudaMemcpyAsync(tmp, Mc.data(), g.V * sizeof(double2), cudaMemcpyHostToDevice, st));
  k_to_prec<R><<<nblk(g.V), 256, 0, st>>>(g.V, tmp, 1.0, b.Mc);
  VOX_TRY(wait_stream(st));
  dfree(tmp);
  auto up_tw = [&](int n, Cx<R>** dst) -> vox_status {
    std::vector<double2> w = twiddles(n);
    std::vector<Cx<R>> wc(n);
    for (int i = 0; i < n; i++) wc[i] = from_d2<Cx<R>>(w[i]);
    VOX_TRY(dalloc(dst, n));
    VOX_CUDA(cudaMemcpyAsync(*dst, wc.data(), n * sizeof(Cx<R>), cudaMemcpyHostToDevice,
                             st));
    return VOX_OK;
  };
  VOX_TRY(up_tw(g.Px, &b.twX));
  VOX_TRY(up_tw(g.Py, &b.twY));
  VOX_TRY(up_tw(g.Pz, &b.twZ));
  const long long tsz = plane_elems(g);
  VOX_TRY(dalloc(&b.T1, tsz * op->K));
  VOX_TRY(dalloc(&b.T2, tsz * op->K));
  if (g.split) VOX_TRY(dalloc(&b.TY, planey_elems(g) * op->K));
  VOX_TRY(set_smem_attrs<R>());
  return VOX_OK;
}

template <typename R>
static void free_bufs(OpBuffers<R>& b) {
  dfree(b.fN);
  dfree(b.Mr);
  dfree(b.Mc);
  dfree(b.twX);
  dfree(b.twY);
  dfree(b.twZ);
  dfree(b.T1);
  dfree(b.T2);
  dfree(b.TY);
  b = OpBuffers<R>();
}

static void pc_release(vox_precond_s* p);
static void lanes_release(vox_op_s* op);

static void destroy_op(vox_op_s* op) {
  if (!op) return;
  DeviceGuard dg(op->device);
  // teardown waits without a limit: freeing memory under queued kernels would
  // fault the context
  cudaDeviceSynchronize();
  // lanes and preconditioners use the operator's state: they go with it
  lanes_release(op);
  // preconditioners hold the operator's index map: they go with it
  std::vector<vox_precond_s*> pcs = op->pcs;
  for (vox_precond_s* p : pcs) pc_release(p);
  op->pcs.clear();
  op->wd.release();
  op->wf.release();
  free_bufs(op->d);
  free_bufs(op->f);
  dfree(op->vmap);
  if (op->h_in) cudaFreeHost(op->h_in);
  if (op->h_out) cudaFreeHost(op->h_out);
  dfree(op->d_in);
  dfree(op->d_out);
  dfree(op->f_in);
  dfree(op->f_out);
  if (op->own_stream) cudaStreamDestroy(op->own_stream);
  delete op;
}

}  // namespace vox

// =================================================================== C ABI
extern "C" {

const char* vox_last_error(void) { return vox::last_error(); }
int vox_abi_version(void) { return VOX_ABI_VERSION; }

vox_status vox_set_wait_timeout(double seconds) {
  if (!(seconds >= 0) || seconds > 1e7) {
    vox::set_error("vox_set_wait_timeout: seconds must be in [0, 1e7]");
    return VOX_ERR_BAD_ARG;
  }
  // 0 returns to the default (VOX_WAIT_TIMEOUT_S or 600 s), read on next use
  vox::g_wait_limit_s.store(seconds > 0 ? seconds : -1.0);
  return VOX_OK;
}

double vox_get_wait_timeout(void) { return vox::wait_limit_s(); }

vox_status vox_mem_in_use(int device, long long* bytes) {
  if (!bytes || device < 0 || device >= vox::kMemDevices) {
    vox::set_error("vox_mem_in_use: NULL bytes or device out of range");
    return VOX_ERR_BAD_ARG;
  }
  std::lock_guard<std::mutex> lk(vox::g_mem_mu);
  *bytes = vox::g_mem_bytes[device];
  return VOX_OK;
}

static vox_status create_op(const vox_op_desc* desc, int K, vox_op_t* out);

vox_status vox_op_create(const vox_op_desc* desc, vox_op_t* out) {
  return create_op(desc, 1, out);
}

vox_status vox_op_create_batch(const vox_op_desc* desc, int members, vox_op_t* out) {
  return create_op(desc, members, out);
}

static vox_status create_op(const vox_op_desc* desc, int K, vox_op_t* out) {
  cudaGetLastError();  // drop a stale error left by an unrelated earlier call
  if (!desc || !out) {
    set_error("vox_op_create: NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  *out = nullptr;
  if (K < 1 || K > kMaxMembers) {
    set_error("vox_op_create: members must be 1.." + std::to_string(kMaxMembers));
    return VOX_ERR_BAD_ARG;
  }
  const int L = desc->L, M = desc->M, N = desc->N;
  if (L < 1 || M < 1 || N < 1) {
    set_error("vox_op_create: grid dimensions must be positive");
    return VOX_ERR_BAD_ARG;
  }
  if ((desc->fN_re == nullptr) == (desc->G_re == nullptr)) {
    set_error("vox_op_create: give exactly one of fN_re or G_re");
    return VOX_ERR_BAD_ARG;
  }
  if (!desc->Mc_re || !desc->idx || desc->n_idx < 1) {
    set_error("vox_op_create: Mc and idx are required");
    return VOX_ERR_BAD_ARG;
  }
  const long long V = (long long)L * M * N;
  if (3 * V > 2147483647LL) {
    set_error("vox_op_create: grid too large for 32-bit index maps");
    return VOX_ERR_UNSUPPORTED;
  }
  if (desc->fN_re) {
    if (desc->LfN < 2 * L - 1 || desc->MfN < 2 * M - 1 || desc->NfN < 2 * N - 1) {
      set_error("vox_op_create: fN must be at least (2L-1)x(2M-1)x(2N-1)");
      return VOX_ERR_BAD_ARG;
    }
    if (desc->LfN != 2 * L || desc->MfN != 2 * M || desc->NfN != 2 * N) {
      set_error("vox_op_create: fN must be 2L x 2M x 2N (circulant_nop_const layout)");
      return VOX_ERR_UNSUPPORTED;
    }
  }
  int precs = desc->precisions ? desc->precisions : 3;
  std::unique_ptr<vox_op_s, void (*)(vox_op_s*)> op(new vox_op_s(), destroy_op);
  op->device = desc->device;
  op->K = K;
  DeviceGuard dg(op->device);
  VOX_CUDA(cudaSetDevice(op->device));
  VOX_CUDA(cudaStreamCreateWithFlags(&op->own_stream, cudaStreamNonBlocking));
  op->stream = op->own_stream;
  cudaStream_t st = op->stream;
  OpGeom& g = op->g;
  g.L = L;
  g.M = M;
  g.N = N;
  g.V = V;
  g.n = desc->n_idx;
  g.Px = choose_pad(L);
  g.Py = choose_pad(M);
  g.Pz = choose_pad(N);
  if (!make_fft_plan(g.Px, &op->px) || !make_fft_plan(g.Py, &op->py) ||
      !make_fft_plan(g.Pz, &op->pz)) {
    set_error("vox_op_create: no FFT plan for the padded grid");
    return VOX_ERR_UNSUPPORTED;
  }
  // admission by footprint, before any input array is read or device memory
  // allocated: the FP64 padded circulant built at setup (6 P complex128) plus
  // the index map must fit in the device's free memory
  {
    const double P = (double)g.Px * g.Py * g.Pz;
    const double need = 6.0 * P * sizeof(double2) + 12.0 * (double)V;
    size_t free_b = 0, total_b = 0;
    VOX_CUDA(cudaMemGetInfo(&free_b, &total_b));
    if (need > (double)free_b) {
      set_error("vox_op_create: the operator needs at least " + std::to_string((long long)need) +
                " bytes of device memory at setup; " + std::to_string((long long)free_b) +
                " are free");
      return VOX_ERR_OOM;
    }
  }
  op->gram = desc->gram;
  // index map
  {
    std::vector<int> vmap(3 * V, -1);
    for (long long i = 0; i < desc->n_idx; i++) {
      const double di = desc->idx[i];
      const long long p = (long long)di - 1;
      if (di != std::floor(di) || p < 0 || p >= 3 * V) {
        set_error("vox_op_create: idx[" + std::to_string(i) + "] out of range 1..3*L*M*N");
        return VOX_ERR_BAD_ARG;
      }
      if (vmap[p] >= 0) {
        set_error("vox_op_create: duplicate position in idx");
        return VOX_ERR_BAD_ARG;
      }
      vmap[p] = (int)i;
    }
    VOX_TRY(dalloc(&op->vmap, 3 * V));
    VOX_CUDA(cudaMemcpyAsync(op->vmap, vmap.data(), 3 * V * sizeof(int), cudaMemcpyHostToDevice,
                             st));
  }
  // material arrays
  std::vector<double2> Mr, Mc(V);
  const bool has_Mr = desc->Mr_re != nullptr;
  if (has_Mr) {
    Mr.resize(V);
    for (long long i = 0; i < V; i++)
      Mr[i] = make_double2(desc->Mr_re[i], desc->Mr_im ? desc->Mr_im[i] : 0.0);
  }
  for (long long i = 0; i < V; i++)
    Mc[i] = make_double2(desc->Mc_re[i], desc->Mc_im ? desc->Mc_im[i] : 0.0);
  // padded circulant [comp][x'][y'][z'] in FP64, transformed
  const long long P = (long long)g.Px * g.Py * g.Pz;
  double2* emb;
  VOX_TRY(dalloc(&emb, 6 * P));
  std::unique_ptr<double2, decltype(&dfree)> emb_guard(emb, dfree);
  if (desc->G_re) {
    std::vector<double2> G(6 * V);
    for (long long i = 0; i < 6 * V; i++)
      G[i] = make_double2(desc->G_re[i], desc->G_im ? desc->G_im[i] : 0.0);
    double2* dG;
    VOX_TRY(dalloc(&dG, 6 * V));
    VOX_CUDA(cudaMemcpyAsync(dG, G.data(), 6 * V * sizeof(double2), cudaMemcpyHostToDevice,
                             st));
    k_embed_from_toeplitz<<<nblk(6 * P), 256, 0, st>>>(g, dG, emb);
    VOX_CUDA(cudaGetLastError());
    VOX_TRY(wait_stream(st));
    dfree(dG);
  } else {
    const int L2 = 2 * L, M2 = 2 * M, N2 = 2 * N;
    const long long Q = (long long)L2 * M2 * N2;
    std::vector<double2> F(6 * Q);
    for (long long i = 0; i < 6 * Q; i++)
      F[i] = make_double2(desc->fN_re[i], desc->fN_im ? desc->fN_im[i] : 0.0);
    double2* dF;
    VOX_TRY(dalloc(&dF, 6 * Q));
    std::unique_ptr<double2, decltype(&dfree)> dF_guard(dF, dfree);
    VOX_CUDA(cudaMemcpyAsync(dF, F.data(), 6 * Q * sizeof(double2), cudaMemcpyHostToDevice,
                             st));
    // inverse 3-D FFT (unscaled) of each component: x stride 1, y 2L, z 4LM
    for (int ax = 0; ax < 3; ax++)
      VOX_TRY(fft_axis_d(dF, L2, M2, N2, 1, L2, (long long)L2 * M2, Q, 6, ax, +1, st));
    k_to_prec<double><<<nblk(6 * Q), 256, 0, st>>>(6 * Q, dF, 1.0 / (double)Q, dF);
    k_embed_from_circ<<<nblk(6 * P), 256, 0, st>>>(g, dF, emb);
    VOX_CUDA(cudaGetLastError());
    VOX_TRY(wait_stream(st));
  }
  // forward 3-D FFT of the padded circulant: z stride 1, y Pz, x Py*Pz
  for (int ax = 0; ax < 3; ax++)
    VOX_TRY(fft_axis_d(emb, g.Px, g.Py, g.Pz, (long long)g.Py * g.Pz, g.Pz, 1, P, 6, ax, -1, st));
  // keep one octant when the transformed circulant has the tensor's parity
  {
    unsigned* dd;
    VOX_TRY(dalloc(&dd, 2));
    std::unique_ptr<unsigned, decltype(&dfree)> gd(dd, dfree);
    VOX_CUDA(cudaMemsetAsync(dd, 0, 2 * sizeof(unsigned), st));
    k_sym_defect<<<nblk(6 * P), 256, 0, st>>>(g, emb, dd);
    unsigned hv[2];
    VOX_CUDA(cudaMemcpyAsync(hv, dd, sizeof(hv), cudaMemcpyDeviceToHost, st));
    VOX_TRY(wait_stream(st));
    float defect, fmax;
    std::memcpy(&defect, &hv[0], 4);
    std::memcpy(&fmax, &hv[1], 4);
    g.sym = (fmax > 0.f && defect <= 1e-12f * fmax) ? 1 : 0;
  }
  if (precs & 1) {
    OpGeom gd = g;
    if (!pick_shapes(gd, sizeof(double2))) {
      set_error("vox_op_create: grid planes too large for the complex128 kernels");
      return VOX_ERR_UNSUPPORTED;
    }
    op->d.geo = gd;
    op->d.gram = desc->gram;
    op->d.out_scale = 1.0;
    VOX_TRY(upload_precision<double>(op.get(), emb, Mr, has_Mr, Mc, 1.0));
    op->has_d = true;
  }
  if (precs & 2) {
    // complex64 copy of A/Gram: fN/Gram, Gram -> 1, output rescaled by Gram
    OpGeom gf = g;
    if (!pick_shapes(gf, sizeof(float2))) {
      set_error("vox_op_create: grid planes too large for the complex64 kernels");
      return VOX_ERR_UNSUPPORTED;
    }
    op->f.geo = gf;
    op->f.gram = 1.0f;
    op->f.out_scale = 1.0f;
    VOX_TRY(upload_precision<float>(op.get(), emb, Mr, has_Mr, Mc, 1.0 / desc->gram));
    op->has_f = true;
  }
  // staging for host-buffer entry points
  const long long n = g.n;
  VOX_CUDA(cudaMallocHost((void**)&op->h_in, K * n * sizeof(double2)));
  VOX_CUDA(cudaMallocHost((void**)&op->h_out, K * n * sizeof(double2)));
  VOX_TRY(dalloc(&op->d_in, K * n));
  VOX_TRY(dalloc(&op->d_out, K * n));
  VOX_TRY(dalloc(&op->f_in, n));
  VOX_TRY(dalloc(&op->f_out, n));
  VOX_TRY(wait_stream(st));
  *out = op.release();
  return VOX_OK;
}

void vox_op_destroy(vox_op_t op) { destroy_op(op); }

vox_status vox_op_info(vox_op_t op, int* Px, int* Py, int* Pz, long long* n) {
  if (!op) return VOX_ERR_BAD_ARG;
  if (Px) *Px = op->g.Px;
  if (Py) *Py = op->g.Py;
  if (Pz) *Pz = op->g.Pz;
  if (n) *n = op->g.n;
  return VOX_OK;
}

}  // extern "C"

namespace vox {

template <typename R>
__global__ void k_from_d2(long long n, const double2* __restrict__ a, Cx<R>* b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    b[i] = from_d2<Cx<R>>(a[i]);
}
template <typename R>
__global__ void k_to_d2(long long n, const Cx<R>* __restrict__ a, double scale, double2* b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double2 v = to_d2(a[i]);
    b[i] = make_double2(v.x * scale, v.y * scale);
  }
}

static void split_to_d2(const double* re, const double* im, long long n, double2* dst) {
  for (long long i = 0; i < n; i++) dst[i] = make_double2(re[i], im ? im[i] : 0.0);
}
static void d2_to_split(const double2* src, long long n, double* re, double* im) {
  for (long long i = 0; i < n; i++) {
    re[i] = src[i].x;
    if (im) im[i] = src[i].y;
  }
}

static vox_status check_prec(vox_op_s* op, vox_prec prec) {
  if (prec == VOX_C128 && !op->has_d) {
    set_error("operator has no complex128 copy");
    return VOX_ERR_BAD_ARG;
  }
  if (prec == VOX_C64 && !op->has_f) {
    set_error("operator has no complex64 copy");
    return VOX_ERR_BAD_ARG;
  }
  if (prec != VOX_C128 && prec != VOX_C64) {
    set_error("unknown precision");
    return VOX_ERR_BAD_ARG;
  }
  return VOX_OK;
}

// Host-buffer matvec through the staging buffers.
static vox_status mv_host(vox_op_s* op, int mode, vox_prec prec, const double* in_re,
                          const double* in_im, double* out_re, double* out_im) {
  if (!op || !in_re || !out_re) {
    set_error("NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  VOX_TRY(check_prec(op, prec));
  DeviceGuard dg(op->device);
  const long long n = op->g.n;
  cudaStream_t st = op->stream;
  split_to_d2(in_re, in_im, n, op->h_in);
  VOX_CUDA(cudaMemcpyAsync(op->d_in, op->h_in, n * sizeof(double2), cudaMemcpyHostToDevice, st));
  if (prec == VOX_C128) {
    VOX_TRY(matvec<double>(op, mode, op->d_in, op->d_out, st, nullptr));
  } else {
    k_from_d2<float><<<nblk(n), 256, 0, st>>>(n, op->d_in, op->f_in);
    VOX_TRY(matvec<float>(op, mode, op->f_in, op->f_out, st, nullptr));
    // the complex64 copy computes A x / Gram for MV_AN (and (N-Gram)x/Gram for MV_L)
    k_to_d2<float><<<nblk(n), 256, 0, st>>>(n, op->f_out, op->gram, op->d_out);
  }
  VOX_CUDA(cudaMemcpyAsync(op->h_out, op->d_out, n * sizeof(double2), cudaMemcpyDeviceToHost, st));
  VOX_TRY(wait_stream(st));
  d2_to_split(op->h_out, n, out_re, out_im);
  return VOX_OK;
}

}  // namespace vox

extern "C" {

vox_status vox_mv_AN(vox_op_t op, int transp, vox_prec prec, const double* in_re,
                     const double* in_im, double* out_re, double* out_im) {
  return mv_host(op, transp ? MV_AN_T : MV_AN, prec, in_re, in_im, out_re, out_im);
}

vox_status vox_mv_L(vox_op_t op, vox_prec prec, const double* in_re, const double* in_im,
                    double* out_re, double* out_im) {
  return mv_host(op, MV_L, prec, in_re, in_im, out_re, out_im);
}

vox_status vox_mv_AN_device(vox_op_t op, int transp, vox_prec prec, const void* in, void* out,
                            void* stream) {
  if (!op || !in || !out) {
    set_error("NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  VOX_TRY(check_prec(op, prec));
  DeviceGuard dg(op->device);
  cudaStream_t st = stream ? (cudaStream_t)stream : op->stream;
  const int mode = transp ? MV_AN_T : MV_AN;
  if (prec == VOX_C128)
    return matvec<double>(op, mode, (const double2*)in, (double2*)out, st, nullptr);
  return matvec<float>(op, mode, (const float2*)in, (float2*)out, st, nullptr);
}

vox_status vox_mv_AN_batch_device(vox_op_t op, int transp, vox_prec prec, int count,
                                  const void* in, void* out, void* stream) {
  if (!op || !in || !out) {
    set_error("NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  if (count < 1 || count > op->K) {
    set_error("count must be 1..members of the operator");
    return VOX_ERR_BAD_ARG;
  }
  VOX_TRY(check_prec(op, prec));
  DeviceGuard dg(op->device);
  cudaStream_t st = stream ? (cudaStream_t)stream : op->stream;
  const int mode = transp ? MV_AN_T : MV_AN;
  Members mm;
  mm.km = count;
  mm.vs = op->g.n;
  if (prec == VOX_C128)
    return matvec<double>(op, mode, (const double2*)in, (double2*)out, st, nullptr, mm);
  return matvec<float>(op, mode, (const float2*)in, (float2*)out, st, nullptr, mm);
}

vox_status vox_block_dot(long long n, int a, int b, const void* X, long long ldx, const void* Y,
                         long long ldy, void* C, void* stream) {
  if (!X || !Y || !C || n < 0 || a < 1 || b < 1 || a > kBlkCols || b > kBlkCols ||
      ldx < n || ldy < n) {
    set_error("vox_block_dot: bad sizes or NULL block");
    return VOX_ERR_BAD_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const long long tiles = (n + kBlkRows - 1) / kBlkRows;
  const int ctas = (int)std::max<long long>(1, std::min<long long>(kBlkCtas, tiles));
  double2* partial = nullptr;
  VOX_TRY(smem_cap(k_block_dot_partial));
  VOX_CUDA(cudaMallocAsync((void**)&partial, (size_t)ctas * a * b * sizeof(double2), st));
  k_block_dot_partial<<<ctas, kBlkThreads, block_dot_smem(a, b), st>>>(
      n, a, b, (const double2*)X, ldx, (const double2*)Y, ldy, partial);
  k_block_dot_reduce<<<(a * b + 255) / 256, 256, 0, st>>>(a, b, ctas, partial, (double2*)C);
  const cudaError_t e = cudaGetLastError();
  VOX_CUDA(cudaFreeAsync(partial, st));
  VOX_CUDA(e);
  return VOX_OK;
}

}  // extern "C"

namespace vox {
// host parts of the assembly (assembly.cpp)
void asm_rule(int np, std::vector<double>& w, std::vector<double>& u, std::vector<double>& v);
void asm_tables(double dx, double p1[6][3], double a[6][3], double b[6][3], double P[6][6][6],
                int obs[21], int src[21], int fill[15][4]);
void asm_near_cell(int mx, int my, int mz, const double Ipair[21][2], double ko, double dx,
                   double G[6][2]);
}  // namespace vox

extern "C" {

vox_status vox_assemble_toeplitz_device(int L, int M, int N, double ko, double dx, int device,
                                        double* G_re, double* G_im) {
  if (L < 2 || M < 2 || N < 2 || !G_re || !G_im || dx <= 0) {
    set_error("vox_assemble_toeplitz_device: needs L, M, N >= 2 and output buffers");
    return VOX_ERR_BAD_ARG;
  }
  DeviceGuard dg(device);
  const long long V = (long long)L * M * N;
  CubGeom g;
  asm_tables(dx, g.p1, g.a, g.b, g.P, g.obs, g.src, g.fill);
  // rules: far 4 x 4, medium 10 x 10, near 20 x 20 points per face
  const int nps[3] = {4, 10, 20};
  std::vector<double> host;
  size_t off[3][3];
  for (int r = 0; r < 3; r++) {
    std::vector<double> w, u, v;
    asm_rule(nps[r], w, u, v);
    off[r][0] = host.size();
    host.insert(host.end(), w.begin(), w.end());
    off[r][1] = host.size();
    host.insert(host.end(), u.begin(), u.end());
    off[r][2] = host.size();
    host.insert(host.end(), v.begin(), v.end());
  }
  cudaStream_t st;
  VOX_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct Cleanup {
    cudaStream_t st;
    double* rules = nullptr;
    double2* Ipair = nullptr;
    double2* G = nullptr;
    ~Cleanup() {
      dfree(rules);
      dfree(Ipair);
      dfree(G);
      cudaStreamDestroy(st);
    }
  } c{st};
  VOX_TRY(dalloc(&c.rules, host.size()));
  VOX_TRY(dalloc(&c.Ipair, (size_t)V * 21));
  VOX_TRY(dalloc(&c.G, (size_t)V * 6));
  VOX_CUDA(cudaMemcpyAsync(c.rules, host.data(), host.size() * sizeof(double),
                           cudaMemcpyHostToDevice, st));
  CubRules rr;
  for (int r = 0; r < 3; r++) {
    rr.w[r] = c.rules + off[r][0];
    rr.u[r] = c.rules + off[r][1];
    rr.v[r] = c.rules + off[r][2];
    rr.np[r] = nps[r] * nps[r];
  }
  const long long warps = V * 21;
  const long long blocks = (warps * 32 + 255) / 256;
  k_cubature_pairs<<<(unsigned)blocks, 256, 0, st>>>(L, M, N, std::min(5, L), std::min(5, M),
                                                     std::min(5, N), ko, dx, g, rr, c.Ipair);
  k_cubature_project<<<nblk(V), 256, 0, st>>>(L, M, N, g, c.Ipair, c.G);
  VOX_CUDA(cudaGetLastError());
  std::vector<double2> Gh((size_t)V * 6);
  VOX_CUDA(cudaMemcpyAsync(Gh.data(), c.G, Gh.size() * sizeof(double2), cudaMemcpyDeviceToHost,
                           st));
  // the near cells' pair integrals, for the singular corrections on the host
  double2 In[8][21];
  for (int m = 0; m < 8; m++) {
    const int mx = m & 1, my = (m >> 1) & 1, mz = m >> 2;
    const long long cell = mx + (long long)L * (my + (long long)M * mz);
    VOX_CUDA(cudaMemcpyAsync(In[m], c.Ipair + cell * 21, 21 * sizeof(double2),
                             cudaMemcpyDeviceToHost, st));
  }
  VOX_TRY(wait_stream(st));
  for (long long i = 0; i < V * 6; i++) {
    const long long cell = i % V;
    const int mx = (int)(cell % L), my = (int)((cell / L) % M), mz = (int)(cell / ((long long)L * M));
    if (mx < 2 && my < 2 && mz < 2) continue;
    G_re[i] = Gh[i].x;
    G_im[i] = Gh[i].y;
  }
  for (int m = 0; m < 8; m++) {
    const int mx = m & 1, my = (m >> 1) & 1, mz = m >> 2;
    const long long cell = mx + (long long)L * (my + (long long)M * mz);
    double Ip[21][2], Gc[6][2];
    for (int t = 0; t < 21; t++) {
      Ip[t][0] = In[m][t].x;
      Ip[t][1] = In[m][t].y;
    }
    asm_near_cell(mx, my, mz, Ip, ko, dx, Gc);
    for (int k = 0; k < 6; k++) {
      G_re[cell + V * k] = Gc[k][0];
      G_im[cell + V * k] = Gc[k][1];
    }
  }
  return VOX_OK;
}

vox_status vox_block_update(long long n, int a, int b, const void* X, long long ldx,
                            const void* W, double beta, void* Y, long long ldy, void* stream) {
  if (!X || !W || !Y || n < 0 || a < 1 || b < 1 || a > kBlkCols || b > kBlkCols ||
      ldx < n || ldy < n) {
    set_error("vox_block_update: bad sizes or NULL block");
    return VOX_ERR_BAD_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  k_block_update<<<nblk(n, kBlkThreads), kBlkThreads, 0, st>>>(
      n, a, b, (const double2*)X, ldx, (const double2*)W, beta, (double2*)Y, ldy);
  VOX_CUDA(cudaGetLastError());
  return VOX_OK;
}

}  // extern "C"

#include "solver.cuh"
#include "lane.cuh"
#include "jvie.cuh"

namespace vox {
static void lanes_release(vox_op_s* op) {
  std::vector<vox_lane_s*> ls = op->lanes;
  for (vox_lane_s* l : ls) delete l;
  op->lanes.clear();
}
}  // namespace vox

// ------------------------------------------------ matvec without allocation
// Some callers cannot call cudaMalloc at the point where they need a product:
// code running under an external memory manager that owns every device
// allocation, or inside a callback/region where allocating is forbidden.
// vox_mv_AN_noalloc runs the fused matvec on an operator prepared earlier with
// the two plane intermediates placed in this fixed, file-scope device array
// instead of the operator's own buffers.  The array is part of the module:
// every GPU that loads libvox holds it until the process exits.
namespace vox {

constexpr size_t kNoAllocScratchBytes = 64ull << 20;  // 64 MiB: T1 and T2 together
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static std::mutex g_noalloc_mu;
static std::map<int, void*> g_noalloc_addr;  // device ordinal -> array address

// Device address of the array on `dev` (which must be current).  Looked up
// once per device and kept while that device's primary context lives; a
// host-side reference to the symbol is not a device address.
static vox_status noalloc_scratch(int dev, void** out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  auto it = g_noalloc_addr.find(dev);
  if (it != g_noalloc_addr.end()) {
    *out = it->second;
    return VOX_OK;
  }
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || p == nullptr) {
    cudaGetLastError();
    set_error(std::string("vox_mv_AN_noalloc: cudaGetSymbolAddress failed: ") +
              cudaGetErrorString(e));
    return VOX_ERR_CUDA;
  }
  g_noalloc_addr[dev] = p;
  *out = p;
  return VOX_OK;
}

}  // namespace vox

extern "C" vox_status vox_mv_AN_noalloc(vox_op_t op, int transp, vox_prec prec, const void* in,
                                        void* out, void* stream) {
  if (!op || !in || !out) {
    set_error("vox_mv_AN_noalloc: NULL argument");
    return VOX_ERR_BAD_ARG;
  }
  VOX_TRY(check_prec(op, prec));
  DeviceGuard dg(op->device);
  const OpGeom& g = prec == VOX_C128 ? op->d.geo : op->f.geo;
  const size_t cs = prec == VOX_C128 ? sizeof(double2) : sizeof(float2);
  const size_t half = ((size_t)g.Px * 3 * g.N * g.M * cs + 255) / 256 * 256;
  if (g.split) {
    set_error("vox_mv_AN_noalloc: operators whose planes do not fit in shared memory (split "
              "plane kernels, a third intermediate) are not supported; use vox_mv_AN_device");
    return VOX_ERR_BAD_ARG;
  }
  if (2 * half > kNoAllocScratchBytes) {
    set_error("vox_mv_AN_noalloc: this operator needs " + std::to_string(2 * half) +
              " bytes of scratch; the fixed maximum is " + std::to_string(kNoAllocScratchBytes) +
              " bytes (use vox_mv_AN_device)");
    return VOX_ERR_BAD_ARG;
  }
  void* base = nullptr;
  VOX_TRY(noalloc_scratch(op->device, &base));
  cudaStream_t st = stream ? (cudaStream_t)stream : op->stream;
  const int mode = transp ? MV_AN_T : MV_AN;
  unsigned char* b8 = static_cast<unsigned char*>(base);
  if (prec == VOX_C128) {
    PlaneScratch<double> sc{(double2*)b8, (double2*)(b8 + half)};
    return matvec<double>(op, mode, (const double2*)in, (double2*)out, st, nullptr, Members(),
                          sc);
  }
  PlaneScratch<float> sc{(float2*)b8, (float2*)(b8 + half)};
  return matvec<float>(op, mode, (const float2*)in, (float2*)out, st, nullptr, Members(), sc);
}
