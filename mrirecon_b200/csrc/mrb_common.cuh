// Shared helpers for the mrirecon_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/mrirecon_b200.h"

namespace mrb {

// ---------------------------------------------------------------------------
// error reporting: every entry point returns a status and records a message
// ---------------------------------------------------------------------------
void set_error(const char* fmt, ...);
int fail(int code, const char* fmt, ...);

#define MRB_CUDA_TRY(expr)                                                          \
  do {                                                                              \
    cudaError_t _e = (expr);                                                        \
    if (_e != cudaSuccess)                                                          \
      return ::mrb::fail(MRB_ECUDA, "%s:%d %s: %s", __FILE__, __LINE__, #expr,     \
                         cudaGetErrorString(_e));                                   \
  } while (0)

// every kernel launch of the library goes through MRB_LAUNCH_CHECK, which also
// counts it (host-side; launches recorded into a CUDA graph count once).  A
// kernel launched directly while grouped launches are being recorded would
// run ahead of the recorded ones: its entry point fails (group.cuh).
void count_launch();
bool group_recording();
#define MRB_LAUNCH_CHECK()                                                               \
  do {                                                                                   \
    ::mrb::count_launch();                                                               \
    MRB_CUDA_TRY(cudaGetLastError());                                                    \
    if (::mrb::group_recording())                                                        \
      return ::mrb::fail(MRB_ESTATE, "%s:%d: kernel without a grouped form launched "   \
                         "inside a recording", __FILE__, __LINE__);                      \
  } while (0)

#define MRB_REQUIRE(cond, ...)                                                      \
  do {                                                                              \
    if (!(cond)) return ::mrb::fail(MRB_EINVAL, __VA_ARGS__);                       \
  } while (0)

inline int ceil_div_i(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// Device memory of the plans.  Large blocks (>= 1 MiB) released by one plan
// are kept, per device and up to a cap, for the next plan of a similar size:
// a process that builds operators repeatedly (a new trajectory per scan) then
// does not pay a cudaMalloc / cudaFree of gigabytes each time, whose cost
// varies by orders of magnitude.  A released block joins the cache only after
// the device has finished its work (a device synchronisation, as cudaFree
// itself implies), so a later owner never races the previous one; like
// cudaFree, releasing is not allowed inside a stream capture.
// mrb_release_cached_memory() returns the cached blocks to the driver.
void* dev_alloc(size_t n, size_t* got);   // nullptr on failure
void dev_free(void* p, size_t bytes);

// Device buffer owned by a plan.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  int ensure(size_t n) {
    if (n <= bytes) return 0;
    release();
    if (n == 0) return 0;
    size_t got = 0;
    p = dev_alloc(n, &got);
    if (!p) return fail(MRB_ENOMEM, "device allocation of %zu bytes failed", n);
    bytes = got;
    return 0;
  }
  void release() {
    if (p) dev_free(p, bytes);
    p = nullptr;
    bytes = 0;
  }
  template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

// ---------------------------------------------------------------------------
// Kaiser-Bessel weights of the W = 4 taps.  A sample at grid coordinate x
// meets the nodes floor(x) - 1 + t, t = 0..3, at distances d = f + 1 - t with
// f = x - floor(x) in [0, 1), and the weight of tap t,
//   phi(d) = I0(beta sqrt(1 - (2d/W)^2)) / I0(beta),
// is a smooth function of f alone.  The host fits each tap's phi on [0, 1] by
// Chebyshev interpolation (degree KB_TAP_DEG, in double; the interpolation
// error is below 4e-9, the FP32 Horner rounding below 1e-7) and stores the fit
// as a polynomial in u = 2f - 1, so one tap costs KB_TAP_DEG fused
// multiply-adds instead of the ~19-term I0 series in z = 1 - (2d/W)^2
// (A&S 9.6.10; the reference evaluates I0 directly, ptnufft.py:79-90).
// ---------------------------------------------------------------------------
constexpr int KB_TAP_DEG = 9;

struct KBPoly {
  float tap[4][KB_TAP_DEG + 1];   // tap[t][k]: coefficient of u^k
};

// weight of tap t at fractional offset f = x - floor(x)
__device__ __forceinline__ float kb_tap(const KBPoly& p, int t, float f) {
  const float u = fmaf(2.0f, f, -1.0f);
  float acc = p.tap[t][KB_TAP_DEG];
#pragma unroll
  for (int k = KB_TAP_DEG - 1; k >= 0; --k) acc = fmaf(acc, u, p.tap[t][k]);
  return acc;
}

// Host: fill the tap polynomials for (W = 4, beta).
void kb_poly_init(KBPoly& p, int W, double beta);

// Reference float32 arithmetic for grid coordinates (ptnufft.py:151-153):
// u = w / float32(2pi) + 0.5 ; gx = u * G ; clamp(gx, 0, float32(G - 1e-6)).
__device__ __forceinline__ float ref_grid_coord(float w, float Gf, float gmax) {
  float u = __fadd_rn(__fdiv_rn(w, 6.28318548202514648f), 0.5f);
  float g = __fmul_rn(u, Gf);
  return fminf(fmaxf(g, 0.0f), gmax);
}

__device__ __forceinline__ int wrap_i(int n, int G) {
  int r = n % G;
  return r < 0 ? r + G : r;
}

}  // namespace mrb
