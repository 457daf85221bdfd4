// Error state, KB polynomial set-up and version entry points.
#include <cmath>
#include <cstdarg>
#include <atomic>
#include <cstring>
#include <mutex>
#include <vector>

#include "mrb_common.cuh"

namespace mrb {

static thread_local char g_err[1024] = "";
static std::atomic<long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

// ---------------------------------------------------------------------------
// block cache of dev_alloc / dev_free
// ---------------------------------------------------------------------------
namespace {
constexpr size_t POOL_MIN_BLOCK = 1u << 20;            // smaller blocks go straight to the driver
constexpr size_t POOL_CAP = (size_t)8 << 30;           // bytes kept per device

struct PoolBlock {
  void* p;
  size_t bytes;
  int dev;
};

std::mutex g_pool_mu;
std::vector<PoolBlock> g_pool;

size_t pool_bytes(int dev) {
  size_t t = 0;
  for (const PoolBlock& b : g_pool)
    if (b.dev == dev) t += b.bytes;
  return t;
}
}  // namespace

void* dev_alloc(size_t n, size_t* got) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (n >= POOL_MIN_BLOCK) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    int best = -1;
    for (int i = 0; i < (int)g_pool.size(); ++i) {
      const PoolBlock& b = g_pool[i];
      if (b.dev == dev && b.bytes >= n && b.bytes <= 2 * n && (best < 0 || b.bytes < g_pool[best].bytes)) best = i;
    }
    if (best >= 0) {
      void* p = g_pool[best].p;
      *got = g_pool[best].bytes;
      g_pool.erase(g_pool.begin() + best);
      return p;
    }
  }
  void* p = nullptr;
  if (cudaMalloc(&p, n) != cudaSuccess) {
    cudaGetLastError();
    // the cache may hold the memory: hand it back and try once more
    mrb_release_cached_memory();
    if (cudaMalloc(&p, n) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
  }
  *got = n;
  return p;
}

void dev_free(void* p, size_t bytes) {
  if (!p) return;
  int dev = 0;
  cudaGetDevice(&dev);
  if (bytes >= POOL_MIN_BLOCK) {
    cudaDeviceSynchronize();   // what cudaFree would wait for: no kernel may still use the block
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (pool_bytes(dev) + bytes <= POOL_CAP) {
      g_pool.push_back(PoolBlock{p, bytes, dev});
      return;
    }
  }
  cudaFree(p);
}

// I0 by its power series (A&S 9.6.10), double precision, host only.
static double i0_series(double x) {
  double q = 0.25 * x * x, term = 1.0, sum = 1.0;
  for (int k = 1; k < 200; ++k) {
    term *= q / ((double)k * (double)k);
    sum += term;
    if (term < 1e-18 * sum) break;
  }
  return sum;
}

void kb_poly_init(KBPoly& p, int W, double beta) {
  const double i0b = i0_series(beta);
  auto phi = [&](double d) {
    const double z = 1.0 - (2.0 * d / W) * (2.0 * d / W);
    return z > 0.0 ? i0_series(beta * std::sqrt(z)) / i0b : 1.0 / i0b;
  };
  constexpr int D = KB_TAP_DEG, M = KB_TAP_DEG + 1;
  for (int t = 0; t < 4; ++t) {
    // Chebyshev interpolation at the M first-kind nodes of u in [-1, 1]
    double v[M], a[M];
    for (int j = 0; j < M; ++j) {
      const double u = std::cos(M_PI * (j + 0.5) / M);
      v[j] = phi(0.5 * (u + 1.0) + 1.0 - t);
    }
    for (int k = 0; k < M; ++k) {
      double s = 0.0;
      for (int j = 0; j < M; ++j) s += v[j] * std::cos(M_PI * k * (j + 0.5) / M);
      a[k] = (k == 0 ? 1.0 : 2.0) * s / M;
    }
    // sum a_k T_k(u) as monomials: T_0 = 1, T_1 = u, T_{k+1} = 2u T_k - T_{k-1}
    double mono[M] = {0.0}, tkm1[M] = {0.0}, tk[M] = {0.0}, tkp1[M];
    tkm1[0] = 1.0;
    tk[1] = 1.0;
    mono[0] += a[0];
    for (int i = 0; i < M; ++i) mono[i] += a[1] * tk[i];
    for (int k = 1; k < D; ++k) {
      for (int i = 0; i < M; ++i) tkp1[i] = (i > 0 ? 2.0 * tk[i - 1] : 0.0) - tkm1[i];
      for (int i = 0; i < M; ++i) {
        mono[i] += a[k + 1] * tkp1[i];
        tkm1[i] = tk[i];
        tk[i] = tkp1[i];
      }
    }
    for (int i = 0; i < M; ++i) p.tap[t][i] = (float)mono[i];
  }
}

}  // namespace mrb

extern "C" int mrb_release_cached_memory(void) {
  int cur = 0;
  cudaGetDevice(&cur);
  std::vector<mrb::PoolBlock> keep;
  {
    std::lock_guard<std::mutex> lk(mrb::g_pool_mu);
    keep.swap(mrb::g_pool);
  }
  for (const mrb::PoolBlock& b : keep) {
    cudaSetDevice(b.dev);
    cudaFree(b.p);
  }
  cudaSetDevice(cur);
  return 0;
}

extern "C" int mrb_version(void) { return 1; }
extern "C" int64_t mrb_launch_count(void) { return (int64_t)mrb::g_launches.load(); }
extern "C" const char* mrb_last_error(void) { return mrb::g_err; }
