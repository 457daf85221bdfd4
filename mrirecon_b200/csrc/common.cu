// Error state, KB polynomial set-up and version entry points.
#include <cmath>
#include <cstdarg>
#include <atomic>
#include <cstring>

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
  double i0b = i0_series(beta);
  double q = 0.25 * beta * beta;
  double ck = 1.0 / i0b;
  int n = 0;
  for (int k = 0; k < KB_MAX_TERMS; ++k) {
    if (k > 0) ck *= q / ((double)k * (double)k);
    p.c[k] = (float)ck;
    n = k + 1;
    if (k > 2 && ck < 1e-10) break;
  }
  p.n = n;
  p.inv_half_w2 = (float)(4.0 / ((double)W * (double)W));
}

}  // namespace mrb

extern "C" int mrb_version(void) { return 1; }
extern "C" int64_t mrb_launch_count(void) { return (int64_t)mrb::g_launches.load(); }
extern "C" const char* mrb_last_error(void) { return mrb::g_err; }
