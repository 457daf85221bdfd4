// Objective, Huber-TV and NCG kernels for B200 (sm_100a).
//
// Image tensors are (F, 1, *S) complex64 (frames, size-1 coil slot, nd
// spatial dims), k-space tensors (nb, C, K) complex64.  Regularisers are
// evaluated at z = x + t*d without modifying x; all scalar reductions (dots,
// energies, objective) are accumulated in FP64 with a fixed block partition
// and a fixed final order, so results are bitwise reproducible.
//
// Reference semantics (graspcg = timodelgado/mrirecon):
//   TV             regularization/tv_nd.py:54-88, ops/ndops.py:28-148
//   objective      ops/objective.py:31-45, 184-291
//   Armijo         numerics/line_search.py:24-79
//   FR/PR+/DY      numerics/directions.py:75-162 (FR seeds rho_prev with the
//                  current rho on its first update, so its first beta is 1)
//   converged      solvers/utils.py:40-43
//   history        solvers/utils.py:64-87 (running sums of the norms)

#include <cuda_runtime.h>

#include <algorithm>

#include <cmath>
#include <cstring>
#include <mutex>

#include "mrb_common.cuh"
#include "group.cuh"

namespace {

using mrb::VBlock;
using mrb::hw_block;

constexpr int RED_THREADS = 256;
constexpr int RED_MAX_BLOCKS = 1184;   // 8 x 148 SMs
constexpr int RED_MAX_VALS = 32;

__host__ __device__ inline int red_blocks(long long n, int per_thread) {
  long long b = (n + (long long)RED_THREADS * per_thread - 1) / ((long long)RED_THREADS * per_thread);
  if (b < 1) b = 1;
  if (b > RED_MAX_BLOCKS) b = RED_MAX_BLOCKS;
  return (int)b;
}

// Block-level FP64 reduction of NV values; lane/warp order fixed.
template <int NV>
__device__ __forceinline__ void block_reduce_store(const VBlock& vb, double (&v)[NV], double* __restrict__ partials) {
  __shared__ double sh[RED_THREADS / 32][NV];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    double s = v[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) sh[warp][j] = s;
  }
  __syncthreads();
  if (warp == 0) {
    for (int j = 0; j < NV; ++j) {
      double s = lane < RED_THREADS / 32 ? sh[lane][j] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
      if (lane == 0) partials[(long long)vb.x * NV + j] = s;
    }
  }
}

// out[j] (=|+=) sum over nblocks of partials[b][j]; one warp per value.
__global__ void finalize_kernel(const double* __restrict__ partials, int nblocks, int stride, int nv,
                                double* __restrict__ out, int accumulate, const double* __restrict__ skip) {
  if (skip && *skip != 0.0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int j = warp; j < nv; j += blockDim.x >> 5) {
    double s = 0.0;
    for (int b = lane; b < nblocks; b += 32) s += partials[(long long)b * stride + j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) out[j] = accumulate ? out[j] + s : s;
  }
}

// partials are laid out [block][stride]; the first nv values of each row are summed
int finalize(const double* partials, int nblocks, int stride, int nv, double* out, int accumulate,
             const double* skip, cudaStream_t st) {
  finalize_kernel<<<1, 256, 0, st>>>(partials, nblocks, stride, nv, out, accumulate, skip);
  MRB_LAUNCH_CHECK();
  return 0;
}

__device__ __forceinline__ double skipped(const double* flag) { return flag ? *flag : 0.0; }

// Where a reducing kernel leaves its result: the block partials are summed by
// the last block to finish (a completion counter in the caller's workspace,
// zero between launches), in the same fixed order as finalize_kernel, so the
// separate finalize launch disappears and the result is bit-identical.
struct RedOut {
  double* out;          // nv results
  int nv;
  int accumulate;       // out[j] += sum
  const double* skip;   // out untouched when *skip != 0
  double* copy0;        // optional second destination of out[0]
  unsigned* counter;    // completion counter (zero between launches)
};

template <int NV>
__device__ __forceinline__ void block_reduce_finish(const VBlock& vb, double (&v)[NV], double* __restrict__ partials,
                                                    const RedOut& r) {
  block_reduce_store<NV>(vb, v, partials);
  __shared__ unsigned s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(r.counter, 1u) == vb.nx - 1 ? 1u : 0u;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // the last block: every thread sums a fixed, strided set of block partials
  // (independent loads, values in groups of 8), then one fixed-order block tree
  __shared__ double fin[RED_THREADS / 32][NV];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int GRP = NV < 8 ? NV : 8;
#pragma unroll 1
  for (int j0 = 0; j0 < NV; j0 += GRP) {
    double acc[GRP];
#pragma unroll
    for (int q = 0; q < GRP; ++q) acc[q] = 0.0;
    for (int b = threadIdx.x; b < (int)vb.nx; b += blockDim.x) {
#pragma unroll
      for (int q = 0; q < GRP; ++q)
        if (j0 + q < NV) acc[q] += __ldcg(partials + (long long)b * NV + j0 + q);
    }
#pragma unroll
    for (int q = 0; q < GRP; ++q) {
      double sv = acc[q];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sv += __shfl_down_sync(0xffffffffu, sv, o);
      if (lane == 0 && j0 + q < NV) fin[warp][j0 + q] = sv;
    }
  }
  __syncthreads();
  if (warp == 0) {
    const bool skip = r.skip && *r.skip != 0.0;
    for (int j = 0; j < r.nv; ++j) {
      double sv = lane < RED_THREADS / 32 ? fin[lane][j] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sv += __shfl_down_sync(0xffffffffu, sv, o);
      if (lane == 0 && !skip) {
        const double val = r.accumulate ? r.out[j] + sv : sv;
        r.out[j] = val;
        if (j == 0 && r.copy0) *r.copy0 = val;
      }
    }
    if (lane == 0) *r.counter = 0u;
  }
}

constexpr size_t RED_PART_BYTES = (size_t)RED_MAX_BLOCKS * RED_MAX_VALS * sizeof(double);

__host__ __device__ inline unsigned* ws_counter(void* ws) {
  return reinterpret_cast<unsigned*>(reinterpret_cast<char*>(ws) + RED_PART_BYTES);
}

inline RedOut red_out(void* ws, double* out, int nv, int accumulate, const double* skip, double* copy0 = nullptr) {
  return RedOut{out, nv, accumulate, skip, copy0, ws_counter(ws)};
}

// ---------------------------------------------------------------------------
// generic dots: out[j] = sum Re(conj(a_j) b_j) / diag_j
// ---------------------------------------------------------------------------
struct DotArgs {
  const float2* a[8];
  const float2* b[8];
  const float* diag[8];
  long long ndiag;
  long long n;
  int npairs;
};

template <int NP>
__global__ void __launch_bounds__(RED_THREADS) dots_kernel(DotArgs a, double* __restrict__ partials) {
  const VBlock vb = hw_block();
  double acc[NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) acc[j] = 0.0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      // the 8-wide instance serves npairs 5..8: slots past npairs hold no operands
      if (NP > 4 && j >= a.npairs) continue;
      float2 u = a.a[j][i], v = a.b[j][i];
      float r = u.x * v.x + u.y * v.y;
      if (a.diag[j]) r /= a.diag[j][i % a.ndiag];
      acc[j] += (double)r;
    }
  }
  block_reduce_store<NP>(vb, acc, partials);
}

// ---------------------------------------------------------------------------
// k-space passes
// ---------------------------------------------------------------------------
// mode 0: scalars e_rr = |r|^2, e_rd = Re<r,Ad>, e_dd = |Ad|^2
// mode 1: r = Ax + t*Ad - y, returns |r|^2 (reference residual, objective.py:31-45)
// mode 2: r += t*Ad (accepted step; t from the device), no reduction
struct KSpace {
  static constexpr int NT = RED_THREADS, MINB = 5;
  static constexpr const char* FAMILY = "kspace";
  static constexpr int MAXG = 16;
  static __device__ __forceinline__ void run(const VBlock& vb, int mode, long long n, float2* __restrict__ r,
      const float2* __restrict__ Ad, const float2* __restrict__ Ax, const float2* __restrict__ y,
      const double* t_dev, double t_host, const double* skip, double* __restrict__ partials, const RedOut& ro) {
    double acc[3] = {0.0, 0.0, 0.0};
    if (skipped(skip) != 0.0) return;   // uniform over the grid: no partials, no counter
    const bool sk = false;
    float t = (float)(t_dev ? *t_dev : t_host);
    const long long stride = (long long)vb.nx * blockDim.x;
    if (!sk) {
      for (long long i = (long long)vb.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        if (mode == 0) {
          float2 a = r[i], b = Ad[i];
          acc[0] += (double)(a.x * a.x + a.y * a.y);
          acc[1] += (double)(a.x * b.x + a.y * b.y);
          acc[2] += (double)(b.x * b.x + b.y * b.y);
        } else if (mode == 1) {
          float2 d = Ad ? Ad[i] : make_float2(0.f, 0.f);
          float2 a = Ax[i], yy = y[i];
          // same operation order as the reference: r = Ad; r *= t; r += Ax; r -= y
          float rx = __fadd_rn(__fadd_rn(__fmul_rn(d.x, t), a.x), -yy.x);
          float ry = __fadd_rn(__fadd_rn(__fmul_rn(d.y, t), a.y), -yy.y);
          r[i] = make_float2(rx, ry);
          acc[0] += (double)(rx * rx + ry * ry);
        } else {
          float2 a = r[i], b = Ad[i];
          a.x = fmaf(t, b.x, a.x);
          a.y = fmaf(t, b.y, a.y);
          r[i] = a;
        }
      }
    }
    if (mode == 2) return;
    if (mode == 1) {
      double v1[1] = {acc[0]};
      block_reduce_finish<1>(vb, v1, partials, ro);
    } else {
      block_reduce_finish<3>(vb, acc, partials, ro);
    }
  }
};
__global__ void __launch_bounds__(RED_THREADS) kspace_kernel(int mode, long long n, float2* __restrict__ r,
    const float2* __restrict__ Ad, const float2* __restrict__ Ax, const float2* __restrict__ y,
    const double* t_dev, double t_host, const double* skip, double* __restrict__ partials, RedOut ro) {
  KSpace::run(hw_block(), mode, n, r, Ad, Ax, y, t_dev, t_host, skip, partials, ro);
}

// ---------------------------------------------------------------------------
// Huber TV at z = x + t*d
// ---------------------------------------------------------------------------
// The terms are compiled on the host into
//   slots: the distinct image axes the terms difference along (<= 4), and
//   units: one per isotropic term, one per axis of an anisotropic term
//          (<= 8), each with lambda, eps and a weight per slot (0 = unused).
// A unit's energy density is sqrt(sum_s w_s^2 |D_s z|^2 + eps^2) - eps and its
// flux p_s = w_s D_s z / max(sqrt(.), 1e-12) (ndops.py:66-135, tv_nd.py:59-86);
// the gradient adds -lambda * sum_s (p_s(v) - p_s(v - e_s)), p_s(v - e_s) = 0
// on the first slice (bwd_diff, ndops.py:45-59).  All loops run over the
// compile-time maxima with runtime guards so every array stays in registers.
constexpr int MAX_TERMS = 4;     // user-visible terms (energy slots out[0..3])
constexpr int NSLOT = 4;
constexpr int NUNIT = 8;

struct TVPlan {
  int F;
  unsigned n;                    // voxels (F * prod S), < 2^31
  int ns;                        // slots in use
  unsigned stride[NSLOT];
  int size[NSLOT];
  int nu;                        // units in use
  float w[NUNIT][NSLOT];         // per-slot weight of each unit (0 = not in unit)
  float lam[NUNIT];
  float eps[NUNIT];
  int term_of[NUNIT];            // user term each unit belongs to
  unsigned diag_mask;            // bit (s*NSLOT+s2): some unit couples slots s and s2
  // v / stride and q % size by multiply-shift (numerators < 2^31): magic, shift
  unsigned st_m[NSLOT], sz_m[NSLOT];
  int st_s[NSLOT], sz_s[NSLOT];
};

// q = v / d for v < 2^31 with m = ceil(2^(31+l) / d), l = ceil(log2 d), shift = l - 1
// (m = 0 encodes d = 1): Granlund-Montgomery division by an invariant integer.
__device__ __forceinline__ unsigned magic_div(unsigned v, unsigned m, int sh) {
  return m ? (__umulhi(v, m) >> sh) : v;
}

// coordinate of voxel v along slot s: (v / stride) % size
__device__ __forceinline__ int slot_coord(const TVPlan& P, int s, unsigned v) {
  const unsigned q = magic_div(v, P.st_m[s], P.st_s[s]);
  return (int)(q - magic_div(q, P.sz_m[s], P.sz_s[s]) * (unsigned)P.size[s]);
}

// sqrt(q + e^2) - e = q / (sqrt(q + e^2) + e), without cancellation for q << e^2;
// *inv receives 1 / sqrt(q + e^2)
__device__ __forceinline__ float huber_excess(float q, float e, float* inv) {
  const float s2 = q + e * e;
  const float r = rsqrtf(s2);
  if (inv) *inv = r;
  return __fdividef(q, fmaf(s2, r, e));
}

__device__ __forceinline__ float2 zload(const float2* __restrict__ x, const float2* __restrict__ d, float t,
                                        unsigned i) {
  float2 v = x[i];
  if (d) {
    float2 w = d[i];
    v.x = fmaf(t, w.x, v.x);
    v.y = fmaf(t, w.y, v.y);
  }
  return v;
}

// Gradient pass: g_out = g_base + t*g_dir - sum_u lam_u div p_u  at z = x + t d,
// with FP64 reductions:
//   slot 0..MAX_TERMS-1  E_T = lam_T * sum e_T
//   then gdot = Re<g,d>, rho = <g,g/D>, zn2 = |z|^2, dn2 = |d|^2,
//        gpg = <g_prev,g/D>, gpgp = <g_prev,g_prev/D>, dgp = Re<d,g_prev>
constexpr int GP_NV = MAX_TERMS + 7;

struct GradArgs {
  const float2* x;
  const float2* d;
  const double* t_dev;
  double t_host;
  const float2* g_base;
  const float2* g_dir;
  float2* g_out;
  const float* diag;     // (ndiag) broadcast, or null
  long long ndiag;
  const float2* g_prev;
  const double* skip;
  int skip_if_zero;
};

template <int NS, int NU>
struct TVGrad {
  static constexpr int NT = RED_THREADS, MINB = (NS <= 3 ? 4 : 1);
  static constexpr const char* FAMILY = "tv_grad";
  static constexpr int MAXG = 16;
  static __device__ __forceinline__ void run(const VBlock& vb, const GradArgs& a, const TVPlan& P,
      double* __restrict__ partials, const RedOut& ro) {
    // dot products (which may cancel) accumulate in FP64 per thread; the TV
    // energies (non-negative terms) in FP32 per thread; reductions in FP64
    double acc[GP_NV];
  #pragma unroll
    for (int j = 0; j < GP_NV; ++j) acc[j] = 0.0;
    float eacc[MAX_TERMS];
  #pragma unroll
    for (int j = 0; j < MAX_TERMS; ++j) eacc[j] = 0.f;
    if (a.skip && (a.skip_if_zero ? (*a.skip == 0.0) : (*a.skip != 0.0))) return;   // uniform: out untouched
    const bool sk = false;
    const float t = (float)(a.t_dev ? *a.t_dev : a.t_host);
    const unsigned stride_all = vb.nx * blockDim.x;
    if (!sk) {
      for (unsigned v = vb.x * blockDim.x + threadIdx.x; v < P.n; v += stride_all) {
        int c[NS];
        bool hn[NS], hp[NS];
        float2 zn[NS], zp[NS];
        const float2 zv = zload(a.x, a.d, t, v);
  #pragma unroll
        for (int s = 0; s < NS; ++s) {
          c[s] = 0;
          hn[s] = hp[s] = false;
          zn[s] = zp[s] = make_float2(0.f, 0.f);
          if (s < P.ns) {
            c[s] = slot_coord(P, s, v);
            hn[s] = c[s] + 1 < P.size[s];
            hp[s] = c[s] > 0;
            if (hn[s]) zn[s] = zload(a.x, a.d, t, v + P.stride[s]);
            if (hp[s]) zp[s] = zload(a.x, a.d, t, v - P.stride[s]);
          }
        }
        // forward differences at v
        float2 D[NS];
  #pragma unroll
        for (int s = 0; s < NS; ++s)
          D[s] = hn[s] ? make_float2(zn[s].x - zv.x, zn[s].y - zv.y) : make_float2(0.f, 0.f);
        // forward differences at v - e_s, along every slot s2: Dp[s][s2]
        float2 Dp[NS][NS];
  #pragma unroll
        for (int s = 0; s < NS; ++s) {
  #pragma unroll
          for (int s2 = 0; s2 < NS; ++s2) {
            Dp[s][s2] = make_float2(0.f, 0.f);
            if (!hp[s]) continue;
            if (s2 == s) {
              Dp[s][s2] = make_float2(zv.x - zp[s].x, zv.y - zp[s].y);
            } else if ((P.diag_mask >> (s * NSLOT + s2)) & 1u) {
              if (hn[s2]) {
                float2 zd = zload(a.x, a.d, t, v - P.stride[s] + P.stride[s2]);
                Dp[s][s2] = make_float2(zd.x - zp[s].x, zd.y - zp[s].y);
              }
            }
          }
        }
        float gx = 0.f, gy = 0.f;
        if (a.g_base) { float2 b = a.g_base[v]; gx = b.x; gy = b.y; }
        if (a.g_dir) { float2 b = a.g_dir[v]; gx = fmaf(t, b.x, gx); gy = fmaf(t, b.y, gy); }
  #pragma unroll
        for (int u = 0; u < NU; ++u) {
          if (u >= P.nu) continue;
          const float e2 = P.eps[u] * P.eps[u];
          float ss = 0.f;
  #pragma unroll
          for (int s = 0; s < NS; ++s) {
            const float w = P.w[u][s];
            float2 q = make_float2(w * D[s].x, w * D[s].y);
            ss += q.x * q.x + q.y * q.y;
          }
          float inv;
          const float ex = huber_excess(ss, P.eps[u], &inv);
          const int ti = P.term_of[u];
  #pragma unroll
          for (int tt = 0; tt < MAX_TERMS; ++tt)
            if (tt == ti) eacc[tt] = fmaf(P.lam[u], ex, eacc[tt]);
          float dx = 0.f, dy = 0.f;
  #pragma unroll
          for (int s = 0; s < NS; ++s) {
            const float w = P.w[u][s];
            if (w == 0.f) continue;
            dx += w * D[s].x * inv;
            dy += w * D[s].y * inv;
            if (hp[s]) {
              float ssp = 0.f;
  #pragma unroll
              for (int s2 = 0; s2 < NS; ++s2) {
                const float w2 = P.w[u][s2];
                float2 q = make_float2(w2 * Dp[s][s2].x, w2 * Dp[s][s2].y);
                ssp += q.x * q.x + q.y * q.y;
              }
              const float invp = rsqrtf(ssp + e2);
              dx -= w * Dp[s][s].x * invp;
              dy -= w * Dp[s][s].y * invp;
            }
          }
          gx = fmaf(-P.lam[u], dx, gx);
          gy = fmaf(-P.lam[u], dy, gy);
        }
        if (a.g_out) a.g_out[v] = make_float2(gx, gy);
        float2 dv = a.d ? a.d[v] : make_float2(0.f, 0.f);
        const float Dv = a.diag ? a.diag[v % a.ndiag] : 1.f;
        const int o = MAX_TERMS;
        acc[o + 0] += (double)(gx * dv.x + gy * dv.y);
        acc[o + 1] += (double)((gx * gx + gy * gy) / Dv);
        acc[o + 2] += (double)(zv.x * zv.x + zv.y * zv.y);
        acc[o + 3] += (double)(dv.x * dv.x + dv.y * dv.y);
        if (a.g_prev) {
          float2 gp = a.g_prev[v];
          acc[o + 4] += (double)((gp.x * gx + gp.y * gy) / Dv);
          acc[o + 5] += (double)((gp.x * gp.x + gp.y * gp.y) / Dv);
          acc[o + 6] += (double)(dv.x * gp.x + dv.y * gp.y);
        }
      }
    }
  #pragma unroll
    for (int j = 0; j < MAX_TERMS; ++j) acc[j] = (double)eacc[j];
    block_reduce_finish<GP_NV>(vb, acc, partials, ro);
  }
};
template <int NS, int NU>
__global__ void __launch_bounds__(RED_THREADS, NS <= 3 ? 4 : 1) grad_kernel(GradArgs a, TVPlan P,
    double* __restrict__ partials, RedOut ro) {
  TVGrad<NS, NU>::run(hw_block(), a, P, partials, ro);
}

// Sum of all unit energies at z = x + t_j d for J <= MT_MAX_J step sizes, one
// pass.  Per slot the differences A = D x and B = D d are loaded once; per unit
// |D z(t)|^2 = sum_s w_s^2 |A_s + t B_s|^2 = alpha + 2 beta t + gamma t^2 is a
// quadratic in t whose three coefficients are formed once per voxel, so each
// trial step costs two FMAs and a square root per unit.
constexpr int MT_MAX_J = 24;

template <int NS, int NU, int JMAX>
struct TVMulti {
  static constexpr int NT = RED_THREADS, MINB = (JMAX <= 8 ? 4 : 1);
  static constexpr const char* FAMILY = "tv_multi";
  static constexpr int MAXG = 16;
  static __device__ __forceinline__ void run(const VBlock& vb, const float2* __restrict__ x,
      const float2* __restrict__ d, const double* __restrict__ ts, int J, const TVPlan& P, const double* skip,
      double* __restrict__ partials, const RedOut& ro) {
    // energies are sums of non-negative terms: a thread sums its ~n / (blocks x threads)
    // voxels in FP32, the block and grid reductions run in FP64
    float facc[JMAX];
  #pragma unroll
    for (int j = 0; j < JMAX; ++j) facc[j] = 0.f;
    if (skipped(skip) != 0.0) return;   // uniform over the grid: no partials, no counter
    const bool sk = false;
    __shared__ float tf[MT_MAX_J];   // trial steps, broadcast from shared memory
    if (threadIdx.x < MT_MAX_J) tf[threadIdx.x] = threadIdx.x < J ? (float)ts[threadIdx.x] : 0.f;
    __syncthreads();
    const unsigned stride_all = vb.nx * blockDim.x;
    if (!sk) {
      for (unsigned v = vb.x * blockDim.x + threadIdx.x; v < P.n; v += stride_all) {
        const float2 xv = x[v], dv = d[v];
        float2 A[NS], B[NS];
  #pragma unroll
        for (int s = 0; s < NS; ++s) {
          A[s] = B[s] = make_float2(0.f, 0.f);
          if (s < P.ns && slot_coord(P, s, v) + 1 < P.size[s]) {
            const float2 xn = x[v + P.stride[s]], dn = d[v + P.stride[s]];
            A[s] = make_float2(xn.x - xv.x, xn.y - xv.y);
            B[s] = make_float2(dn.x - dv.x, dn.y - dv.y);
          }
        }
        float al[NU], be2[NU], ga[NU];
  #pragma unroll
        for (int u = 0; u < NU; ++u) {
          al[u] = be2[u] = ga[u] = 0.f;
          if (u >= P.nu) continue;
  #pragma unroll
          for (int s = 0; s < NS; ++s) {
            const float w2 = P.w[u][s] * P.w[u][s];
            al[u] = fmaf(w2, A[s].x * A[s].x + A[s].y * A[s].y, al[u]);
            be2[u] = fmaf(2.f * w2, A[s].x * B[s].x + A[s].y * B[s].y, be2[u]);
            ga[u] = fmaf(w2, B[s].x * B[s].x + B[s].y * B[s].y, ga[u]);
          }
        }
  #pragma unroll
        for (int j = 0; j < JMAX; ++j) {
          if (j >= J) continue;
          const float t = tf[j];
          float e = 0.f;
  #pragma unroll
          for (int u = 0; u < NU; ++u) {
            if (u >= P.nu) continue;
            const float q = fmaxf(fmaf(t, fmaf(t, ga[u], be2[u]), al[u]), 0.f);
            e = fmaf(P.lam[u], huber_excess(q, P.eps[u], nullptr), e);
          }
          facc[j] += e;
        }
      }
    }
    double acc[JMAX];
  #pragma unroll
    for (int j = 0; j < JMAX; ++j) acc[j] = (double)facc[j];
    block_reduce_finish<JMAX>(vb, acc, partials, ro);
  }
};
template <int NS, int NU, int JMAX>
__global__ void __launch_bounds__(RED_THREADS, JMAX <= 8 ? 4 : 1) tv_multi_kernel(const float2* __restrict__ x,
    const float2* __restrict__ d, const double* __restrict__ ts, int J, TVPlan P, const double* skip,
    double* __restrict__ partials, RedOut ro) {
  TVMulti<NS, NU, JMAX>::run(hw_block(), x, d, ts, J, P, skip, partials, ro);
}

// ---------------------------------------------------------------------------
// NCG controller kernels (single thread; scalar slots in `s`)
// ---------------------------------------------------------------------------
enum Slot {
  S_T = 0, S_LS_OK, S_DONE, S_REASON, S_ITER, S_F0, S_G0D, S_FT, S_GDT,
  S_ERR, S_ERD, S_EDD, S_RHO_PREV, S_RHO_INIT, S_BETA,
  S_CUM_X, S_CUM_G, S_CUM_S, S_NTRIAL, S_NRESTART, S_NOMORE,
  S_GQ0, S_GQ1, S_GQ2,   // quadratic (graph Laplacian) energy and its slope / curvature along d
  S_RED = 24,            // reduction outputs of the gradient pass (GP_NV values)
  S_EJ = 48,             // multi-t energies (MT_MAX_J values)
  S_G0D_NEXT = 80,
  S_COUNT = 96
};

struct NCGCfg {
  double c1;
  double ls_beta;
  int ls_max_iter;
  int max_iter;
  double tol_g;
  double tol_step;
  int stop_window;       // 0 = off
  double stop_tol;
  int direction;         // 0 FR, 1 PR+, 2 DY
  int nhist;             // history row capacity
};

constexpr int HIST_COLS = 11;  // f0, gdot0, gdot_t, t, cum_x, cum_g, cum_s, xn, gn, sn, f_t

// cfg lives in device memory (so a captured graph sees later edits)
__device__ __forceinline__ NCGCfg load_cfg(const double* c) {
  NCGCfg g;
  g.c1 = c[0];
  g.ls_beta = c[1];
  g.ls_max_iter = (int)c[2];
  g.max_iter = (int)c[3];
  g.tol_g = c[4];
  g.tol_step = c[5];
  g.stop_window = (int)c[6];
  g.stop_tol = c[7];
  g.direction = (int)c[8];
  g.nhist = (int)c[9];
  return g;
}

// Armijo selection on the multi-t energies: t_0 = 0, t_j = beta^(j-1).
struct ArmijoSelect {
  static constexpr int NT = 32, MINB = 1;
  static constexpr const char* FAMILY = "armijo_select";
  static constexpr int MAXG = 16;
  static __device__ __forceinline__ void run(const VBlock& vb, double* s, const double* cfg_dev) {
    if (threadIdx.x != 0) return;
    const NCGCfg cfg = load_cfg(cfg_dev);
    if (s[S_DONE] != 0.0) {
      s[S_LS_OK] = 0.0;
      return;
    }
    const double err = s[S_ERR], erd = s[S_ERD], edd = s[S_EDD];
    const double f0 = 0.5 * err + s[S_EJ + 0];
    const double g0d = s[S_G0D];
    s[S_F0] = f0;
    bool bad = !(g0d < 0.0) || isnan(g0d) || isinf(g0d);
    if (bad) {
      s[S_LS_OK] = 0.0;
      s[S_DONE] = 1.0;
      s[S_REASON] = 1.0;
      s[S_T] = 0.0;
      return;
    }
    double t = 1.0;
    const int jmax = cfg.ls_max_iter < MT_MAX_J - 1 ? cfg.ls_max_iter : MT_MAX_J - 1;
    for (int j = 1; j <= jmax; ++j) {
      double ft = 0.5 * (err + 2.0 * t * erd + t * t * edd) + s[S_EJ + j];
      if (ft <= f0 + cfg.c1 * t * g0d) {
        s[S_T] = t;
        s[S_FT] = ft;
        s[S_LS_OK] = 1.0;
        s[S_NTRIAL] = (double)j;
        return;
      }
      t *= cfg.ls_beta;
    }
    s[S_T] = t;
    s[S_LS_OK] = 0.0;
    s[S_DONE] = 1.0;
    s[S_REASON] = 1.0;
  }
};
__global__ void armijo_select_kernel(double* s, const double* cfg_dev) {
  ArmijoSelect::run(hw_block(), s, cfg_dev);
}

// Two-phase Armijo selection over the same backtracking sequence: phase 1
// tries j = 1 .. J1-1 on the energies of a first tv_multi pass over J1 steps;
// when none satisfies f(t) <= f(0) + c1 t f'(0) it clears S_NOMORE and phase 2,
// after a second tv_multi pass over the remaining steps, continues at j = J1.
// S_NOMORE = 1 whenever the second pass and phase 2 have nothing to do.
struct ArmijoPhase {
  static constexpr int NT = 32, MINB = 1;
  static constexpr const char* FAMILY = "armijo_phase";
  static constexpr int MAXG = 16;
  static __device__ __forceinline__ void run(const VBlock& vb, double* s, const double* cfg_dev, int J1,
      int phase) {
    if (threadIdx.x != 0) return;
    const NCGCfg cfg = load_cfg(cfg_dev);
    const int jmax = cfg.ls_max_iter < MT_MAX_J - 1 ? cfg.ls_max_iter : MT_MAX_J - 1;
    const double err = s[S_ERR], erd = s[S_ERD], edd = s[S_EDD];
    double t;
    int j0, j1;
    if (phase == 1) {
      s[S_NOMORE] = 1.0;
      if (s[S_DONE] != 0.0) {
        s[S_LS_OK] = 0.0;
        return;
      }
      const double f0 = 0.5 * err + s[S_EJ + 0];
      const double g0d = s[S_G0D];
      s[S_F0] = f0;
      if (!(g0d < 0.0) || isnan(g0d) || isinf(g0d)) {
        s[S_LS_OK] = 0.0;
        s[S_DONE] = 1.0;
        s[S_REASON] = 1.0;
        s[S_T] = 0.0;
        return;
      }
      t = 1.0;
      j0 = 1;
      j1 = J1 - 1 < jmax ? J1 - 1 : jmax;
    } else {
      if (s[S_NOMORE] != 0.0) return;
      s[S_NOMORE] = 1.0;
      t = s[S_T];
      j0 = J1;
      j1 = jmax;
    }
    const double f0 = s[S_F0], g0d = s[S_G0D];
    for (int j = j0; j <= j1; ++j) {
      double ft = 0.5 * (err + 2.0 * t * erd + t * t * edd) + s[S_EJ + j];
      if (ft <= f0 + cfg.c1 * t * g0d) {
        s[S_T] = t;
        s[S_FT] = ft;
        s[S_LS_OK] = 1.0;
        s[S_NTRIAL] = (double)j;
        return;
      }
      t *= cfg.ls_beta;
    }
    s[S_T] = t;
    s[S_LS_OK] = 0.0;
    if (phase == 1 && j1 < jmax) {
      s[S_NOMORE] = 0.0;   // the remaining steps decide
      return;
    }
    s[S_DONE] = 1.0;
    s[S_REASON] = 1.0;
  }
};
__global__ void armijo_phase_kernel(double* s, const double* cfg_dev, int J1, int phase) {
  ArmijoPhase::run(hw_block(), s, cfg_dev, J1, phase);
}

// After the gradient pass at the accepted t: history row, stopping tests and
// the direction coefficient beta.
struct NCGControl {
  static constexpr int NT = 32, MINB = 1;
  static constexpr const char* FAMILY = "ncg_control";
  static constexpr int MAXG = 16;
  static __device__ __forceinline__ void run(const VBlock& vb, double* s, double* hist, const double* cfg_dev,
      int nterms, int have_ft) {
    if (threadIdx.x != 0) return;
    const NCGCfg cfg = load_cfg(cfg_dev);
    if (s[S_LS_OK] == 0.0) return;
    const double* r = s + S_RED;
    double Esum = 0.0;
    for (int i = 0; i < nterms; ++i) Esum += r[i];
    const double gdot = r[MAX_TERMS + 0], rho = r[MAX_TERMS + 1];
    const double xn = sqrt(fmax(r[MAX_TERMS + 2], 0.0)), sn = sqrt(fmax(r[MAX_TERMS + 3], 0.0));
    const double gn = sqrt(fmax(rho, 0.0));
    if (!have_ft) {
      // objective at the accepted point from the k-space scalars
      double t = s[S_T];
      s[S_FT] = 0.5 * (s[S_ERR] + 2.0 * t * s[S_ERD] + t * t * s[S_EDD]) + Esum;
    }
    s[S_GDT] = gdot;
    s[S_CUM_X] += xn;
    s[S_CUM_G] += gn;
    s[S_CUM_S] += sn;
    int k = (int)s[S_ITER];
    if (k < cfg.nhist) {
      double* h = hist + (long long)k * HIST_COLS;
      h[0] = s[S_F0];
      h[1] = s[S_G0D];
      h[2] = gdot;
      h[3] = s[S_T];
      h[4] = s[S_CUM_X];
      h[5] = s[S_CUM_G];
      h[6] = s[S_CUM_S];
      h[7] = xn;
      h[8] = gn;
      h[9] = sn;
      h[10] = s[S_FT];
    }
    s[S_ITER] = (double)(k + 1);
    // reference convergence test (solvers/utils.py:40-43)
    if (gn <= (1.0 + xn) * cfg.tol_g && sn <= (1.0 + xn) * cfg.tol_step) {
      s[S_DONE] = 1.0;
      s[S_REASON] = 2.0;
      return;
    }
    // windowed relative objective change on the accepted objectives
    if (cfg.stop_window > 0 && k + 1 >= cfg.stop_window && k < cfg.nhist) {
      double fk = hist[(long long)k * HIST_COLS + 10];
      int kk = k + 1 - cfg.stop_window;    // accepted-objective index kk-1 ... use f0 of row kk
      double fw = hist[(long long)kk * HIST_COLS + 0];
      if ((fw - fk) <= cfg.stop_window * cfg.stop_tol * fabs(fk)) {
        s[S_DONE] = 1.0;
        s[S_REASON] = 3.0;
        return;
      }
    }
    if (k + 1 >= cfg.max_iter) {
      s[S_DONE] = 1.0;
      s[S_REASON] = 4.0;
      return;
    }
    double beta;
    if (cfg.direction == 0) {
      if (s[S_RHO_INIT] == 0.0) {
        s[S_RHO_PREV] = rho;
        s[S_RHO_INIT] = 1.0;
      }
      beta = rho / fmax(s[S_RHO_PREV], 1e-20);
      s[S_RHO_PREV] = rho;
    } else if (cfg.direction == 1) {
      double num = rho - r[MAX_TERMS + 4];
      double den = r[MAX_TERMS + 5];
      beta = fmax(num / fmax(den, 1e-20), 0.0);
    } else {
      double num = rho;
      double den = gdot - r[MAX_TERMS + 6];
      beta = num / fmax(den, 1e-20);
    }
    s[S_BETA] = beta;
  }
};
__global__ void ncg_control_kernel(double* s, double* hist, const double* cfg_dev, int nterms, int have_ft) {
  NCGControl::run(hw_block(), s, hist, cfg_dev, nterms, have_ft);
}

// Accept + direction update (one pass):
//   x += t d ; gr += t gAd (if gr) ; then, unless done: d = beta d - g/D,
//   g_prev = g (if g_prev), and Re<g, d_new> for the next slope at t = 0.
struct NCGUpdate {
  static constexpr int NT = RED_THREADS, MINB = 4;
  static constexpr const char* FAMILY = "ncg_update";
  static constexpr int MAXG = 16;
  static __device__ __forceinline__ void run(const VBlock& vb, long long n, float2* __restrict__ x,
      float2* __restrict__ d, const float2* __restrict__ g, float2* __restrict__ gr,
      const float2* __restrict__ gAd, float2* __restrict__ g_prev, const float* __restrict__ diag,
      long long ndiag, const double* __restrict__ s, double* __restrict__ partials, const RedOut& ro) {
    double acc[1] = {0.0};
    const bool ok = s[S_LS_OK] != 0.0;
    const bool upd_dir = ok && s[S_DONE] == 0.0;
    const float t = (float)s[S_T];
    const float beta = (float)s[S_BETA];
    const long long stride = (long long)vb.nx * blockDim.x;
    // one element: its loaded values in, its stores and its term of <g, d> out
    auto element = [&](long long i, float2 dv, float2 xv, float2 a, float2 b, float2 gv, float Dv) {
      // x.add_(d * t) (cg.py:205-207)
      xv.x = __fadd_rn(xv.x, __fmul_rn(dv.x, t));
      xv.y = __fadd_rn(xv.y, __fmul_rn(dv.y, t));
      x[i] = xv;
      if (gr) {
        a.x = fmaf(t, b.x, a.x);
        a.y = fmaf(t, b.y, a.y);
        gr[i] = a;
      }
      if (upd_dir) {
        // d.mul_(beta); d.addcdiv_(g, D, value=-1)  (directions.py:158-161)
        float nx = __fadd_rn(__fmul_rn(dv.x, beta), -(gv.x / Dv));
        float ny = __fadd_rn(__fmul_rn(dv.y, beta), -(gv.y / Dv));
        d[i] = make_float2(nx, ny);
        if (g_prev) g_prev[i] = gv;
        acc[0] += (double)(gv.x * nx + gv.y * ny);
      }
    };
    const float2 z2 = make_float2(0.f, 0.f);
    if (ok) {
      // two elements of the grid-stride sequence per pass, all their loads issued
      // before either is stored (the buffers are distinct): the same values and
      // summation order as one element per pass
      long long i = (long long)vb.x * blockDim.x + threadIdx.x;
      for (; i + stride < n; i += 2 * stride) {
        const long long j = i + stride;
        const float2 dv0 = d[i], dv1 = d[j], xv0 = x[i], xv1 = x[j];
        const float2 a0 = gr ? gr[i] : z2, b0 = gr ? gAd[i] : z2, a1 = gr ? gr[j] : z2, b1 = gr ? gAd[j] : z2;
        const float2 g0 = upd_dir ? g[i] : z2, g1 = upd_dir ? g[j] : z2;
        const float D0 = upd_dir && diag ? diag[i % ndiag] : 1.f, D1 = upd_dir && diag ? diag[j % ndiag] : 1.f;
        element(i, dv0, xv0, a0, b0, g0, D0);
        element(j, dv1, xv1, a1, b1, g1, D1);
      }
      if (i < n) {
        element(i, d[i], x[i], gr ? gr[i] : z2, gr ? gAd[i] : z2, upd_dir ? g[i] : z2,
                upd_dir && diag ? diag[i % ndiag] : 1.f);
      }
    }
    block_reduce_finish<1>(vb, acc, partials, ro);
  }
};
__global__ void __launch_bounds__(RED_THREADS) ncg_update_kernel(long long n, float2* __restrict__ x,
    float2* __restrict__ d, const float2* __restrict__ g, float2* __restrict__ gr,
    const float2* __restrict__ gAd, float2* __restrict__ g_prev, const float* __restrict__ diag,
    long long ndiag, const double* __restrict__ s, double* __restrict__ partials, RedOut ro) {
  NCGUpdate::run(hw_block(), n, x, d, g, gr, gAd, g_prev, diag, ndiag, s, partials, ro);
}

// d = -g/D (priming: cg.py:182-185) and Re<g,d>
struct Steepest {
  static constexpr int NT = RED_THREADS, MINB = 5;
  static constexpr const char* FAMILY = "steepest";
  static constexpr int MAXG = 16;
  static __device__ __forceinline__ void run(const VBlock& vb, long long n, float2* __restrict__ d,
      const float2* __restrict__ g, float2* __restrict__ g_prev, const float* __restrict__ diag,
      long long ndiag, double* __restrict__ partials, const RedOut& ro) {
    double acc[1] = {0.0};
    const long long stride = (long long)vb.nx * blockDim.x;
    for (long long i = (long long)vb.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      float2 gv = g[i];
      float Dv = diag ? diag[i % ndiag] : 1.f;
      float2 dv = make_float2(-(gv.x / Dv), -(gv.y / Dv));
      d[i] = dv;
      if (g_prev) g_prev[i] = gv;
      acc[0] += (double)(gv.x * dv.x + gv.y * dv.y);
    }
    block_reduce_finish<1>(vb, acc, partials, ro);
  }
};
__global__ void __launch_bounds__(RED_THREADS) steepest_kernel(long long n, float2* __restrict__ d,
    const float2* __restrict__ g, float2* __restrict__ g_prev, const float* __restrict__ diag, long long ndiag,
    double* __restrict__ partials, RedOut ro) {
  Steepest::run(hw_block(), n, d, g, g_prev, diag, ndiag, partials, ro);
}

// Optional restart (not in the reference): when the updated direction is not a
// descent direction (Re<g, d> >= 0 or not finite) it becomes steepest descent
// -g/D.  The direction pass leaves the slots alone so that every block sees the
// same decision; restart_slot_kernel then sets the slope to -<g, g/D> (the rho
// of the gradient pass) and counts the restart.
__device__ __forceinline__ bool needs_restart(const double* s) {
  return s[S_LS_OK] != 0.0 && s[S_DONE] == 0.0 && !(s[S_G0D] < 0.0);
}

struct RestartDir {
  static constexpr int NT = RED_THREADS, MINB = 5;
  static constexpr const char* FAMILY = "restart_dir";
  static constexpr int MAXG = 16;
  static __device__ __forceinline__ void run(const VBlock& vb, long long n, float2* __restrict__ d,
      const float2* __restrict__ g, const float* __restrict__ diag, long long ndiag,
      const double* __restrict__ s) {
    if (!needs_restart(s)) return;
    const long long stride = (long long)vb.nx * blockDim.x;
    for (long long i = (long long)vb.x * blockDim.x + threadIdx.x; i < n; i += stride) {
      const float2 gv = g[i];
      const float Dv = diag ? diag[i % ndiag] : 1.f;
      d[i] = make_float2(-(gv.x / Dv), -(gv.y / Dv));
    }
  }
};
__global__ void __launch_bounds__(RED_THREADS) restart_dir_kernel(long long n, float2* __restrict__ d,
    const float2* __restrict__ g, const float* __restrict__ diag, long long ndiag, const double* __restrict__ s) {
  RestartDir::run(hw_block(), n, d, g, diag, ndiag, s);
}

struct RestartSlot {
  static constexpr int NT = 32, MINB = 1;
  static constexpr const char* FAMILY = "restart_slot";
  static constexpr int MAXG = 16;
  static __device__ __forceinline__ void run(const VBlock& vb, double* s) {
    if (threadIdx.x != 0 || !needs_restart(s)) return;
    s[S_G0D] = -s[S_RED + MAX_TERMS + 1];
    s[S_G0D_NEXT] = s[S_G0D];
    s[S_NRESTART] += 1.0;
  }
};
__global__ void restart_slot_kernel(double* s) {
  RestartSlot::run(hw_block(), s);
}

// ||r||^2 after an accepted step when r is not kept (Toeplitz schedule):
// ||r + t Ad||^2 = err + 2 t Re<r, Ad> + t^2 ||Ad||^2.
struct ErrStep {
  static constexpr int NT = 32, MINB = 1;
  static constexpr const char* FAMILY = "err_step";
  static constexpr int MAXG = 16;
  static __device__ __forceinline__ void run(const VBlock& vb, double* s) {
    if (threadIdx.x != 0 || s[S_LS_OK] == 0.0) return;
    const double t = s[S_T];
    s[S_ERR] += 2.0 * t * s[S_ERD] + t * t * s[S_EDD];
  }
};
__global__ void err_step_kernel(double* s) {
  ErrStep::run(hw_block(), s);
}

struct SetSteps {
  static constexpr int NT = 32, MINB = 1;
  static constexpr const char* FAMILY = "set_steps";
  static constexpr int MAXG = 16;
  static __device__ __forceinline__ void run(const VBlock& vb, double* ts, int J, double beta) {
    if (threadIdx.x == 0) {
      ts[0] = 0.0;
      double t = 1.0;
      for (int j = 1; j < J; ++j) {
        ts[j] = t;
        t *= beta;
      }
    }
  }
};
__global__ void set_steps_kernel(double* ts, int J, double beta) {
  SetSteps::run(hw_block(), ts, J, beta);
}

// Kernel instance for the plan's slot / unit counts (rounded up), so the
// unrolled per-voxel loops keep only the accumulators in use.
struct GradLaunch {
  template <int NS, int NU, class... A>
  static int go(int nb, cudaStream_t st, A... args) {
    return mrb::launch<TVGrad<NS, NU>>(grad_kernel<NS, NU>, dim3(nb), 0, st, args...);
  }
};
// trial steps per launch: up to 8 (the first Armijo phase) or up to MT_MAX_J
template <int JMAX>
struct MultiLaunch {
  template <int NS, int NU, class... A>
  static int go(int nb, cudaStream_t st, A... args) {
    return mrb::launch<TVMulti<NS, NU, JMAX>>(tv_multi_kernel<NS, NU, JMAX>, dim3(nb), 0, st, args...);
  }
};

template <class L, int NS, class... A>
int launch_tv_nu(const TVPlan& P, int nb, cudaStream_t st, A... args) {
  if (P.nu <= 1) return L::template go<NS, 1>(nb, st, args...);
  if (P.nu <= 2) return L::template go<NS, 2>(nb, st, args...);
  if (P.nu <= 4) return L::template go<NS, 4>(nb, st, args...);
  return L::template go<NS, NUNIT>(nb, st, args...);
}

template <class L, class... A>
int launch_tv(const TVPlan& P, int nb, cudaStream_t st, A... args) {
  if (P.ns <= 1) return launch_tv_nu<L, 1>(P, nb, st, args...);
  if (P.ns <= 2) return launch_tv_nu<L, 2>(P, nb, st, args...);
  if (P.ns <= 3) return launch_tv_nu<L, 3>(P, nb, st, args...);
  return launch_tv_nu<L, NSLOT>(P, nb, st, args...);
}

// grid of the TV passes: one wave of `per_sm` resident 256-thread blocks on every SM
int tv_grid(int per_sm = 3) {
  static int sms = 0;
  if (!sms) {
    int dev = 0, n = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    sms = n;
  }
  return std::max(1, std::min(RED_MAX_BLOCKS, per_sm * sms));
}

int build_plan(TVPlan& P, int nd, const int* S, int F, const mrb_tv_term* terms, int nterms) {
  MRB_REQUIRE(nd >= 1 && nd <= 3, "spatial nd must be 1..3");
  MRB_REQUIRE(F >= 1, "frames must be positive");
  MRB_REQUIRE(nterms >= 0 && nterms <= MAX_TERMS, "at most %d TV terms", MAX_TERMS);
  MRB_REQUIRE(nterms == 0 || terms != nullptr, "null terms");
  memset(&P, 0, sizeof(P));
  P.F = F;
  // axis geometry of (F, 1, *S): axis 0 = frames, 2.. = spatial
  long long astride[5] = {0, 0, 0, 0, 0};
  int asize[5] = {F, 1, 1, 1, 1};
  long long st = 1;
  for (int a = 2 + nd - 1; a >= 2; --a) {
    MRB_REQUIRE(S[a - 2] >= 1, "bad spatial size");
    asize[a] = S[a - 2];
    astride[a] = st;
    st *= S[a - 2];
  }
  astride[0] = st;
  long long n = st * F;
  MRB_REQUIRE(n < (1LL << 31), "image too large for the TV kernels (%lld voxels)", n);
  P.n = (unsigned)n;
  int slot_of[5] = {-1, -1, -1, -1, -1};
  int period = 0;
  for (int i = 0; i < nterms; ++i)
    if (terms[i].enabled && terms[i].frame_period > 0) {
      MRB_REQUIRE(period == 0 || period == terms[i].frame_period, "TV terms disagree on the frame period");
      MRB_REQUIRE(F % terms[i].frame_period == 0, "frame period %d does not divide %d frames",
                  terms[i].frame_period, F);
      period = terms[i].frame_period;
    }
  if (period > 0) asize[0] = period;   // coordinates along frames are taken within a series
  int k = 0;
  for (int i = 0; i < nterms; ++i) {
    const mrb_tv_term& t = terms[i];
    if (!t.enabled || t.weight == 0.f) continue;
    MRB_REQUIRE(t.naxes >= 0 && t.naxes <= 4, "at most 4 axes per TV term");
    int ax[4], na = 0;
    float aw[4];
    for (int q = 0; q < t.naxes; ++q) {
      int a = t.axes[q];
      MRB_REQUIRE(a >= 0 && a < 2 + nd, "TV axis %d out of range", a);
      if (a == 1 || asize[a] == 1) continue;      // size-1 axis: forward difference is zero
      if (slot_of[a] < 0) {
        MRB_REQUIRE(P.ns < NSLOT, "too many distinct TV axes");
        slot_of[a] = P.ns;
        P.stride[P.ns] = (unsigned)astride[a];
        P.size[P.ns] = asize[a];
        P.ns++;
      }
      ax[na] = slot_of[a];
      aw[na] = t.axis_weights[q];
      ++na;
    }
    if (na == 0) continue;
    if (t.isotropic) {
      MRB_REQUIRE(P.nu < NUNIT, "too many TV units");
      int u = P.nu++;
      P.lam[u] = t.weight;
      P.eps[u] = t.eps;
      P.term_of[u] = k;
      for (int q = 0; q < na; ++q) P.w[u][ax[q]] = aw[q];
      for (int q = 0; q < na; ++q)
        for (int q2 = 0; q2 < na; ++q2)
          if (ax[q] != ax[q2]) P.diag_mask |= 1u << (ax[q] * NSLOT + ax[q2]);
    } else {
      for (int q = 0; q < na; ++q) {
        MRB_REQUIRE(P.nu < NUNIT, "too many TV units");
        int u = P.nu++;
        P.lam[u] = t.weight;
        P.eps[u] = t.eps;
        P.term_of[u] = k;
        P.w[u][ax[q]] = aw[q];
      }
    }
    ++k;
  }
  auto magic = [](unsigned dv, unsigned* m, int* sh) {
    if (dv <= 1) {
      *m = 0;
      *sh = 0;
      return;
    }
    int l = 0;
    while ((1ull << l) < dv) ++l;                                  // ceil(log2 dv)
    const unsigned long long p2 = 1ull << (31 + l);
    *m = (unsigned)((p2 + dv - 1) / dv);
    *sh = l - 1;
  };
  for (int q = 0; q < P.ns; ++q) {
    magic(P.stride[q], &P.st_m[q], &P.st_s[q]);
    magic((unsigned)P.size[q], &P.sz_m[q], &P.sz_s[q]);
  }
  return 0;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" int mrb_workspace_bytes(int64_t* bytes) {
  MRB_REQUIRE(bytes != nullptr, "null pointer");
  *bytes = (int64_t)RED_PART_BYTES + 256;   // block partials + completion counter
  return 0;
}

extern "C" int mrb_ncg_slot_count(int64_t* slots, int64_t* hist_cols) {
  MRB_REQUIRE(slots != nullptr && hist_cols != nullptr, "null pointer");
  *slots = S_COUNT;
  *hist_cols = HIST_COLS;
  return 0;
}

extern "C" int mrb_dots_f64(int64_t n, int npairs, const void* const* a, const void* const* b,
                            const float* const* diag, int64_t ndiag, double* out, void* ws, mrb_stream_t stream) {
  MRB_REQUIRE(n >= 0 && npairs >= 1 && npairs <= 8, "npairs must be 1..8");
  MRB_REQUIRE(a && b && out && ws, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  DotArgs d{};
  for (int j = 0; j < npairs; ++j) {
    MRB_REQUIRE(a[j] && b[j], "null operand %d", j);
    d.a[j] = (const float2*)a[j];
    d.b[j] = (const float2*)b[j];
    d.diag[j] = diag ? diag[j] : nullptr;
  }
  d.ndiag = ndiag > 0 ? ndiag : 1;
  d.n = n;
  d.npairs = npairs;
  int nb = red_blocks(n, 4);
  double* part = (double*)ws;
  switch (npairs) {
    case 1: dots_kernel<1><<<nb, RED_THREADS, 0, st>>>(d, part); break;
    case 2: dots_kernel<2><<<nb, RED_THREADS, 0, st>>>(d, part); break;
    case 3: dots_kernel<3><<<nb, RED_THREADS, 0, st>>>(d, part); break;
    case 4: dots_kernel<4><<<nb, RED_THREADS, 0, st>>>(d, part); break;
    default: dots_kernel<8><<<nb, RED_THREADS, 0, st>>>(d, part); break;
  }
  MRB_LAUNCH_CHECK();
  const int stride = npairs <= 4 ? npairs : 8;
  return finalize(part, nb, stride, npairs, out, 0, nullptr, st);
}

extern "C" int mrb_kspace_pass(int mode, int64_t n, void* r, const void* Ad, const void* Ax, const void* y,
                               const double* t_dev, double t_host, const double* skip, double* out, void* ws,
                               mrb_stream_t stream) {
  MRB_REQUIRE(mode >= 0 && mode <= 2, "bad k-space mode");
  MRB_REQUIRE(r != nullptr && ws != nullptr, "null pointer");
  MRB_REQUIRE(mode != 1 || (Ax && y), "mode 1 needs Ax and y");
  MRB_REQUIRE(mode == 1 || Ad, "modes 0/2 need Ad");
  MRB_REQUIRE(mode == 2 || out, "null output");
  cudaStream_t st = (cudaStream_t)stream;
  int nb = red_blocks(n, 4);
  double* part = (double*)ws;
  return mrb::launch<KSpace>(kspace_kernel, dim3(nb), 0, st, mode, n, (float2*)r, (const float2*)Ad,
                             (const float2*)Ax, (const float2*)y, t_dev, t_host, skip, part,
                             red_out(ws, out, mode == 0 ? 3 : 1, 0, skip));
}

extern "C" int mrb_tv_grad(int nd, const int* S, int F, const mrb_tv_term* terms, int nterms, const void* x,
                           const void* d, const double* t_dev, double t_host, const void* g_base, const void* g_dir,
                           void* g_out, const float* diag, int64_t ndiag, const void* g_prev, const double* skip,
                           int skip_if_zero, double* out, void* ws, mrb_stream_t stream) {
  MRB_REQUIRE(x != nullptr && out != nullptr && ws != nullptr, "null pointer");
  TVPlan P;
  int rc = build_plan(P, nd, S, F, terms, nterms);
  if (rc) return rc;
  GradArgs a{};
  a.x = (const float2*)x;
  a.d = (const float2*)d;
  a.t_dev = t_dev;
  a.t_host = t_host;
  a.g_base = (const float2*)g_base;
  a.g_dir = (const float2*)g_dir;
  a.g_out = (float2*)g_out;
  a.diag = diag;
  a.ndiag = ndiag > 0 ? ndiag : 1;
  a.g_prev = (const float2*)g_prev;
  a.skip = skip;
  a.skip_if_zero = skip_if_zero;
  cudaStream_t st = (cudaStream_t)stream;
  // up to 3 difference axes the gradient pass keeps to 64 registers: 4 blocks per SM
  int nb = std::min(red_blocks(P.n, 2), tv_grid(P.ns <= 3 ? 4 : 3));
  double* part = (double*)ws;
  return launch_tv<GradLaunch>(P, nb, st, a, P, part, red_out(ws, out, GP_NV, 0, nullptr));
}

extern "C" int mrb_tv_multi(int nd, const int* S, int F, const mrb_tv_term* terms, int nterms, const void* x,
                            const void* d, const double* ts, int J, const double* skip, double* out, void* ws,
                            mrb_stream_t stream) {
  MRB_REQUIRE(x != nullptr && d != nullptr && ts != nullptr && out != nullptr && ws != nullptr, "null pointer");
  MRB_REQUIRE(J >= 1 && J <= MT_MAX_J, "J must be 1..%d", MT_MAX_J);
  TVPlan P;
  int rc = build_plan(P, nd, S, F, terms, nterms);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  // up to 8 trial steps the kernel keeps to 64 registers: 4 resident blocks per SM
  int nb = std::min(red_blocks(P.n, 2), tv_grid(J <= 8 ? 4 : 3));
  double* part = (double*)ws;
  if (J <= 8)
    return launch_tv<MultiLaunch<8>>(P, nb, st, (const float2*)x, (const float2*)d, ts, J, P, skip, part,
                                     red_out(ws, out, J, 0, skip));
  return launch_tv<MultiLaunch<MT_MAX_J>>(P, nb, st, (const float2*)x, (const float2*)d, ts, J, P, skip, part,
                                          red_out(ws, out, J, 0, skip));
}

extern "C" int mrb_ncg_armijo_select(double* slots, const double* cfg, mrb_stream_t stream) {
  MRB_REQUIRE(slots != nullptr && cfg != nullptr, "null pointer");
  return mrb::launch<ArmijoSelect>(armijo_select_kernel, dim3(1), 0, (cudaStream_t)stream, slots, cfg);
}

extern "C" int mrb_ncg_armijo_phase(double* slots, const double* cfg, int J1, int phase, mrb_stream_t stream) {
  MRB_REQUIRE(slots != nullptr && cfg != nullptr, "null pointer");
  MRB_REQUIRE(phase == 1 || phase == 2, "phase must be 1 or 2");
  MRB_REQUIRE(J1 >= 2 && J1 <= MT_MAX_J, "J1 out of range");
  return mrb::launch<ArmijoPhase>(armijo_phase_kernel, dim3(1), 0, (cudaStream_t)stream, slots, cfg, J1, phase);
}

extern "C" int mrb_ncg_control(double* slots, double* hist, const double* cfg, int nterms, int have_ft,
                               mrb_stream_t stream) {
  MRB_REQUIRE(slots != nullptr && hist != nullptr && cfg != nullptr, "null pointer");
  return mrb::launch<NCGControl>(ncg_control_kernel, dim3(1), 0, (cudaStream_t)stream, slots, hist, cfg, nterms,
                                 have_ft);
}

extern "C" int mrb_ncg_update(int64_t n, void* x, void* d, const void* g, void* gr, const void* gAd, void* g_prev,
                              const float* diag, int64_t ndiag, double* slots, void* ws, mrb_stream_t stream) {
  MRB_REQUIRE(x && d && g && slots && ws, "null pointer");
  MRB_REQUIRE(!gr || gAd, "gr needs gAd");
  cudaStream_t st = (cudaStream_t)stream;
  int nb = red_blocks(n, 2);
  double* part = (double*)ws;
  // next slope at t = 0 -> S_G0D_NEXT and S_G0D
  return mrb::launch<NCGUpdate>(ncg_update_kernel, dim3(nb), 0, st, n, (float2*)x, (float2*)d, (const float2*)g,
                                (float2*)gr, (const float2*)gAd, (float2*)g_prev, diag, ndiag > 0 ? ndiag : 1, slots,
                                part, red_out(ws, slots + S_G0D_NEXT, 1, 0, nullptr, slots + S_G0D));
}

extern "C" int mrb_ncg_err_step(double* slots, mrb_stream_t stream) {
  MRB_REQUIRE(slots != nullptr, "null slots");
  return mrb::launch<ErrStep>(err_step_kernel, dim3(1), 0, (cudaStream_t)stream, slots);
}

extern "C" int mrb_ncg_restart(int64_t n, void* d, const void* g, const float* diag, int64_t ndiag, double* slots,
                               mrb_stream_t stream) {
  MRB_REQUIRE(d && g && slots, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  if (int rc = mrb::launch<RestartDir>(restart_dir_kernel, dim3(red_blocks(n, 2)), 0, st, n, (float2*)d,
                                      (const float2*)g, diag, ndiag > 0 ? ndiag : 1, slots))
    return rc;
  return mrb::launch<RestartSlot>(restart_slot_kernel, dim3(1), 0, st, slots);
}

extern "C" int mrb_ncg_steepest(int64_t n, void* d, const void* g, void* g_prev, const float* diag, int64_t ndiag,
                                double* out, void* ws, mrb_stream_t stream) {
  MRB_REQUIRE(d && g && out && ws, "null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  int nb = red_blocks(n, 2);
  double* part = (double*)ws;
  return mrb::launch<Steepest>(steepest_kernel, dim3(nb), 0, st, n, (float2*)d, (const float2*)g, (float2*)g_prev,
                               diag, ndiag > 0 ? ndiag : 1, part, red_out(ws, out, 1, 0, nullptr));
}

extern "C" int mrb_ncg_set_steps(double* ts, int J, double beta, mrb_stream_t stream) {
  MRB_REQUIRE(ts != nullptr && J >= 1 && J <= MT_MAX_J, "bad step table");
  return mrb::launch<SetSteps>(set_steps_kernel, dim3(1), 0, (cudaStream_t)stream, ts, J, beta);
}

// ===========================================================================
// Jacobi diagonal D of the NCG preconditioner (d = beta d - g/D).
//
// Data part: D = base + alpha * sum_c |S_c|^2 per pixel, alpha the calibrated
// A^H A gain at the image centre (diag_AHA_scalar, torchkb.py:341-364).
// Regulariser part, one term at a time as RegManager.add_diag adds them
// (graspcg/regularization/manager.py:145-218):
//  * a term whose axes include the frame axis adds its frame profile
//    2 lambda w_0^2 deg(f), deg 1 at both ends of a series and 2 inside
//    (TVND.majorizer_profile, tv_nd.py:187-214), and nothing else;
//  * any other term adds per axis a the lagged diffusivity
//    lambda w_a^2 / sqrt(|D_a x|^2 + eps^2) of the forward difference D_a x
//    (zero on the last slice), once on the first and last slice along a and
//    twice inside (TVND.add_diag, tv_nd.py:113-164).  With frame_profile = 0
//    every term takes this form, the frame axis included (TVND.add_diag
//    called on its own).  The difference is of x
//    itself; the axis weight enters only squared, as in the reference.
// One pass over x and D: elementwise, HBM bound, once per solve.
// ===========================================================================
namespace {

constexpr int PD_MAX_TERMS = 8;

struct PrecondTerms {
  int nt;
  int profile[PD_MAX_TERMS];       // 1: frame profile
  float prof_scale[PD_MAX_TERMS];  // 2 lambda w_0^2 (profile terms)
  float lam[PD_MAX_TERMS];
  float eps2[PD_MAX_TERMS];
  int naxes[PD_MAX_TERMS];
  int axis[PD_MAX_TERMS][4];       // 0 (frames), 1 (size-1 axis) or 2.. (spatial)
  float w2[PD_MAX_TERMS][4];
};

struct PrecondGeom {
  int nd;
  int S[3];
  long long stride[3];  // element strides of the spatial axes
  long long P;          // pixels per frame
  int period;           // frames per series
};

__global__ void __launch_bounds__(256) precond_sense_kernel(long long n, long long P, int C,
                                                             const float2* __restrict__ maps, float alpha,
                                                             float base, float* __restrict__ D) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
    float s = 0.f;
    if (maps) {
      const long long p = v % P;
      for (int c = 0; c < C; ++c) {
        const float2 m = maps[(long long)c * P + p];
        s = fmaf(m.x, m.x, fmaf(m.y, m.y, s));
      }
    }
    D[v] = fmaf(alpha, s, base);
  }
}

__global__ void __launch_bounds__(256) precond_tv_kernel(long long n, PrecondGeom g, PrecondTerms T,
                                                          const float2* __restrict__ x, float* __restrict__ D) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
    const long long f = v / g.P;
    long long p = v - f * g.P;
    int c[3] = {0, 0, 0};
    for (int k = g.nd - 1; k >= 0; --k) {
      c[k] = (int)(p % g.S[k]);
      p /= g.S[k];
    }
    const int fl = (int)(f % g.period);
    const float2 xv = x[v];
    float acc = D[v];
    for (int t = 0; t < T.nt; ++t) {
      if (T.profile[t]) {
        const float deg = (g.period > 2 && fl > 0 && fl < g.period - 1) ? 2.f : 1.f;
        acc += deg * T.prof_scale[t];
        continue;
      }
      for (int q = 0; q < T.naxes[t]; ++q) {
        const int a = T.axis[t][q];
        int na = 1, ca = 0;
        long long sa = 0;
        if (a >= 2) {
          na = g.S[a - 2];
          ca = c[a - 2];
          sa = g.stride[a - 2];
        } else if (a == 0) {  // frames, within a series
          na = g.period;
          ca = fl;
          sa = g.P;
        }
        float dx = 0.f, dy = 0.f;
        if (ca < na - 1) {
          const float2 xn = x[v + sa];
          dx = xn.x - xv.x;
          dy = xn.y - xv.y;
        }
        const float wi = rsqrtf(dx * dx + dy * dy + T.eps2[t]);
        const float s = (T.lam[t] * T.w2[t][q]) * wi;
        acc += (na >= 3 && ca > 0 && ca < na - 1) ? 2.f * s : s;
      }
    }
    D[v] = acc;
  }
}

int precond_blocks(long long n) {
  long long nb = (n + 255) / 256;
  return (int)(nb < 148LL * 16 ? (nb < 1 ? 1 : nb) : 148LL * 16);
}

}  // namespace

extern "C" int mrb_precond_init(int64_t P, int F, int C, const void* maps, float alpha, float base, float* diag,
                                mrb_stream_t stream) {
  MRB_REQUIRE(diag != nullptr, "null diagonal");
  MRB_REQUIRE(P >= 1 && F >= 1, "bad image size");
  MRB_REQUIRE(maps == nullptr || C >= 1, "bad coil count %d", C);
  const long long n = (long long)P * F;
  precond_sense_kernel<<<precond_blocks(n), 256, 0, (cudaStream_t)stream>>>(n, P, C, (const float2*)maps, alpha,
                                                                             base, diag);
  MRB_LAUNCH_CHECK();
  return 0;
}

extern "C" int mrb_tv_add_diag(int nd, const int* S, int F, const mrb_tv_term* terms, int nterms, const void* x,
                               int frame_profile, float* diag, mrb_stream_t stream) {
  MRB_REQUIRE(nd >= 1 && nd <= 3 && S != nullptr && F >= 1, "bad image geometry");
  MRB_REQUIRE(x != nullptr && diag != nullptr, "null pointer");
  MRB_REQUIRE(nterms >= 0 && (nterms == 0 || terms != nullptr), "bad term list");
  PrecondGeom g{};
  g.nd = nd;
  g.P = 1;
  for (int k = nd - 1; k >= 0; --k) {
    MRB_REQUIRE(S[k] >= 1, "bad image size");
    g.S[k] = S[k];
    g.stride[k] = g.P;
    g.P *= S[k];
  }
  g.period = F;
  PrecondTerms T{};
  for (int i = 0; i < nterms; ++i) {
    const mrb_tv_term& t = terms[i];
    if (!t.enabled || t.weight == 0.f || t.naxes == 0) continue;
    MRB_REQUIRE(t.naxes >= 1 && t.naxes <= 4, "at most 4 axes per TV term");
    MRB_REQUIRE(T.nt < PD_MAX_TERMS, "at most %d TV terms", PD_MAX_TERMS);
    if (t.frame_period > 0) {
      MRB_REQUIRE(F % t.frame_period == 0, "frame period %d does not divide %d frames", t.frame_period, F);
      MRB_REQUIRE(g.period == F || g.period == t.frame_period, "TV terms disagree on the frame period");
      g.period = t.frame_period;
    }
    const int k = T.nt++;
    int q0 = -1;
    for (int q = 0; q < t.naxes; ++q) {
      MRB_REQUIRE(t.axes[q] >= 0 && t.axes[q] < 2 + nd, "TV axis %d out of range", t.axes[q]);
      if (t.axes[q] == 0) q0 = q;
    }
    if (q0 >= 0 && frame_profile) {
      const double w0 = t.axis_weights[q0];
      T.profile[k] = 1;
      T.prof_scale[k] = (float)(2.0 * (double)t.weight * w0 * w0);
      continue;
    }
    T.lam[k] = t.weight;
    T.eps2[k] = t.eps * t.eps;
    T.naxes[k] = t.naxes;
    for (int q = 0; q < t.naxes; ++q) {
      T.axis[k][q] = t.axes[q];
      T.w2[k][q] = (float)((double)t.axis_weights[q] * (double)t.axis_weights[q]);
    }
  }
  if (T.nt == 0) return 0;
  const long long n = g.P * F;
  precond_tv_kernel<<<precond_blocks(n), 256, 0, (cudaStream_t)stream>>>(n, g, T, (const float2*)x, diag);
  MRB_LAUNCH_CHECK();
  return 0;
}

// ===========================================================================
// Graph Laplacian over the frame axis (GraphLaplacian,
// graspcg/regularization/graph_laplacian.py:22-321).
//
// E(z) = 1/2 sum_p <z[:, p], L z[:, p]>, gradient L z, with L the B x B real
// matrix that already carries the weights (sum_i lambda_i L_i, L_i = D - W,
// I - D^-1 W or I - D^-1/2 W D^-1/2).  A block stages a tile of 32 pixel
// columns of all B frames in shared memory and every warp forms whole rows
// of L z for them: x (and d) are read once, the accumulator read and written
// once; B^2 FMAs per column stay below the CUDA-core rate up to B = 128.
// ===========================================================================
namespace {

constexpr int GRAPH_MAX_FRAMES = 128;
constexpr int GRAPH_TILE = 32;

// mode 0: z = x + t d (d may be null), y = L z, acc += y, out[0] = 1/2 Re<z, y>
// mode 1: y = L d, acc += y, out[0] = Re<x, y>, out[1] = Re<d, y>
// mode 2: mode 1 for a non-symmetric L: out[0] = Re<x, (L + L^T)/2 d> (the slope
//         of the energy along d; the accumulated L d stays the reference's gradient)
struct GraphPass {
  static constexpr int NT = RED_THREADS, MINB = 1;
  static constexpr const char* FAMILY = "graph_pass";
  static constexpr int MAXG = 16;
  static __device__ __forceinline__ void run(const VBlock& vb, int mode, int B, long long N,
      const float* __restrict__ L, const float2* __restrict__ x, const float2* __restrict__ d,
      const double* t_dev, double t_host, float2* __restrict__ acc, const double* skip,
      double* __restrict__ partials, const RedOut& ro) {
    if (skipped(skip) != 0.0) return;   // uniform over the grid: no partials, no counter
    extern __shared__ __align__(16) unsigned char graph_smem[];
    float2* Z = reinterpret_cast<float2*>(graph_smem);         // B x GRAPH_TILE
    float* Ls = reinterpret_cast<float*>(Z + B * GRAPH_TILE);  // B x B
    for (int i = threadIdx.x; i < B * B; i += blockDim.x) Ls[i] = L[i];
    const float t = (float)(t_dev ? *t_dev : t_host);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double r0 = 0.0, r1 = 0.0;
    const long long ntiles = (N + GRAPH_TILE - 1) / GRAPH_TILE;
    for (long long tile = vb.x; tile < ntiles; tile += vb.nx) {
      const long long p = tile * GRAPH_TILE + lane;
      const bool in = p < N;
      __syncthreads();   // L staged; the previous tile's columns consumed
      for (int f = warp; f < B; f += nw) {
        float2 v = make_float2(0.f, 0.f);
        if (in) {
          const long long i = (long long)f * N + p;
          if (mode == 0) {
            v = x[i];
            if (d) {
              const float2 dv = d[i];
              v.x = __fadd_rn(v.x, __fmul_rn(dv.x, t));
              v.y = __fadd_rn(v.y, __fmul_rn(dv.y, t));
            }
          } else {
            v = d[i];
          }
        }
        Z[f * GRAPH_TILE + lane] = v;
      }
      __syncthreads();
      for (int f = warp; f < B; f += nw) {
        const float* Lr = Ls + f * B;
        float yx = 0.f, yy = 0.f, tx = 0.f, ty = 0.f;
        for (int s2 = 0; s2 < B; ++s2) {
          const float l = Lr[s2];
          const float2 z = Z[s2 * GRAPH_TILE + lane];
          yx = fmaf(l, z.x, yx);
          yy = fmaf(l, z.y, yy);
          if (mode == 2) {
            const float lt = Ls[s2 * B + f];
            tx = fmaf(lt, z.x, tx);
            ty = fmaf(lt, z.y, ty);
          }
        }
        if (in) {
          const long long i = (long long)f * N + p;
          const float2 zf = Z[f * GRAPH_TILE + lane];
          if (acc) {
            float2 a = acc[i];
            a.x += yx;
            a.y += yy;
            acc[i] = a;
          }
          if (mode == 0) {
            r0 += (double)(zf.x * yx + zf.y * yy);
          } else {
            const float2 xv = x[i];
            if (mode == 1)
              r0 += (double)(xv.x * yx + xv.y * yy);
            else
              r0 += 0.5 * (double)(xv.x * (yx + tx) + xv.y * (yy + ty));
            r1 += (double)(zf.x * yx + zf.y * yy);
          }
        }
      }
    }
    double v[2] = {mode == 0 ? 0.5 * r0 : r0, r1};
    block_reduce_finish<2>(vb, v, partials, ro);
  }
};
__global__ void __launch_bounds__(RED_THREADS) graph_kernel(int mode, int B, long long N,
    const float* __restrict__ L, const float2* __restrict__ x, const float2* __restrict__ d,
    const double* t_dev, double t_host, float2* __restrict__ acc, const double* skip,
    double* __restrict__ partials, RedOut ro) {
  GraphPass::run(hw_block(), mode, B, N, L, x, d, t_dev, t_host, acc, skip, partials, ro);
}

// The graph term is quadratic, so the fast schedule carries it beside the
// data term (0.5 (err + 2 t erd + t^2 edd)):
// phase 0 (prime):     err += 2 q0
// phase 1 (iteration): err += 2 q0, erd += q1, edd += q2 (after the k-space scalars)
// phase 2 (update):    q0 += t q1 + t^2 q2 / 2 at the accepted step
struct QuadFold {
  static constexpr int NT = 32, MINB = 1;
  static constexpr const char* FAMILY = "quad_fold";
  static constexpr int MAXG = 16;
  static __device__ __forceinline__ void run(const VBlock& vb, double* s, int phase) {
    if (threadIdx.x != 0) return;
    if (phase == 0) {
      s[S_ERR] += 2.0 * s[S_GQ0];
    } else if (phase == 1) {
      if (s[S_DONE] != 0.0) return;
      s[S_ERR] += 2.0 * s[S_GQ0];
      s[S_ERD] += s[S_GQ1];
      s[S_EDD] += s[S_GQ2];
    } else {
      if (s[S_LS_OK] == 0.0) return;
      const double t = s[S_T];
      s[S_GQ0] += t * s[S_GQ1] + 0.5 * t * t * s[S_GQ2];
    }
  }
};
__global__ void quad_fold_kernel(double* s, int phase) {
  QuadFold::run(hw_block(), s, phase);
}

__global__ void __launch_bounds__(256) diag_frames_kernel(long long n, long long P, const float* __restrict__ v,
                                                           float* __restrict__ D) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) D[i] += v[i / P];
}

}  // namespace

extern "C" int mrb_graph_pass(int mode, int B, int64_t N, const float* L, const void* x, const void* d,
                              const double* t_dev, double t_host, void* acc, const double* skip, double* out,
                              void* ws, mrb_stream_t stream) {
  MRB_REQUIRE(mode >= 0 && mode <= 2, "mode must be 0, 1 or 2");
  MRB_REQUIRE(B >= 1 && B <= GRAPH_MAX_FRAMES, "graph over %d frames (1..%d supported)", B, GRAPH_MAX_FRAMES);
  MRB_REQUIRE(N >= 1, "bad pixel count");
  MRB_REQUIRE(L && x && out && ws, "null pointer");
  MRB_REQUIRE(mode == 0 || d, "modes 1 and 2 need d");
  const size_t smem = (size_t)B * GRAPH_TILE * sizeof(float2) + (size_t)B * B * sizeof(float);
  static bool attr_set[64] = {};
  int dev = 0;
  MRB_CUDA_TRY(cudaGetDevice(&dev));
  if (smem > 48 * 1024 && dev < 64 && !attr_set[dev]) {
    MRB_CUDA_TRY(cudaFuncSetAttribute(graph_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)((size_t)GRAPH_MAX_FRAMES * GRAPH_TILE * sizeof(float2) +
                                            (size_t)GRAPH_MAX_FRAMES * GRAPH_MAX_FRAMES * sizeof(float))));
    attr_set[dev] = true;
  }
  const long long ntiles = (N + GRAPH_TILE - 1) / GRAPH_TILE;
  const int nb = (int)std::min<long long>(ntiles, 148LL * 6);
  double* part = (double*)ws;
  return mrb::launch<GraphPass>(graph_kernel, dim3(nb), smem, (cudaStream_t)stream, mode, B, (long long)N, L,
                                (const float2*)x, (const float2*)d, t_dev, t_host, (float2*)acc, skip, part,
                                red_out(ws, out, mode == 0 ? 1 : 2, 0, skip));
}

extern "C" int mrb_ncg_quad_fold(double* slots, int phase, mrb_stream_t stream) {
  MRB_REQUIRE(slots != nullptr, "null pointer");
  MRB_REQUIRE(phase >= 0 && phase <= 2, "phase must be 0, 1 or 2");
  return mrb::launch<QuadFold>(quad_fold_kernel, dim3(1), 0, (cudaStream_t)stream, slots, phase);
}

// ===========================================================================
// Frame mixing out[r, p] (+)= sum_k M[r, k] in[k, p] over the frame axis
// (TemporalBasisOp u = U V and its adjoint g_V += U^H g_u, mapping.py:112-236;
// per-frame scalings of ScaleOp :44-110 as diagonal M).  Same tiling as the
// graph pass: 32 pixel columns of all input rows staged in shared memory.
// ===========================================================================
namespace {

constexpr int MIX_MAX_ROWS = 128;

// complex data, complex M (row-major rows_out x rows_in, or rows_in x rows_out
// conjugated when conj_t)
__global__ void __launch_bounds__(256) mix_complex_kernel(int Ro, int Ri, long long N, const float2* __restrict__ M,
                                                          int conj_t, const float2* __restrict__ in,
                                                          float2* __restrict__ out, int accumulate) {
  extern __shared__ __align__(16) unsigned char mix_smem[];
  float2* Z = reinterpret_cast<float2*>(mix_smem);          // Ri x 32
  float2* Ms = Z + Ri * GRAPH_TILE;                          // Ro x Ri
  for (int i = threadIdx.x; i < Ro * Ri; i += blockDim.x) {
    const int r = i / Ri, k = i - r * Ri;
    float2 m = conj_t ? M[k * Ro + r] : M[i];
    if (conj_t) m.y = -m.y;
    Ms[i] = m;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const long long ntiles = (N + GRAPH_TILE - 1) / GRAPH_TILE;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long p = tile * GRAPH_TILE + lane;
    const bool ok = p < N;
    __syncthreads();
    for (int k = warp; k < Ri; k += nw) Z[k * GRAPH_TILE + lane] = ok ? in[(long long)k * N + p] : make_float2(0.f, 0.f);
    __syncthreads();
    if (!ok) continue;
    for (int r = warp; r < Ro; r += nw) {
      const float2* Mr = Ms + r * Ri;
      float ax = 0.f, ay = 0.f;
      for (int k = 0; k < Ri; ++k) {
        const float2 m = Mr[k], z = Z[k * GRAPH_TILE + lane];
        ax = fmaf(m.x, z.x, ax);
        ax = fmaf(-m.y, z.y, ax);
        ay = fmaf(m.x, z.y, ay);
        ay = fmaf(m.y, z.x, ay);
      }
      const long long i = (long long)r * N + p;
      if (accumulate) {
        const float2 o = out[i];
        ax += o.x;
        ay += o.y;
      }
      out[i] = make_float2(ax, ay);
    }
  }
}

// real data, real M (row-major rows_out x rows_in, or transposed when trans)
__global__ void __launch_bounds__(256) mix_real_kernel(int Ro, int Ri, long long N, const float* __restrict__ M,
                                                       int trans, const float* __restrict__ in,
                                                       float* __restrict__ out, int accumulate) {
  extern __shared__ __align__(16) unsigned char mix_smem_r[];
  float* Z = reinterpret_cast<float*>(mix_smem_r);  // Ri x 32
  float* Ms = Z + Ri * GRAPH_TILE;                   // Ro x Ri
  for (int i = threadIdx.x; i < Ro * Ri; i += blockDim.x) {
    const int r = i / Ri, k = i - r * Ri;
    Ms[i] = trans ? M[k * Ro + r] : M[i];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const long long ntiles = (N + GRAPH_TILE - 1) / GRAPH_TILE;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long p = tile * GRAPH_TILE + lane;
    const bool ok = p < N;
    __syncthreads();
    for (int k = warp; k < Ri; k += nw) Z[k * GRAPH_TILE + lane] = ok ? in[(long long)k * N + p] : 0.f;
    __syncthreads();
    if (!ok) continue;
    for (int r = warp; r < Ro; r += nw) {
      const float* Mr = Ms + r * Ri;
      float a = 0.f;
      for (int k = 0; k < Ri; ++k) a = fmaf(Mr[k], Z[k * GRAPH_TILE + lane], a);
      const long long i = (long long)r * N + p;
      out[i] = accumulate ? out[i] + a : a;
    }
  }
}

}  // namespace

extern "C" int mrb_frame_mix(int rows_out, int rows_in, int64_t N, const void* M, int conj_transpose, const void* in,
                             void* out, int accumulate, mrb_stream_t stream) {
  MRB_REQUIRE(rows_out >= 1 && rows_out <= MIX_MAX_ROWS && rows_in >= 1 && rows_in <= MIX_MAX_ROWS,
              "frame mix of %d x %d rows (1..%d supported)", rows_out, rows_in, MIX_MAX_ROWS);
  MRB_REQUIRE(N >= 1 && M && in && out, "bad arguments");
  MRB_REQUIRE(in != out, "in and out must not alias");
  const size_t smem = ((size_t)rows_in * GRAPH_TILE + (size_t)rows_out * rows_in) * sizeof(float2);
  if (smem > 48 * 1024)
    MRB_CUDA_TRY(cudaFuncSetAttribute(mix_complex_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long ntiles = (N + GRAPH_TILE - 1) / GRAPH_TILE;
  const int nb = (int)std::min<long long>(ntiles, 148LL * 6);
  mix_complex_kernel<<<nb, 256, smem, (cudaStream_t)stream>>>(rows_out, rows_in, (long long)N, (const float2*)M,
                                                                conj_transpose, (const float2*)in, (float2*)out,
                                                                accumulate);
  MRB_LAUNCH_CHECK();
  return 0;
}

extern "C" int mrb_frame_mix_real(int rows_out, int rows_in, int64_t N, const float* M, int transpose,
                                  const float* in, float* out, int accumulate, mrb_stream_t stream) {
  MRB_REQUIRE(rows_out >= 1 && rows_out <= MIX_MAX_ROWS && rows_in >= 1 && rows_in <= MIX_MAX_ROWS,
              "frame mix of %d x %d rows (1..%d supported)", rows_out, rows_in, MIX_MAX_ROWS);
  MRB_REQUIRE(N >= 1 && M && in && out, "bad arguments");
  MRB_REQUIRE(in != out, "in and out must not alias");
  const size_t smem = ((size_t)rows_in * GRAPH_TILE + (size_t)rows_out * rows_in) * sizeof(float);
  if (smem > 48 * 1024)
    MRB_CUDA_TRY(cudaFuncSetAttribute(mix_real_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long ntiles = (N + GRAPH_TILE - 1) / GRAPH_TILE;
  const int nb = (int)std::min<long long>(ntiles, 148LL * 6);
  mix_real_kernel<<<nb, 256, smem, (cudaStream_t)stream>>>(rows_out, rows_in, (long long)N, M, transpose, in, out,
                                                             accumulate);
  MRB_LAUNCH_CHECK();
  return 0;
}

extern "C" int mrb_diag_add_frames(int64_t P, int F, const float* v, float* diag, mrb_stream_t stream) {
  MRB_REQUIRE(v && diag, "null pointer");
  MRB_REQUIRE(P >= 1 && F >= 1, "bad image size");
  const long long n = (long long)P * F;
  diag_frames_kernel<<<precond_blocks(n), 256, 0, (cudaStream_t)stream>>>(n, P, v, diag);
  MRB_LAUNCH_CHECK();
  return 0;
}

// ===========================================================================
// Allocation-free variant of mrb_dots_f64.
//
// Some callers cannot allocate device memory at the point where they need a
// dot product: code running inside a CUDA stream capture (an allocation is not
// a stream operation and invalidates a global-mode capture), real-time
// reconstruction loops next to the scanner (cudaMalloc/cudaFree synchronise
// the device and stall acquisition), and processes whose device memory is
// handed out by another allocator up front (a stray cudaMalloc can fail).
// This entry point keeps its block partials in a fixed file-scope device
// array instead of a caller workspace, and calls no allocating routine.
// ===========================================================================
namespace {

constexpr int NOALLOC_MAX_PAIRS = 8;
constexpr int NOALLOC_MAX_DEVICES = 64;

// RED_MAX_BLOCKS x 8 doubles = 75,776 bytes; every GPU that loads this
// library holds it until the process exits.
static __device__ __align__(256) double g_noalloc_partials[RED_MAX_BLOCKS * NOALLOC_MAX_PAIRS];

std::mutex g_noalloc_mu;
double* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};

// Device address of the scratch array on the current device.  The host-side
// name g_noalloc_partials is only a stand-in and must never be passed to a
// kernel; the address is looked up with that device current.  Outside a
// stream capture the lookup is repeated on every call (a host-side table
// lookup once the module is loaded), so a cudaDeviceReset, which reloads the
// module at a possibly different address, cannot leave a stale pointer behind;
// inside a capture the address cached by the last call outside one is used,
// so the first call on a device has to come before any capture.
int noalloc_scratch(cudaStream_t st, double** out) {
  int dev = -1;
  MRB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES)
    return mrb::fail(MRB_ERANGE, "device ordinal %d above the %d supported", dev, NOALLOC_MAX_DEVICES);
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  MRB_CUDA_TRY(cudaStreamIsCapturing(st, &cs));
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (cs == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess || p == nullptr)
      return mrb::fail(MRB_ECUDA, "cudaGetSymbolAddress(scratch) failed on device %d: %s", dev,
                       cudaGetErrorString(e));
    g_noalloc_ptr[dev] = (double*)p;
  } else if (!g_noalloc_ptr[dev]) {
    return mrb::fail(MRB_ESTATE, "mrb_dots_f64_noalloc: the first call on device %d must come before "
                                 "any stream capture", dev);
  }
  *out = g_noalloc_ptr[dev];
  return 0;
}

}  // namespace

extern "C" int mrb_dots_f64_noalloc(int64_t n, int npairs, const void* const* a, const void* const* b,
                                    const float* const* diag, int64_t ndiag, double* out, mrb_stream_t stream) {
  if (npairs < 1 || npairs > NOALLOC_MAX_PAIRS)
    return mrb::fail(MRB_ERANGE, "mrb_dots_f64_noalloc: npairs = %d, the fixed scratch holds at most %d pairs",
                     npairs, NOALLOC_MAX_PAIRS);
  MRB_REQUIRE(n >= 0, "mrb_dots_f64_noalloc: negative length");
  MRB_REQUIRE(a && b && out, "mrb_dots_f64_noalloc: null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  double* part = nullptr;
  int rc = noalloc_scratch(st, &part);
  if (rc) return rc;
  DotArgs d{};
  for (int j = 0; j < npairs; ++j) {
    MRB_REQUIRE(a[j] && b[j], "mrb_dots_f64_noalloc: null operand %d", j);
    d.a[j] = (const float2*)a[j];
    d.b[j] = (const float2*)b[j];
    d.diag[j] = diag ? diag[j] : nullptr;
  }
  d.ndiag = ndiag > 0 ? ndiag : 1;
  d.n = n;
  d.npairs = npairs;
  // at most RED_MAX_BLOCKS blocks, each writing its `stride` partials before the
  // final sum reads them: no part of the scratch has to start at zero
  const int nb = red_blocks(n, 4);
  switch (npairs) {
    case 1: dots_kernel<1><<<nb, RED_THREADS, 0, st>>>(d, part); break;
    case 2: dots_kernel<2><<<nb, RED_THREADS, 0, st>>>(d, part); break;
    case 3: dots_kernel<3><<<nb, RED_THREADS, 0, st>>>(d, part); break;
    case 4: dots_kernel<4><<<nb, RED_THREADS, 0, st>>>(d, part); break;
    default: dots_kernel<8><<<nb, RED_THREADS, 0, st>>>(d, part); break;
  }
  MRB_LAUNCH_CHECK();
  const int stride = npairs <= 4 ? npairs : 8;
  return finalize(part, nb, stride, npairs, out, 0, nullptr, st);
}
