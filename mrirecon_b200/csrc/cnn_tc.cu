// Warm-start network convolution on the 5th-generation tensor cores (sm_100a):
// tcgen05.mma with the accumulator in tensor memory, operands staged in shared
// memory by TMA.
//
// 3x3x3 convolution (stride 1, zero padding 1) on channels-last BF16 volumes
// (Nb, D, H, W, C) as an implicit GEMM: M = 128 output voxels per CTA (a
// BH x BW patch of one (n, d) plane), N = output channels (16 .. 256), K = 27
// taps x input channels in chunks of 32.  For tap (dz, dy, dx) the A tile is the
// input patch shifted by the tap: one 5-D TMA box {32 channels, BW, BH, 1, 1} at
// coordinates (c, w0 + dx, h0 + dy, d + dz, n); coordinates outside the volume
// read as zero, which is the zero padding.  B is the weight slice [tap][N][32]
// (K-major).  Both land in 64-byte-swizzled shared tiles that the MMA reads
// through shared-memory descriptors.  A 4-stage ring: one thread issues TMA
// loads (mbarrier transaction counts), one thread issues the MMAs (K = 16 per
// instruction, FP32 accumulation in TMEM) and commits each stage back to the
// producer; the epilogue reads TMEM with tcgen05.ld (warp w owns lanes
// 32w .. 32w+31 = voxels), adds the bias, applies ReLU and stores BF16 and/or
// FP32 (optionally accumulating).  Every mbarrier wait is bounded: on timeout
// the kernel records an error flag, skips the remaining work, releases its
// TMEM and returns.
// No reference counterpart: the reference has no learned component.

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "mrb_common.cuh"

namespace {

typedef __nv_bfloat16 bf16;

constexpr int TC_BM = 128;      // voxels per CTA (UMMA M)
constexpr int TC_BK = 32;       // K per stage (channels): one 64-byte swizzle row
constexpr int TC_STAGES = 4;
constexpr int TC_THREADS = 128;
constexpr long long TC_WAIT_LIMIT = 1LL << 20;   // bounded try_wait rounds of a barrier phase before giving up

__device__ int g_tc_error = 0;   // set when a barrier wait times out

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// try_wait suspends the thread in hardware for a bounded, system-dependent time
// while the phase is incomplete (no busy polling of the issue slots)
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait for the phase with the given parity; false on timeout or when
// another thread of the CTA already gave up
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
  for (long long i = 0; i < TC_WAIT_LIMIT; ++i) {
    if (mbar_test(bar, parity)) return true;
    if (*abort_flag) return false;
    if ((i & 1023) == 1023 && *(volatile int*)&g_tc_error) {   // another CTA gave up: stop too
      *abort_flag = 1;
      return false;
    }
  }
  *abort_flag = 1;
  atomicExch(&g_tc_error, 1);
  return false;
}

__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2,
                                            int c3, int c4) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6, "
      "%7}], [%2];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4)
      : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
      "[%2];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

// Shared-memory matrix descriptor: K-major tile of rows of 64 bytes, 64-byte
// swizzle, 8-row groups 512 bytes apart (start and offsets in 16-byte units;
// descriptor version 1; layout code 4 = 64-byte swizzle).
__device__ __forceinline__ uint64_t sw64_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)1 << 16;                 // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(512 >> 4) << 32;        // stride byte offset: 8 rows x 64 B
  d |= (uint64_t)1 << 46;                 // version
  d |= (uint64_t)4 << 61;                 // 64-byte swizzle
  return d;
}

// Instruction descriptor, kind::f16: D FP32, A and B BF16, both K-major, N, M.
__host__ __device__ constexpr uint32_t f16_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

struct TcArgs {
  int cin;           // K channels (multiple of 32), read at channel offset ci_off
  int ci_off;
  int N;             // output channels computed (multiple of 16, <= 256)
  int cout;          // output channels written
  int flip;          // weight tap = 26 - tap (data gradient)
  const float* bias;
  int relu;
  bf16* yb;
  int cyb, yb_off;
  float* yf;
  int cyf, yf_off, yf_acc;
  int Nb, D, H, W;
  int BW, BH;        // voxel patch of one CTA (BW * BH = 128)
  int ncols;         // TMEM columns allocated (power of two >= 32, >= N)
};

__global__ void __launch_bounds__(TC_THREADS) conv3d_tc_kernel(const __grid_constant__ CUtensorMap xmap,
                                                               const __grid_constant__ CUtensorMap wmap, TcArgs a) {
  extern __shared__ __align__(1024) uint8_t dsm[];
  __shared__ __align__(8) uint64_t full_bar[TC_STAGES], empty_bar[TC_STAGES], done_bar;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // stage buffers, 1024-byte aligned (swizzle atoms)
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(dsm) + 1023) & ~uintptr_t(1023));
  const uint32_t a_bytes = TC_BM * TC_BK * 2;             // 8 KB
  const uint32_t b_bytes = (uint32_t)a.N * TC_BK * 2;      // N x 64 B
  const uint32_t stage_bytes = (a_bytes + b_bytes + 1023) & ~1023u;

  // tile -> (n, d, h0, w0)
  const int tw = a.W / a.BW, th = a.H / a.BH;
  long long t = blockIdx.x;
  const int w0 = (int)(t % tw) * a.BW;
  t /= tw;
  const int h0 = (int)(t % th) * a.BH;
  t /= th;
  const int dd = (int)(t % a.D);
  const int nn = (int)(t / a.D);

  if (threadIdx.x == 0) {
    for (int s = 0; s < TC_STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&done_bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(a.ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem_d = tmem_base;

  const int kch = a.cin / TC_BK;
  const int nk = 27 * kch;

  if (warp == 0 && lane == 0) {
    // producer: TMA loads of A (shifted input patch) and B (weight slice)
    for (int ks = 0; ks < nk; ++ks) {
      const int s = ks % TC_STAGES;
      if (ks >= TC_STAGES && !mbar_wait(&empty_bar[s], ((ks / TC_STAGES) - 1) & 1, &abort_flag)) break;
      const int tap = ks / kch, kc = ks - tap * kch;
      const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
      const int wtap = a.flip ? 26 - tap : tap;
      uint8_t* sa = base + (size_t)s * stage_bytes;
      uint8_t* sb = sa + a_bytes;
      mbar_expect_tx(&full_bar[s], a_bytes + b_bytes);
      tma_load_5d(sa, &xmap, &full_bar[s], a.ci_off + kc * TC_BK, w0 + dx, h0 + dy, dd + dz, nn);
      tma_load_3d(sb, &wmap, &full_bar[s], kc * TC_BK, 0, wtap);
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    const uint32_t idesc = f16_idesc(TC_BM, a.N);
    for (int ks = 0; ks < nk; ++ks) {
      const int s = ks % TC_STAGES;
      if (!mbar_wait(&full_bar[s], (ks / TC_STAGES) & 1, &abort_flag)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t sa = smem_u32(base + (size_t)s * stage_bytes);
      const uint32_t sb = sa + a_bytes;
#pragma unroll
      for (int kk = 0; kk < TC_BK / 16; ++kk) {
        const uint64_t adesc = sw64_desc(sa + kk * 32);
        const uint64_t bdesc = sw64_desc(sb + kk * 32);
        const uint32_t accum = (ks > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&empty_bar[s]))
                   : "memory");
    }
    // arrives once every MMA issued above has completed (also after an abort)
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(&done_bar))
                 : "memory");
  }
  __syncwarp();

  // epilogue: wait for the accumulator, TMEM -> registers -> global
  bool have = mbar_wait(&done_bar, 0, &abort_flag) && !abort_flag;
  have = __all_sync(0xffffffffu, have);   // tcgen05.ld is warp-collective
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (have) {
    const int row = warp * 32 + lane;   // TMEM lane = voxel of the patch
    const int hl = row / a.BW, wl = row - hl * a.BW;
    const long long vox = (((long long)nn * a.D + dd) * a.H + (h0 + hl)) * a.W + (w0 + wl);
    for (int c0 = 0; c0 < a.N; c0 += 16) {
      uint32_t r[16];
      const uint32_t taddr = tmem_d + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
          "%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (c0 >= a.cout) continue;
      float v[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        float x = __uint_as_float(r[j]);
        if (a.bias) x += __ldg(a.bias + c0 + j);
        if (a.relu) x = fmaxf(x, 0.f);
        v[j] = x;
      }
      const int nw = min(16, a.cout - c0);
      if (a.yb) {
        bf16* p = a.yb + vox * a.cyb + a.yb_off + c0;
        if (nw == 16) {
          uint32_t pk[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            __nv_bfloat162 h2 = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
            pk[j] = *reinterpret_cast<uint32_t*>(&h2);
          }
          reinterpret_cast<uint4*>(p)[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
          reinterpret_cast<uint4*>(p)[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
        } else {
          for (int j = 0; j < nw; ++j) p[j] = __float2bfloat16_rn(v[j]);
        }
      }
      if (a.yf) {
        float* p = a.yf + vox * a.cyf + a.yf_off + c0;
        for (int j = 0; j < nw; ++j) p[j] = a.yf_acc ? p[j] + v[j] : v[j];
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_d), "r"(a.ncols) : "memory");
  }
}

// ---------------------------------------------------------------------------
// Weight gradient on tcgen05: dW[tap][ci][co] = sum_v x[v + o(tap)][ci] gz[v][co]
// (o(tap) the (dz, dy, dx) offset; out-of-volume x is zero), the reduction
// over voxels as the GEMM's K.  Both operands must be K-major for the MMA,
// i.e. voxels contiguous, so they are first repacked channels-first
// (wg_pack_kernel).  The operand with more channels is the MMA's M side (128
// rows per tile, channels padded with zeros) and is loaded once per K step;
// the other is the N side (16 .. 256 rows) and carries the tap offset, so a K
// step loads one M tile and one small N tile per tap.  The offset moves only
// the H and D coordinates of a TMA box (out-of-volume rows read as zero) and
// picks one of three copies of the N operand shifted by -1, 0, +1 along W, so
// every box starts at a W coordinate that is a multiple of 32.  With x on the
// M side the N operand is gz shifted the other way (sum_u x[u] gz[u - o]); the
// sums are the same.  A K step is 32 consecutive voxels of one (n, d, h) row.
// A CTA owns a group of TG taps (TG accumulators of N columns in TMEM), an M
// tile and a range of K steps; its partial sums go to part[split][tap][ci][co]
// and are added in a fixed split order (deterministic).
// ---------------------------------------------------------------------------
constexpr int WG_STAGES = 4;
constexpr int WG_KV = 32;   // voxels per K step (one 64-byte swizzle row of BF16)

struct WgArgs {
  int xm;              // 1: x is the M operand (gz shifted), 0: gz is (x shifted)
  int N;               // columns: channels of the N operand (multiple of 16, <= 256)
  int Mreal;           // real channels of the M operand
  int cin, coutp;      // dW is [27][cin][coutp]
  int TG;              // taps per group
  int Nb, D, H, W;
  long long ksteps;    // Nb * D * H * (W / 32)
  long long kper;      // K steps per split
  int ngroups, mtiles;
  float* part;         // [split][27][cin][coutp]
  int ncols;           // TMEM columns allocated
  uint32_t m_bytes, n_bytes;   // tile bytes (multiples of 1024)
};

__global__ void __launch_bounds__(TC_THREADS) wgrad_tc_kernel(const __grid_constant__ CUtensorMap mmap,
                                                              const __grid_constant__ CUtensorMap nmap, WgArgs a) {
  extern __shared__ __align__(1024) uint8_t dsm[];
  __shared__ __align__(8) uint64_t full_bar[WG_STAGES], empty_bar[WG_STAGES], done_bar;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(dsm) + 1023) & ~uintptr_t(1023));
  const uint32_t stage_bytes = a.m_bytes + (uint32_t)a.TG * a.n_bytes;

  // block -> (tap group, M tile, split)
  long long bid = blockIdx.x;
  const int grp = (int)(bid % a.ngroups);
  bid /= a.ngroups;
  const int mt = (int)(bid % a.mtiles);
  const long long split = bid / a.mtiles;
  const int tap0 = grp * a.TG;
  const int ntap = min(a.TG, 27 - tap0);
  const int m0 = mt * 128;
  const long long kb0 = split * a.kper;
  const long long kb1 = min(a.ksteps, kb0 + a.kper);
  const int nk = (int)(kb1 - kb0);
  const uint32_t m_tile = 128u * WG_KV * 2u, n_tile = (uint32_t)a.N * WG_KV * 2u;
  const int sg = a.xm ? -1 : 1;   // the N operand's offset: gz[u - o] or x[v + o]

  if (threadIdx.x == 0) {
    for (int st = 0; st < WG_STAGES; ++st) {
      mbar_init(&full_bar[st], 1);
      mbar_init(&empty_bar[st], 1);
    }
    mbar_init(&done_bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(a.ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem_d = tmem_base;
  const int nwc = a.W / WG_KV;

  if (warp == 0 && lane == 0) {
    // producer: per K step the M tile and one N tile per tap of the group
    for (int ks = 0; ks < nk; ++ks) {
      const int st = ks % WG_STAGES;
      if (ks >= WG_STAGES && !mbar_wait(&empty_bar[st], ((ks / WG_STAGES) - 1) & 1, &abort_flag)) break;
      long long kv = kb0 + ks;
      const int w0 = (int)(kv % nwc) * WG_KV;
      kv /= nwc;
      const int h = (int)(kv % a.H);
      kv /= a.H;
      const int d = (int)(kv % a.D);
      const int n = (int)(kv / a.D);
      uint8_t* sbase = base + (size_t)st * stage_bytes;
      mbar_expect_tx(&full_bar[st], m_tile + (uint32_t)ntap * n_tile);
      tma_load_5d(sbase, &mmap, &full_bar[st], w0, h, d, m0, n);
      for (int t = 0; t < ntap; ++t) {
        const int tap = tap0 + t;
        const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
        tma_load_5d(sbase + a.m_bytes + (size_t)t * a.n_bytes, &nmap, &full_bar[st], w0, h + sg * dy, d + sg * dz,
                    0, n * 3 + sg * dx + 1);
      }
    }
  } else if (warp == 1 && lane == 0) {
    // the N tiles of consecutive taps are contiguous (N x 64 bytes each, whole
    // swizzle atoms) and so are their accumulators (N TMEM columns each): up to
    // 256 / N taps go into one MMA of N' = taps x N columns
    const int ng = 256 / a.N;
    for (int ks = 0; ks < nk; ++ks) {
      const int st = ks % WG_STAGES;
      if (!mbar_wait(&full_bar[st], (ks / WG_STAGES) & 1, &abort_flag)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t sa = smem_u32(base + (size_t)st * stage_bytes);
      for (int t = 0; t < ntap; t += ng) {
        const int nt = min(ng, ntap - t);
        const uint32_t idesc = f16_idesc(128, nt * a.N);
        const uint32_t sb = sa + a.m_bytes + (uint32_t)t * a.n_bytes;
#pragma unroll
        for (int kk = 0; kk < WG_KV / 16; ++kk) {
          const uint64_t adesc = sw64_desc(sa + kk * 32);
          const uint64_t bdesc = sw64_desc(sb + kk * 32);
          const uint32_t accum = (ks > 0 || kk > 0) ? 1u : 0u;
          asm volatile(
              "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
              " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d + (uint32_t)(t * a.N)),
              "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
              : "memory");
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&empty_bar[st]))
                   : "memory");
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(&done_bar))
                 : "memory");
  }
  __syncwarp();

  bool have = nk > 0 && mbar_wait(&done_bar, 0, &abort_flag) && !abort_flag;
  have = __all_sync(0xffffffffu, have);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const int row = warp * 32 + lane;   // TMEM lane = channel m0 + row of the M operand
  const int mch = m0 + row;
  for (int t = 0; t < ntap; ++t) {
    float* pt = a.part + ((size_t)split * 27 + tap0 + t) * (size_t)a.cin * a.coutp;
    for (int c0 = 0; c0 < a.N; c0 += 16) {
      uint32_t r[16];
      if (have) {
        const uint32_t taddr = tmem_d + ((uint32_t)(warp * 32) << 16) + (uint32_t)(t * a.N + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) r[j] = 0u;   // no K steps (or an aborted wait): a zero partial
      }
      if (mch >= a.Mreal) continue;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int nch = c0 + j;
        const float v = __uint_as_float(r[j]);
        if (a.xm) pt[(size_t)mch * a.coutp + nch] = v;   // (ci = m, co = n)
        else pt[(size_t)nch * a.coutp + mch] = v;        // (ci = n, co = m)
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_d), "r"(a.ncols) : "memory");
  }
}

// channels-first repack: out[n][copy][c][d][h][w] = src[n][d][h][w + shift][c_off + c]
// (shift = copy - 1 with three copies, 0 with one; zero outside the volume and
// for nch <= c < chp); a block moves a 32-channel x 64-voxel tile of one row
constexpr int PK_W = 64;

__global__ void __launch_bounds__(256) wg_pack_kernel(const bf16* __restrict__ src, int cs, int c_off, int nch,
                                                      bf16* __restrict__ out, int chp, int ncopies, int D, int H,
                                                      int W) {
  __shared__ bf16 tile[32][PK_W + 3];
  const int nwt = W / PK_W;
  const int wt = blockIdx.x % nwt, ct = blockIdx.x / nwt;
  const int h = blockIdx.y;
  const int nd = blockIdx.z;
  const int n = nd / D, d = nd - n * D;
  const int w0 = wt * PK_W, c0 = ct * 32;
  const long long row = ((long long)nd * H + h) * W;   // voxel index of (n, d, h, 0)
  for (int e = threadIdx.x; e < (PK_W + 2) * 32; e += blockDim.x) {
    const int wl = e >> 5, cl = e & 31;
    const int w = w0 - 1 + wl, c = c0 + cl;
    bf16 v = __float2bfloat16_rn(0.f);
    if (w >= 0 && w < W && c < nch) v = src[(row + w) * cs + c_off + c];
    tile[cl][wl] = v;
  }
  __syncthreads();
  const long long plane = (long long)D * H * W;
  for (int copy = 0; copy < ncopies; ++copy) {
    const int shift = ncopies > 1 ? copy - 1 : 0;
    bf16* ob = out + (((long long)n * ncopies + copy) * chp) * plane + ((long long)d * H + h) * W + w0;
    for (int e = threadIdx.x; e < 32 * PK_W; e += blockDim.x) {
      const int cl = e / PK_W, wl = e - cl * PK_W;
      const int c = c0 + cl;
      if (c < chp) ob[(long long)c * plane + wl] = tile[cl][wl + 1 + shift];
    }
  }
}

// dW[i] = sum over splits in order; dbias[co] likewise from per-split sums
__global__ void wg_sum_kernel(const float* __restrict__ part, int nsplit, long long n, float* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = 0.f;
  for (int k = 0; k < nsplit; ++k) s += part[(long long)k * n + i];
  out[i] = s;
}

// per-split channel sums of gz (bias gradient): block = split, thread = (channel, lane)
__global__ void __launch_bounds__(256) wg_bias_kernel(const bf16* __restrict__ gz, int cg, int cg_off, int coutp,
                                                      long long voxels, long long vper, float* __restrict__ bpart) {
  __shared__ float red[256];
  const long long v0 = (long long)blockIdx.x * vper, v1 = min(voxels, v0 + vper);
  const int lanes = 256 / coutp;   // coutp divides 256
  const int co = threadIdx.x % coutp, l = threadIdx.x / coutp;
  float s = 0.f;
  if (l < lanes)
    for (long long v = v0 + l; v < v1; v += lanes) s += __bfloat162float(gz[v * cg + cg_off + co]);
  red[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x < coutp) {
    float t = 0.f;
    for (int k = 0; k < lanes; ++k) t += red[k * coutp + threadIdx.x];
    bpart[(long long)blockIdx.x * coutp + threadIdx.x] = t;
  }
}

struct WgPlan {
  int xm, N, Mreal, Mpad, TG, ngroups, mtiles, nsplit;
  long long ksteps, kper;
  size_t m_elems, n_elems, part_floats;   // packed M operand (one copy), N operand (three copies)
  uint32_t m_bytes, n_bytes;
};

bool wg_plan(int cin, int coutp, int Nb, int D, int H, int W, WgPlan& p) {
  if (cin <= 0 || coutp <= 0 || cin % 16 != 0 || coutp % 16 != 0 || W % PK_W != 0) return false;
  p.xm = cin > coutp ? 1 : 0;
  p.N = p.xm ? coutp : cin;
  p.Mreal = p.xm ? cin : coutp;
  if (p.N > 256) return false;
  p.mtiles = (p.Mreal + 127) / 128;
  p.Mpad = p.mtiles * 128;
  auto r1k = [](uint32_t b) { return (b + 1023u) & ~1023u; };
  p.m_bytes = r1k(128u * WG_KV * 2u);
  p.n_bytes = (uint32_t)p.N * WG_KV * 2u;   // N % 16 == 0: whole 1024-byte groups, tiles back to back
  const uint32_t budget = 200u * 1024u / WG_STAGES;
  int tg = (int)((budget - p.m_bytes) / p.n_bytes);
  tg = std::min(tg, 512 / p.N);
  tg = std::min(tg, 27);
  if (tg < 1) return false;
  p.ngroups = (27 + tg - 1) / tg;
  p.TG = (27 + p.ngroups - 1) / p.ngroups;   // balance the groups
  p.ksteps = (long long)Nb * D * H * (W / WG_KV);
  // about two CTAs per SM over the whole grid, at least 16 K steps per split
  const long long ctas = (long long)p.ngroups * p.mtiles;
  long long ns = std::max(1LL, (296 + ctas - 1) / ctas);
  ns = std::min(ns, std::max(1LL, p.ksteps / 16));
  p.kper = (p.ksteps + ns - 1) / ns;
  p.nsplit = (int)((p.ksteps + p.kper - 1) / p.kper);
  const long long vox = (long long)Nb * D * H * W;
  p.m_elems = (size_t)p.Mpad * vox;
  p.n_elems = (size_t)3 * p.N * vox;
  p.part_floats = (size_t)p.nsplit * 27 * cin * coutp + (size_t)p.nsplit * coutp;
  return true;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" int mrb_cnn_tc_supported(int cin, int ci_off, int cx, int N, int W, int H) {
  if (cin <= 0 || cin % TC_BK != 0 || ci_off % 8 != 0 || cx % 8 != 0) return 0;
  if (N < 16 || N > 256 || N % 16 != 0) return 0;
  const int BW = W >= TC_BM ? TC_BM : W;
  if (BW <= 0 || TC_BM % BW != 0 || W % BW != 0) return 0;
  const int BH = TC_BM / BW;
  if (H % BH != 0 || BH > 256) return 0;
  return 1;
}

extern "C" int mrb_cnn_conv3d_tc(const void* x, int cx, int ci_off, int cin, const void* wk, int flip, int N, int cout,
                                 const float* bias, int relu, void* yb, int cyb, int yb_off, float* yf, int cyf,
                                 int yf_off, int yf_acc, int Nb, int D, int H, int W, mrb_stream_t stream) {
  MRB_REQUIRE(x && wk && (yb || yf), "null pointer");
  MRB_REQUIRE(Nb >= 1 && D >= 1 && H >= 1 && W >= 1, "bad volume");
  MRB_REQUIRE(mrb_cnn_tc_supported(cin, ci_off, cx, N, W, H), "shape not supported by the tensor-core conv");
  MRB_REQUIRE(cout <= N, "cout > N");
  MRB_REQUIRE(ci_off + cin <= cx, "channel range outside the input");
  MRB_REQUIRE(((uintptr_t)x & 15) == 0 && ((uintptr_t)wk & 15) == 0, "operands must be 16-byte aligned");
  MRB_REQUIRE(!yb || (cyb % 8 == 0 && yb_off % 8 == 0 && ((uintptr_t)yb & 15) == 0), "BF16 output misaligned");
  EncodeTiledFn enc = encode_fn();
  if (!enc) return mrb::fail(MRB_ECUDA, "cuTensorMapEncodeTiled unavailable");
  TcArgs a{};
  a.cin = cin;
  a.ci_off = ci_off;
  a.N = N;
  a.cout = cout;
  a.flip = flip;
  a.bias = bias;
  a.relu = relu;
  a.yb = (bf16*)yb;
  a.cyb = cyb;
  a.yb_off = yb_off;
  a.yf = yf;
  a.cyf = cyf;
  a.yf_off = yf_off;
  a.yf_acc = yf_acc;
  a.Nb = Nb;
  a.D = D;
  a.H = H;
  a.W = W;
  a.BW = W >= TC_BM ? TC_BM : W;
  a.BH = TC_BM / a.BW;
  a.ncols = 32;
  while (a.ncols < N) a.ncols <<= 1;
  // activations: (Nb, D, H, W, cx) bf16, box {32, BW, BH, 1, 1}
  CUtensorMap xmap, wmap;
  cuuint64_t xd[5] = {(cuuint64_t)cx, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)D, (cuuint64_t)Nb};
  cuuint64_t xs[4] = {(cuuint64_t)cx * 2, (cuuint64_t)cx * 2 * W, (cuuint64_t)cx * 2 * W * H,
                      (cuuint64_t)cx * 2 * W * H * D};
  cuuint32_t xb[5] = {(cuuint32_t)TC_BK, (cuuint32_t)a.BW, (cuuint32_t)a.BH, 1, 1};
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  CUresult r = enc(&xmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(x), xd, xs, xb, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return mrb::fail(MRB_ECUDA, "activation tensor map failed (%d)", (int)r);
  // weights: [27][N][cin] bf16 (K-major), box {32, N, 1}
  cuuint64_t wd[3] = {(cuuint64_t)cin, (cuuint64_t)N, 27};
  cuuint64_t ws[2] = {(cuuint64_t)cin * 2, (cuuint64_t)cin * 2 * N};
  cuuint32_t wb[3] = {(cuuint32_t)TC_BK, (cuuint32_t)N, 1};
  r = enc(&wmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(wk), wd, ws, wb, es,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return mrb::fail(MRB_ECUDA, "weight tensor map failed (%d)", (int)r);
  const size_t stage = ((size_t)TC_BM * TC_BK * 2 + (size_t)N * TC_BK * 2 + 1023) & ~(size_t)1023;
  const size_t smem = TC_STAGES * stage + 1024;
  MRB_CUDA_TRY(cudaFuncSetAttribute(conv3d_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long tiles = (long long)Nb * D * (H / a.BH) * (W / a.BW);
  MRB_REQUIRE(tiles < (1LL << 31), "volume too large");
  conv3d_tc_kernel<<<(unsigned)tiles, TC_THREADS, smem, (cudaStream_t)stream>>>(xmap, wmap, a);
  MRB_LAUNCH_CHECK();
  return 0;
}

// Scratch of mrb_cnn_conv3d_wgrad_tc: packed operands (BF16) then FP32 partials.
static size_t wg_scratch_bytes(const WgPlan& p) {
  size_t b = (p.m_elems + p.n_elems) * sizeof(bf16);
  b = (b + 255) & ~(size_t)255;
  return b + p.part_floats * sizeof(float);
}

extern "C" int mrb_cnn_wgrad_tc_scratch_bytes(int cin, int coutp, const int* vol, int64_t* bytes) {
  MRB_REQUIRE(vol && bytes, "null pointer");
  WgPlan p{};
  MRB_REQUIRE(wg_plan(cin, coutp, vol[0], vol[1], vol[2], vol[3], p),
              "shape not supported by the tensor-core weight gradient");
  *bytes = (int64_t)wg_scratch_bytes(p);
  return 0;
}

extern "C" int mrb_cnn_conv3d_wgrad_tc(const void* x, int cx, int ci_off, int cin, const void* gz, int cg, int cg_off,
                                       int coutp, float* dw, float* dbias, void* scratch, int64_t scratch_bytes,
                                       const int* vol, mrb_stream_t stream) {
  MRB_REQUIRE(x && gz && dw && scratch && vol, "null pointer");
  const int Nb = vol[0], D = vol[1], H = vol[2], W = vol[3];
  MRB_REQUIRE(Nb >= 1 && D >= 1 && H >= 1 && W >= 1, "bad volume");
  MRB_REQUIRE(ci_off + cin <= cx && cg_off + coutp <= cg, "channel range outside the tensor");
  MRB_REQUIRE(coutp <= 256 && 256 % coutp == 0, "bias reduction needs coutp dividing 256");
  WgPlan p{};
  MRB_REQUIRE(wg_plan(cin, coutp, Nb, D, H, W, p), "shape not supported by the tensor-core weight gradient");
  MRB_REQUIRE((size_t)scratch_bytes >= wg_scratch_bytes(p), "scratch of %lld bytes, %zu needed",
              (long long)scratch_bytes, wg_scratch_bytes(p));
  MRB_REQUIRE(((uintptr_t)scratch & 255) == 0, "scratch must be 256-byte aligned");
  EncodeTiledFn enc = encode_fn();
  if (!enc) return mrb::fail(MRB_ECUDA, "cuTensorMapEncodeTiled unavailable");
  cudaStream_t st = (cudaStream_t)stream;
  bf16* mpk = (bf16*)scratch;           // M operand, one copy, Mpad channels
  bf16* npk = mpk + p.m_elems;          // N operand, three W-shifted copies
  float* part = (float*)(((uintptr_t)(npk + p.n_elems) + 255) & ~(uintptr_t)255);
  float* bpart = part + (size_t)p.nsplit * 27 * cin * coutp;
  const bf16* msrc = (const bf16*)(p.xm ? x : gz);
  const bf16* nsrc = (const bf16*)(p.xm ? gz : x);
  const int ms = p.xm ? cx : cg, moff = p.xm ? ci_off : cg_off, mch = p.xm ? cin : coutp;
  const int ns = p.xm ? cg : cx, noff = p.xm ? cg_off : ci_off;
  {
    dim3 gm((unsigned)((W / PK_W) * (p.Mpad / 32)), (unsigned)H, (unsigned)(Nb * D));
    wg_pack_kernel<<<gm, 256, 0, st>>>(msrc, ms, moff, mch, mpk, p.Mpad, 1, D, H, W);
    MRB_LAUNCH_CHECK();
    dim3 gn((unsigned)((W / PK_W) * ((p.N + 31) / 32)), (unsigned)H, (unsigned)(Nb * D));
    wg_pack_kernel<<<gn, 256, 0, st>>>(nsrc, ns, noff, p.N, npk, p.N, 3, D, H, W);
    MRB_LAUNCH_CHECK();
  }
  // tensor maps: M (W, H, D, Mpad, Nb), box {32, 1, 1, 128, 1}; N (W, H, D, N, Nb*3), box {32, 1, 1, N, 1}
  const cuuint64_t plane = (cuuint64_t)D * H * W;
  CUtensorMap mmap, nmap;
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  {
    cuuint64_t dims[5] = {(cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)D, (cuuint64_t)p.Mpad, (cuuint64_t)Nb};
    cuuint64_t strd[4] = {(cuuint64_t)W * 2, (cuuint64_t)W * H * 2, plane * 2, plane * p.Mpad * 2};
    cuuint32_t box[5] = {(cuuint32_t)WG_KV, 1, 1, 128, 1};
    CUresult r = enc(&mmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, mpk, dims, strd, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return mrb::fail(MRB_ECUDA, "packed M-operand tensor map failed (%d)", (int)r);
  }
  {
    cuuint64_t dims[5] = {(cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)D, (cuuint64_t)p.N, (cuuint64_t)Nb * 3};
    cuuint64_t strd[4] = {(cuuint64_t)W * 2, (cuuint64_t)W * H * 2, plane * 2, plane * p.N * 2};
    cuuint32_t box[5] = {(cuuint32_t)WG_KV, 1, 1, (cuuint32_t)p.N, 1};
    CUresult r = enc(&nmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, npk, dims, strd, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return mrb::fail(MRB_ECUDA, "packed N-operand tensor map failed (%d)", (int)r);
  }
  WgArgs a{};
  a.xm = p.xm;
  a.N = p.N;
  a.Mreal = p.Mreal;
  a.cin = cin;
  a.coutp = coutp;
  a.TG = p.TG;
  a.Nb = Nb;
  a.D = D;
  a.H = H;
  a.W = W;
  a.ksteps = p.ksteps;
  a.kper = p.kper;
  a.ngroups = p.ngroups;
  a.mtiles = p.mtiles;
  a.part = part;
  a.ncols = 32;
  while (a.ncols < p.TG * p.N) a.ncols <<= 1;
  a.m_bytes = p.m_bytes;
  a.n_bytes = p.n_bytes;
  const size_t smem = WG_STAGES * (size_t)(p.m_bytes + p.TG * p.n_bytes) + 1024;
  MRB_REQUIRE(smem <= 227 * 1024, "weight gradient stages need %zu bytes of shared memory", smem);
  MRB_CUDA_TRY(cudaFuncSetAttribute(wgrad_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long blocks = (long long)p.ngroups * p.mtiles * p.nsplit;
  MRB_REQUIRE(blocks < (1LL << 31), "volume too large");
  wgrad_tc_kernel<<<(unsigned)blocks, TC_THREADS, smem, st>>>(mmap, nmap, a);
  MRB_LAUNCH_CHECK();
  const long long nw = 27LL * cin * coutp;
  wg_sum_kernel<<<(unsigned)((nw + 255) / 256), 256, 0, st>>>(part, p.nsplit, nw, dw);
  MRB_LAUNCH_CHECK();
  if (dbias) {
    const long long vox = (long long)Nb * D * H * W;
    const long long vper = (vox + p.nsplit - 1) / p.nsplit;
    wg_bias_kernel<<<(unsigned)p.nsplit, 256, 0, st>>>((const bf16*)gz, cg, cg_off, coutp, vox, vper, bpart);
    MRB_LAUNCH_CHECK();
    wg_sum_kernel<<<(unsigned)((coutp + 255) / 256), 256, 0, st>>>(bpart, p.nsplit, coutp, dbias);
    MRB_LAUNCH_CHECK();
  }
  return 0;
}

// Reads and clears the timeout flag of the tensor-core conv (synchronous).
extern "C" int mrb_cnn_tc_error(int* out) {
  MRB_REQUIRE(out != nullptr, "null pointer");
  int zero = 0;
  MRB_CUDA_TRY(cudaMemcpyFromSymbol(out, g_tc_error, sizeof(int)));
  MRB_CUDA_TRY(cudaMemcpyToSymbol(g_tc_error, &zero, sizeof(int)));
  return 0;
}
