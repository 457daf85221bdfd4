// Grouped launches: one kernel launch serves many independent problems.
//
// A kernel of the library that may be grouped is written as a body,
//
//   struct Body { static constexpr int NT = threads per block, MINB = ...;
//                 static __device__ void run(const VBlock& vb, args...); };
//
// whose block coordinates come from `vb` instead of blockIdx / gridDim.  The
// grouped kernel grouped_kernel<Body, ...> receives, as one by-value kernel
// parameter (the 32 KB parameter space of CUDA 12.1+, read in place through
// __grid_constant__), a table of up to MAXG argument lists with each list's
// grid and its first block in the combined grid.  A block finds its problem
// by binary search over the first-block table and runs the body on that
// problem's arguments with that problem's own block coordinates.
//
// The grouped kernel reads its arguments from the table where a plain kernel
// reads them as constant operands, so it needs more registers: MINB bounds
// them (__launch_bounds__ minimum blocks per SM) to keep the plain kernel's
// occupancy.  MAXG (default 64) caps the problems per launch, and with it the
// parameter table a launch carries.
//
// Launch sites call launch<Body>(named_kernel, grid, smem, stream, args...).
// Outside a recording that launches the named kernel (a __global__ wrapper
// that passes hw_block()).  The named kernel and the grouped kernel are two
// compilations of one body; they produce the same bits because nothing in a
// body leaves the rounding to the compiler: the files that hold bodies with
// arithmetic the compiler could fuse differently in the two kernels (a
// multiply feeding an add) compile without automatic fusion (-fmad=false,
// build.py) and write every fused multiply-add as fmaf / fma; the interp and
// spread bodies use only explicit fused multiply-adds on such paths.
// Between mrb_group_begin and mrb_group_end the call is recorded for the
// problem selected with mrb_group_select; mrb_group_end replays the records
// step by step (group.cu): FAMILY names the kernel step a body performs (the
// bodies of one step differ only in compile-time shape, e.g. the FFT length),
// the k-th records of a step in every problem form one step of the replay,
// and the records of one step that run the same body form one grouped launch.
// A kernel launched any other way while a recording is open makes its entry
// point fail (MRB_LAUNCH_CHECK).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstring>
#include <type_traits>
#include <vector>

#include "mrb_common.cuh"

namespace mrb {

// block coordinates of a body: the hardware ones in a plain launch, the
// problem-local ones inside a grouped launch
struct VBlock {
  unsigned x, y, z;      // block index
  unsigned nx, ny, nz;   // grid size
};

__device__ __forceinline__ VBlock hw_block() {
  return VBlock{blockIdx.x, blockIdx.y, blockIdx.z, gridDim.x, gridDim.y, gridDim.z};
}

// a kernel's argument list as one trivially copyable value
template <class... A> struct Pack;
template <> struct Pack<> {};
template <class H, class... T> struct Pack<H, T...> {
  H h;
  Pack<T...> t;
};

inline Pack<> make_pack() { return Pack<>{}; }
template <class H, class... T> Pack<H, T...> make_pack(H h, T... t) { return Pack<H, T...>{h, make_pack(t...)}; }

template <int I, class P> __host__ __device__ __forceinline__ const auto& pack_get(const P& p) {
  if constexpr (I == 0) return p.h;
  else return pack_get<I - 1>(p.t);
}

template <int... I> struct Seq {};
template <int N, int... I> struct MakeSeq : MakeSeq<N - 1, N - 1, I...> {};
template <int... I> struct MakeSeq<0, I...> { using type = Seq<I...>; };

template <class T> struct Ident { using type = T; };

// optional body constants
template <class K, class = void> struct BodyMaxG { static constexpr int value = 64; };
template <class K> struct BodyMaxG<K, std::void_t<decltype(K::MAXG)>> { static constexpr int value = K::MAXG; };
template <class K, class = void> struct BodyFamily { static constexpr const char* value = nullptr; };
template <class K> struct BodyFamily<K, std::void_t<decltype(K::FAMILY)>> {
  static constexpr const char* value = K::FAMILY;
};

// kernel parameter space (32764 bytes from CUDA 12.1 on sm_70+), with room to spare
constexpr size_t GROUP_PARAM_BYTES = 32000;

template <class K, class P> constexpr int group_max() {
  constexpr size_t per = sizeof(P) + 4 * sizeof(unsigned);   // arguments, grid and first block
  constexpr size_t m = (GROUP_PARAM_BYTES - 64) / per;
  constexpr int cap = BodyMaxG<K>::value;
  return m > (size_t)cap ? cap : (int)m;
}

template <class P, int M> struct GroupTable {
  int n;                  // problems in this launch
  unsigned first[M + 1];  // first block of each problem in the combined grid; first[n] = total
  unsigned dim[M][3];     // each problem's own grid
  P args[M];
};

template <class K, class P, int M, int... I>
__device__ __forceinline__ void group_run(const GroupTable<P, M>& t, Seq<I...>) {
  const unsigned b = blockIdx.x;
  int lo = 0, hi = t.n - 1;   // the last problem whose first block is <= b
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (t.first[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  const unsigned l = b - t.first[lo];
  const unsigned nx = t.dim[lo][0], ny = t.dim[lo][1], nz = t.dim[lo][2];
  const VBlock vb{l % nx, (l / nx) % ny, l / (nx * ny), nx, ny, nz};
  K::run(vb, pack_get<I>(t.args[lo])...);
}

template <class K, class P, int M, class S>
__global__ void __launch_bounds__(K::NT, K::MINB) grouped_kernel(const __grid_constant__ GroupTable<P, M> t) {
  group_run<K>(t, S{});
}

// one recorded launch
struct LaunchRec {
  const void* key;                  // identifies the body and its argument types
  const char* family;               // the kernel step the body belongs to (its shapes share it), or null
  int occ;                          // earlier records of the same step in this problem's list
  const void* kern;                 // the named kernel
  dim3 grid;
  unsigned threads;
  size_t smem;
  std::vector<unsigned char> args;  // a Pack of the arguments
  int (*single)(const LaunchRec& r, cudaStream_t st);
  int (*group)(const LaunchRec* const* recs, int n, cudaStream_t st);
};

bool group_recording();
int group_record(LaunchRec&& r);
int set_max_smem(const void* fn, size_t bytes, size_t* done);

template <class K, class... A> struct GroupLauncher {
  using P = Pack<A...>;
  static constexpr int M = group_max<K, P>();
  using Table = GroupTable<P, M>;
  using S = typename MakeSeq<(int)sizeof...(A)>::type;
  static_assert(M >= 1, "argument list too large for a grouped launch");
  static_assert(sizeof(Table) <= 32764, "group table exceeds the kernel parameter space");

  static char key_tag;   // its address identifies (K, A...)

  template <int... I> static int launch_named(const LaunchRec& r, cudaStream_t st, Seq<I...>) {
    P p;
    std::memcpy(&p, r.args.data(), sizeof(P));
    void* ptrs[] = {const_cast<void*>(static_cast<const void*>(&pack_get<I>(p)))..., nullptr};
    MRB_CUDA_TRY(cudaLaunchKernel(r.kern, r.grid, dim3(r.threads), ptrs, r.smem, st));
    count_launch();
    return 0;
  }

  static int group(const LaunchRec* const* recs, int n, cudaStream_t st) {
    static size_t smem_done = 0;
    const void* gk = (const void*)grouped_kernel<K, P, M, S>;
    for (int i0 = 0; i0 < n; i0 += M) {
      const int m = n - i0 < M ? n - i0 : M;
      std::vector<unsigned char> buf(sizeof(Table));
      Table* t = reinterpret_cast<Table*>(buf.data());
      t->n = 0;
      unsigned long long total = 0;
      size_t smem = 0;
      for (int i = 0; i < m; ++i) {
        const LaunchRec& r = *recs[i0 + i];
        const unsigned long long nbk = (unsigned long long)r.grid.x * r.grid.y * r.grid.z;
        if (nbk == 0) continue;
        const int j = t->n++;
        t->first[j] = (unsigned)total;
        t->dim[j][0] = r.grid.x;
        t->dim[j][1] = r.grid.y;
        t->dim[j][2] = r.grid.z;
        std::memcpy(&t->args[j], r.args.data(), sizeof(P));
        total += nbk;
        if (r.smem > smem) smem = r.smem;
      }
      if (t->n == 0) continue;
      MRB_REQUIRE(total < (1ull << 31), "grouped launch of %llu blocks", total);
      t->first[t->n] = (unsigned)total;
      if (int rc = set_max_smem(gk, smem, &smem_done)) return rc;
      void* ptrs[] = {buf.data()};
      MRB_CUDA_TRY(cudaLaunchKernel(gk, dim3((unsigned)total), dim3(K::NT), ptrs, smem, st));
      count_launch();
    }
    return 0;
  }

  static int single(const LaunchRec& r, cudaStream_t st) {
    if ((long long)r.grid.x * r.grid.y * r.grid.z == 0) return 0;
    return launch_named(r, st, S{});
  }
};

template <class K, class... A> char GroupLauncher<K, A...>::key_tag = 0;

// Launch (or, inside a recording, record) body K; `kern` is its named kernel.
template <class K, class... A>
int launch(void (*kern)(A...), dim3 grid, size_t smem, cudaStream_t st, typename Ident<A>::type... a) {
  using L = GroupLauncher<K, A...>;
  if (!group_recording()) {
    if ((long long)grid.x * grid.y * grid.z == 0) return 0;
    kern<<<grid, K::NT, smem, st>>>(a...);
    MRB_LAUNCH_CHECK();
    return 0;
  }
  LaunchRec r;
  r.key = &L::key_tag;
  r.family = BodyFamily<K>::value;
  r.occ = 0;
  r.kern = (const void*)kern;
  r.grid = grid;
  r.threads = K::NT;
  r.smem = smem;
  typename L::P p = make_pack<A...>(a...);
  r.args.resize(sizeof(p));
  std::memcpy(r.args.data(), &p, sizeof(p));
  r.single = &L::single;
  r.group = &L::group;
  return group_record(std::move(r));
}

}  // namespace mrb
