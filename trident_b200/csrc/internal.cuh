// internal.cuh — shared internals of libtspg: the context, its stream-ordered
// workspace pool, status plumbing and small device helpers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <mutex>
#include <unordered_map>

#include "tspg.h"

namespace tspg {
// Class limits = table capacities (symbolic: on min(mults, ncols); numeric: on
// the row's nnz).  Symbolic tables hold int32 keys (128 KiB per CTA), numeric
// tables hold key + FP64 value (192 KiB per CTA); a table has T = pow2 >=
// load x the bound slots.
constexpr int64_t kSymLim32 = 512, kSymLim128 = 2048, kSymLim256 = 4096, kSymLim1024 = 24576;
constexpr int64_t kNumLim32 = 256, kNumLim128 = 1024, kNumLim256 = 2048, kNumLim1024 = 8192;

// Runtime row-binning parameters (the autotuned part of the SpGEMM): upper
// bounds of the warp / 128 / 256 / CTA group classes, symbolic on
// min(products, ncols) and numeric on the row's nnz, and the hash-table slots
// per key.  Bounds never exceed the compile-time table capacities
// (kSymLim*, kNumLim*); tspg_ctx_set_tuning checks that.
struct Tune {
  int32_t sym[4];
  int32_t num[4];
  int32_t load;
  int32_t win;   // log2 of the products from which DENSE numeric rows take the window form; 0 = never
  int32_t fill;  // ... when their output also fills >= 1 / 2^fill of the columns
  int32_t cluster;  // CTAs per thread-block cluster working on one such row (0 = one CTA)
};
constexpr int32_t kDefaultWinLog2 = 0, kDefaultWinFillLog2 = 4;  // window form off by default (measured slower)

// A tuning is valid when every bound is positive, non-decreasing over the
// classes and within the table capacity of its class, and load is 2, 4 or 8.
inline bool tune_valid(const Tune &t) {
  const int64_t smax[4] = {kSymLim32, kSymLim128, kSymLim256, kSymLim1024};
  const int64_t nmax[4] = {kNumLim32, kNumLim128, kNumLim256, kNumLim1024};
  for (int i = 0; i < 4; ++i) {
    if (t.sym[i] < 1 || t.sym[i] > smax[i] || t.num[i] < 1 || t.num[i] > nmax[i]) return false;
    if (i > 0 && (t.sym[i] < t.sym[i - 1] || t.num[i] < t.num[i - 1])) return false;
  }
  if (t.win != 0 && (t.win < 10 || t.win > 40)) return false;
  if (t.fill < 0 || t.fill > 12) return false;
  if (t.cluster != 0 && t.cluster != 2 && t.cluster != 4 && t.cluster != 8) return false;
  return t.load == 2 || t.load == 4 || t.load == 8;
}
}  // namespace tspg

struct tspg_ctx {
  int device = 0;
  int num_sms = 0;
  size_t smem_optin = 0;
  cudaMemPool_t pool = nullptr;
  size_t budget = 0;  // 0 = unlimited
  size_t in_use = 0;
  size_t high_water = 0;
  int last_cuda = 0;
  // pinned host words for small read-backs (sizes, flags)
  int64_t *h_words = nullptr;
  // device words: error flag and small counters that live with the context
  int64_t *d_words = nullptr;
  std::unordered_map<void *, size_t> live;
  std::mutex live_mu;  // ws_alloc / ws_free may be called from a releasing thread
  // instrumentation
  int64_t launches = 0;        // library kernels launched (graph nodes included)
  bool phase_timing = false;   // record events around the persistent phases
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  bool ev_sym = false, ev_num = false;
  // per-class cycle accounting of the persistent phases: [phase][2 * 7]
  unsigned long long *d_prof = nullptr;
  // row binning (tspg_ctx_set_tuning); the defaults are the table capacities
  tspg::Tune tune = {{int32_t(tspg::kSymLim32), int32_t(tspg::kSymLim128),
                      int32_t(tspg::kSymLim256), int32_t(tspg::kSymLim1024)},
                     {int32_t(tspg::kNumLim32), int32_t(tspg::kNumLim128),
                      int32_t(tspg::kNumLim256), int32_t(tspg::kNumLim1024)},
                     2,
                     tspg::kDefaultWinLog2,
                     tspg::kDefaultWinFillLog2,
                     0};
};

namespace tspg {

constexpr int kHostWords = 64;
constexpr int kDevWords = 64;
// d_words slots
constexpr int kErrWord = 0;  // device-side error code (0 = ok)

#define TSPG_CUDA(ctx, ...)                                   \
  do {                                                        \
    cudaError_t _e = (__VA_ARGS__);                           \
    if (_e != cudaSuccess) {                                  \
      (ctx)->last_cuda = (int)_e;                             \
      return TSPG_ECUDA;                                      \
    }                                                         \
  } while (0)

#define TSPG_TRY(...)                 \
  do {                                \
    int _s = (__VA_ARGS__);           \
    if (_s != TSPG_OK) return _s;     \
  } while (0)

// Event pair k (0: symbolic phase, 1: numeric phase) around the two persistent
// kernels of a phase (k_phase, then k_groups).
inline void phase_mark(tspg_ctx *ctx, int k, int edge, cudaStream_t s) {
  if (!ctx->phase_timing) return;
  cudaEventRecord(ctx->ev[2 * k + edge], s);
  if (edge == 1) (k == 0 ? ctx->ev_sym : ctx->ev_num) = true;
}

// Stream-ordered workspace from the context pool, with the budget enforced.
int ws_alloc(tspg_ctx *ctx, void **p, size_t bytes, cudaStream_t s);
void ws_free(tspg_ctx *ctx, void *p, cudaStream_t s);

// RAII list of workspace blocks released at scope exit on one stream.
struct Scratch {
  tspg_ctx *ctx;
  cudaStream_t s;
  void *ptrs[32];
  int n = 0;
  Scratch(tspg_ctx *c, cudaStream_t st) : ctx(c), s(st) {}
  template <typename T>
  int get(T **p, size_t count) {
    void *q = nullptr;
    size_t bytes = count * sizeof(T);
    if (bytes == 0) bytes = 16;
    int st = ws_alloc(ctx, &q, bytes, s);
    if (st != TSPG_OK) return st;
    ptrs[n++] = q;
    *p = (T *)q;
    return TSPG_OK;
  }
  ~Scratch() {
    for (int i = n - 1; i >= 0; --i) ws_free(ctx, ptrs[i], s);
  }
};

inline int check_csr(const tspg_csr *M) {
  if (!M) return TSPG_EINVAL;
  if (M->nrows < 0 || M->ncols < 0 || M->nnz < 0) return TSPG_EINVAL;
  if (M->rowptr_bits != 32 && M->rowptr_bits != 64) return TSPG_EINVAL;
  if (M->val_bits != 32 && M->val_bits != 64) return TSPG_EINVAL;
  if (M->ncols > INT32_MAX) return TSPG_EINVAL;  // int32 column indices
  if (M->rowptr_bits == 32 && M->nnz > INT32_MAX) return TSPG_EOVERFLOW;
  if (M->nnz > 0 && (!M->col || !M->val)) return TSPG_EINVAL;
  if (!M->rowptr && M->nrows > 0) return TSPG_EINVAL;
  return TSPG_OK;
}

// ---------------------------------------------------------------- device side

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}

// Inclusive warp scan.
template <typename T>
__device__ __forceinline__ T warp_scan_incl(T v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T w = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += w;
  }
  return v;
}

// Synchronise a group of G threads.  G = 32: the warp.  G = 256 / 128: named
// barriers 1-4 / 5-12, disjoint so that 256- and 128-thread groups of one CTA
// can be active at the same time.  Any other G is a whole block.
template <int G>
__device__ __forceinline__ void group_sync(int gid) {
  if constexpr (G == 32) {
    __syncwarp();
  } else if constexpr (G == 256) {
    asm volatile("bar.sync %0, %1;" ::"r"(gid + 1), "r"(G) : "memory");
  } else if constexpr (G == 128) {
    asm volatile("bar.sync %0, %1;" ::"r"(gid + 5), "r"(G) : "memory");
  } else {
    __syncthreads();
  }
}

// Exclusive scan across a group of G threads; `tmp` holds G/32 + 1 ints of
// shared memory private to the group.  Returns the exclusive prefix; the group
// total goes to *total.
template <int G, typename T>
__device__ __forceinline__ T group_excl_scan(T v, T *tmp, int gid, T *total) {
  const int lane = threadIdx.x & 31;
  T inc = warp_scan_incl(v);
  if constexpr (G == 32) {
    *total = __shfl_sync(0xffffffffu, inc, 31);
    return inc - v;
  } else {
    constexpr int NW = G / 32;
    const int w = (threadIdx.x % G) >> 5;
    if (lane == 31) tmp[w] = inc;
    group_sync<G>(gid);
    if (w == 0) {
      T x = lane < NW ? tmp[lane] : T(0);
      T xi = warp_scan_incl(x);
      if (lane < NW) tmp[lane] = xi - x;
      if (lane == NW - 1) tmp[NW] = xi;
    }
    group_sync<G>(gid);
    T res = tmp[w] + inc - v;
    *total = tmp[NW];
    group_sync<G>(gid);
    return res;
  }
}

template <int G, typename T>
__device__ __forceinline__ T group_sum(T v, T *tmp, int gid) {
  T total;
  group_excl_scan<G, T>(v, tmp, gid, &total);
  return total;
}

// Min and max across a group (tmp: 2 * (G/32) + 2 ints of group-private smem).
template <int G>
__device__ __forceinline__ void group_minmax(int &mn, int &mx, int *tmp, int gid) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if constexpr (G > 32) {
    constexpr int NW = G / 32;
    const int w = (threadIdx.x % G) >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
      tmp[w] = mn;
      tmp[NW + w] = mx;
    }
    group_sync<G>(gid);
    mn = tmp[0];
    mx = tmp[NW];
    for (int i = 1; i < NW; ++i) {
      mn = min(mn, tmp[i]);
      mx = max(mx, tmp[NW + i]);
    }
    group_sync<G>(gid);
  }
}

__device__ __forceinline__ void set_error(int64_t *err, int code) {
  atomicCAS((unsigned long long *)err, 0ull, (unsigned long long)code);
}

// Fire-and-forget global reduction (PTX `red`): no value comes back, so the
// issuing thread never waits on the L2 round trip.
__device__ __forceinline__ void red_add(double *p, double v) {
  asm volatile("red.relaxed.gpu.global.add.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
// L2 eviction-priority policies (PTX createpolicy) and the stores and
// reductions that carry them.  evict_last marks lines that will be hit again
// soon (a DENSE row's values, reduced into while the row is worked on),
// evict_first lines written once (its column indices).
__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ void red_add_hint(double *p, double v, uint64_t pol) {
  asm volatile("red.relaxed.gpu.global.add.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(p), "d"(v),
               "l"(pol) : "memory");
}
__device__ __forceinline__ void red_add_hint(float *p, float v, uint64_t pol) {
  asm volatile("red.relaxed.gpu.global.add.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(v),
               "l"(pol) : "memory");
}
__device__ __forceinline__ void store_hint(double *p, double v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(p), "d"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void store_hint(float *p, float v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void store_hint(int32_t *p, int32_t v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.b32 [%0], %1, %2;" ::"l"(p), "r"(v), "l"(pol) : "memory");
}
// 16 zero bytes at a 16-byte aligned address
__device__ __forceinline__ void store_zero16(void *p, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v4.b32 [%0], {%1, %1, %1, %1}, %2;" ::"l"(p), "r"(0),
               "l"(pol) : "memory");
}
__device__ __forceinline__ void red_add(float *p, float v) {
  asm volatile("red.relaxed.gpu.global.add.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}

}  // namespace tspg
