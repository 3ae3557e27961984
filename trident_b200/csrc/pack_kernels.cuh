// pack_kernels.cuh — device kernels of the bitmask tile pack (masked segment
// counts and the copy pass), shared by tspg_pack and tspg_pack_noalloc.
#pragma once

#include <type_traits>

#include "internal.cuh"

namespace tspg {

// Masked segment lengths (select_ptrs' MaskedTransform, spacomm.cuh:539-553).
template <typename PT>
__global__ void k_pack_counts(const PT *ptr, int64_t len, const uint8_t *mask,
                              int32_t *cnt) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < len) {
    const bool keep = (mask[i >> 3] >> (i & 7)) & 1;
    cnt[i] = keep ? int32_t(int64_t(ptr[i + 1]) - int64_t(ptr[i])) : 0;
  }
}

constexpr int kPackItems = 8;

// Copy pass.  Entry e belongs to the last segment r with ptr[r] <= e (the
// reference's locate_segment_by_pos, spacomm.cuh:714-725); it is kept iff bit
// r is set and goes to newp[r] + (e - ptr[r]).  The pointer region starts at
// kept*(val+4) bytes rounded up to the pointer width (no padding for the
// reference's int32 pointers; at most 4 bytes for int64 ones).
template <typename PT, int VB>
__global__ void __launch_bounds__(256)
    k_pack_copy(const PT *ptr, int64_t len, const int32_t *idx, const void *val,
                const uint8_t *mask, const int64_t *newp, char *out,
                int64_t *kept_dev) {
  using V = typename std::conditional<VB == 8, unsigned long long, unsigned>::type;
  const int64_t kept = newp[len];
  // an empty pointer array (len == 0) may be null and holds no entries
  const int64_t nnz = len > 0 ? int64_t(ptr[len]) : 0;
  V *oval = (V *)out;
  int32_t *oidx = (int32_t *)(out + kept * VB);
  const V *ival = (const V *)val;
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  // entries: thread t covers [t*K, t*K + K) within each sweep
  for (int64_t e0 = t * kPackItems; e0 < nnz; e0 += stride * kPackItems) {
    int64_t lo = 0, hi = len;  // last r in [0, len) with ptr[r] <= e0
    while (hi - lo > 1) {
      const int64_t mid = (lo + hi) >> 1;
      if (int64_t(ptr[mid]) <= e0) lo = mid; else hi = mid;
    }
    int64_t r = lo;
    int64_t rend = ptr[r + 1];
    const int64_t e1 = e0 + kPackItems < nnz ? e0 + kPackItems : nnz;
    for (int64_t e = e0; e < e1; ++e) {
      while (e >= rend) {
        ++r;
        rend = ptr[r + 1];
      }
      if ((mask[r >> 3] >> (r & 7)) & 1) {
        const int64_t o = newp[r] + (e - int64_t(ptr[r]));
        oval[o] = ival[e];
        oidx[o] = idx[e];
      }
    }
  }
  // pointer array of the packed tile
  PT *optr = (PT *)(out + ((kept * (VB + 4) + int64_t(sizeof(PT)) - 1) &
                           ~(int64_t(sizeof(PT)) - 1)));
  for (int64_t i = t; i <= len; i += stride) optr[i] = PT(newp[i]);
  if (t == 0 && kept_dev) *kept_dev = kept;
}

}  // namespace tspg
