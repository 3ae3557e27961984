// spgemm_phase.cuh — the persistent symbolic / numeric kernels.
//
// One 1024-thread CTA per SM (192 KiB of dynamic shared memory) pulls work
// items from a device counter; an item is one DENSE or G1024 row, 4 G256
// rows, 8 G128 rows or 64 G32 rows.  Item numbers run heaviest class first.
#pragma once

#include "spgemm_kernels.cuh"

namespace tspg {

// Product loop: sub-groups of S threads take A entries in turn; the S threads
// of a sub-group stride over that entry's B row.  f(col, a*b) per product.
template <int G, bool NUM, typename PT, typename VT, typename F>
__device__ __forceinline__ void for_products(const int32_t *__restrict__ Aj,
                                             const VT *__restrict__ Ax,
                                             const PT *__restrict__ Bp,
                                             const int32_t *__restrict__ Bj,
                                             const VT *__restrict__ Bx,
                                             int64_t a0, int64_t a1, int S,
                                             int lane, F &&f) {
  const int sub = lane / S, sl = lane - sub * S, nsub = G / S;
  for (int64_t p = a0 + sub; p < a1; p += nsub) {
    const int64_t k = __ldg(Aj + p);
    VT a = VT(0);
    if constexpr (NUM) a = __ldg(Ax + p);
    const int64_t b1 = __ldg(Bp + k + 1);
    for (int64_t q = __ldg(Bp + k) + sl; q < b1; q += S) {
      if constexpr (NUM) f(__ldg(Bj + q), a * __ldg(Bx + q));
      else f(__ldg(Bj + q), VT(0));
    }
  }
}

// Probe bound: tables are sized T >= 2 * (distinct keys), so a probe never
// runs T steps; the bound only turns a broken invariant into an error flag.
__device__ __forceinline__ int sym_insert(int *keys, int32_t col, int logT,
                                          uint32_t mask, int64_t *err) {
  uint32_t h = hash_slot(col, logT);
  for (uint32_t it = 0; it <= mask; ++it) {
    const int k = ((volatile int *)keys)[h];
    if (k == col) return 0;
    if (k == -1) {
      const int old = atomicCAS(keys + h, -1, col);
      if (old == -1) return 1;
      if (old == col) return 0;
    }
    h = (h + 1) & mask;
  }
  set_error(err, 101);
  return 0;
}

__device__ __forceinline__ uint32_t num_insert(int *keys, int32_t col,
                                               int logT, uint32_t mask,
                                               int64_t *err) {
  uint32_t h = hash_slot(col, logT);
  for (uint32_t it = 0; it <= mask; ++it) {
    const int k = ((volatile int *)keys)[h];
    if (k == col) return h;
    if (k == -1) {
      const int old = atomicCAS(keys + h, -1, col);
      if (old == -1 || old == col) return h;
    }
    h = (h + 1) & mask;
  }
  set_error(err, 102);
  return 0;
}

struct PhaseArgs {
  const int64_t *base;
  Sched *S;
  const uint64_t *list;
  const int64_t *rowf;
  int32_t *rowc;
  const int64_t *cp;
  int32_t *curbuf;     // per-CTA cursor scratch for DENSE rows with long A rows
  int64_t cur_stride;  // entries per CTA in curbuf
  int64_t *err;
};

// ---------------------------------------------------------------- symbolic

template <int G, int TMAX, typename PT, typename VT>
__device__ void sym_hash_rows(const ProdDev<PT, VT> *prods,
                              const PhaseArgs &A, int64_t first, int64_t last,
                              unsigned char *smem, int64_t *scan_tmp) {
  constexpr int NG = kThreads / G;
  constexpr int RPI = cls_rows_per_item(
      G == 1024 ? CLS_G1024 : G == 256 ? CLS_G256 : G == 128 ? CLS_G128 : CLS_G32);
  static_assert(NG * TMAX * 4 <= kDynSmem, "symbolic table exceeds shared memory");
  const int gid = threadIdx.x / G, lane = threadIdx.x % G;
  int *keys = (int *)smem + gid * TMAX;
  int64_t *tmp = scan_tmp + gid * 33;
  for (int64_t idx = first + gid; idx < last && idx < first + RPI; idx += NG) {
    const uint64_t e = A.list[idx];
    const int p = int(e >> 40);
    const int64_t r = int64_t(e & ((uint64_t(1) << 40) - 1));
    const int64_t g = A.base[p] + r;
    const ProdDev<PT, VT> &P = prods[p];
    const int64_t f = A.rowf[g];
    const int64_t n = P.n;
    const int64_t fe = f < n ? f : n;
    uint32_t T = pow2_at_least(2 * fe, 32);
    if (T > TMAX) T = TMAX;
    const int logT = ilog2_pow2(T);
    const uint32_t mask = T - 1;
    for (uint32_t s = lane; s < T; s += G) keys[s] = -1;
    group_sync<G>(gid);
    const int64_t a0 = P.Ap[r], a1 = P.Ap[r + 1];
    const int S = subgroup_width(f, a1 - a0, G);
    int cnt = 0;
    for_products<G, false, PT, VT>(P.Aj, P.Ax, P.Bp, P.Bj, P.Bx, a0, a1, S,
                                   lane, [&](int32_t col, VT) {
                                     cnt += sym_insert(keys, col, logT, mask,
                                                       A.err);
                                   });
    group_sync<G>(gid);
    const int64_t total = group_sum<G, int64_t>(int64_t(cnt), tmp, gid);
    if (lane == 0) A.rowc[g] = int32_t(total);
    group_sync<G>(gid);
  }
}

template <typename PT, typename VT>
__device__ void sym_dense_row(const ProdDev<PT, VT> *prods, const PhaseArgs &A,
                              int64_t idx, unsigned char *smem,
                              int64_t *scan_tmp) {
  const int tid = threadIdx.x;
  uint32_t *bm = (uint32_t *)smem;
  const uint64_t e = A.list[idx];
  const int p = int(e >> 40);
  const int64_t r = int64_t(e & ((uint64_t(1) << 40) - 1));
  const int64_t g = A.base[p] + r;
  const ProdDev<PT, VT> &P = prods[p];
  const int64_t n = P.n;
  const int64_t a0 = P.Ap[r], a1 = P.Ap[r + 1];
  const int S = subgroup_width(A.rowf[g], a1 - a0, 32);
  const int64_t W = n < kDenseBits ? n : kDenseBits;
  int64_t total = 0;
  for (int64_t w0 = 0; w0 < n; w0 += W) {
    const int64_t w1 = (w0 + W < n) ? w0 + W : n;
    const int64_t nw = (w1 - w0 + 31) >> 5;
    for (int64_t i = tid; i < nw; i += kThreads) bm[i] = 0u;
    __syncthreads();
    for_products<kThreads, false, PT, VT>(
        P.Aj, P.Ax, P.Bp, P.Bj, P.Bx, a0, a1, S, tid, [&](int32_t col, VT) {
          if (col >= w0 && col < w1) {
            const uint32_t o = uint32_t(col - w0);
            const uint32_t bit = 1u << (o & 31);
            if (!(((volatile uint32_t *)bm)[o >> 5] & bit))
              atomicOr(bm + (o >> 5), bit);
          }
        });
    __syncthreads();
    int64_t local = 0;
    for (int64_t i = tid; i < nw; i += kThreads) local += __popc(bm[i]);
    total += group_sum<kThreads, int64_t>(local, scan_tmp, 0);
  }
  if (tid == 0) A.rowc[g] = int32_t(total);
}

// ---------------------------------------------------------------- numeric

template <int G, int TMAX, typename PT, typename VT>
__device__ void num_hash_rows(const ProdDev<PT, VT> *prods,
                              const PhaseArgs &A, int64_t first, int64_t last,
                              unsigned char *smem, int64_t *scan_tmp) {
  constexpr int NG = kThreads / G;
  constexpr int SLICE = TMAX * 12;  // FP64 value + int32 key per slot
  constexpr int RPI = cls_rows_per_item(
      G == 1024 ? CLS_G1024 : G == 256 ? CLS_G256 : G == 128 ? CLS_G128 : CLS_G32);
  static_assert(NG * SLICE <= kDynSmem, "numeric table exceeds shared memory");
  static_assert(TMAX / 2 <= 8 * G, "compaction keeps 8 first-half slots per thread");
  const int gid = threadIdx.x / G, lane = threadIdx.x % G;
  unsigned char *slice = smem + gid * SLICE;
  VT *vals = (VT *)slice;
  int *keys = (int *)(slice + TMAX * 8);
  int64_t *tmp = scan_tmp + gid * 33;
  for (int64_t idx = first + gid; idx < last && idx < first + RPI; idx += NG) {
    const uint64_t e = A.list[idx];
    const int p = int(e >> 40);
    const int64_t r = int64_t(e & ((uint64_t(1) << 40) - 1));
    const int64_t g = A.base[p] + r;
    const ProdDev<PT, VT> &P = prods[p];
    const int64_t c = A.rowc[g];
    const int64_t off = A.cp[g] - A.cp[A.base[p]];
    uint32_t T = pow2_at_least(2 * c, 32);
    if (T > TMAX) T = TMAX;
    const int logT = ilog2_pow2(T);
    const uint32_t mask = T - 1;
    for (uint32_t s = lane; s < T; s += G) {
      keys[s] = -1;
      vals[s] = VT(0);
    }
    group_sync<G>(gid);
    const int64_t a0 = P.Ap[r], a1 = P.Ap[r + 1];
    const int S = subgroup_width(A.rowf[g], a1 - a0, G);
    for_products<G, true, PT, VT>(P.Aj, P.Ax, P.Bp, P.Bj, P.Bx, a0, a1, S,
                                  lane, [&](int32_t col, VT v) {
                                    const uint32_t h =
                                        num_insert(keys, col, logT, mask, A.err);
                                    atomicAdd(vals + h, v);
                                  });
    group_sync<G>(gid);
    // In-place compaction into [0, c): the targets lie in the first half of
    // the table (c <= T/2), so only first-half slots are read into registers
    // before the group barrier inside the scan; second-half slots are never
    // overwritten and are read after it.
    const uint32_t H = T >> 1;
    int rk[8];
    VT rv[8];
    int64_t mine = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const uint32_t s = lane + i * G;
      rk[i] = -1;
      rv[i] = VT(0);
      if (s < H) {
        rk[i] = keys[s];
        rv[i] = vals[s];
      }
      mine += rk[i] != -1;
    }
    for (uint32_t s = H + lane; s < T; s += G) mine += keys[s] != -1;
    int64_t tot;
    int64_t pos = group_excl_scan<G, int64_t>(mine, tmp, gid, &tot);
    group_sync<G>(gid);
    if (lane == 0 && tot != c) set_error(A.err, 103);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if (rk[i] != -1) {
        keys[pos] = rk[i];
        vals[pos] = rv[i];
        ++pos;
      }
    }
    for (uint32_t s = H + lane; s < T; s += G) {
      const int k = keys[s];
      if (k != -1) {
        const VT v = vals[s];
        keys[pos] = k;
        vals[pos] = v;
        ++pos;
      }
    }
    group_sync<G>(gid);
    for (uint32_t s = uint32_t(c) + lane; s < H; s += G) keys[s] = INT32_MAX;
    group_sync<G>(gid);
    // Bitonic sort of the H = pow2 >= c compacted pairs by column.
    for (uint32_t k = 2; k <= H; k <<= 1) {
      for (uint32_t j = k >> 1; j > 0; j >>= 1) {
        for (uint32_t t = lane; t < (H >> 1); t += G) {
          const uint32_t i = 2 * t - (t & (j - 1));
          const uint32_t l = i + j;
          const bool up = (i & k) == 0;
          const int ki = keys[i], kl = keys[l];
          if ((ki > kl) == up) {
            keys[i] = kl;
            keys[l] = ki;
            const VT vi = vals[i];
            vals[i] = vals[l];
            vals[l] = vi;
          }
        }
        group_sync<G>(gid);
      }
    }
    int32_t *__restrict__ Cj = P.Cj + off;
    VT *__restrict__ Cx = P.Cx + off;
    for (int64_t s = lane; s < c; s += G) {
      Cj[s] = keys[s];
      Cx[s] = vals[s];
    }
    group_sync<G>(gid);
  }
}

// DENSE numeric row: sweep the columns in windows of kDenseW.  Each A entry j
// keeps a cursor into its (sorted) B row, so every B entry is read once; the
// window's accumulator is dense FP64 plus a presence bitmap, and the window
// is emitted in column order.  With unsorted B every window rescans the rows.
template <typename PT, typename VT>
__device__ void num_dense_row(const ProdDev<PT, VT> *prods, const PhaseArgs &A,
                              int64_t idx, unsigned char *smem,
                              int64_t *scan_tmp) {
  const int tid = threadIdx.x, lane = tid & 31;
  VT *acc = (VT *)smem;
  uint32_t *bm = (uint32_t *)(smem + kDenseW * 8);
  int32_t *cur_s = (int32_t *)(smem + kDenseW * 8 + kDenseW / 8);
  const uint64_t e = A.list[idx];
  const int p = int(e >> 40);
  const int64_t r = int64_t(e & ((uint64_t(1) << 40) - 1));
  const int64_t g = A.base[p] + r;
  const ProdDev<PT, VT> &P = prods[p];
  const int64_t n = P.n;
  const int64_t a0 = P.Ap[r], a1 = P.Ap[r + 1], na = a1 - a0;
  int32_t *cur = na <= kDenseCurSmem ? cur_s : A.curbuf + blockIdx.x * A.cur_stride;
  const bool sorted = P.b_sorted != 0;
  for (int64_t j = tid; j < na; j += kThreads) cur[j] = 0;
  for (int i = tid; i < kDenseW; i += kThreads) acc[i] = VT(0);
  for (int i = tid; i < kDenseW / 32; i += kThreads) bm[i] = 0u;
  __syncthreads();
  int64_t out = A.cp[g] - A.cp[A.base[p]];
  const int S = subgroup_width(A.rowf[g], na, 32);
  const int sl = lane % S;
  const int subid = tid / S, nsub = kThreads / S;
  const unsigned submask =
      S == 32 ? 0xffffffffu : (((1u << S) - 1u) << ((lane / S) * S));
  const int32_t *__restrict__ Aj = P.Aj;
  const VT *__restrict__ Ax = P.Ax;
  const PT *__restrict__ Bp = P.Bp;
  const int32_t *__restrict__ Bj = P.Bj;
  const VT *__restrict__ Bx = P.Bx;
  for (int64_t w0 = 0; w0 < n; w0 += kDenseW) {
    const int64_t w1 = (w0 + kDenseW < n) ? w0 + kDenseW : n;
    for (int64_t j = subid; j < na; j += nsub) {
      const int64_t k = __ldg(Aj + a0 + j);
      const VT a = __ldg(Ax + a0 + j);
      const int64_t b0 = __ldg(Bp + k), b1 = __ldg(Bp + k + 1);
      if (sorted) {
        int64_t q = b0 + cur[j];
        while (q < b1) {
          const int64_t qq = q + sl;
          const bool valid = qq < b1;
          const int32_t col = valid ? __ldg(Bj + qq) : INT32_MAX;
          const bool in = valid && col < w1;
          const unsigned bal = __ballot_sync(submask, in);
          if (in) {
            const uint32_t o = uint32_t(col - w0);
            atomicAdd(acc + o, a * __ldg(Bx + qq));
            const uint32_t bit = 1u << (o & 31);
            if (!(((volatile uint32_t *)bm)[o >> 5] & bit)) atomicOr(bm + (o >> 5), bit);
          }
          const int nin = __popc(bal);
          q += nin;
          if (nin < S) break;
        }
        if (sl == 0) cur[j] = int32_t(q - b0);
      } else {
        for (int64_t q = b0 + sl; q < b1; q += S) {
          const int32_t col = __ldg(Bj + q);
          if (col >= w0 && col < w1) {
            const uint32_t o = uint32_t(col - w0);
            atomicAdd(acc + o, a * __ldg(Bx + q));
            const uint32_t bit = 1u << (o & 31);
            if (!(((volatile uint32_t *)bm)[o >> 5] & bit)) atomicOr(bm + (o >> 5), bit);
          }
        }
      }
    }
    __syncthreads();
    uint32_t word = tid < kDenseW / 32 ? bm[tid] : 0u;
    int64_t tot;
    int64_t pos = group_excl_scan<kThreads, int64_t>(int64_t(__popc(word)),
                                                     scan_tmp, 0, &tot);
    int32_t *__restrict__ Cj = P.Cj + out;
    VT *__restrict__ Cx = P.Cx + out;
    while (word) {
      const int b = __ffs(word) - 1;
      word &= word - 1;
      const int o = tid * 32 + b;
      Cj[pos] = int32_t(w0 + o);
      Cx[pos] = acc[o];
      acc[o] = VT(0);
      ++pos;
    }
    if (tid < kDenseW / 32) bm[tid] = 0u;
    out += tot;
    __syncthreads();
  }
}

template <typename PT, typename VT, bool NUM>
__global__ void __launch_bounds__(kThreads, 1)
    k_phase(const ProdDev<PT, VT> *prods, PhaseArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ int64_t s_items[NCLS + 1], s_off[NCLS], s_cnt[NCLS];
  __shared__ unsigned long long s_item;
  __shared__ int64_t s_scan[16 * 33];
  const int tid = threadIdx.x;
  if (tid <= NCLS) s_items[tid] = A.S->items[tid];
  if (tid < NCLS) {
    s_off[tid] = A.S->off[tid];
    s_cnt[tid] = A.S->cnt[tid];
  }
  __syncthreads();
  const int64_t total = s_items[NCLS];
  while (true) {
    if (tid == 0) s_item = atomicAdd(&A.S->work, 1ull);
    __syncthreads();
    const int64_t item = (int64_t)s_item;
    if (item >= total) break;
    int c = 0;
    while (item >= s_items[c + 1]) ++c;
    const int64_t first = s_off[c] + (item - s_items[c]) * cls_rows_per_item(c);
    const int64_t last = s_off[c] + s_cnt[c];
    if constexpr (!NUM) {
      switch (c) {
        case CLS_DENSE: sym_dense_row<PT, VT>(prods, A, first, smem, s_scan); break;
        case CLS_G1024: sym_hash_rows<1024, kSymT1024, PT, VT>(prods, A, first, last, smem, s_scan); break;
        case CLS_G256: sym_hash_rows<256, kSymT256, PT, VT>(prods, A, first, last, smem, s_scan); break;
        case CLS_G128: sym_hash_rows<128, kSymT128, PT, VT>(prods, A, first, last, smem, s_scan); break;
        default: sym_hash_rows<32, kSymT32, PT, VT>(prods, A, first, last, smem, s_scan); break;
      }
    } else {
      switch (c) {
        case CLS_DENSE: num_dense_row<PT, VT>(prods, A, first, smem, s_scan); break;
        case CLS_G1024: num_hash_rows<1024, kNumT1024, PT, VT>(prods, A, first, last, smem, s_scan); break;
        case CLS_G256: num_hash_rows<256, kNumT256, PT, VT>(prods, A, first, last, smem, s_scan); break;
        case CLS_G128: num_hash_rows<128, kNumT128, PT, VT>(prods, A, first, last, smem, s_scan); break;
        default: num_hash_rows<32, kNumT32, PT, VT>(prods, A, first, last, smem, s_scan); break;
      }
    }
    __syncthreads();
  }
}

}  // namespace tspg
