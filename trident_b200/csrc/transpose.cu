// transpose.cu — CSR transpose on the device: T = M^T, rows of T sorted.
//
// Replaces cusparse_csc_to_csr (include/cusparse_helpers.cuh:607-705) and
// LocalMatrix::csc_to_csr (include/KokkosWrap.hpp:442-531), which call
// cusparseCsr2cscEx2: a CSC matrix is the CSR of its transpose, so CSC -> CSR
// is one transpose of the compressed arrays.  Also builds R = P^T for the
// Galerkin product.
//
// Steps: column counts (atomics), the device scan, an atomic scatter of every
// entry into its column segment, then each segment is sorted by source row.
// Segments of up to 32 entries are sorted by one warp in registers (bitonic);
// segments of up to kSegCta entries in shared memory by one CTA (stable radix
// sort on the row index), over a device-built list of them; longer ones are
// cut into sorted runs of kSegCta that are merged pairwise in global memory
// (each element finds its place by binary search in the other run), which
// keeps the result deterministic and independent of the scatter order.
#include "spgemm_phase.cuh"

namespace tspg {

constexpr int kSegCta = 4096;   // segment sorted in one CTA (512 threads x 8)
constexpr int kSegThreads = 512;

template <typename PT>
__global__ void k_col_counts(const PT *rp, const int32_t *col, int64_t m, int32_t *cnt) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = warp; r < m; r += nwarps)
    for (int64_t p = int64_t(rp[r]) + lane; p < int64_t(rp[r + 1]); p += 32)
      atomicAdd(cnt + col[p], 1);
}

template <typename PT, typename VT>
__global__ void k_col_scatter(const PT *rp, const int32_t *col, const VT *val, int64_t m,
                              const int64_t *tp, int32_t *cursor, int32_t *trow, VT *tval) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = warp; r < m; r += nwarps)
    for (int64_t p = int64_t(rp[r]) + lane; p < int64_t(rp[r + 1]); p += 32) {
      const int32_t j = col[p];
      const int64_t o = tp[j] + atomicAdd(cursor + j, 1);
      trow[o] = int32_t(r);
      tval[o] = val[p];
    }
}

// The same two passes for a matrix whose row r is the single entry r (a COO
// sequence): one thread per entry.
__global__ void k_seq_counts(const int32_t *col, int64_t nnz, int32_t *cnt) {
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < nnz; p += stride)
    atomicAdd(cnt + col[p], 1);
}

template <typename VT>
__global__ void k_seq_scatter(const int32_t *col, const VT *val, int64_t nnz, const int64_t *tp,
                              int32_t *cursor, int32_t *trow, VT *tval) {
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; p < nnz; p += stride) {
    const int32_t j = col[p];
    const int64_t o = tp[j] + atomicAdd(cursor + j, 1);
    trow[o] = int32_t(p);
    tval[o] = val[p];
  }
}

// Segments of 2..32 entries: one warp each, sorted in registers.
template <typename VT>
__global__ void k_sort_short(const int64_t *tp, int64_t nseg, int32_t *key, VT *val) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t s = warp; s < nseg; s += nwarps) {
    const int64_t b = tp[s], n = tp[s + 1] - b;
    if (n < 2 || n > 32) continue;  // uniform over the warp
    int k = lane < n ? key[b + lane] : INT32_MAX;
    VT v = lane < n ? val[b + lane] : VT(0);
    warp_bitonic32<VT>(k, v, lane);
    if (lane < n) {
      key[b + lane] = k;
      val[b + lane] = v;
    }
  }
}

// Segments of more than 32 entries (sorted by CTAs) and of more than lim
// (merged after): two lists, their lengths and the longest length in
// n[0], n[1], n[2].
__global__ void k_list_segs(const int64_t *tp, int64_t nseg, int64_t lim, int64_t *mid,
                            int64_t *lng, unsigned long long *n) {
  const int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  const int64_t len = tp[s + 1] - tp[s];
  if (len > 32) mid[atomicAdd(n, 1ull)] = s;
  if (len > lim) {
    lng[atomicAdd(n + 1, 1ull)] = s;
    atomicMax(n + 2, (unsigned long long)len);
  }
}

// One CTA per listed segment (grid-stride over the list): sort up to kSegCta pairs
// of a segment (or one run of a longer segment) by key.
constexpr int kSortSmem = 2 * kSegCta * 4 + 2 * kSegCta * 8 + 64 * 8 * (kSegThreads / 32) * 2;

template <typename VT>
__global__ void __launch_bounds__(kSegThreads)
    k_sort_runs(const int64_t *tp, const int64_t *segs, const unsigned long long *nsegs,
                int32_t *key, VT *val) {
  extern __shared__ __align__(16) unsigned char dsm[];
  VT *vs = (VT *)dsm;                                   // 2 x kSegCta values
  int *ks = (int *)(dsm + 2 * kSegCta * 8);             // 2 x kSegCta keys
  uint16_t *cnt = (uint16_t *)(dsm + 2 * kSegCta * 12);  // digit counters
  __shared__ int64_t tmp[33];
  const int tid = threadIdx.x;
  const int64_t nseg = int64_t(*nsegs);
  for (int64_t i = blockIdx.x; i < nseg; i += gridDim.x) {
    const int64_t s = segs[i];
    const int64_t b = tp[s], e = tp[s + 1];
    for (int64_t r0 = b; r0 < e; r0 += kSegCta) {
      const int n = int(min(int64_t(kSegCta), e - r0));
      if (n <= 1) continue;
      int mn = INT32_MAX, mx = 0;
      for (int i = tid; i < n; i += kSegThreads) {
        ks[i] = key[r0 + i];
        vs[i] = val[r0 + i];
        mn = min(mn, ks[i]);
        mx = max(mx, ks[i]);
      }
      int *itmp = (int *)tmp;
      group_minmax<kSegThreads>(mn, mx, itmp, 0);
      for (int i = tid; i < n; i += kSegThreads) ks[i] -= mn;
      __syncthreads();
      const int bits = mx > mn ? 32 - __clz(mx - mn) : 0;
      const int src = radix_pairs<kSegThreads, 8, 6, VT>(ks, vs, ks + kSegCta, vs + kSegCta, n,
                                                         bits, cnt, tmp, 0, tid);
      const int *ko = src ? ks + kSegCta : ks;
      const VT *vo = src ? vs + kSegCta : vs;
      for (int i = tid; i < n; i += kSegThreads) {
        key[r0 + i] = ko[i] + mn;
        val[r0 + i] = vo[i];
      }
      __syncthreads();
    }
  }
}

// Merge pass over segments longer than `run`: runs [x, x+run) and
// [x+run, x+2run) of every such segment are merged from (key, val) into
// (k2, v2); each element's position = its index in its run + the number of
// elements of the other run ordered before it (ties: left run first).
template <typename VT>
__global__ void k_merge_runs(const int64_t *tp, const int64_t *longseg, int64_t nlong, int64_t run,
                             const int32_t *key, const VT *val, int32_t *k2, VT *v2) {
  for (int64_t ls = blockIdx.x; ls < nlong; ls += gridDim.x) {
    const int64_t s = longseg[ls];
    const int64_t b = tp[s], e = tp[s + 1];
    for (int64_t i = b + threadIdx.x; i < e; i += blockDim.x) {
      const int64_t rel = i - b;
      const int64_t x = b + (rel / (2 * run)) * (2 * run);  // pair start
      const int64_t mid = min(e, x + run), hi = min(e, x + 2 * run);
      const int32_t k = key[i];
      int64_t pos;
      if (i < mid) {  // left run: count right-run keys < k
        int64_t lo = mid, up = hi;
        while (lo < up) {
          const int64_t md = (lo + up) >> 1;
          if (key[md] < k) lo = md + 1; else up = md;
        }
        pos = x + (i - x) + (lo - mid);
      } else {  // right run: count left-run keys <= k
        int64_t lo = x, up = mid;
        while (lo < up) {
          const int64_t md = (lo + up) >> 1;
          if (key[md] <= k) lo = md + 1; else up = md;
        }
        pos = x + (i - mid) + (lo - x);
      }
      k2[pos] = k;
      v2[pos] = val[i];
    }
  }
}

__global__ void k_narrow(const int64_t *src, int64_t n, int32_t *dst) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = int32_t(src[i]);
}


template <typename T>
__global__ void k_copy_segs(const int64_t *tp, const int64_t *longseg, int64_t nlong, const T *src,
                            T *dst) {
  for (int64_t ls = blockIdx.x; ls < nlong; ls += gridDim.x) {
    const int64_t s = longseg[ls];
    for (int64_t i = tp[s] + threadIdx.x; i < tp[s + 1]; i += blockDim.x) dst[i] = src[i];
  }
}

// seq: row r of M is the single entry r (rowptr = 0, 1, ..., nnz); the count
// and scatter passes then run one thread per entry.
template <typename PT, typename VT>
static int transpose_impl(tspg_ctx *ctx, cudaStream_t s, const tspg_csr *M, tspg_csr_out *T,
                          bool seq = false) {
  const int64_t m = M->nrows, n = M->ncols, nnz = M->nnz;
  Scratch sc(ctx, s);
  int32_t *cnt, *cursor;
  int64_t *tp, *partial, *longseg, *midseg;
  unsigned long long *nlong;
  Sched *dummy;
  const int64_t nb = (n + kScanTile - 1) / kScanTile;
  TSPG_TRY(sc.get(&cnt, n));
  TSPG_TRY(sc.get(&cursor, n));
  TSPG_TRY(sc.get(&tp, n + 1));
  TSPG_TRY(sc.get(&partial, nb + 1));
  TSPG_TRY(sc.get(&dummy, 1));
  TSPG_TRY(sc.get(&nlong, 3));
  TSPG_TRY(sc.get(&longseg, n));
  TSPG_TRY(sc.get(&midseg, n));
  TSPG_CUDA(ctx, cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (n > 0 ? n : 1), s));
  TSPG_CUDA(ctx, cudaMemsetAsync(cursor, 0, sizeof(int32_t) * (n > 0 ? n : 1), s));
  TSPG_CUDA(ctx, cudaMemsetAsync(tp, 0, sizeof(int64_t), s));
  TSPG_CUDA(ctx, cudaMemsetAsync(nlong, 0, 3 * sizeof(unsigned long long), s));
  const unsigned gw = (unsigned)std::max<int64_t>(1, std::min<int64_t>((m * 32 + 255) / 256,
                                                                       int64_t(ctx->num_sms) * 16));
  const unsigned ge = (unsigned)std::max<int64_t>(1, std::min<int64_t>((nnz + 255) / 256,
                                                                       int64_t(ctx->num_sms) * 8));
  if (m > 0 && nnz > 0) {
    if (seq) k_seq_counts<<<ge, 256, 0, s>>>(M->col, nnz, cnt);
    else k_col_counts<PT><<<gw, 256, 0, s>>>((const PT *)M->rowptr, M->col, m, cnt);
  }
  if (n > 0) {
    k_scan_reduce<<<(unsigned)nb, kScanThreads, 0, s>>>(cnt, n, partial);
    k_scan_partials<<<1, 1024, 0, s>>>(partial, nb);
    k_scan_final<<<(unsigned)nb, kScanThreads, 0, s>>>(cnt, n, partial, nb, tp, dummy, nullptr);
  }
  ctx->launches += (m > 0 && nnz > 0) + (n > 0 ? 3 : 0);
  T->nnz = nnz;
  if (T->capacity < nnz) {
    if (!T->alloc) return TSPG_ENOMEM;
    void *cj = T->alloc(T->alloc_user, size_t(nnz) * 4, s);
    void *cx = T->alloc(T->alloc_user, size_t(nnz) * sizeof(VT), s);
    if (!cj || !cx) return TSPG_ENOMEM;
    T->col = (int32_t *)cj;
    T->val = cx;
    T->capacity = nnz;
  }
  if (m > 0 && nnz > 0) {
    if (seq)
      k_seq_scatter<VT><<<ge, 256, 0, s>>>(M->col, (const VT *)M->val, nnz, tp, cursor, T->col,
                                           (VT *)T->val);
    else
      k_col_scatter<PT, VT><<<gw, 256, 0, s>>>((const PT *)M->rowptr, M->col, (const VT *)M->val,
                                               m, tp, cursor, T->col, (VT *)T->val);
    const unsigned gs = (unsigned)std::max<int64_t>(1, std::min<int64_t>(n, int64_t(ctx->num_sms) * 2));
    const unsigned gq = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n * 32 + 255) / 256,
                                                                         int64_t(ctx->num_sms) * 16));
    TSPG_CUDA(ctx, cudaFuncSetAttribute(k_sort_runs<VT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        kSortSmem));
    k_list_segs<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(tp, n, kSegCta, midseg, longseg, nlong);
    k_sort_short<VT><<<gq, 256, 0, s>>>(tp, n, T->col, (VT *)T->val);
    k_sort_runs<VT><<<gs, kSegThreads, kSortSmem, s>>>(tp, midseg, nlong, T->col, (VT *)T->val);
    ctx->launches += 4;
    int64_t *h = ctx->h_words;
    TSPG_CUDA(ctx, cudaMemcpyAsync(h, nlong + 1, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    TSPG_CUDA(ctx, cudaStreamSynchronize(s));
    const int64_t nl = h[0], longest = h[1];
    if (nl > 0) {
      int32_t *k2;
      VT *v2;
      TSPG_TRY(sc.get(&k2, nnz));
      TSPG_TRY(sc.get(&v2, nnz));
      int32_t *ka = T->col, *kb = k2;
      VT *va = (VT *)T->val, *vb = v2;
      // merge passes until a run covers the longest segment
      for (int64_t run = kSegCta; run < longest; run *= 2) {
        k_merge_runs<VT><<<(unsigned)std::min<int64_t>(nl, int64_t(ctx->num_sms) * 8), 256, 0, s>>>(
            tp, longseg, nl, run, ka, va, kb, vb);
        std::swap(ka, kb);
        std::swap(va, vb);
        ctx->launches += 1;
      }
      if (ka != T->col) {
        k_copy_segs<int32_t><<<(unsigned)std::min<int64_t>(nl, 1024), 256, 0, s>>>(tp, longseg, nl, ka, T->col);
        k_copy_segs<VT><<<(unsigned)std::min<int64_t>(nl, 1024), 256, 0, s>>>(tp, longseg, nl, va,
                                                                             (VT *)T->val);
        ctx->launches += 2;
      }
    }
  }
  // row offsets of T in the requested width
  if (T->rowptr_bits == 64) {
    TSPG_CUDA(ctx, cudaMemcpyAsync(T->rowptr, tp, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToDevice, s));
  } else {
    k_narrow<<<(unsigned)((n + 1 + 255) / 256), 256, 0, s>>>(tp, n + 1, (int32_t *)T->rowptr);
    ctx->launches += 1;
  }
  TSPG_CUDA(ctx, cudaGetLastError());
  return TSPG_OK;
}

// ---------------------------------------------------------------- COO -> CSR / CSC

// Any index outside [0, n) sets flag (the scatter passes index arrays by it).
__global__ void k_coo_check(const int32_t *maj, const int32_t *mnr, int64_t nnz, int64_t nmaj,
                            int64_t nmin, unsigned long long *flag) {
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  bool bad = false;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nnz; i += stride) {
    const int32_t a = maj[i], b = mnr[i];
    bad |= a < 0 || a >= nmaj || b < 0 || b >= nmin;
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1ull);
}

__global__ void k_iota64(int64_t *p, int64_t n) {
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) p[i] = i;
}

// dst[i] = src[idx[i]]
__global__ void k_gather32(const int32_t *src, const int32_t *idx, int64_t n, int32_t *dst) {
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    dst[i] = src[idx[i]];
}

// out[u] = mnr[pos1[out[u]]]: the positions left by the second pass become
// minor indices, in place
__global__ void k_minor_of(const int32_t *mnr, const int32_t *pos1, int64_t n, int32_t *out) {
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = mnr[pos1[out[i]]];
}

// COO -> compressed by `maj`, as two stable counting sorts (least significant
// key first): the COO seen as a CSR with one entry per row (identity row
// offsets) is transposed by its minor index, so every minor segment lists the
// input positions in increasing order; that sequence, seen the same way, is
// transposed by its major index.  The result is ordered by (major, minor,
// input position), deterministic with repeated entries; the second transpose
// writes the output's offsets and values, a gather its minor indices.
template <typename VT>
static int coo_impl(tspg_ctx *ctx, cudaStream_t s, int64_t nmaj, int64_t nmin, int64_t nnz,
                    const int32_t *maj, const int32_t *mnr, const VT *val, tspg_csr_out *out) {
  Scratch sc(ctx, s);
  const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>((nnz + 255) / 256,
                                                                      int64_t(ctx->num_sms) * 8));
  unsigned long long *flag;
  int64_t *idrp, *tp1;
  int32_t *pos1, *maj2;
  VT *val1;
  TSPG_TRY(sc.get(&flag, 1));
  TSPG_CUDA(ctx, cudaMemsetAsync(flag, 0, sizeof(unsigned long long), s));
  if (nnz > 0) {
    k_coo_check<<<g, 256, 0, s>>>(maj, mnr, nnz, nmaj, nmin, flag);
    ctx->launches += 1;
  }
  int64_t *h = ctx->h_words;
  TSPG_CUDA(ctx, cudaMemcpyAsync(h, flag, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  TSPG_CUDA(ctx, cudaStreamSynchronize(s));
  if (h[0] != 0) return TSPG_EINVAL;
  TSPG_TRY(sc.get(&idrp, nnz + 1));
  TSPG_TRY(sc.get(&tp1, nmin + 1));
  TSPG_TRY(sc.get(&pos1, nnz));
  TSPG_TRY(sc.get(&maj2, nnz));
  TSPG_TRY(sc.get(&val1, nnz));
  k_iota64<<<g, 256, 0, s>>>(idrp, nnz + 1);
  ctx->launches += 1;
  const int vb = int(sizeof(VT) * 8);
  // pass 1: by minor index
  auto seq = [&](int64_t ncols, const int32_t *key, const VT *v) {
    tspg_csr m{};
    m.nrows = nnz;
    m.ncols = ncols;
    m.nnz = nnz;
    m.rowptr = idrp;
    m.rowptr_bits = 64;
    m.val_bits = vb;
    m.col = key;
    m.val = v;
    return m;
  };
  const tspg_csr m1 = seq(nmin, mnr, val);
  tspg_csr_out t1{};
  t1.nrows = nmin;
  t1.ncols = nnz;
  t1.rowptr = tp1;
  t1.rowptr_bits = 64;
  t1.val_bits = vb;
  t1.col = pos1;
  t1.val = val1;
  t1.capacity = nnz;
  TSPG_TRY(transpose_impl<int64_t, VT>(ctx, s, &m1, &t1, true));
  // pass 2: by major index, into the output
  if (nnz > 0) {
    k_gather32<<<g, 256, 0, s>>>(maj, pos1, nnz, maj2);
    ctx->launches += 1;
  }
  const tspg_csr m2 = seq(nmaj, maj2, val1);
  TSPG_TRY(transpose_impl<int64_t, VT>(ctx, s, &m2, out, true));
  if (nnz > 0) {
    k_minor_of<<<g, 256, 0, s>>>(mnr, pos1, nnz, out->col);
    ctx->launches += 1;
  }
  TSPG_CUDA(ctx, cudaGetLastError());
  return TSPG_OK;
}

}  // namespace tspg

using namespace tspg;

extern "C" int tspg_transpose(tspg_ctx *ctx, void *stream, const tspg_csr *M, tspg_csr_out *T) {
  if (!ctx || !T) return TSPG_EINVAL;
  TSPG_TRY(check_csr(M));
  if (M->nrows > INT32_MAX) return TSPG_EINVAL;  // rows become int32 column indices
  if (!T->rowptr || T->nrows != M->ncols || T->ncols != M->nrows || T->val_bits != M->val_bits ||
      (T->rowptr_bits != 32 && T->rowptr_bits != 64))
    return TSPG_EINVAL;
  if (T->rowptr_bits == 32 && M->nnz > INT32_MAX) return TSPG_EOVERFLOW;
  TSPG_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  if (M->val_bits == 64)
    return M->rowptr_bits == 32 ? transpose_impl<int32_t, double>(ctx, s, M, T)
                                : transpose_impl<int64_t, double>(ctx, s, M, T);
  return M->rowptr_bits == 32 ? transpose_impl<int32_t, float>(ctx, s, M, T)
                              : transpose_impl<int64_t, float>(ctx, s, M, T);
}

extern "C" int tspg_coo_to_csx(tspg_ctx *ctx, void *stream, int64_t nrows, int64_t ncols,
                               int64_t nnz, const int32_t *row, const int32_t *col,
                               const void *val, int val_bits, int major, tspg_csr_out *out) {
  if (!ctx || !out) return TSPG_EINVAL;
  if (nrows < 0 || ncols < 0 || nnz < 0 || nrows > INT32_MAX || ncols > INT32_MAX ||
      nnz > INT32_MAX)
    return TSPG_EINVAL;
  if ((val_bits != 32 && val_bits != 64) || (major != TSPG_ROWS && major != TSPG_COLS))
    return TSPG_EINVAL;
  if (nnz > 0 && (!row || !col || !val)) return TSPG_EINVAL;
  const int64_t nmaj = major == TSPG_ROWS ? nrows : ncols, nmin = major == TSPG_ROWS ? ncols : nrows;
  if (!out->rowptr || out->nrows != nmaj || out->ncols != nmin || out->val_bits != val_bits ||
      (out->rowptr_bits != 32 && out->rowptr_bits != 64))
    return TSPG_EINVAL;
  TSPG_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  const int32_t *maj = major == TSPG_ROWS ? row : col, *mnr = major == TSPG_ROWS ? col : row;
  return val_bits == 64 ? coo_impl<double>(ctx, s, nmaj, nmin, nnz, maj, mnr, (const double *)val, out)
                        : coo_impl<float>(ctx, s, nmaj, nmin, nnz, maj, mnr, (const float *)val, out);
}
