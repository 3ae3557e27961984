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
// Segments of up to kSegCta entries are sorted in shared memory by one CTA
// (stable radix sort on the row index); longer ones are cut into sorted runs
// of kSegCta that are merged pairwise in global memory (each element finds its
// place by binary search in the other run), which keeps the result
// deterministic and independent of the scatter order.
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

// One CTA per segment (grid-stride over segments): sort up to kSegCta pairs
// of a segment (or one run of a longer segment) by key.
constexpr int kSortSmem = 2 * kSegCta * 4 + 2 * kSegCta * 8 + 64 * 8 * (kSegThreads / 32) * 2;

template <typename VT>
__global__ void __launch_bounds__(kSegThreads)
    k_sort_runs(const int64_t *tp, int64_t nseg, int32_t *key, VT *val) {
  extern __shared__ __align__(16) unsigned char dsm[];
  VT *vs = (VT *)dsm;                                   // 2 x kSegCta values
  int *ks = (int *)(dsm + 2 * kSegCta * 8);             // 2 x kSegCta keys
  uint16_t *cnt = (uint16_t *)(dsm + 2 * kSegCta * 12);  // digit counters
  __shared__ int64_t tmp[33];
  const int tid = threadIdx.x;
  for (int64_t s = blockIdx.x; s < nseg; s += gridDim.x) {
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

__global__ void k_list_long(const int64_t *tp, int64_t nseg, int64_t lim, int64_t *out,
                            unsigned long long *n) {
  const int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s < nseg && tp[s + 1] - tp[s] > lim) out[atomicAdd(n, 1ull)] = s;
}

template <typename T>
__global__ void k_copy_segs(const int64_t *tp, const int64_t *longseg, int64_t nlong, const T *src,
                            T *dst) {
  for (int64_t ls = blockIdx.x; ls < nlong; ls += gridDim.x) {
    const int64_t s = longseg[ls];
    for (int64_t i = tp[s] + threadIdx.x; i < tp[s + 1]; i += blockDim.x) dst[i] = src[i];
  }
}

template <typename PT, typename VT>
static int transpose_impl(tspg_ctx *ctx, cudaStream_t s, const tspg_csr *M, tspg_csr_out *T) {
  const int64_t m = M->nrows, n = M->ncols, nnz = M->nnz;
  Scratch sc(ctx, s);
  int32_t *cnt, *cursor;
  int64_t *tp, *partial, *longseg;
  unsigned long long *nlong;
  Sched *dummy;
  const int64_t nb = (n + kScanTile - 1) / kScanTile;
  TSPG_TRY(sc.get(&cnt, n));
  TSPG_TRY(sc.get(&cursor, n));
  TSPG_TRY(sc.get(&tp, n + 1));
  TSPG_TRY(sc.get(&partial, nb + 1));
  TSPG_TRY(sc.get(&dummy, 1));
  TSPG_TRY(sc.get(&nlong, 1));
  TSPG_TRY(sc.get(&longseg, n));
  TSPG_CUDA(ctx, cudaMemsetAsync(cnt, 0, sizeof(int32_t) * (n > 0 ? n : 1), s));
  TSPG_CUDA(ctx, cudaMemsetAsync(cursor, 0, sizeof(int32_t) * (n > 0 ? n : 1), s));
  TSPG_CUDA(ctx, cudaMemsetAsync(tp, 0, sizeof(int64_t), s));
  TSPG_CUDA(ctx, cudaMemsetAsync(nlong, 0, sizeof(unsigned long long), s));
  const unsigned gw = (unsigned)std::max<int64_t>(1, std::min<int64_t>((m * 32 + 255) / 256,
                                                                       int64_t(ctx->num_sms) * 16));
  if (m > 0 && nnz > 0)
    k_col_counts<PT><<<gw, 256, 0, s>>>((const PT *)M->rowptr, M->col, m, cnt);
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
    k_col_scatter<PT, VT><<<gw, 256, 0, s>>>((const PT *)M->rowptr, M->col, (const VT *)M->val, m,
                                             tp, cursor, T->col, (VT *)T->val);
    const unsigned gs = (unsigned)std::max<int64_t>(1, std::min<int64_t>(n, int64_t(ctx->num_sms) * 2));
    TSPG_CUDA(ctx, cudaFuncSetAttribute(k_sort_runs<VT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        kSortSmem));
    k_sort_runs<VT><<<gs, kSegThreads, kSortSmem, s>>>(tp, n, T->col, (VT *)T->val);
    k_list_long<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(tp, n, kSegCta, longseg, nlong);
    ctx->launches += 3;
    int64_t *h = ctx->h_words;
    TSPG_CUDA(ctx, cudaMemcpyAsync(h, nlong, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    TSPG_CUDA(ctx, cudaStreamSynchronize(s));
    const int64_t nl = h[0];
    if (nl > 0) {
      int32_t *k2;
      VT *v2;
      TSPG_TRY(sc.get(&k2, nnz));
      TSPG_TRY(sc.get(&v2, nnz));
      int32_t *ka = T->col, *kb = k2;
      VT *va = (VT *)T->val, *vb = v2;
      // merge passes until a run covers any segment (a column has <= m entries)
      for (int64_t run = kSegCta; run < m; run *= 2) {
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
