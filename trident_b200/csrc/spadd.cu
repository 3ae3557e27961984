// spadd.cu — merge of partial C tiles, C = A + B with the union pattern.
//
// Replaces cusparse_spgeam (include/cusparse_helpers.cuh:799-905: csrgeam2
// bufferSize + Nnz + compute, five stream syncs, the nnz through the host) and
// LocalMatrix::spadd (include/KokkosWrap.hpp:394-439: KK spadd symbolic +
// numeric).  Rows are sorted and duplicate-free, so every entry finds its
// output slot from its rank in the other row.  Rows with up to kMergeHeavy
// entries in A and B together: one warp per row, merging 32-column chunks of
// both rows in registers (merge_row_warp; per-entry binary searches of the
// other row, as first built, took twice as long).  Longer rows (the hub rows of
// partial C tiles reach 10^5 entries, and one warp per such row left the merge
// waiting on a handful of warps) are listed and merged by a whole CTA: its
// warps take the ranges between merge-path cuts of the row.
#include "internal.cuh"
#include "spgemm_kernels.cuh"

namespace tspg {

constexpr int64_t kMergeHeavy = 4096;  // rows above this go to the CTA merge
constexpr int kMergeThreads = 512;

// Chunked warp merge of one light row.  Each iteration loads the next 32
// columns of A and of B (coalesced).  Every entry up to lim, the smaller of
// the two chunk maxima, is final this iteration (entries past a full chunk are
// larger than its maximum); its output position is its index in its chunk
// plus its rank in the other chunk (a 5-step search over the other chunk's
// registers by shuffles) minus the columns of both rows below it.  A column in
// both rows leaves once, from A, with the two values added.  At least 32
// entries leave per iteration and no global load depends on another.
// WRITE = false returns the size of the union only; WRITE = true writes no
// position at or past cap (the row's size from the count pass), so rows that
// break the sorted / duplicate-free contract cannot write outside their row.
template <bool WRITE, typename VT>
__device__ __forceinline__ int64_t merge_row_warp(const int32_t *__restrict__ Aj,
                                                  const VT *__restrict__ Ax, int64_t a0,
                                                  int64_t a1, const int32_t *__restrict__ Bj,
                                                  const VT *__restrict__ Bx, int64_t b0,
                                                  int64_t b1, int32_t *__restrict__ cj,
                                                  VT *__restrict__ cx, int64_t cap, int lane) {
  constexpr unsigned FULL = 0xffffffffu;
  const unsigned below = (1u << lane) - 1u;
  int64_t pa = a0, pb = b0, out = 0;
  while (pa < a1 || pb < b1) {
    const bool va = pa + lane < a1, vb = pb + lane < b1;
    const int32_t ai = va ? __ldg(Aj + pa + lane) : INT32_MAX;  // no column is INT32_MAX
    const int32_t bi = vb ? __ldg(Bj + pb + lane) : INT32_MAX;
    VT av = VT(0), bv = VT(0);
    if constexpr (WRITE) {
      if (va) av = __ldg(Ax + pa + lane);
      if (vb) bv = __ldg(Bx + pb + lane);
    }
    const int32_t lastA = __shfl_sync(FULL, ai, 31), lastB = __shfl_sync(FULL, bi, 31);
    const int32_t lim = min(pa + 32 <= a1 ? lastA : INT32_MAX, pb + 32 <= b1 ? lastB : INT32_MAX);
    int ra = 0, rb = 0;  // entries of the other chunk below this lane's entry
#pragma unroll
    for (int st = 16; st > 0; st >>= 1) {
      if (__shfl_sync(FULL, bi, ra + st - 1) < ai) ra += st;
      if (__shfl_sync(FULL, ai, rb + st - 1) < bi) rb += st;
    }
    if (ra == 31 && lastB < ai) ra = 32;
    if (rb == 31 && lastA < bi) rb = 32;
    const int32_t bat = __shfl_sync(FULL, bi, ra & 31), aat = __shfl_sync(FULL, ai, rb & 31);
    const bool ca = va && ai <= lim, cb = vb && bi <= lim;
    const bool dupa = ca && ra < 32 && bat == ai, dupb = cb && rb < 32 && aat == bi;
    const unsigned dm = __ballot_sync(FULL, dupa);
    const int na = __popc(__ballot_sync(FULL, ca)), nb = __popc(__ballot_sync(FULL, cb));
    if constexpr (WRITE) {
      const VT bvat = __shfl_sync(FULL, bv, ra & 31);
      if (ca) {
        const int64_t pos = out + lane + ra - __popc(dm & below);
        if (pos < cap) {
          cj[pos] = ai;
          cx[pos] = dupa ? av + bvat : av;
        }
      }
      if (cb && !dupb) {
        const unsigned mk = rb >= 32 ? FULL : ((1u << rb) - 1u);
        const int64_t pos = out + lane + rb - __popc(dm & mk);
        if (pos < cap) {
          cj[pos] = bi;
          cx[pos] = bv;
        }
      }
    }
    out += na + nb - __popc(dm);
    pa += na;
    pb += nb;
  }
  return out;
}

template <typename PTA, typename PTB>
__global__ void __launch_bounds__(256)
    k_spadd_count(int64_t m, const PTA *Ap, const int32_t *Aj, const PTB *Bp,
                  const int32_t *Bj, int32_t *rowc, int64_t *heavy, int64_t *nheavy) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = warp; r < m; r += nwarps) {
    const int64_t a0 = Ap[r], a1 = Ap[r + 1], b0 = Bp[r], b1 = Bp[r + 1];
    if ((a1 - a0) + (b1 - b0) > kMergeHeavy) {
      if (lane == 0) heavy[atomicAdd((unsigned long long *)nheavy, 1ull)] = r;
      continue;
    }
    const int64_t n = merge_row_warp<false, double>(Aj, nullptr, a0, a1, Bj, nullptr, b0, b1,
                                                    nullptr, nullptr, 0, lane);
    if (lane == 0) rowc[r] = int32_t(n);
  }
}

template <typename PTA, typename PTB, typename VT>
__global__ void __launch_bounds__(256)
    k_spadd_fill(int64_t m, const PTA *Ap, const int32_t *Aj, const VT *Ax,
                 const PTB *Bp, const int32_t *Bj, const VT *Bx,
                 const int64_t *cp, void *Cp, int cp_bits, int32_t *Cj, VT *Cx) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = warp; r < m; r += nwarps) {
    const int64_t a0 = Ap[r], a1 = Ap[r + 1], b0 = Bp[r], b1 = Bp[r + 1];
    const int64_t o = cp[r];
    if (lane == 0) {
      if (cp_bits == 32) ((int32_t *)Cp)[r] = int32_t(o);
      else ((int64_t *)Cp)[r] = o;
      if (r == m - 1) {
        if (cp_bits == 32) ((int32_t *)Cp)[m] = int32_t(cp[m]);
        else ((int64_t *)Cp)[m] = cp[m];
      }
    }
    if ((a1 - a0) + (b1 - b0) > kMergeHeavy) continue;  // merged by k_spadd_heavy
    merge_row_warp<true, VT>(Aj, Ax, a0, a1, Bj, Bx, b0, b1, Cj + o, Cx + o, cp[r + 1] - o, lane);
  }
}

// Heavy rows: one CTA of kMergeWarps warps per row.  The merged sequence is
// cut at kMergeWarps + 1 diagonals (merge path: the A entries among the first
// d merged entries, A before B on equal columns); a column present in both
// rows whose A entry falls before a cut and B entry after it moves whole to
// the earlier range, so every range merges on its own.  Each warp merges its
// range with merge_row_warp.  The count pass keeps the cuts and the per-warp
// counts (meta: kMergeWarps counts, then kMergeWarps + 1 pairs of cuts per
// listed row) for the fill pass.
constexpr int kMergeWarps = kMergeThreads / 32;
constexpr int kHeavyMeta = kMergeWarps + 2 * (kMergeWarps + 1);

__device__ __forceinline__ void merge_cut(const int32_t *__restrict__ aj, int64_t la,
                                          const int32_t *__restrict__ bj, int64_t lb, int64_t d,
                                          int64_t &i, int64_t &j) {
  int64_t lo = d > lb ? d - lb : 0, hi = d < la ? d : la;
  while (lo < hi) {
    const int64_t mid = (lo + hi + 1) >> 1;
    if (__ldg(aj + mid - 1) <= __ldg(bj + d - mid)) lo = mid; else hi = mid - 1;
  }
  i = lo;
  j = d - lo;
  // the B entry that follows an equal A entry: the diagonal after d takes it
  // first (A is strictly increasing), so the next cut's j stays >= this one
  if (i > 0 && j < lb && __ldg(aj + i - 1) == __ldg(bj + j)) ++j;
}

template <bool WRITE, typename PTA, typename PTB, typename VT>
__global__ void __launch_bounds__(kMergeThreads)
    k_spadd_heavy(const int64_t *heavy, const int64_t *nheavy, const PTA *Ap,
                  const int32_t *Aj, const VT *Ax, const PTB *Bp, const int32_t *Bj,
                  const VT *Bx, int32_t *rowc, const int64_t *cp, int64_t *meta, int32_t *Cj,
                  VT *Cx) {
  __shared__ int64_t cnt[kMergeWarps];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t nh = *nheavy;
  for (int64_t h = blockIdx.x; h < nh; h += gridDim.x) {
    const int64_t r = heavy[h];
    const int64_t a0 = Ap[r], a1 = Ap[r + 1], b0 = Bp[r], b1 = Bp[r + 1];
    const int64_t la = a1 - a0, lb = b1 - b0;
    int64_t *mt = meta + h * kHeavyMeta;
    int64_t *cuts = mt + kMergeWarps;  // (i, j) per diagonal
    if constexpr (!WRITE) {
      if (threadIdx.x <= kMergeWarps) {
        int64_t i, j;
        merge_cut(Aj + a0, la, Bj + b0, lb, (la + lb) * threadIdx.x / kMergeWarps, i, j);
        cuts[2 * threadIdx.x] = i;
        cuts[2 * threadIdx.x + 1] = j;
      }
      __syncthreads();  // the cuts are read back through L1-bypassing loads below
      const int64_t i0 = __ldcg(cuts + 2 * w), j0 = __ldcg(cuts + 2 * w + 1);
      const int64_t i1 = __ldcg(cuts + 2 * w + 2), j1 = __ldcg(cuts + 2 * w + 3);
      const int64_t n = merge_row_warp<false, VT>(Aj + a0, nullptr, i0, i1, Bj + b0, nullptr, j0,
                                                  j1, nullptr, nullptr, 0, lane);
      if (lane == 0) {
        mt[w] = n;
        cnt[w] = n;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        int64_t t = 0;
        for (int k = 0; k < kMergeWarps; ++k) t += cnt[k];
        rowc[r] = int32_t(t);
      }
    } else {
      const int64_t i0 = cuts[2 * w], j0 = cuts[2 * w + 1];
      const int64_t i1 = cuts[2 * w + 2], j1 = cuts[2 * w + 3];
      int64_t off = cp[r];
      for (int k = 0; k < w; ++k) off += mt[k];
      merge_row_warp<true, VT>(Aj + a0, Ax + a0, i0, i1, Bj + b0, Bx + b0, j0, j1, Cj + off,
                               Cx + off, mt[w], lane);
    }
    __syncthreads();
  }
}

template <typename PTA, typename PTB, typename VT>
static int spadd_impl(tspg_ctx *ctx, cudaStream_t s, const tspg_csr *A,
                      const tspg_csr *B, tspg_csr_out *C) {
  const int64_t m = A->nrows;
  Scratch sc(ctx, s);
  int32_t *rowc;
  int64_t *cp, *partial, *heavy, *meta;
  const int64_t nb = (m + kScanTile - 1) / kScanTile;
  Sched *dummy;
  TSPG_TRY(sc.get(&rowc, m));
  TSPG_TRY(sc.get(&cp, m + 1));
  TSPG_TRY(sc.get(&partial, nb + 1));
  TSPG_TRY(sc.get(&dummy, 1));
  // heavy[0] = count of listed rows, heavy[1..] = the rows
  const int64_t max_heavy = (A->nnz + B->nnz) / (kMergeHeavy + 1) + 1;
  TSPG_TRY(sc.get(&heavy, max_heavy + 1));
  TSPG_TRY(sc.get(&meta, max_heavy * kHeavyMeta));
  TSPG_CUDA(ctx, cudaMemsetAsync(heavy, 0, sizeof(int64_t), s));
  TSPG_CUDA(ctx, cudaMemsetAsync(cp, 0, sizeof(int64_t), s));
  TSPG_CUDA(ctx, cudaMemsetAsync(dummy, 0, sizeof(Sched), s));
  const unsigned grid = (unsigned)std::min<int64_t>((m * 32 + 255) / 256, int64_t(ctx->num_sms) * 16);
  if (m > 0) {
    k_spadd_count<PTA, PTB><<<grid, 256, 0, s>>>(m, (const PTA *)A->rowptr, A->col,
                                                 (const PTB *)B->rowptr, B->col, rowc,
                                                 heavy + 1, heavy);
    k_spadd_heavy<false, PTA, PTB, VT><<<ctx->num_sms * 2, kMergeThreads, 0, s>>>(
        heavy + 1, heavy, (const PTA *)A->rowptr, A->col, (const VT *)A->val,
        (const PTB *)B->rowptr, B->col, (const VT *)B->val, rowc, nullptr, meta, nullptr, nullptr);
    k_scan_reduce<<<(unsigned)nb, kScanThreads, 0, s>>>(rowc, m, partial);
    k_scan_partials<<<1, 1024, 0, s>>>(partial, nb);
    k_scan_final<<<(unsigned)nb, kScanThreads, 0, s>>>(rowc, m, partial, nb, cp, dummy, nullptr);
    ctx->launches += 5;
  }
  TSPG_CUDA(ctx, cudaGetLastError());
  int64_t *h = ctx->h_words;
  TSPG_CUDA(ctx, cudaMemcpyAsync(h, cp + m, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  TSPG_CUDA(ctx, cudaStreamSynchronize(s));
  const int64_t nnz = h[0];
  if (C->rowptr_bits == 32 && nnz > INT32_MAX) return TSPG_EOVERFLOW;
  C->nnz = nnz;
  if (C->capacity < nnz) {
    if (!C->alloc) return TSPG_ENOMEM;
    void *cj = C->alloc(C->alloc_user, size_t(nnz) * 4, s);
    void *cx = C->alloc(C->alloc_user, size_t(nnz) * sizeof(VT), s);
    if (!cj || !cx) return TSPG_ENOMEM;
    C->col = (int32_t *)cj;
    C->val = cx;
    C->capacity = nnz;
  }
  if (m == 0) {
    TSPG_CUDA(ctx, cudaMemsetAsync(C->rowptr, 0, C->rowptr_bits / 8, s));
    return TSPG_OK;
  }
  k_spadd_fill<PTA, PTB, VT><<<grid, 256, 0, s>>>(
      m, (const PTA *)A->rowptr, A->col, (const VT *)A->val, (const PTB *)B->rowptr,
      B->col, (const VT *)B->val, cp, C->rowptr, C->rowptr_bits, C->col, (VT *)C->val);
  k_spadd_heavy<true, PTA, PTB, VT><<<ctx->num_sms * 2, kMergeThreads, 0, s>>>(
      heavy + 1, heavy, (const PTA *)A->rowptr, A->col, (const VT *)A->val,
      (const PTB *)B->rowptr, B->col, (const VT *)B->val, nullptr, cp, meta, C->col, (VT *)C->val);
  ctx->launches += 2;
  TSPG_CUDA(ctx, cudaGetLastError());
  return TSPG_OK;
}

}  // namespace tspg

using namespace tspg;

extern "C" int tspg_spadd(tspg_ctx *ctx, void *stream, const tspg_csr *A,
                          const tspg_csr *B, tspg_csr_out *C) {
  if (!ctx || !C) return TSPG_EINVAL;
  TSPG_TRY(check_csr(A));
  TSPG_TRY(check_csr(B));
  if (A->nrows != B->nrows || A->ncols != B->ncols || A->val_bits != B->val_bits)
    return TSPG_EINVAL;
  if (!C->rowptr || C->nrows != A->nrows || C->ncols != A->ncols ||
      C->val_bits != A->val_bits || (C->rowptr_bits != 32 && C->rowptr_bits != 64))
    return TSPG_EINVAL;
  cudaStream_t s = (cudaStream_t)stream;
  TSPG_CUDA(ctx, cudaSetDevice(ctx->device));
  const int a = A->rowptr_bits, b = B->rowptr_bits;
  if (A->val_bits == 64) {
    if (a == 32 && b == 32) return spadd_impl<int32_t, int32_t, double>(ctx, s, A, B, C);
    if (a == 32 && b == 64) return spadd_impl<int32_t, int64_t, double>(ctx, s, A, B, C);
    if (a == 64 && b == 32) return spadd_impl<int64_t, int32_t, double>(ctx, s, A, B, C);
    return spadd_impl<int64_t, int64_t, double>(ctx, s, A, B, C);
  } else {
    if (a == 32 && b == 32) return spadd_impl<int32_t, int32_t, float>(ctx, s, A, B, C);
    if (a == 32 && b == 64) return spadd_impl<int32_t, int64_t, float>(ctx, s, A, B, C);
    if (a == 64 && b == 32) return spadd_impl<int64_t, int32_t, float>(ctx, s, A, B, C);
    return spadd_impl<int64_t, int64_t, float>(ctx, s, A, B, C);
  }
}
