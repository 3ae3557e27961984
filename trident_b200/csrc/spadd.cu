// spadd.cu — merge of partial C tiles, C = A + B with the union pattern.
//
// Replaces cusparse_spgeam (include/cusparse_helpers.cuh:799-905: csrgeam2
// bufferSize + Nnz + compute, five stream syncs, the nnz through the host) and
// LocalMatrix::spadd (include/KokkosWrap.hpp:394-439: KK spadd symbolic +
// numeric).  Rows are sorted and duplicate-free, so every entry finds its
// output slot independently: an A entry at row position i lands at
// i + |{b in B row : b < a}|, a B entry that is not in A at
// j + |{a in A row : a < b}|.  Rows with up to kMergeHeavy entries in A and B
// together: one warp per row; lanes take entries and binary search the other
// row (which sits in L1 after the first probes).  Longer rows (the hub rows of
// partial C tiles reach 10^5 entries, and one warp per such row left the merge
// waiting on a handful of warps) are listed and merged by a whole CTA along a
// merge path: thread t takes steps [t, t+1) x (|A|+|B|) / threads of the
// merged sequence (A before B on equal columns).
#include "internal.cuh"
#include "spgemm_kernels.cuh"

namespace tspg {

template <typename IT>
__device__ __forceinline__ int64_t lower_bound_row(const int32_t *col, int64_t lo,
                                                   int64_t hi, int32_t x) {
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (__ldg(col + mid) < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

constexpr int64_t kMergeHeavy = 4096;  // rows above this go to the CTA merge
constexpr int kMergeThreads = 512;

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
    int dup = 0;
    if (b1 > b0) {
      for (int64_t p = a0 + lane; p < a1; p += 32) {
        const int32_t x = __ldg(Aj + p);
        const int64_t q = lower_bound_row<int>(Bj, b0, b1, x);
        dup += (q < b1 && __ldg(Bj + q) == x);
      }
    }
    dup = warp_sum(dup);
    if (lane == 0) rowc[r] = int32_t((a1 - a0) + (b1 - b0) - dup);
  }
}

// Output rank of a column x of the union row: |{a < x}| + |{b < x}| minus
// the columns below x present in both rows.  The fill walks A's row in warp
// chunks, flags A entries that also occur in B (binary search), keeps the
// running exclusive count of those flags in dpre[] (one int per A entry) and
// writes every A entry; B entries absent from A then look their rank up
// through dpre at their lower bound in A.
template <typename PTA, typename PTB, typename VT>
__global__ void __launch_bounds__(256)
    k_spadd_fill(int64_t m, const PTA *Ap, const int32_t *Aj, const VT *Ax,
                 const PTB *Bp, const int32_t *Bj, const VT *Bx,
                 const int64_t *cp, void *Cp, int cp_bits, int32_t *Cj, VT *Cx,
                 int32_t *dpre) {
  const int lane = threadIdx.x & 31;
  const unsigned below = (1u << lane) - 1u;
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
    int running = 0;
    for (int64_t base = a0; base < a1; base += 32) {
      const int64_t p = base + lane;
      bool dup = false;
      int32_t x = 0;
      int64_t q = b0;
      if (p < a1) {
        x = __ldg(Aj + p);
        q = lower_bound_row<int>(Bj, b0, b1, x);
        dup = q < b1 && __ldg(Bj + q) == x;
      }
      const unsigned bal = __ballot_sync(0xffffffffu, dup);
      const int pre = running + __popc(bal & below);
      if (p < a1) {
        dpre[p] = pre;
        VT v = __ldg(Ax + p);
        if (dup) v += __ldg(Bx + q);
        const int64_t pos = o + (p - a0) + (q - b0) - pre;
        Cj[pos] = x;
        Cx[pos] = v;
      }
      running += __popc(bal);
    }
    __syncwarp();
    for (int64_t q = b0 + lane; q < b1; q += 32) {
      const int32_t x = __ldg(Bj + q);
      const int64_t p = lower_bound_row<int>(Aj, a0, a1, x);
      if (p < a1 && __ldg(Aj + p) == x) continue;
      const int common = p < a1 ? dpre[p] : running;
      const int64_t pos = o + (q - b0) + (p - a0) - common;
      Cj[pos] = x;
      Cx[pos] = __ldg(Bx + q);
    }
    __syncwarp();
  }
}

// Merge path of one heavy row inside a CTA.  Thread t covers the merged
// steps [d0, d1); an A entry equal to the B entry at the B cursor takes that
// B value too (it may lie past the thread's range), and a B entry equal to the
// A entry before it is skipped, so a column present in both rows is emitted
// once whichever thread holds either half.  WRITE = false counts the row's
// union size; WRITE = true writes the row at (cj, cx).
template <bool WRITE, typename VT>
__device__ int64_t merge_row_cta(const int32_t *__restrict__ aj, const VT *__restrict__ ax,
                                 int64_t la, const int32_t *__restrict__ bj,
                                 const VT *__restrict__ bx, int64_t lb, int64_t *tmp,
                                 int32_t *cj, VT *cx) {
  const int tid = threadIdx.x;
  const int64_t tot = la + lb;
  const int64_t d0 = tot * tid / kMergeThreads, d1 = tot * (tid + 1) / kMergeThreads;
  // largest i with A[i-1] <= B[d0-i]: the A entries among the first d0 steps
  int64_t lo = d0 > lb ? d0 - lb : 0, hi = d0 < la ? d0 : la;
  while (lo < hi) {
    const int64_t mid = (lo + hi + 1) >> 1;
    if (__ldg(aj + mid - 1) <= __ldg(bj + d0 - mid)) lo = mid; else hi = mid - 1;
  }
  int64_t i = lo, j = d0 - lo;
  auto step = [&](bool emit, int64_t pos) -> int {  // 1 if the step makes an output
    const bool take_a = i < la && (j >= lb || __ldg(aj + i) <= __ldg(bj + j));
    if (take_a) {
      if (emit) {
        const int32_t x = __ldg(aj + i);
        VT v = __ldg(ax + i);
        if (j < lb && __ldg(bj + j) == x) v += __ldg(bx + j);
        cj[pos] = x;
        cx[pos] = v;
      }
      ++i;
      return 1;
    }
    const int32_t x = __ldg(bj + j);
    const bool dup = i > 0 && __ldg(aj + i - 1) == x;
    if (emit && !dup) {
      cj[pos] = x;
      cx[pos] = __ldg(bx + j);
    }
    ++j;
    return dup ? 0 : 1;
  };
  const int64_t si = i, sj = j;
  int64_t n = 0;
  for (int64_t d = d0; d < d1; ++d) n += step(false, 0);
  int64_t all;
  const int64_t base = group_excl_scan<kMergeThreads, int64_t>(n, tmp, 0, &all);
  if constexpr (WRITE) {
    i = si;
    j = sj;
    int64_t pos = base;
    for (int64_t d = d0; d < d1; ++d) pos += step(true, pos);
  }
  return all;
}

// The listed heavy rows, one CTA each (persistent over the list).
template <bool WRITE, typename PTA, typename PTB, typename VT>
__global__ void __launch_bounds__(kMergeThreads)
    k_spadd_heavy(const int64_t *heavy, const int64_t *nheavy, const PTA *Ap,
                  const int32_t *Aj, const VT *Ax, const PTB *Bp, const int32_t *Bj,
                  const VT *Bx, int32_t *rowc, const int64_t *cp, int32_t *Cj, VT *Cx) {
  __shared__ int64_t tmp[kMergeThreads / 32 + 1];
  const int64_t nh = *nheavy;
  for (int64_t h = blockIdx.x; h < nh; h += gridDim.x) {
    const int64_t r = heavy[h];
    const int64_t a0 = Ap[r], a1 = Ap[r + 1], b0 = Bp[r], b1 = Bp[r + 1];
    if constexpr (WRITE) {
      merge_row_cta<true, VT>(Aj + a0, Ax + a0, a1 - a0, Bj + b0, Bx + b0, b1 - b0, tmp,
                              Cj + cp[r], Cx + cp[r]);
    } else {
      const int64_t n = merge_row_cta<false, VT>(Aj + a0, nullptr, a1 - a0, Bj + b0, nullptr,
                                                 b1 - b0, tmp, nullptr, nullptr);
      if (threadIdx.x == 0) rowc[r] = int32_t(n);
    }
    __syncthreads();
  }
}

template <typename PTA, typename PTB, typename VT>
static int spadd_impl(tspg_ctx *ctx, cudaStream_t s, const tspg_csr *A,
                      const tspg_csr *B, tspg_csr_out *C) {
  const int64_t m = A->nrows;
  Scratch sc(ctx, s);
  int32_t *rowc, *dpre;
  int64_t *cp, *partial, *heavy;
  const int64_t nb = (m + kScanTile - 1) / kScanTile;
  Sched *dummy;
  TSPG_TRY(sc.get(&rowc, m));
  TSPG_TRY(sc.get(&dpre, A->nnz));
  TSPG_TRY(sc.get(&cp, m + 1));
  TSPG_TRY(sc.get(&partial, nb + 1));
  TSPG_TRY(sc.get(&dummy, 1));
  // heavy[0] = count of listed rows, heavy[1..] = the rows
  const int64_t max_heavy = (A->nnz + B->nnz) / (kMergeHeavy + 1) + 1;
  TSPG_TRY(sc.get(&heavy, max_heavy + 1));
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
        (const PTB *)B->rowptr, B->col, (const VT *)B->val, rowc, nullptr, nullptr, nullptr);
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
      B->col, (const VT *)B->val, cp, C->rowptr, C->rowptr_bits, C->col, (VT *)C->val, dpre);
  k_spadd_heavy<true, PTA, PTB, VT><<<ctx->num_sms * 2, kMergeThreads, 0, s>>>(
      heavy + 1, heavy, (const PTA *)A->rowptr, A->col, (const VT *)A->val,
      (const PTB *)B->rowptr, B->col, (const VT *)B->val, nullptr, cp, C->col, (VT *)C->val);
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
