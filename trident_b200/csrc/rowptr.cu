// rowptr.cu — in-place conversions of a pointer array on the device: row
// offsets <-> row counts (the wire step around the node gather of B tiles,
// rowptrs_to_rownnz / rownnz_to_rowptrs, include/utils.cuh:412-448, used at
// include/tile_holder.cuh:283-327), and the masked pointer pack of a tile
// (select_ptrs, include/spacomm.cuh:556-623) built from them.
#include <algorithm>

#include "spgemm_kernels.cuh"

namespace tspg {
namespace {

// dst[0] = src[0], dst[i] = src[i] - src[i - 1] (the left difference of
// cub::DeviceAdjacentDifference::SubtractLeft) over n1 entries.
template <typename PT>
__global__ void k_adjdiff(const PT *src, PT *dst, int64_t n1) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n1) dst[i] = i ? PT(src[i] - src[i - 1]) : src[0];
}

// counts of segments whose mask bit is clear become 0 (cnt = ptr + 1)
template <typename PT>
__global__ void k_mask_counts(PT *cnt, int64_t len, const uint8_t *mask) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < len && !((mask[i >> 3] >> (i & 7)) & 1)) cnt[i] = PT(0);
}

// per tile of kScanTile entries: the sum
template <typename PT>
__global__ void __launch_bounds__(kScanThreads) k_tile_sum(const PT *in, int64_t n, int64_t *partial) {
  __shared__ int64_t tmp[kScanThreads / 32 + 1];
  const int64_t t0 = int64_t(blockIdx.x) * kScanTile;
  int64_t s = 0;
  for (int i = 0; i < kScanItems; ++i) {
    const int64_t j = t0 + int64_t(i) * kScanThreads + threadIdx.x;
    if (j < n) s += int64_t(in[j]);
  }
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) tmp[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    int64_t v = threadIdx.x < kScanThreads / 32 ? tmp[threadIdx.x] : 0;
    v = warp_sum(v);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
  }
}

// inclusive scan in place; each thread owns kScanItems consecutive entries
// (read before the block scan, written after it, so in place is safe); an
// int32 result above INT32_MAX raises *ovf
template <typename PT>
__global__ void __launch_bounds__(kScanThreads)
    k_tile_scan(PT *io, int64_t n, const int64_t *partial, int64_t *ovf) {
  __shared__ int64_t tmp[kScanThreads / 32 + 1];
  const int64_t j0 = int64_t(blockIdx.x) * kScanTile + int64_t(threadIdx.x) * kScanItems;
  int64_t v[kScanItems];
  int64_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    v[i] = j0 + i < n ? int64_t(io[j0 + i]) : 0;
    s += v[i];
  }
  int64_t tot;
  int64_t run = group_excl_scan<kScanThreads, int64_t>(s, tmp, 0, &tot) + partial[blockIdx.x];
  bool over = false;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    run += v[i];
    if (j0 + i < n) {
      if (sizeof(PT) == 4 && run > INT32_MAX) over = true;
      io[j0 + i] = PT(run);
    }
  }
  if (over) atomicExch((unsigned long long *)ovf, 1ull);
}

template <typename PT>
int to_rownnz(tspg_ctx *ctx, cudaStream_t s, PT *ptr, int64_t nrows) {
  Scratch sc(ctx, s);
  PT *copy;
  TSPG_TRY(sc.get(&copy, nrows + 1));
  TSPG_CUDA(ctx, cudaMemcpyAsync(copy, ptr, sizeof(PT) * size_t(nrows + 1), cudaMemcpyDeviceToDevice, s));
  k_adjdiff<PT><<<(unsigned)((nrows + 1 + 255) / 256), 256, 0, s>>>(copy, ptr, nrows + 1);
  ctx->launches += 1;
  TSPG_CUDA(ctx, cudaGetLastError());
  return TSPG_OK;
}

// ptr[1..nrows] := inclusive scan of ptr[1..nrows]; synchronises s to report
// an int32 overflow
template <typename PT>
int to_rowptrs(tspg_ctx *ctx, cudaStream_t s, PT *ptr, int64_t nrows) {
  if (nrows == 0) return TSPG_OK;
  Scratch sc(ctx, s);
  const int64_t nb = (nrows + kScanTile - 1) / kScanTile;
  int64_t *partial, *ovf;
  TSPG_TRY(sc.get(&partial, nb + 1));
  TSPG_TRY(sc.get(&ovf, 1));
  TSPG_CUDA(ctx, cudaMemsetAsync(ovf, 0, sizeof(int64_t), s));
  k_tile_sum<PT><<<(unsigned)nb, kScanThreads, 0, s>>>(ptr + 1, nrows, partial);
  k_scan_partials<<<1, 1024, 0, s>>>(partial, nb);
  k_tile_scan<PT><<<(unsigned)nb, kScanThreads, 0, s>>>(ptr + 1, nrows, partial, ovf);
  ctx->launches += 3;
  TSPG_CUDA(ctx, cudaGetLastError());
  TSPG_CUDA(ctx, cudaMemcpyAsync(ctx->h_words, ovf, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  TSPG_CUDA(ctx, cudaStreamSynchronize(s));
  return ctx->h_words[0] ? TSPG_EOVERFLOW : TSPG_OK;
}

template <typename PT>
int select_ptrs_impl(tspg_ctx *ctx, cudaStream_t s, PT *ptr, int64_t len, const uint8_t *mask) {
  TSPG_TRY(to_rownnz<PT>(ctx, s, ptr, len));
  if (len > 0) {
    k_mask_counts<PT><<<(unsigned)((len + 255) / 256), 256, 0, s>>>(ptr + 1, len, mask);
    ctx->launches += 1;
    TSPG_CUDA(ctx, cudaGetLastError());
  }
  return to_rowptrs<PT>(ctx, s, ptr, len);
}

// products of row r of A·B: sum over A's entries (r, k) of nnz(B row k); one
// warp per row
template <typename PA, typename PB>
__global__ void __launch_bounds__(256)
    k_row_products(const PA *Ap, const int32_t *Aj, const PB *Bp, int64_t m, int64_t *out) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; r < m; r += nw) {
    int64_t f = 0;
    for (int64_t q = int64_t(Ap[r]) + lane; q < int64_t(Ap[r + 1]); q += 32) {
      const int32_t k = Aj[q];
      f += int64_t(Bp[k + 1]) - int64_t(Bp[k]);
    }
    f = warp_sum(f);
    if (lane == 0) out[r] = f;
  }
}

template <typename PA, typename PB>
int row_products_impl(tspg_ctx *ctx, cudaStream_t s, const tspg_csr *A, const tspg_csr *B, int64_t *out) {
  if (A->nrows == 0) return TSPG_OK;
  const int64_t blocks = std::min<int64_t>((A->nrows * 32 + 255) / 256, int64_t(ctx->num_sms) * 16);
  k_row_products<PA, PB><<<(unsigned)blocks, 256, 0, s>>>((const PA *)A->rowptr, A->col, (const PB *)B->rowptr,
                                                         A->nrows, out);
  ctx->launches += 1;
  TSPG_CUDA(ctx, cudaGetLastError());
  return TSPG_OK;
}

int check_ptr_args(tspg_ctx *ctx, void *ptr, int ptr_bits, int64_t n) {
  if (!ctx || !ptr || n < 0) return TSPG_EINVAL;
  if (ptr_bits != 32 && ptr_bits != 64) return TSPG_EINVAL;
  return TSPG_OK;
}

}  // namespace
}  // namespace tspg

using namespace tspg;

extern "C" int tspg_rowptrs_to_rownnz(tspg_ctx *ctx, void *stream, void *ptr, int ptr_bits,
                                      int64_t nrows) {
  TSPG_TRY(check_ptr_args(ctx, ptr, ptr_bits, nrows));
  TSPG_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  return ptr_bits == 32 ? to_rownnz<int32_t>(ctx, s, (int32_t *)ptr, nrows)
                        : to_rownnz<int64_t>(ctx, s, (int64_t *)ptr, nrows);
}

extern "C" int tspg_rownnz_to_rowptrs(tspg_ctx *ctx, void *stream, void *ptr, int ptr_bits,
                                      int64_t nrows) {
  TSPG_TRY(check_ptr_args(ctx, ptr, ptr_bits, nrows));
  TSPG_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  return ptr_bits == 32 ? to_rowptrs<int32_t>(ctx, s, (int32_t *)ptr, nrows)
                        : to_rowptrs<int64_t>(ctx, s, (int64_t *)ptr, nrows);
}

extern "C" int tspg_select_ptrs(tspg_ctx *ctx, void *stream, void *ptr, int ptr_bits, int64_t len,
                                const uint8_t *mask) {
  TSPG_TRY(check_ptr_args(ctx, ptr, ptr_bits, len));
  if (len > 0 && !mask) return TSPG_EINVAL;
  TSPG_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  return ptr_bits == 32 ? select_ptrs_impl<int32_t>(ctx, s, (int32_t *)ptr, len, mask)
                        : select_ptrs_impl<int64_t>(ctx, s, (int64_t *)ptr, len, mask);
}

extern "C" int tspg_spgemm_row_products(tspg_ctx *ctx, void *stream, const tspg_csr *A,
                                        const tspg_csr *B, int64_t *out) {
  if (!ctx || !out) return TSPG_EINVAL;
  TSPG_TRY(check_csr(A));
  TSPG_TRY(check_csr(B));
  if (A->ncols != B->nrows) return TSPG_EINVAL;
  if (A->nnz > 0 && B->nrows > 0 && !B->rowptr) return TSPG_EINVAL;
  TSPG_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  if (A->rowptr_bits == 32)
    return B->rowptr_bits == 32 ? row_products_impl<int32_t, int32_t>(ctx, s, A, B, out)
                                : row_products_impl<int32_t, int64_t>(ctx, s, A, B, out);
  return B->rowptr_bits == 32 ? row_products_impl<int64_t, int32_t>(ctx, s, A, B, out)
                              : row_products_impl<int64_t, int64_t>(ctx, s, A, B, out);
}
