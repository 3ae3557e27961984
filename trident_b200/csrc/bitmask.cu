// bitmask.cu — sparsity bitmasks and the bitmask tile pack / unpack.
//
// Reference behaviour (include/spacomm.cuh):
//   gen_bitmask (:29-117)        thrust transform + cub segmented reduce +
//                                a host round trip to narrow int -> uint8;
//   intersect_bitmasks (:126-148) thrust copy of a zipped AND;
//   select_entries_cuda (:808-889) per-block select with cub::BlockScan, a
//                                host scan of block counts, then a compaction
//                                kernel — run once for values, once for
//                                indices;
//   select_ptrs (:556-623)       two cub passes in place on the pointer array.
// Here: gen is one ballot per 32 segments; the pack is one masked-count pass
// over the pointer array, the device scan, and one copy pass in which each
// thread walks a run of consecutive entries (segment found once by binary
// search, then advanced), writing values and indices together.  The kept
// count never leaves the device unless the caller asks for it.
#include "internal.cuh"
#include "pack_kernels.cuh"
#include "spgemm_kernels.cuh"

namespace tspg {

template <typename PT>
__global__ void k_bitmask_gen(const PT *ptr, int64_t n, uint8_t *out) {
  const int64_t nbytes = (n + 7) >> 3;
  const int lane = threadIdx.x & 31;
  for (int64_t i0 = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) & ~int64_t(31);
       i0 < n; i0 += int64_t(gridDim.x) * blockDim.x) {
    const int64_t i = i0 + lane;
    const bool ne = i < n && ptr[i] != ptr[i + 1];
    const unsigned bal = __ballot_sync(0xffffffffu, ne);
    if (lane < 4) {
      const int64_t byte = (i0 >> 3) + lane;
      if (byte < nbytes) out[byte] = uint8_t((bal >> (8 * lane)) & 0xffu);
    }
  }
}

__global__ void k_bitmask_and(const uint8_t *a, const uint8_t *b,
                              int64_t nbytes, uint8_t *out, int vec) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  int64_t done = 0;
  if (vec) {
    const int64_t nv = nbytes >> 4;
    const uint4 *a4 = (const uint4 *)a, *b4 = (const uint4 *)b;
    uint4 *o4 = (uint4 *)out;
    for (int64_t i = t; i < nv; i += stride) {
      const uint4 x = a4[i], y = b4[i];
      o4[i] = make_uint4(x.x & y.x, x.y & y.y, x.z & y.z, x.w & y.w);
    }
    done = nv << 4;
  }
  for (int64_t i = done + t; i < nbytes; i += stride) out[i] = a[i] & b[i];
}

template <typename PT>
static int pack_impl(tspg_ctx *ctx, cudaStream_t s, const tspg_csr *M,
                     int64_t len, const uint8_t *mask, void *out_buf,
                     int64_t *kept_dev, int64_t *kept_host) {
  Scratch sc(ctx, s);
  int32_t *cnt;
  int64_t *newp, *partial;
  Sched *dummy;
  const int64_t nb = (len + kScanTile - 1) / kScanTile;
  TSPG_TRY(sc.get(&cnt, len));
  TSPG_TRY(sc.get(&newp, len + 1));
  TSPG_TRY(sc.get(&partial, nb + 1));
  TSPG_TRY(sc.get(&dummy, 1));
  TSPG_CUDA(ctx, cudaMemsetAsync(newp, 0, sizeof(int64_t), s));
  TSPG_CUDA(ctx, cudaMemsetAsync(dummy, 0, sizeof(Sched), s));
  const PT *ptr = (const PT *)M->rowptr;
  if (len > 0) {
    k_pack_counts<PT><<<(unsigned)((len + 255) / 256), 256, 0, s>>>(ptr, len, mask, cnt);
    k_scan_reduce<<<(unsigned)nb, kScanThreads, 0, s>>>(cnt, len, partial);
    k_scan_partials<<<1, 1024, 0, s>>>(partial, nb);
    k_scan_final<<<(unsigned)nb, kScanThreads, 0, s>>>(cnt, len, partial, nb, newp, dummy, nullptr);
    ctx->launches += 4;
  }
  ctx->launches += 1;
  const int64_t work = (M->nnz + kPackItems - 1) / kPackItems;
  const int64_t w = work > len + 1 ? work : len + 1;
  const unsigned grid = (unsigned)std::min<int64_t>((w + 255) / 256, int64_t(ctx->num_sms) * 32);
  if (M->val_bits == 64)
    k_pack_copy<PT, 8><<<grid, 256, 0, s>>>(ptr, len, M->col, M->val, mask, newp,
                                            (char *)out_buf, kept_dev);
  else
    k_pack_copy<PT, 4><<<grid, 256, 0, s>>>(ptr, len, M->col, M->val, mask, newp,
                                            (char *)out_buf, kept_dev);
  TSPG_CUDA(ctx, cudaGetLastError());
  if (kept_host) {
    TSPG_CUDA(ctx, cudaMemcpyAsync(ctx->h_words, newp + len, sizeof(int64_t),
                                   cudaMemcpyDeviceToHost, s));
    TSPG_CUDA(ctx, cudaStreamSynchronize(s));
    *kept_host = ctx->h_words[0];
  }
  return TSPG_OK;
}

}  // namespace tspg

using namespace tspg;

extern "C" int tspg_bitmask_gen(tspg_ctx *ctx, void *stream, const void *ptr,
                                int ptr_bits, int64_t n, uint8_t *mask_out) {
  if (!ctx || n < 0 || (ptr_bits != 32 && ptr_bits != 64)) return TSPG_EINVAL;
  if (n == 0) return TSPG_OK;
  if (!ptr || !mask_out) return TSPG_EINVAL;
  TSPG_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned grid = (unsigned)std::min<int64_t>((n + 255) / 256, int64_t(ctx->num_sms) * 32);
  if (ptr_bits == 32)
    k_bitmask_gen<int32_t><<<grid, 256, 0, s>>>((const int32_t *)ptr, n, mask_out);
  else
    k_bitmask_gen<int64_t><<<grid, 256, 0, s>>>((const int64_t *)ptr, n, mask_out);
  ctx->launches += 1;
  TSPG_CUDA(ctx, cudaGetLastError());
  return TSPG_OK;
}

extern "C" int tspg_bitmask_and(tspg_ctx *ctx, void *stream, const uint8_t *a,
                                const uint8_t *b, int64_t nbytes, uint8_t *out) {
  if (!ctx || nbytes < 0) return TSPG_EINVAL;
  if (nbytes == 0) return TSPG_OK;
  if (!a || !b || !out) return TSPG_EINVAL;
  TSPG_CUDA(ctx, cudaSetDevice(ctx->device));
  const int vec = ((((uintptr_t)a) | ((uintptr_t)b) | ((uintptr_t)out)) & 15) == 0;
  const int64_t work = vec ? (nbytes >> 4) + 16 : nbytes;
  const unsigned grid = (unsigned)std::min<int64_t>((work + 255) / 256, int64_t(ctx->num_sms) * 32);
  k_bitmask_and<<<grid, 256, 0, (cudaStream_t)stream>>>(a, b, nbytes, out, vec);
  ctx->launches += 1;
  TSPG_CUDA(ctx, cudaGetLastError());
  return TSPG_OK;
}

static inline size_t packed_ptr_offset(int64_t nnz, int val_bits, int ptr_bits) {
  const size_t pb = size_t(ptr_bits / 8);
  return (size_t(nnz) * size_t(val_bits / 8 + 4) + pb - 1) & ~(pb - 1);
}

extern "C" size_t tspg_packed_bytes(int64_t nnz, int64_t ptr_len, int val_bits,
                                    int ptr_bits) {
  return packed_ptr_offset(nnz, val_bits, ptr_bits) +
         size_t(ptr_len + 1) * size_t(ptr_bits / 8);
}

extern "C" int tspg_pack(tspg_ctx *ctx, void *stream, const tspg_csr *M,
                         int major, const uint8_t *mask, void *out_buf,
                         size_t cap, int64_t *nnz_kept_dev,
                         int64_t *nnz_kept_host) {
  if (!ctx || !out_buf) return TSPG_EINVAL;
  TSPG_TRY(check_csr(M));
  if (major != TSPG_ROWS && major != TSPG_COLS) return TSPG_EINVAL;
  const int64_t len = major == TSPG_ROWS ? M->nrows : M->ncols;
  // the pointer array has len + 1 entries: no segments means no entries, and
  // a non-empty pointer array must be given
  if ((len == 0 && M->nnz > 0) || (len > 0 && !M->rowptr)) return TSPG_EINVAL;
  if (len > 0 && !mask) return TSPG_EINVAL;
  if ((uintptr_t)out_buf & 7) return TSPG_EINVAL;
  if (cap < tspg_packed_bytes(M->nnz, len, M->val_bits, M->rowptr_bits)) return TSPG_ENOMEM;
  TSPG_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  if (M->rowptr_bits == 32)
    return pack_impl<int32_t>(ctx, s, M, len, mask, out_buf, nnz_kept_dev, nnz_kept_host);
  return pack_impl<int64_t>(ctx, s, M, len, mask, out_buf, nnz_kept_dev, nnz_kept_host);
}

extern "C" int tspg_unpack(const void *buf, int64_t nrows, int64_t ncols,
                           int major, int64_t nnz, int val_bits, int ptr_bits,
                           tspg_csr *out) {
  if (!buf || !out || nnz < 0) return TSPG_EINVAL;
  if ((val_bits != 32 && val_bits != 64) || (ptr_bits != 32 && ptr_bits != 64))
    return TSPG_EINVAL;
  if (major != TSPG_ROWS && major != TSPG_COLS) return TSPG_EINVAL;
  const char *b = (const char *)buf;
  out->nrows = nrows;
  out->ncols = ncols;
  out->nnz = nnz;
  out->val_bits = val_bits;
  out->rowptr_bits = ptr_bits;
  out->val = b;
  out->col = (const int32_t *)(b + nnz * (val_bits / 8));
  out->rowptr = b + packed_ptr_offset(nnz, val_bits, ptr_bits);
  return TSPG_OK;
}
