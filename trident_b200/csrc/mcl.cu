// mcl.cu — the per-iteration matrix updates of Markov clustering on the device.
//
// The reference's MCL driver (src/mcl.cu:56-149) copies its tile to the host
// for each of prune, normalize and inflation, loops over the rows there and
// copies the result back.  Here each is one or a few kernels on the caller's
// stream: normalize and inflation rewrite the values in place (one warp per
// row: its sum, then the scaled values), prune compacts the kept entries into
// a new CSR (count pass, device scan, order-preserving fill).  The row sums
// are over this tile's rows only: the reference then adds the partial sums of
// the ranks of a process row (MPI_Allreduce on the row communicator), a step
// that does not exist on one GPU.
#include "spgemm_kernels.cuh"

namespace tspg {

// Rows scaled to sum 1 (entries of a row whose sum is <= 1e-20 become 0),
// after raising every value to `power` when do_pow (inflation).
template <typename PT, typename VT>
__global__ void k_mcl_rows(const PT *rp, const VT *val, int64_t m, VT power, int do_pow,
                           VT *out) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = warp; r < m; r += nwarps) {
    const int64_t a0 = int64_t(rp[r]), a1 = int64_t(rp[r + 1]);
    VT sum = VT(0);
    for (int64_t p = a0 + lane; p < a1; p += 32) {
      VT v = val[p];
      if (do_pow) {
        v = pow(v, power);
        out[p] = v;
      }
      sum += v;
    }
    sum = warp_sum(sum);
    __syncwarp();  // the powered values written above are read back below
    const bool keep = sum > VT(1e-20);
    for (int64_t p = a0 + lane; p < a1; p += 32) {
      const VT v = do_pow ? out[p] : val[p];
      out[p] = keep ? v / sum : VT(0);
    }
  }
}

// Prune, pass 1: entries per row with |v| > tol.
template <typename PT, typename VT>
__global__ void k_prune_count(const PT *rp, const VT *val, int64_t m, VT tol, int32_t *cnt) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = warp; r < m; r += nwarps) {
    const int64_t a0 = int64_t(rp[r]), a1 = int64_t(rp[r + 1]);
    int c = 0;
    for (int64_t p0 = a0; p0 < a1; p0 += 32) {
      const int64_t p = p0 + lane;
      c += __popc(__ballot_sync(0xffffffffu, p < a1 && fabs(val[p]) > tol));
    }
    if (lane == 0) cnt[r] = c;
  }
}

// Prune, pass 2: the kept entries of every row, in their order, at the row's
// new offset.
template <typename PT, typename VT>
__global__ void k_prune_fill(const PT *rp, const int32_t *col, const VT *val, int64_t m, VT tol,
                             const int64_t *np, int32_t *ocol, VT *oval) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t r = warp; r < m; r += nwarps) {
    const int64_t a0 = int64_t(rp[r]), a1 = int64_t(rp[r + 1]);
    int64_t o = np[r];
    for (int64_t p0 = a0; p0 < a1; p0 += 32) {
      const int64_t p = p0 + lane;
      const VT v = p < a1 ? val[p] : VT(0);
      const bool k = p < a1 && fabs(v) > tol;
      const unsigned b = __ballot_sync(0xffffffffu, k);
      if (k) {
        const int64_t q = o + __popc(b & ((1u << lane) - 1u));
        ocol[q] = col[p];
        oval[q] = v;
      }
      o += __popc(b);
    }
  }
}

__global__ void k_offsets32(const int64_t *src, int64_t n, int32_t *dst) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = int32_t(src[i]);
}

static unsigned warp_grid(tspg_ctx *ctx, int64_t rows) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>((rows * 32 + 255) / 256,
                                                          int64_t(ctx->num_sms) * 16));
}

template <typename PT, typename VT>
static int mcl_rows_impl(tspg_ctx *ctx, cudaStream_t s, const tspg_csr *M, double power,
                         int do_pow, void *val_out) {
  if (M->nrows > 0 && M->nnz > 0) {
    k_mcl_rows<PT, VT><<<warp_grid(ctx, M->nrows), 256, 0, s>>>(
        (const PT *)M->rowptr, (const VT *)M->val, M->nrows, VT(power), do_pow, (VT *)val_out);
    ctx->launches += 1;
  }
  TSPG_CUDA(ctx, cudaGetLastError());
  return TSPG_OK;
}

template <typename PT, typename VT>
static int prune_impl(tspg_ctx *ctx, cudaStream_t s, const tspg_csr *M, double tol,
                      tspg_csr_out *out) {
  const int64_t m = M->nrows, nb = (m + kScanTile - 1) / kScanTile;
  Scratch sc(ctx, s);
  int32_t *cnt;
  int64_t *np, *partial;
  Sched *dummy;
  TSPG_TRY(sc.get(&cnt, m));
  TSPG_TRY(sc.get(&np, m + 1));
  TSPG_TRY(sc.get(&partial, nb + 1));
  TSPG_TRY(sc.get(&dummy, 1));
  TSPG_CUDA(ctx, cudaMemsetAsync(np, 0, sizeof(int64_t) * (m + 1), s));
  const unsigned g = warp_grid(ctx, m);
  if (m > 0) {
    k_prune_count<PT, VT><<<g, 256, 0, s>>>((const PT *)M->rowptr, (const VT *)M->val, m, VT(tol), cnt);
    k_scan_reduce<<<(unsigned)nb, kScanThreads, 0, s>>>(cnt, m, partial);
    k_scan_partials<<<1, 1024, 0, s>>>(partial, nb);
    k_scan_final<<<(unsigned)nb, kScanThreads, 0, s>>>(cnt, m, partial, nb, np, dummy, nullptr);
    ctx->launches += 4;
  }
  int64_t *h = ctx->h_words;
  TSPG_CUDA(ctx, cudaMemcpyAsync(h, np + m, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  TSPG_CUDA(ctx, cudaStreamSynchronize(s));
  const int64_t nnz = h[0];
  out->nnz = nnz;
  if (out->rowptr_bits == 32 && nnz > INT32_MAX) return TSPG_EOVERFLOW;
  if (out->capacity < nnz) {
    if (!out->alloc) return TSPG_ENOMEM;
    void *cj = out->alloc(out->alloc_user, size_t(nnz) * 4, s);
    void *cx = out->alloc(out->alloc_user, size_t(nnz) * sizeof(VT), s);
    if (!cj || !cx) return TSPG_ENOMEM;
    out->col = (int32_t *)cj;
    out->val = cx;
    out->capacity = nnz;
  }
  if (m > 0 && nnz > 0) {
    k_prune_fill<PT, VT><<<g, 256, 0, s>>>((const PT *)M->rowptr, M->col, (const VT *)M->val, m,
                                           VT(tol), np, out->col, (VT *)out->val);
    ctx->launches += 1;
  }
  if (out->rowptr_bits == 64) {
    TSPG_CUDA(ctx, cudaMemcpyAsync(out->rowptr, np, sizeof(int64_t) * (m + 1), cudaMemcpyDeviceToDevice, s));
  } else {
    k_offsets32<<<(unsigned)((m + 1 + 255) / 256), 256, 0, s>>>(np, m + 1, (int32_t *)out->rowptr);
    ctx->launches += 1;
  }
  TSPG_CUDA(ctx, cudaGetLastError());
  return TSPG_OK;
}

}  // namespace tspg

using namespace tspg;

static int mcl_rows(tspg_ctx *ctx, void *stream, const tspg_csr *M, double power, int do_pow,
                    void *val_out) {
  if (!ctx) return TSPG_EINVAL;
  TSPG_TRY(check_csr(M));
  if (!val_out && M->nnz > 0) return TSPG_EINVAL;
  TSPG_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  if (M->val_bits == 64)
    return M->rowptr_bits == 32 ? mcl_rows_impl<int32_t, double>(ctx, s, M, power, do_pow, val_out)
                                : mcl_rows_impl<int64_t, double>(ctx, s, M, power, do_pow, val_out);
  return M->rowptr_bits == 32 ? mcl_rows_impl<int32_t, float>(ctx, s, M, power, do_pow, val_out)
                              : mcl_rows_impl<int64_t, float>(ctx, s, M, power, do_pow, val_out);
}

extern "C" int tspg_mcl_normalize(tspg_ctx *ctx, void *stream, const tspg_csr *M, void *val_out) {
  return mcl_rows(ctx, stream, M, 1.0, 0, val_out);
}

extern "C" int tspg_mcl_inflate(tspg_ctx *ctx, void *stream, const tspg_csr *M, double power,
                                void *val_out) {
  return mcl_rows(ctx, stream, M, power, 1, val_out);
}

extern "C" int tspg_mcl_prune(tspg_ctx *ctx, void *stream, const tspg_csr *M, double tol,
                              tspg_csr_out *out) {
  if (!ctx || !out) return TSPG_EINVAL;
  TSPG_TRY(check_csr(M));
  if (!out->rowptr || out->nrows != M->nrows || out->ncols != M->ncols ||
      out->val_bits != M->val_bits || (out->rowptr_bits != 32 && out->rowptr_bits != 64))
    return TSPG_EINVAL;
  TSPG_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  if (M->val_bits == 64)
    return M->rowptr_bits == 32 ? prune_impl<int32_t, double>(ctx, s, M, tol, out)
                                : prune_impl<int64_t, double>(ctx, s, M, tol, out);
  return M->rowptr_bits == 32 ? prune_impl<int32_t, float>(ctx, s, M, tol, out)
                              : prune_impl<int64_t, float>(ctx, s, M, tol, out);
}
