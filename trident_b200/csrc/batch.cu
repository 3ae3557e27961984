// batch.cu — many independent products C_i = A_i·B_i in one persistent launch
// per phase.
//
// All rows of all products form one flat row space (row g of product p is
// base[p] + r).  The same binning / persistent kernels as the single
// product path run once over that space, so the device work queue interleaves
// rows of every product, heaviest class first; a product of 1k rows and one of
// 200k rows cost one launch each phase together.  Outputs land in one slab
// (int32 columns, values, int64 row offsets with one extra entry per product).
//
// A run is two CUDA graphs around one host sync (the output size):
//   graph 1: sortedness check, mults, binning, symbolic k_phase + k_groups, scan,
//            per-product offsets -> pinned host;
//   graph 2: output pointers, numeric binning, numeric k_phase + k_groups.
// The graphs are captured on the first run and replayed while the batch's
// operands are unchanged; tspg_batch_add / clear drop them.
#include <cstring>
#include <new>
#include <vector>

#include "spgemm_cluster.cuh"

namespace tspg {

// Flattened B-row sortedness check over all products (one warp per B row).
template <typename PT, typename VT>
__global__ void k_check_sorted_batch(ProdDev<PT, VT> *prods, const int64_t *bbase,
                                     int nprod, int64_t RB) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  for (int64_t g = warp; g < RB; g += nwarps) {
    const int p = find_prod(bbase, nprod, g);
    const int64_t r = g - bbase[p];
    const PT *Bp = prods[p].Bp;
    const int32_t *Bj = prods[p].Bj;
    const int64_t b0 = Bp[r], b1 = Bp[r + 1];
    bool bad = false;
    for (int64_t q = b0 + lane; q + 1 < b1; q += 32)
      if (Bj[q] >= Bj[q + 1]) bad = true;
    if (__any_sync(0xffffffffu, bad) && lane == 0) prods[p].b_sorted = 0;
  }
}

// Per-product output offsets (cp at each product's first row) and the total.
__global__ void k_gather_offsets(const int64_t *cp, const int64_t *base, int nprod,
                                 int64_t *out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p <= nprod) out[p] = cp[base[p]];
}

template <typename PT, typename VT>
__global__ void k_set_batch_out(ProdDev<PT, VT> *prods, const int64_t *base,
                                const int64_t *cp, int nprod, int32_t *Cj, VT *Cx,
                                int64_t *Cp) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < nprod) {
    const int64_t o = cp[base[p]];
    prods[p].Cj = Cj + o;
    prods[p].Cx = Cx + o;
    prods[p].Cp = Cp + base[p] + p;
    prods[p].cp_bits = 64;
  }
}

// Operands of one product for the batched flop-count pass (either offset width).
struct CountDesc {
  const void *Ap;
  const int32_t *Aj;
  const void *Bp;
  int64_t n;
  int a64, b64;
};

// Flop count and output upper bound of every product of a batch in one launch:
// one thread per row of the flat row space (rows of a product are contiguous,
// so the products of a warp's 32 rows are non-decreasing over its lanes), a
// segmented inclusive warp sum per product and one 64-bit atomic per segment.
// out[2p] = sum of products, out[2p + 1] = sum over rows of min(products, ncols).
__global__ void k_count_batch(const CountDesc *d, const int64_t *base, int nprod, int64_t R,
                              unsigned long long *out) {
  const int lane = threadIdx.x & 31;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t w0 = int64_t(blockIdx.x) * blockDim.x + threadIdx.x - lane; w0 < R; w0 += stride) {
    const int64_t g = w0 + lane;
    int p = -1;
    long long mu = 0, up = 0;
    if (g < R) {
      p = find_prod(base, nprod, g);
      const int64_t r = g - base[p];
      const CountDesc c = d[p];
      const int64_t a0 = c.a64 ? ((const int64_t *)c.Ap)[r] : ((const int32_t *)c.Ap)[r];
      const int64_t a1 = c.a64 ? ((const int64_t *)c.Ap)[r + 1] : ((const int32_t *)c.Ap)[r + 1];
      for (int64_t q = a0; q < a1; ++q) {
        const int32_t k = __ldg(c.Aj + q);
        mu += c.b64 ? ((const int64_t *)c.Bp)[k + 1] - ((const int64_t *)c.Bp)[k]
                    : ((const int32_t *)c.Bp)[k + 1] - ((const int32_t *)c.Bp)[k];
      }
      up = mu < c.n ? mu : c.n;
    }
    for (int o = 1; o < 32; o <<= 1) {
      const long long m2 = __shfl_up_sync(0xffffffffu, mu, o);
      const long long u2 = __shfl_up_sync(0xffffffffu, up, o);
      const int p2 = __shfl_up_sync(0xffffffffu, p, o);
      if (lane >= o && p2 == p) {
        mu += m2;
        up += u2;
      }
    }
    const int pn = __shfl_down_sync(0xffffffffu, p, 1);
    if (p >= 0 && (lane == 31 || pn != p)) {
      atomicAdd(out + 2 * p, (unsigned long long)mu);
      atomicAdd(out + 2 * p + 1, (unsigned long long)up);
    }
  }
}

}  // namespace tspg

using namespace tspg;

struct tspg_batch {
  tspg_ctx *ctx = nullptr;
  std::vector<tspg_csr> A, B;
  int pt_bits = 0, vt_bits = 0;
  // host copies of the layout
  std::vector<int64_t> base, bbase;
  std::vector<int64_t> c_off;  // nprod + 1 output offsets
  int64_t R = 0, RB = 0, total_nnz = 0, max_a_row = 0;
  // device state (pool-backed, grow-only)
  void *prods = nullptr;
  size_t prods_bytes = 0;
  int64_t *d_base = nullptr, *d_bbase = nullptr, *rowf = nullptr, *cp = nullptr,
          *partial = nullptr, *offs = nullptr;
  int32_t *rowc = nullptr;
  uint64_t *list = nullptr;
  Sched *sched = nullptr;
  Tune tune{};  // row binning the graphs were captured with
  int32_t *curbuf = nullptr;
  int64_t cur_stride = 0;
  int32_t *Cj = nullptr;
  void *Cx = nullptr;
  int64_t *Cp = nullptr;
  int64_t *wide = nullptr;  // int32 row offsets widened when the batch runs as int64
  int64_t cap_wide = 0, cap_cp = 0;
  int64_t cap_rows = 0, cap_nnz = 0, cap_cur = 0, cap_prod = 0;
  int64_t *h_offs = nullptr;  // pinned, cap_prod + 1
  size_t h_offs_cap = 0;
  int64_t *h_cnt = nullptr;  // pinned, 2 per product (tspg_batch_count)
  size_t h_cnt_cap = 0;
  cudaGraphExec_t g1 = nullptr, g2 = nullptr;
  // graphs are captured and launched on a batch-private stream (capture is
  // not allowed on the legacy default stream); events join it to the caller's
  cudaStream_t own = nullptr;
  cudaEvent_t join_in = nullptr, join_out = nullptr;
  int g1_kernels = 0, g2_kernels = 0;
  cudaStream_t gstream = nullptr;
  bool dirty = true;

  void drop_graphs() {
    if (g1) cudaGraphExecDestroy(g1);
    if (g2) cudaGraphExecDestroy(g2);
    g1 = g2 = nullptr;
  }
  void free_dev(cudaStream_t s) {
    void *ps[] = {prods, d_base, d_bbase, rowf, cp, partial, offs, rowc, list, sched,
                  curbuf, Cj, Cx, Cp, wide};
    for (void *p : ps) ws_free(ctx, p, s);
    prods = nullptr;
    d_base = d_bbase = rowf = cp = partial = offs = nullptr;
    rowc = nullptr;
    list = nullptr;
    sched = nullptr;
    curbuf = nullptr;
    Cj = nullptr;
    Cx = nullptr;
    Cp = nullptr;
    wide = nullptr;
    cap_rows = cap_nnz = cap_cur = cap_prod = cap_wide = cap_cp = 0;
    prods_bytes = 0;
  }
};

namespace tspg {

template <typename T>
static int regrow(tspg_ctx *ctx, T **p, int64_t count, cudaStream_t s) {
  ws_free(ctx, *p, s);
  *p = nullptr;
  void *q = nullptr;
  TSPG_TRY(ws_alloc(ctx, &q, size_t(count > 0 ? count : 1) * sizeof(T), s));
  *p = (T *)q;
  return TSPG_OK;
}

template <typename PT, typename VT>
static int batch_run_impl(tspg_batch *b, cudaStream_t s, int flags);

// Join the caller's stream to the batch stream, run, and join back.
template <typename PT, typename VT>
static int batch_run_joined(tspg_batch *b, cudaStream_t caller, int flags) {
  tspg_ctx *ctx = b->ctx;
  if (!b->own) {
    TSPG_CUDA(ctx, cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking));
    TSPG_CUDA(ctx, cudaEventCreateWithFlags(&b->join_in, cudaEventDisableTiming));
    TSPG_CUDA(ctx, cudaEventCreateWithFlags(&b->join_out, cudaEventDisableTiming));
  }
  TSPG_CUDA(ctx, cudaEventRecord(b->join_in, caller));
  TSPG_CUDA(ctx, cudaStreamWaitEvent(b->own, b->join_in, 0));
  const int st = batch_run_impl<PT, VT>(b, b->own, flags);
  TSPG_CUDA(ctx, cudaEventRecord(b->join_out, b->own));
  TSPG_CUDA(ctx, cudaStreamWaitEvent(caller, b->join_out, 0));
  return st;
}

template <typename PT, typename VT>
static int batch_run_impl(tspg_batch *b, cudaStream_t s, int flags) {
  tspg_ctx *ctx = b->ctx;
  const int nprod = (int)b->A.size();
  TSPG_CUDA(ctx, cudaFuncSetAttribute(k_phase<PT, VT, false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, kDynSmem));
  TSPG_CUDA(ctx, cudaFuncSetAttribute(k_phase<PT, VT, true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, kDynSmem));
  TSPG_CUDA(ctx, cudaFuncSetAttribute(k_dense_rank<PT, VT>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, kDynSmem));
  TSPG_CUDA(ctx, cudaFuncSetAttribute(k_groups<PT, VT, false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, kGroupDynSmem));
  TSPG_CUDA(ctx, cudaFuncSetAttribute(k_groups<PT, VT, true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, kGroupDynSmem));
  // the cluster form must be launchable before it is captured (k_phase leaves
  // its rows alone)
  if (ctx->tune.cluster && cluster_slots<PT, VT>(ctx->device, ctx->tune.cluster) <= 0)
    return TSPG_EINVAL;
  // the graphs hold the row binning of their capture: a new tuning re-captures
  const bool retune = std::memcmp(&b->tune, &ctx->tune, sizeof(Tune)) != 0;
  const bool rebuild = b->dirty || !b->g1 || b->gstream != s || retune;
  b->tune = ctx->tune;
  if (rebuild) {
    b->drop_graphs();
    // layout
    b->base.assign(nprod + 1, 0);
    b->bbase.assign(nprod + 1, 0);
    for (int p = 0; p < nprod; ++p) {
      b->base[p + 1] = b->base[p] + b->A[p].nrows;
      b->bbase[p + 1] = b->bbase[p] + b->B[p].nrows;
    }
    b->R = b->base[nprod];
    b->RB = b->bbase[nprod];
    if (b->R > b->cap_rows || nprod > b->cap_prod) {
      const int64_t R = b->R > b->cap_rows ? b->R : b->cap_rows;
      TSPG_TRY(regrow(ctx, &b->rowf, R, s));
      TSPG_TRY(regrow(ctx, &b->rowc, R, s));
      TSPG_TRY(regrow(ctx, &b->cp, R + 1, s));
      TSPG_TRY(regrow(ctx, &b->list, R, s));
      TSPG_TRY(regrow(ctx, &b->partial, (R + kScanTile - 1) / kScanTile + 1, s));
      b->cap_rows = R;
    }
    if (nprod > b->cap_prod) {
      TSPG_TRY(regrow(ctx, (ProdDev<PT, VT> **)&b->prods, nprod, s));
      TSPG_TRY(regrow(ctx, &b->d_base, nprod + 1, s));
      TSPG_TRY(regrow(ctx, &b->d_bbase, nprod + 1, s));
      TSPG_TRY(regrow(ctx, &b->offs, nprod + 1, s));
      TSPG_TRY(regrow(ctx, &b->sched, 2, s));
      b->cap_prod = nprod;
    }
    if (size_t(nprod + 1) > b->h_offs_cap) {
      if (b->h_offs) cudaFreeHost(b->h_offs);
      b->h_offs = nullptr;
      TSPG_CUDA(ctx, cudaMallocHost((void **)&b->h_offs, sizeof(int64_t) * (nprod + 4)));
      b->h_offs_cap = nprod + 1;
    }
    // operands with int32 offsets in an int64 batch are widened first
    int64_t nwide = 0;
    if (sizeof(PT) == 8)
      for (int p = 0; p < nprod; ++p) {
        if (b->A[p].rowptr_bits == 32) nwide += b->A[p].nrows + 1;
        if (b->B[p].rowptr_bits == 32) nwide += b->B[p].nrows + 1;
      }
    if (nwide > b->cap_wide) {
      TSPG_TRY(regrow(ctx, &b->wide, nwide, s));
      b->cap_wide = nwide;
    }
    std::vector<const void *> arow(nprod), brow(nprod);
    int64_t wo = 0;
    for (int p = 0; p < nprod; ++p) {
      const tspg_csr *M[2] = {&b->A[p], &b->B[p]};
      const void **dst[2] = {&arow[p], &brow[p]};
      for (int t = 0; t < 2; ++t) {
        *dst[t] = M[t]->rowptr;
        if (sizeof(PT) == 8 && M[t]->rowptr_bits == 32) {
          const int64_t n = M[t]->nrows + 1;
          k_widen<<<(unsigned)((n + 255) / 256), 256, 0, s>>>((const int32_t *)M[t]->rowptr, n,
                                                              b->wide + wo);
          ctx->launches += 1;
          *dst[t] = b->wide + wo;
          wo += n;
        }
      }
    }
    std::vector<ProdDev<PT, VT>> hp(nprod);
    for (int p = 0; p < nprod; ++p) {
      ProdDev<PT, VT> v{};
      v.Ap = (const PT *)arow[p];
      v.Aj = b->A[p].col;
      v.Ax = (const VT *)b->A[p].val;
      v.Bp = (const PT *)brow[p];
      v.Bj = b->B[p].col;
      v.Bx = (const VT *)b->B[p].val;
      v.m = b->A[p].nrows;
      v.n = b->B[p].ncols;
      v.cp_bits = 64;
      v.b_sorted = 1;
      hp[p] = v;
    }
    // descriptor upload (pageable source: staged before the call returns)
    TSPG_CUDA(ctx, cudaMemcpyAsync(b->prods, hp.data(), sizeof(ProdDev<PT, VT>) * nprod,
                                   cudaMemcpyHostToDevice, s));
    TSPG_CUDA(ctx, cudaMemcpyAsync(b->d_base, b->base.data(), sizeof(int64_t) * (nprod + 1),
                                   cudaMemcpyHostToDevice, s));
    TSPG_CUDA(ctx, cudaMemcpyAsync(b->d_bbase, b->bbase.data(), sizeof(int64_t) * (nprod + 1),
                                   cudaMemcpyHostToDevice, s));
    TSPG_CUDA(ctx, cudaStreamSynchronize(s));
  }
  ProdDev<PT, VT> *prods = (ProdDev<PT, VT> *)b->prods;
  const int64_t R = b->R;
  const int64_t nb = (R + kScanTile - 1) / kScanTile;
  int64_t *errw = ctx->d_words + kErrWord;

  // ---- graph 1: symbolic
  if (rebuild) {
    cudaGraph_t g;
    TSPG_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(b->sched, 0, 2 * sizeof(Sched), s);
    k_set_tune<<<1, 32, 0, s>>>(b->sched, 2, ctx->tune);
    cudaMemsetAsync(b->rowc, 0, sizeof(int32_t) * (R > 0 ? R : 1), s);
    cudaMemsetAsync(b->cp, 0, sizeof(int64_t), s);
    if (!(flags & TSPG_F_B_SORTED) && b->RB > 0)
      k_check_sorted_batch<PT, VT><<<(unsigned)std::min<int64_t>((b->RB * 32 + 255) / 256,
                                                                 int64_t(ctx->num_sms) * 16),
                                     256, 0, s>>>(prods, b->d_bbase, nprod, b->RB);
    if (R > 0) {
      k_row_mults<PT, VT><<<(unsigned)std::min<int64_t>((R * 32 + 255) / 256,
                                                        int64_t(ctx->num_sms) * 16),
                            256, 0, s>>>(prods, b->d_base, nprod, R, b->rowf, b->sched);
      k_sched_offsets<<<1, 32, 0, s>>>(b->sched);
      k_scatter<PT, VT, 0><<<(unsigned)((R + 255) / 256), 256, 0, s>>>(
          prods, b->d_base, nprod, R, b->rowf, b->rowc, b->cp, b->sched, b->list);
      PhaseArgs pa{b->d_base, b->sched, b->list, b->rowf, b->rowc, b->cp, nullptr, 0, errw,
                   ctx->d_prof};
      phase_mark(ctx, 0, 0, s);
      k_phase<PT, VT, false><<<ctx->num_sms, kSymThreads, kDynSmem, s>>>(prods, pa);
      k_groups<PT, VT, false><<<ctx->num_sms, kGroupThreads, kGroupDynSmem, s>>>(prods, pa);
      phase_mark(ctx, 0, 1, s);
      k_scan_reduce<<<(unsigned)nb, kScanThreads, 0, s>>>(b->rowc, R, b->partial);
      k_scan_partials<<<1, 1024, 0, s>>>(b->partial, nb);
      k_scan_final<<<(unsigned)nb, kScanThreads, 0, s>>>(b->rowc, R, b->partial, nb, b->cp,
                                                         b->sched + 1, b->rowf);
    }
    k_gather_offsets<<<(nprod + 256) / 256, 256, 0, s>>>(b->cp, b->d_base, nprod, b->offs);
    b->g1_kernels = 2 + (!(flags & TSPG_F_B_SORTED) && b->RB > 0) + (R > 0 ? 8 : 0);
    cudaMemcpyAsync(b->h_offs, b->offs, sizeof(int64_t) * (nprod + 1), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(b->h_offs + nprod + 1, &b->sched[0].max_a_row, sizeof(int64_t),
                    cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(b->h_offs + nprod + 2, errw, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (e != cudaSuccess) {
      ctx->last_cuda = (int)e;
      return TSPG_ECUDA;
    }
    e = cudaGraphInstantiate(&b->g1, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      ctx->last_cuda = (int)e;
      return TSPG_ECUDA;
    }
    b->gstream = s;
  }
  TSPG_CUDA(ctx, cudaGraphLaunch(b->g1, s));
  ctx->launches += b->g1_kernels;
  TSPG_CUDA(ctx, cudaStreamSynchronize(s));
  if (b->h_offs[nprod + 2] != 0) {
    cudaMemsetAsync(errw, 0, sizeof(int64_t), s);
    return TSPG_ECUDA;
  }
  b->c_off.assign(b->h_offs, b->h_offs + nprod + 1);
  b->total_nnz = b->c_off[nprod];
  b->max_a_row = b->h_offs[nprod + 1];

  // ---- output slab and graph 2: numeric
  bool regraph = rebuild;
  if (b->total_nnz > b->cap_nnz || !b->Cj) {
    // grows by at least half its size, so a batch reused for larger and
    // larger admissions (a server lane) maps new memory only a few times
    const int64_t want = b->total_nnz > 0 ? b->total_nnz : 1;
    const int64_t nnz = b->Cj && want < b->cap_nnz + b->cap_nnz / 2 ? b->cap_nnz + b->cap_nnz / 2 : want;
    TSPG_TRY(regrow(ctx, &b->Cj, nnz, s));
    TSPG_TRY(regrow(ctx, (VT **)&b->Cx, nnz, s));
    b->cap_nnz = nnz;
    regraph = true;
  }
  if (R + nprod > b->cap_cp || !b->Cp) {  // one row-offset array per product
    TSPG_TRY(regrow(ctx, &b->Cp, R + nprod, s));
    b->cap_cp = R + nprod;
    regraph = true;
  }
  if (b->max_a_row > kDenseCurSmem && b->max_a_row > b->cap_cur) {
    TSPG_TRY(regrow(ctx, &b->curbuf, 2 * int64_t(ctx->num_sms) * b->max_a_row, s));
    b->cap_cur = b->max_a_row;
    b->cur_stride = b->max_a_row;
    regraph = true;
  }
  if (regraph || !b->g2) {
    if (b->g2) cudaGraphExecDestroy(b->g2);
    b->g2 = nullptr;
    cudaGraph_t g;
    TSPG_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    k_set_batch_out<PT, VT><<<(nprod + 255) / 256, 256, 0, s>>>(prods, b->d_base, b->cp, nprod,
                                                                b->Cj, (VT *)b->Cx, b->Cp);
    if (R > 0) {
      k_sched_offsets<<<1, 32, 0, s>>>(b->sched + 1);
      k_scatter<PT, VT, 1><<<(unsigned)((R + 255) / 256), 256, 0, s>>>(
          prods, b->d_base, nprod, R, b->rowf, b->rowc, b->cp, b->sched + 1, b->list);
      PhaseArgs pa{b->d_base, b->sched + 1, b->list, b->rowf, b->rowc, b->cp,
                   b->curbuf, b->cur_stride, errw, ctx->d_prof ? ctx->d_prof + kProfPerPhase : nullptr};
      phase_mark(ctx, 1, 0, s);
      launch_dense_cluster<PT, VT>(ctx, s, prods, pa);  // launchable: checked above
      k_dense_rank<PT, VT><<<ctx->num_sms, kRankThreads, kDynSmem, s>>>(prods, pa);
      k_phase<PT, VT, true><<<ctx->num_sms, kThreads, kDynSmem, s>>>(prods, pa);
      k_groups<PT, VT, true><<<ctx->num_sms, kGroupThreads, kGroupDynSmem, s>>>(prods, pa);
      phase_mark(ctx, 1, 1, s);
    }
    k_zero_rowptr<PT, VT><<<(nprod + 31) / 32, 32, 0, s>>>(prods, nprod);
    b->g2_kernels = 2 + (R > 0 ? 5 + (ctx->tune.cluster ? 1 : 0) : 0);
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (e != cudaSuccess) {
      ctx->last_cuda = (int)e;
      return TSPG_ECUDA;
    }
    e = cudaGraphInstantiate(&b->g2, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      ctx->last_cuda = (int)e;
      return TSPG_ECUDA;
    }
  }
  TSPG_CUDA(ctx, cudaGraphLaunch(b->g2, s));
  ctx->launches += b->g2_kernels;
  b->dirty = false;
  return TSPG_OK;
}

}  // namespace tspg

extern "C" int tspg_batch_create(tspg_ctx *ctx, tspg_batch **out) {
  if (!ctx || !out) return TSPG_EINVAL;
  tspg_batch *b = new (std::nothrow) tspg_batch();
  if (!b) return TSPG_ENOMEM;
  b->ctx = ctx;
  *out = b;
  return TSPG_OK;
}

extern "C" int tspg_batch_destroy(tspg_batch *b) {
  if (!b) return TSPG_EINVAL;
  cudaSetDevice(b->ctx->device);
  cudaDeviceSynchronize();
  b->drop_graphs();
  b->free_dev(nullptr);
  if (b->h_offs) cudaFreeHost(b->h_offs);
  if (b->h_cnt) cudaFreeHost(b->h_cnt);
  if (b->join_in) cudaEventDestroy(b->join_in);
  if (b->join_out) cudaEventDestroy(b->join_out);
  if (b->own) cudaStreamDestroy(b->own);
  delete b;
  return TSPG_OK;
}

extern "C" int tspg_batch_clear(tspg_batch *b) {
  if (!b) return TSPG_EINVAL;
  b->A.clear();
  b->B.clear();
  b->pt_bits = b->vt_bits = 0;
  b->dirty = true;
  return TSPG_OK;
}

extern "C" int tspg_batch_add(tspg_batch *b, const tspg_csr *A, const tspg_csr *B,
                              int *index_out) {
  if (!b) return TSPG_EINVAL;
  TSPG_TRY(check_csr(A));
  TSPG_TRY(check_csr(B));
  if (A->ncols != B->nrows || A->val_bits != B->val_bits) return TSPG_EINVAL;
  if (!b->A.empty() && A->val_bits != b->vt_bits) return TSPG_EINVAL;
  if (b->A.size() >= (size_t(1) << 23) || A->nrows >= (int64_t(1) << 40)) return TSPG_EINVAL;
  // the batch runs with int64 offsets as soon as any operand has them
  if (b->A.empty()) b->pt_bits = 32;
  if (A->rowptr_bits == 64 || B->rowptr_bits == 64) b->pt_bits = 64;
  b->vt_bits = A->val_bits;
  if (index_out) *index_out = (int)b->A.size();
  b->A.push_back(*A);
  b->B.push_back(*B);
  b->dirty = true;
  return TSPG_OK;
}

extern "C" int tspg_batch_run(tspg_batch *b, void *stream, int flags, int64_t *total_nnz) {
  if (!b) return TSPG_EINVAL;
  if (b->A.empty()) {
    if (total_nnz) *total_nnz = 0;
    return TSPG_OK;
  }
  TSPG_CUDA(b->ctx, cudaSetDevice(b->ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  int st;
  if (b->pt_bits == 32 && b->vt_bits == 64) st = batch_run_joined<int32_t, double>(b, s, flags);
  else if (b->pt_bits == 64 && b->vt_bits == 64) st = batch_run_joined<int64_t, double>(b, s, flags);
  else if (b->pt_bits == 32) st = batch_run_joined<int32_t, float>(b, s, flags);
  else st = batch_run_joined<int64_t, float>(b, s, flags);
  if (st == TSPG_OK && total_nnz) *total_nnz = b->total_nnz;
  return st;
}

extern "C" int tspg_batch_count(tspg_batch *b, void *stream, int64_t *mults,
                                int64_t *c_nnz_upper) {
  if (!b) return TSPG_EINVAL;
  const int nprod = (int)b->A.size();
  if (nprod == 0) return TSPG_OK;
  if (!mults || !c_nnz_upper) return TSPG_EINVAL;
  tspg_ctx *ctx = b->ctx;
  TSPG_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<CountDesc> hd(nprod);
  std::vector<int64_t> base(nprod + 1, 0);
  for (int p = 0; p < nprod; ++p) {
    hd[p] = CountDesc{b->A[p].rowptr, b->A[p].col, b->B[p].rowptr, b->B[p].ncols,
                      b->A[p].rowptr_bits == 64, b->B[p].rowptr_bits == 64};
    base[p + 1] = base[p] + b->A[p].nrows;
  }
  const int64_t R = base[nprod];
  if (size_t(2 * nprod) > b->h_cnt_cap) {
    if (b->h_cnt) cudaFreeHost(b->h_cnt);
    b->h_cnt = nullptr;
    b->h_cnt_cap = 0;
    TSPG_CUDA(ctx, cudaMallocHost((void **)&b->h_cnt, sizeof(int64_t) * 2 * nprod));
    b->h_cnt_cap = 2 * nprod;
  }
  Scratch sc(ctx, s);
  CountDesc *dd;
  int64_t *dbase;
  unsigned long long *dout;
  TSPG_TRY(sc.get(&dd, nprod));
  TSPG_TRY(sc.get(&dbase, nprod + 1));
  TSPG_TRY(sc.get(&dout, 2 * nprod));
  // pageable sources: staged before the calls return
  TSPG_CUDA(ctx, cudaMemcpyAsync(dd, hd.data(), sizeof(CountDesc) * nprod, cudaMemcpyHostToDevice, s));
  TSPG_CUDA(ctx, cudaMemcpyAsync(dbase, base.data(), sizeof(int64_t) * (nprod + 1),
                                 cudaMemcpyHostToDevice, s));
  TSPG_CUDA(ctx, cudaMemsetAsync(dout, 0, sizeof(int64_t) * 2 * nprod, s));
  if (R > 0) {
    k_count_batch<<<(unsigned)std::min<int64_t>((R + 255) / 256, int64_t(ctx->num_sms) * 8), 256, 0,
                    s>>>(dd, dbase, nprod, R, dout);
    ctx->launches += 1;
    TSPG_CUDA(ctx, cudaGetLastError());
  }
  TSPG_CUDA(ctx, cudaMemcpyAsync(b->h_cnt, dout, sizeof(int64_t) * 2 * nprod, cudaMemcpyDeviceToHost, s));
  TSPG_CUDA(ctx, cudaStreamSynchronize(s));
  for (int p = 0; p < nprod; ++p) {
    mults[p] = b->h_cnt[2 * p];
    c_nnz_upper[p] = b->h_cnt[2 * p + 1];
  }
  return TSPG_OK;
}

extern "C" int tspg_batch_result(const tspg_batch *b, int i, tspg_csr *out) {
  if (!b || !out || i < 0 || size_t(i) >= b->A.size() || b->dirty ||
      b->c_off.size() != b->A.size() + 1)
    return TSPG_EINVAL;
  const int64_t o = b->c_off[i];
  out->nrows = b->A[i].nrows;
  out->ncols = b->B[i].ncols;
  out->nnz = b->c_off[i + 1] - o;
  out->rowptr = b->Cp + b->base[i] + i;
  out->rowptr_bits = 64;
  out->val_bits = b->vt_bits;
  out->col = b->Cj + o;
  out->val = (char *)b->Cx + o * (b->vt_bits / 8);
  return TSPG_OK;
}
