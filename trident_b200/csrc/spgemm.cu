// spgemm.cu — host side of the two-phase SpGEMM (C = A·B, C = C_in + A·B).
//
// Call sequence of one product on the caller's stream:
//   k_set_prod, [k_check_sorted_rows], k_row_mults, k_sched_offsets,
//   k_scatter<sym>, k_phase + k_groups <symbolic>, k_scan_reduce / k_scan_partials /
//   k_scan_final, one 2-word device->host read + stream sync (nnz(C), longest
//   A row), then k_set_out, k_sched_offsets, k_scatter<num>, k_phase + k_groups <numeric>.
// KokkosSparse::spgemm (include/KokkosWrap.hpp:375) and the cuSPARSE paths
// (include/cusparse_helpers.cuh:908-1344) do the same job with library-owned
// allocation and ~10 stream syncs per call.
#include <algorithm>
#include <new>

#include "spgemm_cluster.cuh"

namespace tspg {

// The dynamic shared-memory limit is a per-device attribute of a kernel: it
// is raised once per device (the caller has made ctx->device current), so a
// process that drives several GPUs sets it on each of them.
template <typename PT, typename VT>
static int set_smem_attr(int device) {
  constexpr int kMaxDev = 64;
  static bool done[kMaxDev] = {};  // per device and instantiation; benign if raced
  const bool cached = device >= 0 && device < kMaxDev;
  if (!cached || !done[device]) {
    cudaError_t e1 = cudaFuncSetAttribute(k_phase<PT, VT, false>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          kDynSmem);
    cudaError_t e2 = cudaFuncSetAttribute(k_phase<PT, VT, true>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          kDynSmem);
    cudaError_t e3 = cudaFuncSetAttribute(k_groups<PT, VT, false>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          kGroupDynSmem);
    cudaError_t e4 = cudaFuncSetAttribute(k_groups<PT, VT, true>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          kGroupDynSmem);
    cudaError_t e5 = cudaFuncSetAttribute(k_onepass<PT, VT>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          kGroupDynSmem);
    cudaError_t e6 = cudaFuncSetAttribute(k_dense_rank<PT, VT>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          kDynSmem);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess || e4 != cudaSuccess ||
        e5 != cudaSuccess || e6 != cudaSuccess)
      return TSPG_ECUDA;
    if (cached) done[device] = true;
  }
  return TSPG_OK;
}

}  // namespace tspg

using namespace tspg;

struct tspg_plan {
  tspg_ctx *ctx = nullptr;
  cudaStream_t stream = nullptr;
  int pt_bits = 32, vt_bits = 64;
  int64_t m = 0, k = 0, n = 0;
  int64_t a_nnz = 0, b_nnz = 0;
  int64_t c_nnz = 0;
  int64_t mults = 0;
  int64_t max_a_row = 0;
  void *prods = nullptr;
  int64_t *base = nullptr;
  int64_t *rowf = nullptr;
  int32_t *rowc = nullptr;
  int64_t *cp = nullptr;
  uint64_t *list = nullptr;
  Sched *sched = nullptr;  // [0] symbolic, [1] numeric, [2] deferred one-pass rows
  int64_t *partial = nullptr;
  int64_t nb = 0;
  int32_t *curbuf = nullptr;
  int64_t cur_stride = 0;
  int64_t *wide_a = nullptr, *wide_b = nullptr;  // widened row offsets (mixed widths)
  tspg_csr E{};        // addend of C = E + A·B (tspg_spgemm_acc), E.col == nullptr if none
  int64_t onepass = 0;  // entries of the one-pass rows' scratch (0: none)
  int32_t *oj = nullptr;
  void *ox = nullptr;
  uint64_t *defer = nullptr;
  void *blocks[16];
  int nblocks = 0;

  template <typename T>
  int get(T **p, size_t count) {
    void *q = nullptr;
    size_t bytes = count * sizeof(T);
    if (bytes == 0) bytes = 16;
    if (nblocks == int(sizeof(blocks) / sizeof(blocks[0]))) return TSPG_ENOMEM;
    int st = ws_alloc(ctx, &q, bytes, stream);
    if (st != TSPG_OK) return st;
    blocks[nblocks++] = q;
    *p = (T *)q;
    return TSPG_OK;
  }
  ~tspg_plan() {
    for (int i = nblocks - 1; i >= 0; --i) ws_free(ctx, blocks[i], stream);
  }
};

namespace tspg {

// Internal flag of the one-shot product (tspg_spgemm): warp rows may be
// multiplied whole in the symbolic launch (one-pass rows).  A plan that is
// kept for numeric calls with new values cannot use it.
constexpr int kFlagOnePass = 1 << 30;
// ... and only on products of at least this many rows (it adds a scan and a
// host round trip before the symbolic launch), with a scratch of at most
// this many entries.
constexpr int64_t kOnePassMinRows = 1 << 16;
constexpr int64_t kOnePassMaxEntries = int64_t(1) << 30;

static inline unsigned grid_for(int64_t work, int per_block, int cap) {
  int64_t g = (work + per_block - 1) / per_block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (unsigned)g;
}

template <typename PT, typename VT>
static int symbolic_impl(tspg_ctx *ctx, cudaStream_t s, const tspg_csr *A,
                         const tspg_csr *B, int flags, tspg_plan *P) {
  TSPG_TRY(set_smem_attr<PT, VT>(ctx->device));
  const int64_t m = A->nrows, n = B->ncols, k = A->ncols;
  P->m = m;
  P->n = n;
  P->k = k;
  P->a_nnz = A->nnz;
  P->b_nnz = B->nnz;
  P->nb = (m + kScanTile - 1) / kScanTile;
  ProdDev<PT, VT> *prods;
  TSPG_TRY(P->get(&prods, 1));
  P->prods = prods;
  TSPG_TRY(P->get(&P->base, 2));
  TSPG_TRY(P->get(&P->rowf, m));
  TSPG_TRY(P->get(&P->rowc, m));
  TSPG_TRY(P->get(&P->cp, m + 1));
  TSPG_TRY(P->get(&P->list, m));
  TSPG_TRY(P->get(&P->sched, 3));
  TSPG_TRY(P->get(&P->partial, P->nb + 1));
  bool onepass = (flags & kFlagOnePass) && !(P->E.col && P->E.nnz > 0) && m >= kOnePassMinRows;
  TSPG_CUDA(ctx, cudaMemsetAsync(P->sched, 0, 3 * sizeof(Sched), s));
  k_set_tune<<<1, 32, 0, s>>>(P->sched, 3, ctx->tune, onepass ? 1 : 0);
  TSPG_CUDA(ctx, cudaMemsetAsync(P->rowc, 0, (m > 0 ? m : 1) * sizeof(int32_t), s));
  TSPG_CUDA(ctx, cudaMemsetAsync(P->cp, 0, sizeof(int64_t), s));

  ProdDev<PT, VT> v{};
  v.Ap = (const PT *)A->rowptr;
  v.Aj = A->col;
  v.Ax = (const VT *)A->val;
  v.Bp = (const PT *)B->rowptr;
  v.Bj = B->col;
  v.Bx = (const VT *)B->val;
  v.m = m;
  v.n = n;
  v.cp_bits = 64;
  v.b_sorted = 1;
  if (P->E.col && P->E.nnz > 0) {
    v.Ep = P->E.rowptr;
    v.Ej = P->E.col;
    v.Ex = (const VT *)P->E.val;
    v.ep_bits = P->E.rowptr_bits;
  }
  k_set_prod<PT, VT><<<1, 1, 0, s>>>(prods, v, P->base, m);
  if (!(flags & TSPG_F_B_SORTED) && B->nnz > 0 && B->nrows > 0) {
    k_check_sorted_rows<PT><<<grid_for(B->nrows * 32, 256, ctx->num_sms * 16), 256,
                              0, s>>>(v.Bp, v.Bj, B->nrows, &prods->b_sorted);
  }
  int extra = 0;
  if (m > 0) {
    k_row_mults<PT, VT><<<grid_for(m * 32, 256, ctx->num_sms * 16), 256, 0, s>>>(
        prods, P->base, 1, m, P->rowf, P->sched, onepass ? P->rowc : nullptr);
    if (onepass) {
      // the one-pass rows' scratch offsets: a scan of their output bounds
      k_scan_reduce<<<(unsigned)P->nb, kScanThreads, 0, s>>>(P->rowc, m, P->partial);
      k_scan_partials<<<1, 1024, 0, s>>>(P->partial, P->nb);
      k_scan_final<<<(unsigned)P->nb, kScanThreads, 0, s>>>(P->rowc, m, P->partial, P->nb,
                                                            P->cp, P->sched + 1, nullptr);
      extra += 3;
      int64_t *h = ctx->h_words;
      TSPG_CUDA(ctx, cudaMemcpyAsync(h, P->cp + m, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
      TSPG_CUDA(ctx, cudaMemcpyAsync(h + 1, &P->sched[0].cnt[CLS_ONEPASS], sizeof(int64_t),
                                     cudaMemcpyDeviceToHost, s));
      TSPG_CUDA(ctx, cudaStreamSynchronize(s));
      const int64_t tot = h[0], rows = h[1];
      // one pass when most rows take it (R-MAT 20: a tenth of the rows, and
      // those with more than 32 outputs need their second attempt: +0.9 ms
      // of symbolic phase; Galerkin A·P: every row, -0.9 ms per call)
      if (tot > 0 && 2 * rows >= m && tot <= kOnePassMaxEntries &&
          P->get(&P->oj, size_t(tot)) == TSPG_OK && P->get((VT **)&P->ox, size_t(tot)) == TSPG_OK &&
          P->get(&P->defer, size_t(rows)) == TSPG_OK) {
        P->onepass = tot;
      } else {  // every row two-pass: the one-pass rows back to their classes
        onepass = false;
        k_fold_onepass<<<1, 32, 0, s>>>(P->sched);
        TSPG_CUDA(ctx, cudaMemsetAsync(P->rowc, 0, m * sizeof(int32_t), s));
        extra += 1;
      }
    }
    k_sched_offsets<<<1, 32, 0, s>>>(P->sched);
    k_scatter<PT, VT, 0><<<grid_for(m, 256, INT32_MAX), 256, 0, s>>>(
        prods, P->base, 1, m, P->rowf, P->rowc, P->cp, P->sched, P->list);
    PhaseArgs pa{P->base, P->sched, P->list, P->rowf, P->rowc, P->cp,
                 nullptr, 0, ctx->d_words + kErrWord, ctx->d_prof};
    pa.oj = P->oj;
    pa.ox = P->ox;
    pa.defer = P->defer;
    phase_mark(ctx, 0, 0, s);
    k_phase<PT, VT, false><<<ctx->num_sms, kSymThreads, kDynSmem, s>>>(prods, pa);
    k_groups<PT, VT, false><<<ctx->num_sms, kGroupThreads, kGroupDynSmem, s>>>(prods, pa);
    if (onepass) {
      k_onepass<PT, VT><<<ctx->num_sms, kGroupThreads, kGroupDynSmem, s>>>(prods, pa);
      // the rows sent back (too many columns for their 64-slot attempt and
      // too large for a warp's full table): their symbolic count, as
      // 256-thread rows of their own record
      Sched *D = P->sched + 2;
      k_defer_setup<<<1, 32, 0, s>>>(P->sched, D);
      k_sched_offsets<<<1, 32, 0, s>>>(D);
      PhaseArgs pd = pa;
      pd.S = D;
      pd.list = P->defer;
      k_groups<PT, VT, false><<<ctx->num_sms, kGroupThreads, kGroupDynSmem, s>>>(prods, pd);
      extra += 4;
    }
    phase_mark(ctx, 0, 1, s);
    k_scan_reduce<<<(unsigned)P->nb, kScanThreads, 0, s>>>(P->rowc, m, P->partial);
    k_scan_partials<<<1, 1024, 0, s>>>(P->partial, P->nb);
    k_scan_final<<<(unsigned)P->nb, kScanThreads, 0, s>>>(P->rowc, m, P->partial,
                                                          P->nb, P->cp, P->sched + 1, P->rowf);
  }
  TSPG_CUDA(ctx, cudaGetLastError());
  ctx->launches += 2 + (!(flags & TSPG_F_B_SORTED) && B->nnz > 0 && B->nrows > 0) + (m > 0 ? 8 : 0) +
                   extra;
  int64_t *h = ctx->h_words;
  TSPG_CUDA(ctx, cudaMemcpyAsync(h, P->cp + m, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  TSPG_CUDA(ctx, cudaMemcpyAsync(h + 1, &P->sched[0].total, 4 * sizeof(int64_t),
                                 cudaMemcpyDeviceToHost, s));
  TSPG_CUDA(ctx, cudaMemcpyAsync(h + 5, ctx->d_words + kErrWord, sizeof(int64_t),
                                 cudaMemcpyDeviceToHost, s));
  TSPG_CUDA(ctx, cudaStreamSynchronize(s));
  P->c_nnz = h[0];
  P->mults = h[1];
  P->max_a_row = h[3];
  if (h[5] != 0) {
    cudaMemsetAsync(ctx->d_words + kErrWord, 0, sizeof(int64_t), s);
    return TSPG_ECUDA;
  }
  return TSPG_OK;
}

template <typename PT, typename VT>
static int numeric_impl(tspg_ctx *ctx, cudaStream_t s, tspg_plan *P,
                        tspg_csr_out *C) {
  const int64_t m = P->m;
  ProdDev<PT, VT> *prods = (ProdDev<PT, VT> *)P->prods;
  k_set_out<PT, VT><<<1, 1, 0, s>>>(prods, C->col, (VT *)C->val, C->rowptr,
                                    C->rowptr_bits);
  if (m == 0) {
    k_zero_rowptr<PT, VT><<<1, 32, 0, s>>>(prods, 1);
    ctx->launches += 2;
    TSPG_CUDA(ctx, cudaGetLastError());
    return TSPG_OK;
  }
  if (P->max_a_row > kDenseCurSmem && !P->curbuf) {
    P->cur_stride = P->max_a_row;
    TSPG_TRY(P->get(&P->curbuf, 2 * size_t(ctx->num_sms) * P->cur_stride));
  }
  k_sched_offsets<<<1, 32, 0, s>>>(P->sched + 1);
  k_scatter<PT, VT, 1><<<grid_for(m, 256, INT32_MAX), 256, 0, s>>>(
      prods, P->base, 1, m, P->rowf, P->rowc, P->cp, P->sched + 1, P->list);
  PhaseArgs pa{P->base, P->sched + 1, P->list, P->rowf, P->rowc, P->cp,
               P->curbuf, P->cur_stride, ctx->d_words + kErrWord,
               ctx->d_prof ? ctx->d_prof + kProfPerPhase : nullptr};
  phase_mark(ctx, 1, 0, s);
  TSPG_CUDA(ctx, launch_dense_cluster<PT, VT>(ctx, s, prods, pa));
  k_dense_rank<PT, VT><<<ctx->num_sms, kRankThreads, kDynSmem, s>>>(prods, pa);
  k_phase<PT, VT, true><<<ctx->num_sms, kThreads, kDynSmem, s>>>(prods, pa);
  k_groups<PT, VT, true><<<ctx->num_sms, kGroupThreads, kGroupDynSmem, s>>>(prods, pa);
  if (P->onepass)
    k_onepass_copy<PT, VT><<<grid_for(m * 32, 256, ctx->num_sms * 16), 256, 0, s>>>(
        prods, P->rowf, P->rowc, P->cp, P->oj, (const VT *)P->ox, m);
  phase_mark(ctx, 1, 1, s);
  ctx->launches += 6 + (P->onepass ? 1 : 0);
  TSPG_CUDA(ctx, cudaGetLastError());
  return TSPG_OK;
}

// Output capacity: use the caller's buffers, grow through its allocator, or
// report the needed size (CsxBuffers::ensure_async semantics).
static int ensure_out(tspg_csr_out *C, int64_t nnz, int vbytes, cudaStream_t s) {
  C->nnz = nnz;
  if (C->capacity >= nnz) return TSPG_OK;
  if (!C->alloc) return TSPG_ENOMEM;
  void *cj = C->alloc(C->alloc_user, size_t(nnz) * 4, s);
  void *cx = C->alloc(C->alloc_user, size_t(nnz) * vbytes, s);
  if (!cj || !cx) return TSPG_ENOMEM;
  C->col = (int32_t *)cj;
  C->val = cx;
  C->capacity = nnz;
  return TSPG_OK;
}

static int check_pair(const tspg_csr *A, const tspg_csr *B) {
  TSPG_TRY(check_csr(A));
  TSPG_TRY(check_csr(B));
  if (A->ncols != B->nrows) return TSPG_EINVAL;
  if (A->val_bits != B->val_bits) return TSPG_EINVAL;
  return TSPG_OK;
}

static int check_out(const tspg_csr_out *C, int64_t m, int64_t n, int vbits) {
  if (!C || !C->rowptr) return TSPG_EINVAL;
  if (C->nrows != m || C->ncols != n) return TSPG_EINVAL;
  if (C->rowptr_bits != 32 && C->rowptr_bits != 64) return TSPG_EINVAL;
  if (C->val_bits != vbits) return TSPG_EINVAL;
  return TSPG_OK;
}

template <typename F>
static int dispatch(int pt_bits, int vt_bits, F &&f) {
  if (pt_bits == 32 && vt_bits == 64) return f((int32_t *)0, (double *)0);
  if (pt_bits == 64 && vt_bits == 64) return f((int64_t *)0, (double *)0);
  if (pt_bits == 32 && vt_bits == 32) return f((int32_t *)0, (float *)0);
  if (pt_bits == 64 && vt_bits == 32) return f((int64_t *)0, (float *)0);
  return TSPG_EINVAL;
}

}  // namespace tspg

extern "C" int tspg_plan_destroy(tspg_plan *plan) {
  if (!plan) return TSPG_EINVAL;
  cudaSetDevice(plan->ctx->device);
  delete plan;
  return TSPG_OK;
}

static int plan_get(tspg_ctx *, void *plan, int64_t **p, int64_t n) {
  return ((tspg_plan *)plan)->get(p, size_t(n));
}

// Symbolic phase of A·B, or of E + A·B when E is given (its entries join
// their rows as products with coefficient 1).
static int symbolic_entry(tspg_ctx *ctx, void *stream, const tspg_csr *A_in,
                          const tspg_csr *B_in, const tspg_csr *E, int flags,
                          tspg_plan **plan, int64_t *c_nnz) {
  if (!ctx || !plan) return TSPG_EINVAL;
  *plan = nullptr;
  TSPG_TRY(check_pair(A_in, B_in));
  cudaStream_t s = (cudaStream_t)stream;
  TSPG_CUDA(ctx, cudaSetDevice(ctx->device));
  tspg_plan *P = new (std::nothrow) tspg_plan();
  if (!P) return TSPG_ENOMEM;
  P->ctx = ctx;
  P->stream = s;
  if (E) P->E = *E;
  tspg_csr a = *A_in, b = *B_in;
  const tspg_csr *A = &a, *B = &b;
  if (a.rowptr_bits != b.rowptr_bits) {
    tspg_csr *M = a.rowptr_bits == 32 ? &a : &b;
    int64_t **buf = M == &a ? &P->wide_a : &P->wide_b;
    int st = P->get(buf, size_t(M->nrows + 1));
    if (st != TSPG_OK) {
      delete P;
      return st;
    }
    k_widen<<<(unsigned)((M->nrows + 1 + 255) / 256), 256, 0, s>>>((const int32_t *)M->rowptr,
                                                                    M->nrows + 1, *buf);
    ctx->launches += 1;
    M->rowptr = *buf;
    M->rowptr_bits = 64;
  }
  P->pt_bits = A->rowptr_bits;
  P->vt_bits = A->val_bits;
  int st = dispatch(P->pt_bits, P->vt_bits, [&](auto pt, auto vt) {
    using PT = std::remove_pointer_t<decltype(pt)>;
    using VT = std::remove_pointer_t<decltype(vt)>;
    return symbolic_impl<PT, VT>(ctx, s, A, B, flags, P);
  });
  if (st != TSPG_OK) {
    delete P;
    return st;
  }
  if (c_nnz) *c_nnz = P->c_nnz;
  *plan = P;
  return TSPG_OK;
}

extern "C" int tspg_spgemm_symbolic(tspg_ctx *ctx, void *stream,
                                    const tspg_csr *A_in, const tspg_csr *B_in,
                                    int flags, tspg_plan **plan,
                                    int64_t *c_nnz) {
  return symbolic_entry(ctx, stream, A_in, B_in, nullptr, flags, plan, c_nnz);
}

extern "C" int tspg_spgemm_numeric(tspg_ctx *ctx, void *stream,
                                   tspg_plan *plan, const tspg_csr *A_in,
                                   const tspg_csr *B_in, tspg_csr_out *C) {
  if (!ctx || !plan) return TSPG_EINVAL;
  TSPG_TRY(check_pair(A_in, B_in));
  tspg_csr a = *A_in, b = *B_in;
  const tspg_csr *A = &a, *B = &b;
  if (a.rowptr_bits != b.rowptr_bits) {
    tspg_csr *M = a.rowptr_bits == 32 ? &a : &b;
    int64_t *buf = M == &a ? plan->wide_a : plan->wide_b;
    if (!buf) return TSPG_EINVAL;  // the symbolic call had matching widths
    k_widen<<<(unsigned)((M->nrows + 1 + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        (const int32_t *)M->rowptr, M->nrows + 1, buf);
    ctx->launches += 1;
    M->rowptr = buf;
    M->rowptr_bits = 64;
  }
  if (A->nrows != plan->m || B->ncols != plan->n || A->nnz != plan->a_nnz ||
      B->nnz != plan->b_nnz || A->rowptr_bits != plan->pt_bits ||
      A->val_bits != plan->vt_bits)
    return TSPG_EINVAL;
  TSPG_TRY(check_out(C, plan->m, plan->n, plan->vt_bits));
  if (C->rowptr_bits == 32 && plan->c_nnz > INT32_MAX) return TSPG_EOVERFLOW;
  cudaStream_t s = (cudaStream_t)stream;
  TSPG_CUDA(ctx, cudaSetDevice(ctx->device));
  TSPG_TRY(ensure_out(C, plan->c_nnz, plan->vt_bits / 8, s));
  // the plan's prods descriptor points at the symbolic call's operands; the
  // numeric call may pass new value arrays of the same pattern
  return dispatch(plan->pt_bits, plan->vt_bits, [&](auto pt, auto vt) {
    using PT = std::remove_pointer_t<decltype(pt)>;
    using VT = std::remove_pointer_t<decltype(vt)>;
    ProdDev<PT, VT> v{};
    v.Ap = (const PT *)A->rowptr;
    v.Aj = A->col;
    v.Ax = (const VT *)A->val;
    v.Bp = (const PT *)B->rowptr;
    v.Bj = B->col;
    v.Bx = (const VT *)B->val;
    v.m = A->nrows;
    v.n = B->ncols;
    v.cp_bits = 64;
    ProdDev<PT, VT> *prods = (ProdDev<PT, VT> *)plan->prods;
    k_set_operands<PT, VT><<<1, 1, 0, s>>>(prods, v);
    ctx->launches += 1;
    return numeric_impl<PT, VT>(ctx, s, plan, C);
  });
}

extern "C" int tspg_spgemm(tspg_ctx *ctx, void *stream, const tspg_csr *A,
                           const tspg_csr *B, tspg_csr_out *C, int flags) {
  if (!ctx) return TSPG_EINVAL;
  TSPG_TRY(check_pair(A, B));
  TSPG_TRY(check_out(C, A->nrows, B->ncols, A->val_bits));
  tspg_plan *plan = nullptr;
  int64_t nnz = 0;
  TSPG_TRY(symbolic_entry(ctx, stream, A, B, nullptr, (flags & ~kFlagOnePass) | kFlagOnePass, &plan,
                          &nnz));
  int st = TSPG_OK;
  if (C->rowptr_bits == 32 && nnz > INT32_MAX) st = TSPG_EOVERFLOW;
  if (st == TSPG_OK) st = ensure_out(C, nnz, A->val_bits / 8, (cudaStream_t)stream);
  if (st == TSPG_OK) {
    st = dispatch(plan->pt_bits, plan->vt_bits, [&](auto pt, auto vt) {
      using PT = std::remove_pointer_t<decltype(pt)>;
      using VT = std::remove_pointer_t<decltype(vt)>;
      return numeric_impl<PT, VT>(ctx, (cudaStream_t)stream, plan, C);
    });
  }
  tspg_plan_destroy(plan);
  return st;
}

extern "C" int tspg_spgemm_count(tspg_ctx *ctx, void *stream,
                                 const tspg_csr *A, const tspg_csr *B,
                                 int64_t *mults, int64_t *c_nnz_upper) {
  if (!ctx) return TSPG_EINVAL;
  TSPG_TRY(check_pair(A, B));
  cudaStream_t s = (cudaStream_t)stream;
  TSPG_CUDA(ctx, cudaSetDevice(ctx->device));
  Scratch sc(ctx, s);
  tspg_csr a = *A, b = *B;
  if (a.rowptr_bits != b.rowptr_bits) {
    tspg_csr *M = a.rowptr_bits == 32 ? &a : &b;
    int64_t *buf;
    TSPG_TRY(sc.get(&buf, M->nrows + 1));
    k_widen<<<(unsigned)((M->nrows + 1 + 255) / 256), 256, 0, s>>>((const int32_t *)M->rowptr,
                                                                    M->nrows + 1, buf);
    ctx->launches += 1;
    M->rowptr = buf;
    M->rowptr_bits = 64;
  }
  A = &a;
  B = &b;
  return dispatch(A->rowptr_bits, A->val_bits, [&](auto pt, auto vt) -> int {
    using PT = std::remove_pointer_t<decltype(pt)>;
    using VT = std::remove_pointer_t<decltype(vt)>;
    const int64_t m = A->nrows;
    ProdDev<PT, VT> *prods;
    int64_t *base, *rowf;
    Sched *sched;
    TSPG_TRY(sc.get(&prods, 1));
    TSPG_TRY(sc.get(&base, 2));
    TSPG_TRY(sc.get(&rowf, m));
    TSPG_TRY(sc.get(&sched, 1));
    TSPG_CUDA(ctx, cudaMemsetAsync(sched, 0, sizeof(Sched), s));
    k_set_tune<<<1, 32, 0, s>>>(sched, 1, ctx->tune);
    ProdDev<PT, VT> v{};
    v.Ap = (const PT *)A->rowptr;
    v.Aj = A->col;
    v.Bp = (const PT *)B->rowptr;
    v.m = m;
    v.n = B->ncols;
    k_set_prod<PT, VT><<<1, 1, 0, s>>>(prods, v, base, m);
    if (m > 0)
      k_row_mults<PT, VT><<<grid_for(m * 32, 256, ctx->num_sms * 16), 256, 0, s>>>(
          prods, base, 1, m, rowf, sched);
    ctx->launches += 2 + (m > 0);
    TSPG_CUDA(ctx, cudaGetLastError());
    int64_t *h = ctx->h_words;
    TSPG_CUDA(ctx, cudaMemcpyAsync(h, &sched->total, 2 * sizeof(int64_t),
                                   cudaMemcpyDeviceToHost, s));
    TSPG_CUDA(ctx, cudaStreamSynchronize(s));
    if (mults) *mults = h[0];
    if (c_nnz_upper) *c_nnz_upper = h[1];
    return TSPG_OK;
  });
}

namespace tspg {

// Flop count of A·B fused with the SUMMA stage mask: one warp per row of A;
// entry (i, k) adds nnz(B row k) to the row's products and, when that row of B
// is non-empty, sets bit k of the word mask.  Bit k ends up set exactly when
// column k of A holds an entry and row k of B is non-empty, i.e. the AND of
// the column mask of A and the row mask of B.
template <typename APT, typename BPT>
__global__ void k_count_mask(const APT *Ap, const int32_t *Aj, const BPT *Bp, int64_t m,
                             int64_t n, uint32_t *mask, unsigned long long *tot) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  unsigned long long wm = 0, wu = 0;
  for (int64_t r = warp; r < m; r += nwarps) {
    const int64_t a0 = int64_t(Ap[r]), a1 = int64_t(Ap[r + 1]);
    int64_t sum = 0;
    for (int64_t q = a0 + lane; q < a1; q += 32) {
      const int32_t k = __ldg(Aj + q);
      const int64_t len = int64_t(Bp[k + 1]) - int64_t(Bp[k]);
      sum += len;
      if (len > 0) {
        const uint32_t bit = 1u << (k & 31);
        if (!(*(volatile uint32_t *)(mask + (k >> 5)) & bit)) atomicOr(mask + (k >> 5), bit);
      }
    }
    sum = warp_sum(sum);
    wm += (unsigned long long)sum;
    wu += (unsigned long long)(sum < n ? sum : n);
  }
  if (lane == 0 && (wm | wu)) {
    atomicAdd(tot, wm);
    atomicAdd(tot + 1, wu);
  }
}

// Word mask -> LSB-first byte mask: byte i holds bits k = 8i .. 8i + 7.
__global__ void k_mask_bytes(const uint32_t *w, int64_t nbytes, uint8_t *out) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < nbytes) out[i] = uint8_t(w[i >> 2] >> ((i & 3) * 8));
}

template <typename APT, typename BPT>
static void launch_count_mask(tspg_ctx *ctx, cudaStream_t s, const tspg_csr *A, const tspg_csr *B,
                              uint32_t *words, unsigned long long *tot) {
  k_count_mask<APT, BPT><<<grid_for(A->nrows * 32, 256, ctx->num_sms * 16), 256, 0, s>>>(
      (const APT *)A->rowptr, A->col, (const BPT *)B->rowptr, A->nrows, B->ncols, words, tot);
}

}  // namespace tspg

extern "C" int tspg_spgemm_count_mask(tspg_ctx *ctx, void *stream, const tspg_csr *A,
                                      const tspg_csr *B, uint8_t *mask, int64_t *mults,
                                      int64_t *c_nnz_upper) {
  if (!ctx) return TSPG_EINVAL;
  TSPG_TRY(check_pair(A, B));
  const int64_t kdim = A->ncols, nbytes = (kdim + 7) / 8;
  if (nbytes > 0 && !mask) return TSPG_EINVAL;
  cudaStream_t s = (cudaStream_t)stream;
  TSPG_CUDA(ctx, cudaSetDevice(ctx->device));
  Scratch sc(ctx, s);
  uint32_t *words;
  unsigned long long *tot;
  TSPG_TRY(sc.get(&words, (kdim + 31) / 32));
  TSPG_TRY(sc.get(&tot, 2));
  TSPG_CUDA(ctx, cudaMemsetAsync(words, 0, sizeof(uint32_t) * ((kdim + 31) / 32 > 0 ? (kdim + 31) / 32 : 1), s));
  TSPG_CUDA(ctx, cudaMemsetAsync(tot, 0, 2 * sizeof(unsigned long long), s));
  if (A->nrows > 0) {
    if (A->rowptr_bits == 32 && B->rowptr_bits == 32) launch_count_mask<int32_t, int32_t>(ctx, s, A, B, words, tot);
    else if (A->rowptr_bits == 32) launch_count_mask<int32_t, int64_t>(ctx, s, A, B, words, tot);
    else if (B->rowptr_bits == 32) launch_count_mask<int64_t, int32_t>(ctx, s, A, B, words, tot);
    else launch_count_mask<int64_t, int64_t>(ctx, s, A, B, words, tot);
    ctx->launches += 1;
  }
  if (nbytes > 0) {
    k_mask_bytes<<<(unsigned)((nbytes + 255) / 256), 256, 0, s>>>(words, nbytes, mask);
    ctx->launches += 1;
  }
  TSPG_CUDA(ctx, cudaGetLastError());
  int64_t *h = ctx->h_words;
  TSPG_CUDA(ctx, cudaMemcpyAsync(h, tot, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  TSPG_CUDA(ctx, cudaStreamSynchronize(s));
  if (mults) *mults = h[0];
  if (c_nnz_upper) *c_nnz_upper = h[1];
  return TSPG_OK;
}

// C_out = C_in + A·B: the product goes to pool workspace, then the union merge
// writes C_out (sp_mma_hybrid, include/cusparse_helpers.cuh:708-739, does the
// same with KokkosKernels + csrgeam2).
extern "C" int tspg_spgemm_acc(tspg_ctx *ctx, void *stream, const tspg_csr *A,
                               const tspg_csr *B, const tspg_csr *C_in,
                               tspg_csr_out *C_out, int flags) {
  if (!ctx) return TSPG_EINVAL;
  TSPG_TRY(check_pair(A, B));
  const bool have_in = C_in && C_in->nnz > 0;
  const int pflags = flags & TSPG_F_B_SORTED;
  if (!have_in) return tspg_spgemm(ctx, stream, A, B, C_out, pflags);
  TSPG_TRY(check_csr(C_in));
  if (C_in->nrows != A->nrows || C_in->ncols != B->ncols ||
      C_in->val_bits != A->val_bits)
    return TSPG_EINVAL;
  TSPG_TRY(check_out(C_out, A->nrows, B->ncols, A->val_bits));
  const bool fuse = (flags & TSPG_F_ACC_FUSE) ||
                    (!(flags & TSPG_F_ACC_SPLIT) && C_in->nnz <= A->nnz + B->nnz);
  if (fuse) {
    // one SpGEMM in which C_in's entries join their rows as products with
    // coefficient 1
    tspg_plan *plan = nullptr;
    TSPG_TRY(symbolic_entry(ctx, stream, A, B, C_in, pflags, &plan, nullptr));
    const int st = tspg_spgemm_numeric(ctx, stream, plan, A, B, C_out);
    tspg_plan_destroy(plan);
    return st;
  }
  // the product into workspace, then the merge into C_out
  cudaStream_t s = (cudaStream_t)stream;
  tspg_plan *plan = nullptr;
  int64_t nnz = 0;
  TSPG_TRY(tspg_spgemm_symbolic(ctx, stream, A, B, pflags, &plan, &nnz));
  const int vb = A->val_bits / 8;
  const int pb = nnz > INT32_MAX ? 64 : C_in->rowptr_bits;
  void *rp = nullptr, *cj = nullptr, *cx = nullptr;
  int st = ws_alloc(ctx, &rp, size_t(A->nrows + 1) * (pb / 8), s);
  if (st == TSPG_OK) st = ws_alloc(ctx, &cj, size_t(nnz > 0 ? nnz : 1) * 4, s);
  if (st == TSPG_OK) st = ws_alloc(ctx, &cx, size_t(nnz > 0 ? nnz : 1) * vb, s);
  tspg_csr_out T{};
  if (st == TSPG_OK) {
    T.nrows = A->nrows;
    T.ncols = B->ncols;
    T.rowptr = rp;
    T.rowptr_bits = pb;
    T.val_bits = A->val_bits;
    T.col = (int32_t *)cj;
    T.val = cx;
    T.capacity = nnz;
    st = tspg_spgemm_numeric(ctx, stream, plan, A, B, &T);
  }
  tspg_plan_destroy(plan);
  if (st == TSPG_OK) {
    tspg_csr prod{T.nrows, T.ncols, T.nnz, T.rowptr, T.rowptr_bits, T.val_bits,
                  T.col, T.val};
    st = tspg_spadd(ctx, stream, &prod, C_in, C_out);
  }
  ws_free(ctx, cx, s);
  ws_free(ctx, cj, s);
  ws_free(ctx, rp, s);
  return st;
}
