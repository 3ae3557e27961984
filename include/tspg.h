/*
 * tspg.h — C ABI of the B200 (sm_100a) on-node SpGEMM path for Trident.
 *
 * The library replaces the three library-backed pieces of Trident's per-stage
 * local compute:
 *   - the local tile SpGEMM  C = A·B  and the accumulate form  C = C + A·B
 *     (KokkosSparse::spgemm in include/KokkosWrap.hpp:331,375, and the
 *      cusparseSpGEMM* paths in include/cusparse_helpers.cuh:908-1344);
 *   - the merge of partial C tiles  C = A + B  with the union pattern
 *     (KokkosSparse::spadd_* in include/KokkosWrap.hpp:343-349,420-425 and
 *      cusparseScsrgeam2* in include/cusparse_helpers.cuh:799-905);
 *   - the bitmask tile pack / unpack of the sparsity-aware exchange
 *     (SpaComm::gen_bitmask, intersect_bitmasks, select_entries_cuda,
 *      select_ptrs and SpaCommHandler::Compress in include/spacomm.cuh:29-148,
 *      556-623, 808-889, 962-1091).
 *
 * Conventions
 *   - All matrix pointers are DEVICE pointers, 0-based CSR (or CSC where a
 *     function says so).  Column indices are int32.  Row offsets are int32 or
 *     int64 (rowptr_bits 32|64).  Values are FP64 (val_bits 64, the graded
 *     path) or FP32 (val_bits 32, the twin that the unchanged <int32_t,float>
 *     Trident drivers link against).
 *   - Every call is stream-ordered on the caller's stream (a cudaStream_t
 *     passed as void*; NULL is the legacy default stream).  Calls that must
 *     return a size to the host synchronise that stream and say so.
 *   - A context owns its workspace pool; it is not thread-safe.  Use one
 *     context per host thread (Trident's main and accumulation threads each
 *     get their own).  There is no global mutable state.
 *   - Functions return a TSPG_* status; nothing in the library exits.
 *   - Output rows of SpGEMM, SpGEMM-accumulate and spadd are sorted by column
 *     with no duplicate columns.  Structural zeros are kept (an entry whose
 *     value cancels to 0.0 stays in the pattern), matching KokkosKernels and
 *     csrgeam2 as Trident uses them.  spadd requires sorted, duplicate-free
 *     rows; the C_in operand of tspg_spgemm_acc may have either.
 */
#ifndef TSPG_H
#define TSPG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TSPG_ABI_VERSION 1

/* Status codes. */
enum {
  TSPG_OK = 0,
  TSPG_EINVAL = 1,     /* bad argument (null pointer, bad bits, shape mismatch) */
  TSPG_ENOMEM = 2,     /* workspace beyond the context budget, or an output
                          buffer too small and no allocator given (the needed
                          size is still reported) */
  TSPG_EOVERFLOW = 3,  /* int32 row offsets requested but nnz > INT32_MAX */
  TSPG_ETIMEOUT = 4,   /* a bounded device wait gave up */
  TSPG_ECUDA = 5,      /* a CUDA runtime call failed (see tspg_last_cuda_error) */
  TSPG_EUNSORTED = 6,  /* an operand that must have sorted rows does not */
  TSPG_ESCRATCH = 7    /* larger than the static scratch of tspg_pack_noalloc */
};

/* Major dimension of a compressed sparse matrix (mmio::MajorDim). */
enum { TSPG_ROWS = 0, TSPG_COLS = 1 };

/* Flags for the SpGEMM entry points. */
enum {
  TSPG_F_NONE = 0,
  /* Skip the device check that B's rows are sorted; the caller promises they
     are.  Without it the library checks and, for unsorted B, uses the
     cursor-free form of the long-row kernel. */
  TSPG_F_B_SORTED = 1,
  /* tspg_spgemm_acc: force one SpGEMM with C_in's entries as products
     (ACC_FUSE) or a product followed by the merge (ACC_SPLIT).  Default: fuse
     when nnz(C_in) <= nnz(A) + nnz(B) — a large accumulator merges faster
     (sequential) than it re-enters the hash / bitmap passes. */
  TSPG_F_ACC_FUSE = 2,
  TSPG_F_ACC_SPLIT = 4
};

/* Read-only sparse operand (CSR; for the pack, the compressed dimension is
   given separately). */
typedef struct tspg_csr {
  int64_t nrows;
  int64_t ncols;
  int64_t nnz;
  const void *rowptr;  /* (major dim + 1) offsets, int32 or int64 */
  int32_t rowptr_bits; /* 32 | 64 */
  int32_t val_bits;    /* 32 | 64 */
  const int32_t *col;  /* nnz column (or row, for CSC) indices */
  const void *val;     /* nnz values */
} tspg_csr;

/* Device allocator callback: returns a device pointer of at least `bytes`
   bytes usable on `stream`, or NULL.  The library never frees it. */
typedef void *(*tspg_alloc_fn)(void *user, size_t bytes, void *stream);

/* Sparse result.  The caller provides rowptr (nrows+1 entries of
   rowptr_bits).  col/val either point to `capacity` entries each, or are
   allocated through `alloc` when capacity < nnz (mirrors
   CsxBuffers::ensure_async in include/utils.cuh:685-728).  On return nnz holds
   the result size, also when the call fails with TSPG_ENOMEM because the
   capacity was short and alloc is NULL. */
typedef struct tspg_csr_out {
  int64_t nrows;
  int64_t ncols;
  int64_t nnz;      /* out */
  void *rowptr;
  int32_t rowptr_bits;
  int32_t val_bits;
  int32_t *col;
  void *val;
  int64_t capacity; /* entries available in col and val */
  tspg_alloc_fn alloc;
  void *alloc_user;
} tspg_csr_out;

typedef struct tspg_ctx tspg_ctx;
typedef struct tspg_plan tspg_plan;

/* ---- library and context -------------------------------------------------
 * Replaces: the cusparseHandle_t + CsxBuffers temp buffers + setup_mempool
 * (include/mempool.cuh:9-22) that every Trident rank holds.  The context owns
 * a cudaMemPool with release threshold UINT64_MAX, so workspace stays
 * resident between calls; `pool_budget` bytes (0 = no limit) caps what the
 * library itself may hold. */
int tspg_abi_version(void);
const char *tspg_strerror(int status);
int tspg_last_cuda_error(const tspg_ctx *ctx);
int tspg_ctx_create(int device, size_t pool_budget, tspg_ctx **out);
int tspg_ctx_destroy(tspg_ctx *ctx);
/* Bytes of workspace the context holds now / at most so far. */
int tspg_ctx_mem(const tspg_ctx *ctx, size_t *in_use, size_t *high_water);
/* Instrumentation.  tspg_ctx_stats: library kernels launched through this
 * context so far (kernels inside replayed CUDA graphs included).
 * tspg_ctx_phase_timing: when enabled, every SpGEMM call records CUDA events
 * on its stream around its persistent symbolic and numeric kernels;
 * tspg_ctx_phase_ms waits for and returns those two durations of the last
 * call (the NVTX / CUDA_TIMER_* role of the reference, src/hns_spgemm.cu
 * :755-1042). */
int tspg_ctx_stats(const tspg_ctx *ctx, int64_t *launches);
int tspg_ctx_phase_timing(tspg_ctx *ctx, int enable);
int tspg_ctx_phase_ms(tspg_ctx *ctx, float *symbolic_ms, float *numeric_ms);
/* Row binning of the SpGEMM (no counterpart in the reference, whose binning
 * lives inside KokkosKernels / cuSPARSE): rows go to warp / 128-thread /
 * 256-thread / CTA groups by the upper bounds sym_lim[] (symbolic phase, on
 * min(products, ncols)) and num_lim[] (numeric phase, on the row's nnz); rows
 * above the last bound are DENSE rows.  hash_load = hash-table slots per key
 * (2, 4 or 8).  Bounds must be positive, non-decreasing and at most the table
 * capacities sym <= {512, 2048, 4096, 24576}, num <= {256, 1024, 2048, 8192}
 * (the defaults); otherwise TSPG_EINVAL.  dense_win_log2: numeric DENSE
 * rows with at least 2^dense_win_log2 products, an output filling at least
 * 1/2^dense_win_fill_log2 of the columns and sorted B rows take the
 * column-window form (a shared-memory FP64 accumulator per window of
 * columns, written to C once) instead of the whole-row rank form;
 * dense_win_log2 = 0 (the default: on R-MAT 20 A·A the form took 450 ms per
 * numeric phase against 261 ms for the rank form) turns it off, otherwise
 * 10..40;
 * dense_win_fill_log2 0..12 (default 4).  dense_win_cluster: 0 (default) —
 * one CTA per such row; 2, 4 or 8 — a thread-block cluster of that many CTAs
 * per row, the window spread over their shared memories (distributed shared
 * memory) so it spans that many times the columns.  Applies to calls made
 * after it; results do not depend on it. */
typedef struct tspg_tuning {
  int32_t sym_lim[4];
  int32_t num_lim[4];
  int32_t hash_load;
  int32_t dense_win_log2;
  int32_t dense_win_fill_log2;
  int32_t dense_win_cluster;
} tspg_tuning;
int tspg_ctx_set_tuning(tspg_ctx *ctx, const tspg_tuning *t);
int tspg_ctx_get_tuning(const tspg_ctx *ctx, tspg_tuning *t);

/* Per-class accounting of the persistent phases (off by default): SM cycles
 * and rows per row class, accumulated over calls since enabling.  out64 =
 * symbolic[32], numeric[32]; each half holds cycles x 8, rows x 8 (classes
 * DENSE0 (>= 2^20 products), DENSE1 (>= 2^17), DENSE2, G1024, G256, G128,
 * G32, then the one-pass warp rows, counted in the symbolic half), then
 * sub-phase cycles: [16..20] the whole-row DENSE rows' bitmap pass, block
 * scan, zero fill, column emission and value pass; [21..24] the windowed
 * DENSE rows' set-up, short-entry walks, long-entry walks and emission;
 * [25..29] the group rows' set-up, products, compaction, sort and write
 * (symbolic: set-up, products, count).  Reading synchronises the device. */
int tspg_ctx_class_profile(tspg_ctx *ctx, int enable);
int tspg_ctx_class_cycles(tspg_ctx *ctx, uint64_t *out64);

/* ---- SpGEMM ----------------------------------------------------------------
 * tspg_spgemm_count — the flop-count pass.  mults = sum over A's nonzeros
 * (i,k) of nnz(B row k) (cusparseSpGEMM_getNumProducts,
 * include/cusparse_helpers.cuh:981-985,1251-1257); c_nnz_upper =
 * sum_i min(mults_i, ncols(B)), the admission bound on nnz(C).  Synchronises
 * `stream`. */
int tspg_spgemm_count(tspg_ctx *ctx, void *stream, const tspg_csr *A,
                      const tspg_csr *B, int64_t *mults, int64_t *c_nnz_upper);

/* tspg_spgemm_count_mask — the flop-count pass fused with the stage mask of a
 * SUMMA step on one GPU (the single-GPU form of SpaComm::spcomm_2D,
 * include/spacomm.cuh:165-352): besides mults and c_nnz_upper it writes
 * mask[ceil(ncols(A) / 8)] (device, LSB-first bytes) with bit k set exactly
 * when column k of A holds an entry and row k of B is non-empty — the same
 * bytes as SpaComm::intersect_bitmasks(gen_bitmask(colptr(A)),
 * gen_bitmask(rowptr(B))) (spacomm.cuh:29-148), in one pass over A with no
 * CSC copy of A.  Synchronises `stream`. */
int tspg_spgemm_count_mask(tspg_ctx *ctx, void *stream, const tspg_csr *A,
                           const tspg_csr *B, uint8_t *mask, int64_t *mults,
                           int64_t *c_nnz_upper);

/* tspg_spgemm_row_products — products per row of A·B into the device int64
 * array out[nrows(A)]: out[i] = sum over A's entries (i, k) of nnz(B row k).
 * Stream-ordered.  Its prefix sum cuts A's rows into panels of equal work for
 * the row-panel split of one product over several GPUs (no reference
 * counterpart: the reference splits by tiles, src/hns_spgemm.cu). */
int tspg_spgemm_row_products(tspg_ctx *ctx, void *stream, const tspg_csr *A,
                             const tspg_csr *B, int64_t *out);

/* tspg_spgemm — C = A·B, two-phase inside (symbolic, then numeric).
 * Replaces LocalMatrix::spgemm (include/KokkosWrap.hpp:367-391) and
 * cusparse_spgemm / _reuse / _mem (include/cusparse_helpers.cuh:908-1344).
 * A's row offsets need not start at 0: a view of rows [r0, r1) of a larger
 * CSR (rowptr advanced by r0, col and val unchanged) is a valid A, which is
 * how a row panel of one product is computed on its own GPU.
 * Empty operands give an empty C with a zeroed rowptr (the num_prods == 0
 * exit, include/cusparse_helpers.cuh:1251-1257).  Synchronises `stream` once
 * (to learn nnz(C)); twice when A has at least 65,536 rows.  Such a product
 * whose rows are mostly short (or repeat their columns) computes those rows
 * whole in its first launch, into a workspace of 4 + val_bits / 8 bytes per
 * entry they may write (at most 32 per row, or the row's bound when smaller;
 * at most 2^30 entries) taken from the context's pool, and copies them into
 * C in the second; when the budget refuses that
 * workspace, or the product has few such rows, every row takes the two-pass
 * path.  Results are the same either way; a plan (tspg_spgemm_symbolic)
 * always takes the two-pass path, since its numeric calls may bring new
 * values. */
int tspg_spgemm(tspg_ctx *ctx, void *stream, const tspg_csr *A,
                const tspg_csr *B, tspg_csr_out *C, int flags);

/* Split form for structure reuse (cusparse_spgemm_reuse,
 * include/cusparse_helpers.cuh:1023-1189): the symbolic phase returns nnz(C)
 * and keeps the row structure in `plan`; numeric may then run any number of
 * times for operands with the same pattern and new values.  The plan borrows
 * nothing; destroy it with tspg_plan_destroy. */
int tspg_spgemm_symbolic(tspg_ctx *ctx, void *stream, const tspg_csr *A,
                         const tspg_csr *B, int flags, tspg_plan **plan,
                         int64_t *c_nnz);
int tspg_spgemm_numeric(tspg_ctx *ctx, void *stream, tspg_plan *plan,
                        const tspg_csr *A, const tspg_csr *B,
                        tspg_csr_out *C);
int tspg_plan_destroy(tspg_plan *plan);

/* tspg_spgemm_acc — C_out = C_in + A·B with the union pattern.  Replaces
 * LocalMatrix::sp_mma (include/KokkosWrap.hpp:315-364), sp_mma_hybrid
 * (include/cusparse_helpers.cuh:708-739) and cusparse_spmma
 * (include/cusparse_helpers.cuh:744-796).  C_in may be NULL or empty (the
 * "first product" case, KokkosWrap.hpp:334-338); then C_out = A·B.  Either
 * one SpGEMM in which C_in's entries join their rows as products with
 * coefficient 1, or the product followed by tspg_spadd (flags
 * TSPG_F_ACC_FUSE / TSPG_F_ACC_SPLIT; by default by size).  C_out's arrays
 * must not overlap C_in's. */
int tspg_spgemm_acc(tspg_ctx *ctx, void *stream, const tspg_csr *A,
                    const tspg_csr *B, const tspg_csr *C_in,
                    tspg_csr_out *C_out, int flags);

/* tspg_transpose — T = M^T with sorted rows (T is the CSC of M).  Replaces
 * cusparse_csc_to_csr (include/cusparse_helpers.cuh:607-705) and
 * LocalMatrix::csc_to_csr (include/KokkosWrap.hpp:442-531): a CSC tile
 * passed as the CSR of its transpose comes back as the CSR of the tile.
 * T->nrows = M->ncols, T->ncols = M->nrows; output capacity / allocator as
 * for SpGEMM.  Synchronises `stream` once. */
int tspg_transpose(tspg_ctx *ctx, void *stream, const tspg_csr *M,
                   tspg_csr_out *T);

/* tspg_coo_to_csx — device COO (int32 row and column indices, values) to a
 * compressed matrix: CSR for major = TSPG_ROWS (out: nrows x ncols), CSC for
 * TSPG_COLS (out: the CSR of the transpose, ncols x nrows).  Replaces the host
 * builders coo_to_row_csx / coo_to_col_csx(_contig) and coo_to_kokkos_crs /
 * _ccs (include/cusparse_helpers.cuh:17-131, include/kokkos_helpers.cuh:52-352),
 * which sort the triples on the host by the major index only and copy the
 * result to the device.  Same pointer array and the same multiset of entries
 * per segment, repeated entries kept; inside a segment entries come ordered
 * by minor index, then input position (the reference leaves that order to
 * std::sort).  Indices outside the shape: TSPG_EINVAL, nothing written.
 * Output capacity / allocator as for SpGEMM.  Synchronises `stream`. */
int tspg_coo_to_csx(tspg_ctx *ctx, void *stream, int64_t nrows, int64_t ncols,
                    int64_t nnz, const int32_t *row, const int32_t *col,
                    const void *val, int val_bits, int major,
                    tspg_csr_out *out);

/* ---- merge ------------------------------------------------------------------
 * tspg_spadd — C = A + B, union pattern, alpha = beta = 1.  Replaces
 * cusparse_spgeam (include/cusparse_helpers.cuh:799-905) and
 * LocalMatrix::spadd (include/KokkosWrap.hpp:394-439).  Rows of A and B must
 * be sorted and duplicate-free.  Synchronises `stream` once. */
int tspg_spadd(tspg_ctx *ctx, void *stream, const tspg_csr *A,
               const tspg_csr *B, tspg_csr_out *C);

/* ---- bitmask tile pack --------------------------------------------------------
 * tspg_bitmask_gen — mask byte w bit b (LSB first) is set iff segment 8w+b of
 * `ptr` is non-empty (ptr[i] != ptr[i+1]); n segments, ceil(n/8) bytes out.
 * Replaces SpaComm::gen_bitmask (include/spacomm.cuh:29-117) with
 * MASK_SIZE = 8, BMASK_TYPE = uint8_t (include/common.h:63-65). */
int tspg_bitmask_gen(tspg_ctx *ctx, void *stream, const void *ptr,
                     int ptr_bits, int64_t n, uint8_t *mask_out);

/* tspg_bitmask_and — out = a & b bytewise (SpaComm::intersect_bitmasks,
 * include/spacomm.cuh:126-148).  `out` may alias a or b. */
int tspg_bitmask_and(tspg_ctx *ctx, void *stream, const uint8_t *a,
                     const uint8_t *b, int64_t nbytes, uint8_t *out);

/* tspg_pack — SpaCommHandler::Compress (include/spacomm.cuh:962-1091) on one
 * tile: keep the entries of every segment (row for TSPG_ROWS, column for
 * TSPG_COLS) whose mask bit is set, in their original order; the pointer
 * array keeps its full length with masked segments made empty
 * (select_ptrs, include/spacomm.cuh:556-623).  Output wire layout in
 * `out_buf` (TileHolder::set_csx_ptrs, include/tile_holder.cuh:80-89):
 *     [ val[nnz_kept] | idx int32[nnz_kept] | ptr[len+1] ]
 * with val of M->val_bits and ptr of M->rowptr_bits.  `cap` must be at least
 * the unpacked tile's size, nnz*(val+4) + (len+1)*ptr bytes.  When
 * `nnz_kept_host` is non-NULL the call synchronises `stream` and stores the
 * kept count there; it is always also written to `nnz_kept_dev` when that is
 * non-NULL (device int64). */
int tspg_pack(tspg_ctx *ctx, void *stream, const tspg_csr *M, int major,
              const uint8_t *mask, void *out_buf, size_t cap,
              int64_t *nnz_kept_dev, int64_t *nnz_kept_host);

/* tspg_pack_noalloc — the same pack as tspg_pack for callers that cannot
 * allocate device memory, e.g. a communication thread that packs the next
 * tile while compute and transfers run on other streams, where the implicit
 * device synchronisation of cudaMalloc / cudaFree would stall that overlap.
 * No counterpart in the reference (its select_entries_cuda / select_ptrs
 * allocate per call).  Takes no context, allocates nothing and never
 * synchronises; the kept count is written to the device int64 *nnz_kept_dev
 * when non-NULL.  Scratch is one static device array in the library (about
 * 3 MiB per GPU, held until exit) sized for tiles of up to
 * TSPG_PACK_NOALLOC_MAX_SEGMENTS segments; larger tiles return
 * TSPG_ESCRATCH.  The first call on a device looks up that array's device
 * address (make it before any stream capture).  The device current on the
 * calling thread must own `stream` and the buffers; an output buffer on
 * another device returns TSPG_EINVAL.  All calls share the array: calls that
 * overlap on the GPU race and must be serialised by the caller. */
#define TSPG_PACK_NOALLOC_MAX_SEGMENTS 262144
int tspg_pack_noalloc(void *stream, const tspg_csr *M, int major,
                      const uint8_t *mask, void *out_buf, size_t cap,
                      int64_t *nnz_kept_dev);

/* tspg_select_ptrs — the pointer array of a packed tile, in place
 * (SpaComm::select_ptrs, include/spacomm.cuh:556-623): the counts of the
 * `len` segments whose mask bit is clear become 0 and ptr[1..len] becomes the
 * inclusive scan of the counts; the length stays len + 1.  Synchronises
 * `stream`; TSPG_EOVERFLOW when an int32 offset would pass INT32_MAX. */
int tspg_select_ptrs(tspg_ctx *ctx, void *stream, void *ptr, int ptr_bits,
                     int64_t len, const uint8_t *mask);

/* Row offsets <-> row counts, in place on nrows + 1 entries, around the
 * gather of B tiles (rowptrs_to_rownnz / rownnz_to_rowptrs,
 * include/utils.cuh:412-448, used at include/tile_holder.cuh:283-327).
 * tspg_rowptrs_to_rownnz: ptr[i] := ptr[i] - ptr[i-1] for i >= 1 (ptr[0]
 * kept); stream-ordered.  tspg_rownnz_to_rowptrs: ptr[1..nrows] := its
 * inclusive scan (ptr[0] kept); synchronises `stream` and returns
 * TSPG_EOVERFLOW when an int32 offset would pass INT32_MAX. */
int tspg_rowptrs_to_rownnz(tspg_ctx *ctx, void *stream, void *ptr, int ptr_bits,
                           int64_t nrows);
int tspg_rownnz_to_rowptrs(tspg_ctx *ctx, void *stream, void *ptr, int ptr_bits,
                           int64_t nrows);

/* Size in bytes of a packed tile (CSX_buf_size / compute_message_size,
 * src/hns_spgemm.cu:23-26). */
size_t tspg_packed_bytes(int64_t nnz, int64_t ptr_len, int val_bits,
                         int ptr_bits);

/* tspg_unpack — the receiver side: wrap a packed buffer as a CSX view
 * (TileHolder::form_mmiocsx, include/tile_holder.cuh:212-233).  Host-only
 * pointer arithmetic; the view borrows `buf`. */
int tspg_unpack(const void *buf, int64_t nrows, int64_t ncols, int major,
                int64_t nnz, int val_bits, int ptr_bits, tspg_csr *out);

/* ---- Markov clustering updates -----------------------------------------------------
 * The per-iteration matrix updates of the reference's MCL driver
 * (src/mcl.cu:56-149), which copies its tile to the host for each of them.
 * Row sums are over the rows of M alone (the reference then adds the partial
 * sums of a process row with MPI_Allreduce; on one GPU the tile holds whole
 * rows).
 * tspg_mcl_normalize: every row divided by its sum; a row whose sum is
 *   <= 1e-20 becomes zeros (normalize, mcl.cu:97-127).
 * tspg_mcl_inflate: every value raised to `power`, then normalized
 *   (inflation, mcl.cu:130-149).
 * Both write M's values (same pattern) to val_out, which may be M->val.
 * tspg_mcl_prune: the entries with |v| > tol, in their order, as a new CSR
 *   (prune, mcl.cu:56-93); output capacity / allocator as for SpGEMM;
 *   synchronises `stream`. */
int tspg_mcl_normalize(tspg_ctx *ctx, void *stream, const tspg_csr *M,
                       void *val_out);
int tspg_mcl_inflate(tspg_ctx *ctx, void *stream, const tspg_csr *M,
                     double power, void *val_out);
int tspg_mcl_prune(tspg_ctx *ctx, void *stream, const tspg_csr *M, double tol,
                   tspg_csr_out *out);

/* ---- batched products ----------------------------------------------------------
 * Many independent products C_i = A_i·B_i of uneven sizes in one persistent
 * launch per phase, fed by a device work queue; each phase is a CUDA graph
 * captured on the first run and replayed while the batch is unchanged.
 * Outputs go to one slab owned by the batch (context pool, reused across
 * runs); read each result with tspg_batch_result, valid until the next run,
 * clear or destroy.  All products of a batch share the value width; row
 * offsets may mix int32 and int64 (the batch then runs with int64 offsets).
 * The batch borrows its operands: they must stay valid and unchanged in
 * shape while it is used. */
typedef struct tspg_batch tspg_batch;
int tspg_batch_create(tspg_ctx *ctx, tspg_batch **out);
int tspg_batch_destroy(tspg_batch *b);
int tspg_batch_clear(tspg_batch *b);
int tspg_batch_add(tspg_batch *b, const tspg_csr *A, const tspg_csr *B,
                   int *index_out);
/* Runs all products; synchronises `stream` once (for the output size). */
int tspg_batch_run(tspg_batch *b, void *stream, int flags,
                   int64_t *total_nnz);
/* The flop-count pass of tspg_spgemm_count for every product of the batch in
 * one launch: mults[i] and c_nnz_upper[i] for product i (arrays of the
 * batch's size).  Synchronises `stream` once; does not run the products. */
int tspg_batch_count(tspg_batch *b, void *stream, int64_t *mults,
                     int64_t *c_nnz_upper);
/* View of result i (device pointers into the batch's slab, int64 rowptr). */
int tspg_batch_result(const tspg_batch *b, int i, tspg_csr *out);

/* ---- serving ---------------------------------------------------------------------
 * A continuous-batching server for C = A·B and Galerkin C = R·(A·P) requests
 * with device-resident operands (borrowed until the request completes).
 * Submission does no device work.  A bounding thread bounds the outputs of
 * the submitted requests, in order, with batched flop-count passes; each of
 * `lanes` worker threads (own context and stream) then admits from the head
 * of that FIFO, in submission order, the requests (up to max_batch) that fit
 * `mem_budget` bytes and runs them as one batched product per stage, so
 * batches formed while others run overlap on the device.  A result (int64
 * row offsets) is a view into the output slab of the batch that computed it,
 * not a copy; it stays valid until release, and a batch is reused only once
 * every request it computed has been released. */
enum { TSPG_REQ_AB = 0, TSPG_REQ_RAP = 1 };
typedef struct tspg_server tspg_server;
typedef struct tspg_server_config {
  size_t mem_budget; /* admission budget, bytes */
  int lanes;         /* concurrent worker lanes (1..16) */
  int max_batch;     /* requests per batch */
} tspg_server_config;
/* The server uses ctx's device; it creates its own contexts and streams,
 * which take ctx's row binning (tspg_ctx_set_tuning) at creation. */
int tspg_server_create(tspg_ctx *ctx, const tspg_server_config *cfg,
                       tspg_server **out);
/* Finishes the batches on the device, drops requests still waiting for
 * admission and frees every result not yet released. */
int tspg_server_destroy(tspg_server *s);
/* kind TSPG_REQ_AB: C = A·B (R unused); TSPG_REQ_RAP: C = R·(A·B) with B the
 * prolongator.  Checks the shapes and enqueues; a request whose output bound
 * alone exceeds the budget completes with TSPG_ENOMEM (from
 * tspg_server_wait).  Thread-safe. */
int tspg_server_submit(tspg_server *s, int kind, const tspg_csr *A,
                       const tspg_csr *B, const tspg_csr *R, int64_t *ticket);
/* Wait up to timeout_ms (< 0: forever) for a ticket; TSPG_ETIMEOUT if not
 * done.  latency_ms = completion - submission (host clock). */
int tspg_server_wait(tspg_server *s, int64_t ticket, int timeout_ms,
                     tspg_csr *result, double *latency_ms);
int tspg_server_release(tspg_server *s, int64_t ticket);
int tspg_server_stats(tspg_server *s, int64_t *batches, int64_t *completed,
                      int64_t *queued, size_t *reserved);

#ifdef __cplusplus
}
#endif
#endif /* TSPG_H */
