// tspg_trident.hpp — C++ host mirror of Trident's on-node operator interface
// on top of the libtspg C ABI (tspg.h).
//
// The reference drivers call LocalMatrix::spgemm / sp_mma / spadd
// (include/KokkosWrap.hpp:60-66), sp_mma_hybrid and cusparse_spgeam
// (include/cusparse_helpers.cuh:708,799), and SpaComm::gen_bitmask /
// intersect_bitmasks / select_ptrs / SpaCommHandler::Compress
// (include/spacomm.cuh:29,126,556,962) on mmio::CSX tiles and CsxBuffers
// (include/utils.cuh:527).  This header keeps those names, argument meanings
// and the reference's error behaviour (a failing call prints and exits, as
// CUSPARSE_CHECK does, include/utils.cuh:3-10), with the arithmetic done by
// the B200 kernels.  Kokkos and cuSPARSE types are replaced by plain device
// CSR (Csx); the drivers' KokkosWrap::LocalMatrix wrapper maps onto
// tspg_trident::LocalMatrix one to one.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <type_traits>
#include <utility>

#include "tspg.h"

namespace tspg_trident {

#define TSPG_TRIDENT_CHECK(call)                                                       \
  do {                                                                                 \
    const int _st = (call);                                                            \
    if (_st != TSPG_OK) {                                                              \
      std::fprintf(stderr, "libtspg error %s (%d) at %s:%d\n", tspg_strerror(_st), _st, \
                   __FILE__, __LINE__);                                                \
      std::exit(EXIT_FAILURE);                                                         \
    }                                                                                  \
  } while (0)

#define TSPG_TRIDENT_CUDA(call)                                                          \
  do {                                                                                   \
    const cudaError_t _e = (call);                                                       \
    if (_e != cudaSuccess) {                                                             \
      std::fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(_e), __FILE__, \
                   __LINE__);                                                            \
      std::exit(EXIT_FAILURE);                                                           \
    }                                                                                    \
  } while (0)

enum class MajorDim { ROWS = TSPG_ROWS, COLS = TSPG_COLS };

// mmio::CSX: device arrays of a compressed tile; contig tiles live in one
// [val | idx | ptr] buffer (TileHolder::set_csx_ptrs layout).
template <typename IT, typename VT>
struct Csx {
  static_assert(std::is_same<IT, int32_t>::value, "int32 indices (mmio::CSX<int32_t, VT>)");
  MajorDim majordim = MajorDim::ROWS;
  IT nrows = 0, ncols = 0, nnz = 0;
  IT *ptr_vec = nullptr;
  IT *idx_vec = nullptr;
  VT *val = nullptr;
  bool contig = false;
  char *buf = nullptr;
  size_t buf_size = 0;

  IT ptr_len() const { return majordim == MajorDim::ROWS ? nrows : ncols; }
  tspg_csr abi() const {
    tspg_csr c;
    c.nrows = nrows;
    c.ncols = ncols;
    c.nnz = nnz;
    c.rowptr = ptr_vec;
    c.rowptr_bits = 32;
    c.val_bits = int32_t(sizeof(VT) * 8);
    c.col = idx_vec;
    c.val = val;
    return c;
  }
};

// Library context (one per host thread, like the reference's cusparseHandle_t
// + CsxBuffers temp buffers + setup_mempool).
class Context {
 public:
  explicit Context(int device = 0, size_t budget = 0) {
    TSPG_TRIDENT_CHECK(tspg_ctx_create(device, budget, &ctx_));
  }
  ~Context() {
    if (ctx_) tspg_ctx_destroy(ctx_);
  }
  Context(const Context &) = delete;
  Context &operator=(const Context &) = delete;
  tspg_ctx *get() const { return ctx_; }

 private:
  tspg_ctx *ctx_ = nullptr;
};

// utils.cuh CsxBuffers: grow-only device CSR.  `ensure` keeps the reference's
// semantics (nnz becomes the requested size, arrays grow, never shrink).
template <typename IT, typename VT>
struct CsxBuffers {
  uint64_t nnz = 0, max_nnz = 0, ptr_dim = 0, other_dim = 0;
  VT *d_node_vals = nullptr;
  IT *d_node_colinds = nullptr;
  IT *d_node_rowptrs = nullptr;
  cudaStream_t stream = nullptr;

  CsxBuffers() = default;
  CsxBuffers(uint64_t nnz_cap, uint64_t ptr_dim_, uint64_t other_dim_, cudaStream_t s = nullptr)
      : stream(s) {
    ensure(nnz_cap, ptr_dim_, other_dim_);
    nnz = 0;
    TSPG_TRIDENT_CUDA(cudaMemset(d_node_rowptrs, 0, sizeof(IT) * ptr_dim));
  }
  CsxBuffers(const CsxBuffers &) = delete;
  CsxBuffers &operator=(const CsxBuffers &) = delete;
  ~CsxBuffers() { explicitFree(); }

  void ensure(uint64_t input_nnz, uint64_t input_ptr_dim, uint64_t other) {
    nnz = input_nnz;
    other_dim = other;
    if (input_nnz > max_nnz || !d_node_vals) {
      cudaFree(d_node_vals);
      cudaFree(d_node_colinds);
      max_nnz = input_nnz > max_nnz ? input_nnz : max_nnz;
      TSPG_TRIDENT_CUDA(cudaMalloc(&d_node_vals, sizeof(VT) * (max_nnz ? max_nnz : 1)));
      TSPG_TRIDENT_CUDA(cudaMalloc(&d_node_colinds, sizeof(IT) * (max_nnz ? max_nnz : 1)));
    }
    if (input_ptr_dim > ptr_dim || !d_node_rowptrs) {
      cudaFree(d_node_rowptrs);
      ptr_dim = input_ptr_dim > ptr_dim ? input_ptr_dim : ptr_dim;
      TSPG_TRIDENT_CUDA(cudaMalloc(&d_node_rowptrs, sizeof(IT) * ptr_dim));
      TSPG_TRIDENT_CUDA(cudaMemset(d_node_rowptrs, 0, sizeof(IT) * ptr_dim));
    }
  }

  void explicitFree() {
    cudaFree(d_node_vals);
    cudaFree(d_node_colinds);
    cudaFree(d_node_rowptrs);
    d_node_vals = nullptr;
    d_node_colinds = nullptr;
    d_node_rowptrs = nullptr;
    nnz = max_nnz = ptr_dim = 0;
  }

  IT nrows() const { return IT(ptr_dim ? ptr_dim - 1 : 0); }
  Csx<IT, VT> view() const {
    Csx<IT, VT> c;
    c.nrows = nrows();
    c.ncols = IT(other_dim);
    c.nnz = IT(nnz);
    c.ptr_vec = d_node_rowptrs;
    c.idx_vec = d_node_colinds;
    c.val = d_node_vals;
    return c;
  }
  tspg_csr abi() const { return view().abi(); }

  // Output descriptor that grows these buffers through the allocator hook.
  tspg_csr_out out(IT rows, IT cols) {
    ensure(0, uint64_t(rows) + 1, uint64_t(cols));
    tspg_csr_out o{};
    o.nrows = rows;
    o.ncols = cols;
    o.rowptr = d_node_rowptrs;
    o.rowptr_bits = 32;
    o.val_bits = int32_t(sizeof(VT) * 8);
    o.col = d_node_colinds;
    o.val = d_node_vals;
    o.capacity = int64_t(max_nnz);
    o.alloc = &CsxBuffers::grow;
    o.alloc_user = this;
    pending_ = 0;
    return o;
  }
  // after a call that used out(): record the result size
  void commit(const tspg_csr_out &o) {
    nnz = uint64_t(o.nnz);
    d_node_colinds = o.col;
    d_node_vals = (VT *)o.val;
  }

 private:
  int pending_ = 0;
  // first call: column indices, second call: values (tspg_csr_out contract)
  static void *grow(void *user, size_t bytes, void *) {
    CsxBuffers *b = (CsxBuffers *)user;
    void *p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    if (b->pending_ == 0) {
      cudaFree(b->d_node_colinds);
      b->d_node_colinds = (IT *)p;
      b->max_nnz = bytes / sizeof(IT);
    } else {
      cudaFree(b->d_node_vals);
      b->d_node_vals = (VT *)p;
    }
    b->pending_ ^= 1;
    return p;
  }
};

// KokkosWrap::LocalMatrix: a CSR tile owned through CsxBuffers.
template <typename IT, typename VT>
struct LocalMatrix {
  bool initialized = false;
  CsxBuffers<IT, VT> storage;

  // C = A·B (LocalMatrix::spgemm, KokkosWrap.hpp:367-391)
  static void spgemm(Context &ctx, const Csx<IT, VT> &A, const Csx<IT, VT> &B,
                     LocalMatrix &C, cudaStream_t s = nullptr) {
    const tspg_csr a = A.abi(), b = B.abi();
    tspg_csr_out o = C.storage.out(A.nrows, B.ncols);
    TSPG_TRIDENT_CHECK(tspg_spgemm(ctx.get(), s, &a, &b, &o, TSPG_F_NONE));
    C.storage.commit(o);
    C.initialized = true;
  }

  // C = C + A·B (LocalMatrix::sp_mma, KokkosWrap.hpp:315-364); the first call
  // sets C = A·B.
  static void sp_mma(Context &ctx, const Csx<IT, VT> &A, const Csx<IT, VT> &B,
                     LocalMatrix &C, cudaStream_t s = nullptr) {
    if (!C.initialized) {
      spgemm(ctx, A, B, C, s);
      return;
    }
    const tspg_csr a = A.abi(), b = B.abi(), cin = C.storage.abi();
    LocalMatrix acc;
    tspg_csr_out o = acc.storage.out(A.nrows, B.ncols);
    TSPG_TRIDENT_CHECK(tspg_spgemm_acc(ctx.get(), s, &a, &b, &cin, &o, TSPG_F_NONE));
    acc.storage.commit(o);
    std::swap(C.storage.d_node_vals, acc.storage.d_node_vals);
    std::swap(C.storage.d_node_colinds, acc.storage.d_node_colinds);
    std::swap(C.storage.d_node_rowptrs, acc.storage.d_node_rowptrs);
    std::swap(C.storage.nnz, acc.storage.nnz);
    std::swap(C.storage.max_nnz, acc.storage.max_nnz);
    std::swap(C.storage.ptr_dim, acc.storage.ptr_dim);
  }

  // C = A + C (LocalMatrix::spadd, KokkosWrap.hpp:394-439): no-op for an
  // empty A; C := A when C is not initialised.
  static void spadd(Context &ctx, const Csx<IT, VT> &A, LocalMatrix &C, cudaStream_t s = nullptr) {
    if (A.nnz == 0) return;
    LocalMatrix acc;
    const tspg_csr a = A.abi();
    tspg_csr empty{};
    empty.nrows = A.nrows;
    empty.ncols = A.ncols;
    empty.rowptr_bits = 32;
    empty.val_bits = int32_t(sizeof(VT) * 8);
    IT *zero = nullptr;
    if (!C.initialized) {
      TSPG_TRIDENT_CUDA(cudaMalloc(&zero, sizeof(IT) * (A.nrows + 1)));
      TSPG_TRIDENT_CUDA(cudaMemset(zero, 0, sizeof(IT) * (A.nrows + 1)));
      empty.rowptr = zero;
    }
    const tspg_csr c = C.initialized ? C.storage.abi() : empty;
    tspg_csr_out o = acc.storage.out(A.nrows, A.ncols);
    TSPG_TRIDENT_CHECK(tspg_spadd(ctx.get(), s, &a, &c, &o));
    acc.storage.commit(o);
    if (zero) cudaFree(zero);
    std::swap(C.storage.d_node_vals, acc.storage.d_node_vals);
    std::swap(C.storage.d_node_colinds, acc.storage.d_node_colinds);
    std::swap(C.storage.d_node_rowptrs, acc.storage.d_node_rowptrs);
    std::swap(C.storage.nnz, acc.storage.nnz);
    std::swap(C.storage.max_nnz, acc.storage.max_nnz);
    std::swap(C.storage.ptr_dim, acc.storage.ptr_dim);
    C.initialized = true;
  }

  // LocalMatrix::csc_to_csr (KokkosWrap.hpp:442-531): a CSC tile is the CSR
  // of its transpose, so one device transpose gives the CSR tile.
  static void csc_to_csr(Context &ctx, const Csx<IT, VT> &csc, LocalMatrix &C,
                         cudaStream_t s = nullptr) {
    tspg_csr t = csc.abi();
    t.nrows = csc.ncols;  // compressed dimension of the CSC
    t.ncols = csc.nrows;
    tspg_csr_out o = C.storage.out(csc.nrows, csc.ncols);
    TSPG_TRIDENT_CHECK(tspg_transpose(ctx.get(), s, &t, &o));
    C.storage.commit(o);
    C.initialized = true;
  }

  Csx<IT, VT> get_csx() const { return storage.view(); }
};

// coo_to_row_csx / coo_to_col_csx (cusparse_helpers.cuh:17-131) and
// coo_to_kokkos_crs / coo_to_kokkos_ccs (kokkos_helpers.cuh:52-352): triples
// sorted by the major index and compressed — here on the device, from device
// COO arrays, into a grow-only buffer (CSC comes out as the CSR of the
// transpose: ptr over columns, row indices).  Repeated entries are kept.
template <typename IT, typename VT>
void coo_to_csx(Context &ctx, MajorDim major, IT nrows, IT ncols, IT nnz, const IT *d_row,
                const IT *d_col, const VT *d_val, CsxBuffers<IT, VT> &out,
                cudaStream_t s = nullptr) {
  const bool rows = major == MajorDim::ROWS;
  tspg_csr_out o = out.out(rows ? nrows : ncols, rows ? ncols : nrows);
  TSPG_TRIDENT_CHECK(tspg_coo_to_csx(ctx.get(), s, nrows, ncols, nnz, d_row, d_col, d_val,
                                     int(sizeof(VT) * 8), int(major), &o));
  out.commit(o);
}
template <typename IT, typename VT>
void coo_to_row_csx(Context &ctx, IT nrows, IT ncols, IT nnz, const IT *d_row, const IT *d_col,
                    const VT *d_val, CsxBuffers<IT, VT> &out, cudaStream_t s = nullptr) {
  coo_to_csx(ctx, MajorDim::ROWS, nrows, ncols, nnz, d_row, d_col, d_val, out, s);
}
template <typename IT, typename VT>
void coo_to_col_csx(Context &ctx, IT nrows, IT ncols, IT nnz, const IT *d_row, const IT *d_col,
                    const VT *d_val, CsxBuffers<IT, VT> &out, cudaStream_t s = nullptr) {
  coo_to_csx(ctx, MajorDim::COLS, nrows, ncols, nnz, d_row, d_col, d_val, out, s);
}

// cusparse_spgeam (cusparse_helpers.cuh:799-905): C_accum = C_prod + C_local.
template <typename IT, typename VT>
void cusparse_spgeam(Context &ctx, const Csx<IT, VT> &C_prod, CsxBuffers<IT, VT> &C_local,
                     CsxBuffers<IT, VT> &C_accum, cudaStream_t s = nullptr) {
  const tspg_csr p = C_prod.abi(), l = C_local.abi();
  tspg_csr_out o = C_accum.out(C_prod.nrows, C_prod.ncols);
  TSPG_TRIDENT_CHECK(tspg_spadd(ctx.get(), s, &p, &l, &o));
  C_accum.commit(o);
}

// sp_mma_hybrid (cusparse_helpers.cuh:708-739): C_accum = C_local + A·B, then
// swap, skipping an empty product.
template <typename IT, typename VT>
void sp_mma_hybrid(Context &ctx, const Csx<IT, VT> &A, const Csx<IT, VT> &B,
                   CsxBuffers<IT, VT> **C_local, CsxBuffers<IT, VT> **C_accum, bool &did_first,
                   cudaStream_t s = nullptr) {
  LocalMatrix<IT, VT> prod;
  LocalMatrix<IT, VT>::spgemm(ctx, A, B, prod, s);
  if (prod.storage.nnz == 0) return;
  did_first = true;
  cusparse_spgeam(ctx, prod.get_csx(), **C_local, **C_accum, s);
  std::swap(*C_local, *C_accum);
}

namespace SpaComm {

// gen_bitmask (spacomm.cuh:29-117); MASK_SIZE = 8.  Caller frees the result.
template <typename IT>
uint8_t *gen_bitmask(Context &ctx, const IT *ptr_d, int n, int mask_size = 8,
                     cudaStream_t s = nullptr) {
  if (mask_size != 8) {
    std::fprintf(stderr, "libtspg: MASK_SIZE must be 8 (BMASK_TYPE uint8_t)\n");
    std::exit(EXIT_FAILURE);
  }
  uint8_t *out = nullptr;
  TSPG_TRIDENT_CUDA(cudaMalloc(&out, size_t((n + 7) / 8 > 0 ? (n + 7) / 8 : 1)));
  TSPG_TRIDENT_CHECK(tspg_bitmask_gen(ctx.get(), s, ptr_d, int(sizeof(IT) * 8), n, out));
  TSPG_TRIDENT_CUDA(cudaStreamSynchronize(s));
  return out;
}

// intersect_bitmasks (spacomm.cuh:126-148).  Caller frees the result.
template <typename T>
T *intersect_bitmasks(Context &ctx, const T *a, const T *b, int n, cudaStream_t s = nullptr) {
  T *out = nullptr;
  TSPG_TRIDENT_CUDA(cudaMalloc(&out, sizeof(T) * (n > 0 ? n : 1)));
  TSPG_TRIDENT_CHECK(tspg_bitmask_and(ctx.get(), s, (const uint8_t *)a, (const uint8_t *)b,
                                      int64_t(n) * int64_t(sizeof(T)), (uint8_t *)out));
  TSPG_TRIDENT_CUDA(cudaStreamSynchronize(s));
  return out;
}

// SpaCommHandler::Compress (spacomm.cuh:962-1091) on one tile: the packed
// tile in `buf` (capacity >= the unpacked tile's size), wrapped as a contig
// Csx that borrows `buf`.
template <typename IT, typename VT>
Csx<IT, VT> Compress(Context &ctx, const Csx<IT, VT> &M, const uint8_t *mask, char *buf,
                     size_t cap, cudaStream_t s = nullptr) {
  const tspg_csr m = M.abi();
  int64_t kept = 0;
  TSPG_TRIDENT_CHECK(tspg_pack(ctx.get(), s, &m, int(M.majordim), mask, buf, cap, nullptr, &kept));
  tspg_csr v{};
  TSPG_TRIDENT_CHECK(tspg_unpack(buf, m.nrows, m.ncols, int(M.majordim), kept, m.val_bits, 32, &v));
  Csx<IT, VT> out = M;
  out.nnz = IT(kept);
  out.contig = true;
  out.buf = buf;
  out.buf_size = tspg_packed_bytes(kept, M.ptr_len(), m.val_bits, 32);
  out.val = (VT *)v.val;
  out.idx_vec = (IT *)v.col;
  out.ptr_vec = (IT *)v.rowptr;
  return out;
}

}  // namespace SpaComm
}  // namespace tspg_trident
