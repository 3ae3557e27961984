// tspg_trident.hpp — Trident's on-node operators with the reference's own
// signatures, on top of the libtspg C ABI (tspg.h).
//
// A Trident driver includes this header in place of the operator bodies of
// include/KokkosWrap.hpp, include/cusparse_helpers.cuh and include/spacomm.cuh
// and keeps its call sites as they are:
//
//   KokkosWrap::LocalMatrix<KIT,DIT,VT>  ::spgemm / ::sp_mma / ::spadd / ::csc_to_csr
//                                         (KokkosWrap.hpp:44-77, 315-531)
//   CsxBuffers<IT,VT>                     (utils.cuh:527-784)
//   CusparseCSX<IT,VT>                    (cusparse_helpers.cuh:134-484)
//   sp_mma_hybrid(cusparseHandle_t*, const LocalMatrix&, const LocalMatrix&,
//                 CusparseCSX**, CusparseCSX**, bool&)      (cusparse_helpers.cuh:708-739)
//   cusparse_spmma(cusparseHandle_t*, CusparseCSX*, CusparseCSX*,
//                  CusparseCSX**, CusparseCSX**, CusparseCSX**, bool)  (:744-796)
//   cusparse_spgeam(cusparseHandle_t*, CusparseCSX*, CusparseCSX*, CusparseCSX*)  (:799-905)
//   SpaComm::gen_bitmask / intersect_bitmasks / select_ptrs  (spacomm.cuh:29-148, 556-623)
//   SpaComm::SpaCommBuffers, SpaComm::SpaCommHandler::Compress(const mmio::CSX*, int,
//                  SpaCommBuffers*, cudaStream_t, MPI_Comm)  (spacomm.cuh:634-712, 962-1091)
//   rownnz_to_rowptrs / rowptrs_to_rownnz (utils.cuh:412-448)
//   coo_to_row_csx(_contig) / coo_to_col_csx(_contig)  (cusparse_helpers.cuh:17-131,
//                  kokkos_helpers.cuh:125-352)
//
// The arithmetic runs in the B200 kernels of libtspg; no cuSPARSE, Kokkos or
// CUB call remains.  Every call gets its library context from a thread-local
// (one per host thread and device, created on first use with the device that
// is current), which matches the reference's use of one cuSPARSE handle and
// cudaStreamPerThread per thread (include/common.h:13).  Failing calls print
// and exit, like CUSPARSE_CHECK / CUDA_CHECK (include/utils.cuh:3-10).
//
// The data types the drivers bring from dmmio (mmio::CSX, mmio::MajorDim,
// CSX_buf_size, CSX_get_ptrs) and the cuSPARSE / MPI handle types are used as
// they are when the build has them (define TSPG_TRIDENT_HAVE_DMMIO; cusparse.h
// and mpi.h are picked up when present); otherwise this header declares
// stand-ins with the same names and fields, so it also compiles alone.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <type_traits>
#include <utility>

#include "tspg.h"

#if defined(__has_include)
#if __has_include(<cusparse.h>)
#include <cusparse.h>
#define TSPG_TRIDENT_HAVE_CUSPARSE_TYPES 1
#endif
#if __has_include(<mpi.h>)
#include <mpi.h>
#define TSPG_TRIDENT_HAVE_MPI_TYPES 1
#endif
#endif

#ifndef TSPG_TRIDENT_HAVE_CUSPARSE_TYPES
struct cusparseContext;
typedef struct cusparseContext *cusparseHandle_t;
#endif
#ifndef TSPG_TRIDENT_HAVE_MPI_TYPES
typedef int MPI_Comm;
#define MPI_COMM_WORLD 0
#endif

#ifndef BMASK_TYPE
#define BMASK_TYPE uint8_t  // include/common.h:63-65
#endif
#ifndef MASK_SIZE
#define MASK_SIZE 8
#endif

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

// ---------------------------------------------------------------------------
// dmmio stand-ins (the reference takes them from the distributed_mmio submodule)
#ifndef TSPG_TRIDENT_HAVE_DMMIO
namespace mmio {
enum class MajorDim { ROWS = TSPG_ROWS, COLS = TSPG_COLS };

template <typename IT, typename VT>
struct CSX {
  MajorDim majordim;
  IT nrows, ncols, nnz;
  IT *ptr_vec;
  IT *idx_vec;
  VT *val;
  bool contig;
  char *buf;
  size_t buf_size;
};

// Bytes of a contiguous tile [val[nnz] | idx[nnz] | ptr[major + 1]]
// (TileHolder::set_csx_ptrs layout, include/tile_holder.cuh:80-89).
template <typename IT, typename VT>
size_t CSX_buf_size(IT nrows, IT ncols, IT nnz, MajorDim majordim) {
  const size_t len = size_t(majordim == MajorDim::ROWS ? nrows : ncols) + 1;
  return size_t(nnz) * (sizeof(VT) + sizeof(IT)) + len * sizeof(IT);
}
template <typename IT, typename VT>
size_t CSX_buf_size(const CSX<IT, VT> *m) {
  return CSX_buf_size<IT, VT>(m->nrows, m->ncols, m->nnz, m->majordim);
}
// Host COO triples of a tile (mmio::COO).
template <typename IT, typename VT>
struct COO {
  IT nrows, ncols, nnz;
  IT *row;
  IT *col;
  VT *val;
};
template <typename IT, typename VT>
void CSX_get_ptrs(IT, IT, IT nnz, char *buf, IT **ptr, IT **idx, VT **val) {
  *val = (VT *)buf;
  *idx = (IT *)(buf + size_t(nnz) * sizeof(VT));
  *ptr = (IT *)(buf + size_t(nnz) * (sizeof(VT) + sizeof(IT)));
}
}  // namespace mmio
#endif

namespace tspg_trident {

// The calling thread's library context on the current device (created on
// first use, destroyed when the thread exits).
inline tspg_ctx *thread_ctx() {
  struct Holder {
    tspg_ctx *ctx = nullptr;
    int dev = -1;
    ~Holder() {
      if (ctx) tspg_ctx_destroy(ctx);
    }
  };
  thread_local Holder h;
  int dev = 0;
  TSPG_TRIDENT_CUDA(cudaGetDevice(&dev));
  if (!h.ctx || h.dev != dev) {
    if (h.ctx) tspg_ctx_destroy(h.ctx);
    h.ctx = nullptr;
    TSPG_TRIDENT_CHECK(tspg_ctx_create(dev, 0, &h.ctx));
    h.dev = dev;
  }
  return h.ctx;
}

template <typename IT, typename VT>
tspg_csr abi_of(IT nrows, IT ncols, IT nnz, const IT *ptr, const IT *idx, const VT *val) {
  static_assert(std::is_same<IT, int32_t>::value, "int32 indices, as the reference instantiates");
  tspg_csr c{};
  c.nrows = nrows;
  c.ncols = ncols;
  c.nnz = nnz;
  c.rowptr = ptr;
  c.rowptr_bits = 32;
  c.val_bits = int32_t(sizeof(VT) * 8);
  c.col = idx;
  c.val = val;
  return c;
}

// Device CSR arrays owned through a shared block (the refcounted Kokkos views
// of the reference), or borrowed (unmanaged views over caller memory).
template <typename IT, typename VT>
struct DeviceArrays {
  IT *ptr = nullptr;
  IT *idx = nullptr;
  VT *val = nullptr;
  bool owned = false;
  ~DeviceArrays() {
    if (owned) {
      cudaFree(ptr);
      cudaFree(idx);
      cudaFree(val);
    }
  }
};

// Output descriptor whose column / value arrays are allocated on demand
// (cudaMalloc, first call columns, second values) into `dst`.
template <typename IT, typename VT>
struct FreshOut {
  std::shared_ptr<DeviceArrays<IT, VT>> dst = std::make_shared<DeviceArrays<IT, VT>>();
  int calls = 0;
  static void *alloc(void *user, size_t bytes, void *) {
    FreshOut *f = (FreshOut *)user;
    void *p = nullptr;
    if (cudaMalloc(&p, bytes ? bytes : 1) != cudaSuccess) return nullptr;
    if (f->calls++ == 0) f->dst->idx = (IT *)p;
    else f->dst->val = (VT *)p;
    return p;
  }
  tspg_csr_out make(IT rows, IT cols) {
    dst->owned = true;
    TSPG_TRIDENT_CUDA(cudaMalloc(&dst->ptr, sizeof(IT) * (size_t(rows) + 1)));
    tspg_csr_out o{};
    o.nrows = rows;
    o.ncols = cols;
    o.rowptr = dst->ptr;
    o.rowptr_bits = 32;
    o.val_bits = int32_t(sizeof(VT) * 8);
    o.capacity = 0;
    o.alloc = &FreshOut::alloc;
    o.alloc_user = this;
    return o;
  }
};

}  // namespace tspg_trident

// ---------------------------------------------------------------------------
// CsxBuffers (include/utils.cuh:527-784): grow-only device CSR; `nnz` is a
// host field; the row offsets start zeroed.
template <typename IT, typename VT>
struct CsxBuffers {
  uint64_t nnz = 0;
  uint64_t max_nnz = 0;
  uint64_t ptr_dim = 0;
  uint64_t other_dim = 0;
  uint64_t nbufs = 1;
  int initialized = 0;
  VT *d_node_vals = nullptr;
  IT *d_node_colinds = nullptr;
  IT *d_node_rowptrs = nullptr;
  cudaStream_t *stream = nullptr;
  bool async_csx = false;

  CsxBuffers() = default;
  CsxBuffers(uint64_t input_nnz, uint64_t input_ptr_dim, uint64_t _other_dim,
             cudaStream_t *_stream = nullptr, uint64_t _nbufs = 1, bool _async_csx = false) {
    init(input_nnz, input_ptr_dim, _other_dim, _stream, _nbufs, _async_csx);
  }
  CsxBuffers(const CsxBuffers &) = delete;
  CsxBuffers &operator=(const CsxBuffers &) = delete;
  ~CsxBuffers() {
    if (initialized) explicitFree();
  }

  cudaStream_t s() const { return stream ? *stream : cudaStreamPerThread; }

  void init(uint64_t input_nnz, uint64_t input_ptr_dim, uint64_t _other_dim, cudaStream_t *_stream,
            uint64_t _nbufs, bool _async_csx) {
    initialized = 1;
    nnz = 0;
    max_nnz = input_nnz;
    ptr_dim = input_ptr_dim;
    other_dim = _other_dim;
    nbufs = _nbufs;
    stream = _stream;
    async_csx = _async_csx;
    d_node_vals = (VT *)alloc_bytes(sizeof(VT) * (max_nnz ? max_nnz : 1));
    d_node_colinds = (IT *)alloc_bytes(sizeof(IT) * (max_nnz ? max_nnz : 1));
    d_node_rowptrs = (IT *)alloc_bytes(sizeof(IT) * (ptr_dim ? ptr_dim : 1));
    TSPG_TRIDENT_CUDA(cudaMemsetAsync(d_node_rowptrs, 0, sizeof(IT) * (ptr_dim ? ptr_dim : 1), s()));
    if (async_csx) TSPG_TRIDENT_CUDA(cudaStreamSynchronize(s()));
  }

  void *alloc_bytes(size_t b) {
    void *p = nullptr;
    if (async_csx) TSPG_TRIDENT_CUDA(cudaMallocAsync(&p, b, s()));
    else TSPG_TRIDENT_CUDA(cudaMalloc(&p, b));
    return p;
  }
  void free_bytes(void *p) {
    if (!p) return;
    if (async_csx) cudaFreeAsync(p, s());
    else cudaFree(p);
  }

  // ensure / ensure_async: nnz becomes the requested size; the arrays grow
  // (contents not kept), never shrink; a grown row-offset array is zeroed.
  void ensure(uint64_t input_nnz, uint64_t input_ptr_dim, uint64_t _other_dim) {
    nnz = input_nnz;
    other_dim = _other_dim;
    if (!initialized) {
      init(input_nnz, input_ptr_dim, _other_dim, stream, nbufs, async_csx);
      nnz = input_nnz;
      return;
    }
    if (input_nnz > max_nnz) {
      free_bytes(d_node_vals);
      free_bytes(d_node_colinds);
      max_nnz = input_nnz;
      d_node_vals = (VT *)alloc_bytes(sizeof(VT) * max_nnz);
      d_node_colinds = (IT *)alloc_bytes(sizeof(IT) * max_nnz);
    }
    if (input_ptr_dim > ptr_dim) {
      free_bytes(d_node_rowptrs);
      ptr_dim = input_ptr_dim;
      d_node_rowptrs = (IT *)alloc_bytes(sizeof(IT) * ptr_dim);
      TSPG_TRIDENT_CUDA(cudaMemsetAsync(d_node_rowptrs, 0, sizeof(IT) * ptr_dim, s()));
    }
    if (async_csx) TSPG_TRIDENT_CUDA(cudaStreamSynchronize(s()));
  }
  void ensure_async(uint64_t input_nnz, uint64_t input_ptr_dim, uint64_t _other_dim) {
    ensure(input_nnz, input_ptr_dim, _other_dim);
  }

  size_t total_size() const {
    return sizeof(VT) * max_nnz + sizeof(IT) * max_nnz + sizeof(IT) * ptr_dim;
  }

  mmio::CSX<IT, VT> *to_mmio_csx() {
    mmio::CSX<IT, VT> *csx = (mmio::CSX<IT, VT> *)std::calloc(1, sizeof(mmio::CSX<IT, VT>));
    csx->majordim = mmio::MajorDim::ROWS;
    csx->nnz = IT(nnz);
    csx->nrows = IT(ptr_dim - 1);
    csx->ncols = IT(other_dim);
    csx->val = d_node_vals;
    csx->ptr_vec = d_node_rowptrs;
    csx->idx_vec = d_node_colinds;
    return csx;
  }

  void explicitFree() {
    if (initialized) {
      free_bytes(d_node_colinds);
      free_bytes(d_node_rowptrs);
      free_bytes(d_node_vals);
      if (async_csx) cudaStreamSynchronize(s());
      d_node_vals = nullptr;
      d_node_colinds = nullptr;
      d_node_rowptrs = nullptr;
      initialized = 0;
      ptr_dim = nnz = max_nnz = 0;
    }
  }

  tspg_csr abi() const {
    return tspg_trident::abi_of<IT, VT>(IT(ptr_dim ? ptr_dim - 1 : 0), IT(other_dim), IT(nnz),
                                        d_node_rowptrs, d_node_colinds, d_node_vals);
  }

  // An output descriptor into these buffers for a rows x cols result: the
  // library reports the size and, when the arrays are short, grows them
  // through `grow` (the ensure_async step of the reference's calls).
  tspg_csr_out out(IT rows, IT cols) {
    if (!initialized) init(0, uint64_t(rows) + 1, uint64_t(cols), stream, nbufs, async_csx);
    if (uint64_t(rows) + 1 > ptr_dim) ensure(nnz, uint64_t(rows) + 1, uint64_t(cols));
    other_dim = uint64_t(cols);
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
  void commit(const tspg_csr_out &o) { nnz = uint64_t(o.nnz); }

 private:
  int pending_ = 0;
  static void *grow(void *user, size_t bytes, void *) {
    CsxBuffers *b = (CsxBuffers *)user;
    void *p = b->alloc_bytes(bytes ? bytes : 1);
    if (b->pending_ == 0) {
      b->free_bytes(b->d_node_colinds);
      b->d_node_colinds = (IT *)p;
      b->max_nnz = bytes / sizeof(IT);
    } else {
      b->free_bytes(b->d_node_vals);
      b->d_node_vals = (VT *)p;
    }
    b->pending_ ^= 1;
    return p;
  }
};

// ---------------------------------------------------------------------------
namespace KokkosWrap {

using MajorDim = mmio::MajorDim;

// The CrsMatrix storage of a LocalMatrix: row offsets, entries, values on the
// device, with the numRows / numCols / nnz accessors the drivers use.
template <typename VT, typename KIT>
struct CrsStorage {
  KIT nrows_ = 0, ncols_ = 0, nnz_ = 0;
  std::shared_ptr<tspg_trident::DeviceArrays<KIT, VT>> arrays;
  KIT numRows() const { return nrows_; }
  KIT numCols() const { return ncols_; }
  KIT nnz() const { return nnz_; }
  KIT *row_map() const { return arrays ? arrays->ptr : nullptr; }
  KIT *entries() const { return arrays ? arrays->idx : nullptr; }
  VT *values() const { return arrays ? arrays->val : nullptr; }
  tspg_csr abi() const {
    return tspg_trident::abi_of<KIT, VT>(nrows_, ncols_, nnz_, row_map(), entries(), values());
  }
};

template <typename KIT, typename DIT, typename VT>
struct LocalMatrix {
  static_assert(std::is_same<KIT, DIT>::value, "KIT == DIT, as the reference instantiates");
  using KokkosCrs = CrsStorage<VT, KIT>;

  bool initialized = false;
  KokkosCrs storage;

  LocalMatrix() = default;
  // From a device tile; a CSC tile is converted to CSR (KokkosWrap.hpp:205-236).
  LocalMatrix(cusparseHandle_t &handle, mmio::CSX<DIT, VT> *mmio_csx,
              CsxBuffers<DIT, VT> *buffs = nullptr)
      : initialized(true) {
    if (mmio_csx->majordim == MajorDim::ROWS) storage = wrap(mmio_csx);
    else storage = csc_to_csr(handle, mmio_csx, buffs);
  }
  // Unmanaged view over a device CSR tile (KokkosWrap.hpp:265-286).
  explicit LocalMatrix(mmio::CSX<DIT, VT> *mmio_csx) : initialized(true), storage(wrap(mmio_csx)) {}
  LocalMatrix(DIT nrows, DIT ncols, DIT nnz, DIT *ptrvec, DIT *idxvec, VT *values, MajorDim layout)
      : initialized(true) {
    mmio::CSX<DIT, VT> c{};
    c.majordim = layout;
    c.nrows = nrows;
    c.ncols = ncols;
    c.nnz = nnz;
    c.ptr_vec = ptrvec;
    c.idx_vec = idxvec;
    c.val = values;
    storage = wrap(&c);
  }

  // C = C + A·B; the first call sets C = A·B (KokkosWrap.hpp:315-364).
  static void sp_mma(const LocalMatrix &A, const LocalMatrix &B, LocalMatrix &C) {
    if (!C.initialized) {
      C.storage = spgemm(A, B).storage;
      C.initialized = true;
      return;
    }
    const tspg_csr a = A.storage.abi(), b = B.storage.abi(), c = C.storage.abi();
    tspg_trident::FreshOut<KIT, VT> f;
    tspg_csr_out o = f.make(A.storage.numRows(), B.storage.numCols());
    TSPG_TRIDENT_CHECK(tspg_spgemm_acc(tspg_trident::thread_ctx(), cudaStreamPerThread, &a, &b, &c, &o,
                                       TSPG_F_NONE));
    C.storage = result(f, o);
  }

  // C = A·B (KokkosWrap.hpp:367-391).
  static LocalMatrix spgemm(const LocalMatrix &A, const LocalMatrix &B) {
    const tspg_csr a = A.storage.abi(), b = B.storage.abi();
    tspg_trident::FreshOut<KIT, VT> f;
    tspg_csr_out o = f.make(A.storage.numRows(), B.storage.numCols());
    TSPG_TRIDENT_CHECK(tspg_spgemm(tspg_trident::thread_ctx(), cudaStreamPerThread, &a, &b, &o,
                                   TSPG_F_NONE));
    LocalMatrix r;
    r.storage = result(f, o);
    r.initialized = true;
    return r;
  }

  // C = A + C; nothing for an empty A; C := A when C is not initialised
  // (KokkosWrap.hpp:394-439).
  static void spadd(const LocalMatrix &A, LocalMatrix &C) {
    if (A.storage.nnz() == 0) return;
    if (!C.initialized) {
      C.storage = A.storage;
      C.initialized = true;
      return;
    }
    const tspg_csr a = A.storage.abi(), c = C.storage.abi();
    tspg_trident::FreshOut<KIT, VT> f;
    tspg_csr_out o = f.make(A.storage.numRows(), A.storage.numCols());
    TSPG_TRIDENT_CHECK(tspg_spadd(tspg_trident::thread_ctx(), cudaStreamPerThread, &a, &c, &o));
    C.storage = result(f, o);
  }

  // CSC tile -> CSR (KokkosWrap.hpp:442-531): a CSC tile is the CSR of its
  // transpose, so one device transpose gives the CSR.
  KokkosCrs csc_to_csr(cusparseHandle_t &, mmio::CSX<DIT, VT> *csc,
                       CsxBuffers<DIT, VT> * = nullptr) {
    tspg_csr t = tspg_trident::abi_of<KIT, VT>(csc->ncols, csc->nrows, csc->nnz, csc->ptr_vec,
                                               csc->idx_vec, csc->val);
    tspg_trident::FreshOut<KIT, VT> f;
    tspg_csr_out o = f.make(csc->nrows, csc->ncols);
    TSPG_TRIDENT_CHECK(tspg_transpose(tspg_trident::thread_ctx(), cudaStreamPerThread, &t, &o));
    return result(f, o);
  }

  mmio::CSX<DIT, VT> *get_csx() {
    mmio::CSX<DIT, VT> *csx = (mmio::CSX<DIT, VT> *)std::calloc(1, sizeof(mmio::CSX<DIT, VT>));
    csx->majordim = MajorDim::ROWS;
    csx->nnz = storage.nnz();
    csx->nrows = storage.numRows();
    csx->ncols = storage.numCols();
    csx->val = storage.values();
    csx->ptr_vec = storage.row_map();
    csx->idx_vec = storage.entries();
    return csx;
  }

  // Releases the arrays (KokkosWrap.hpp:294-302 frees the raw pointers): an
  // owned result drops this reference, a borrowed view frees caller memory as
  // the reference does.
  void freeBuffers() {
    if (!initialized) return;
    if (storage.arrays && !storage.arrays->owned) {
      cudaFree(storage.arrays->ptr);
      cudaFree(storage.arrays->idx);
      cudaFree(storage.arrays->val);
    }
    storage.arrays.reset();
    initialized = false;
  }

 private:
  static KokkosCrs wrap(const mmio::CSX<DIT, VT> *m) {
    KokkosCrs s;
    s.nrows_ = m->nrows;
    s.ncols_ = m->ncols;
    s.nnz_ = m->nnz;
    s.arrays = std::make_shared<tspg_trident::DeviceArrays<KIT, VT>>();
    s.arrays->ptr = m->ptr_vec;
    s.arrays->idx = m->idx_vec;
    s.arrays->val = m->val;
    return s;
  }
  static KokkosCrs result(tspg_trident::FreshOut<KIT, VT> &f, const tspg_csr_out &o) {
    KokkosCrs s;
    s.nrows_ = KIT(o.nrows);
    s.ncols_ = KIT(o.ncols);
    s.nnz_ = KIT(o.nnz);
    s.arrays = f.dst;
    return s;
  }
};

// rawptr_get (KokkosWrap.hpp:89-131): a malloc'ed CSX view of the storage.
template <typename KIT, typename VT>
mmio::CSX<KIT, VT> *rawptr_get(LocalMatrix<KIT, KIT, VT> &m) {
  return m.get_csx();
}

}  // namespace KokkosWrap

using KokkosWrap::LocalMatrix;

// ---------------------------------------------------------------------------
// CusparseCSX (cusparse_helpers.cuh:134-484): a tile held as a CSX ("Mat"),
// as CsxBuffers ("Buffs") or both; the cuSPARSE descriptors of the reference
// have no counterpart (nothing here calls cuSPARSE).
template <typename IT, typename VT>
struct CusparseCSX {
  enum class State { Mat, Buffs, Null, Both };

  mmio::CSX<IT, VT> *mat = nullptr;
  CsxBuffers<IT, VT> *buffers = nullptr;
  State state = State::Null;

  CusparseCSX() = default;
  explicit CusparseCSX(mmio::CSX<IT, VT> *m) : mat(m), state(State::Mat) {}
  // Views the product of a LocalMatrix (state Both; the buffers alias the
  // storage and free nothing).
  explicit CusparseCSX(LocalMatrix<IT, IT, VT> &local)
      : mat(local.get_csx()), buffers(new CsxBuffers<IT, VT>()), state(State::Both) {
    buffers->d_node_vals = mat->val;
    buffers->d_node_colinds = mat->idx_vec;
    buffers->d_node_rowptrs = mat->ptr_vec;
    buffers->nnz = uint64_t(mat->nnz);
    buffers->max_nnz = uint64_t(mat->nnz);
    buffers->ptr_dim = uint64_t(mat->nrows) + 1;
    buffers->other_dim = uint64_t(mat->ncols);
  }
  // A received tile; a CSC tile is converted to CSR into storage this object
  // owns (cusparse_helpers.cuh:204-229).
  CusparseCSX(cusparseHandle_t *, mmio::CSX<IT, VT> *m, CsxBuffers<IT, VT> *)
      : state(State::Mat) {
    if (m->majordim == mmio::MajorDim::COLS) {
      tspg_csr t = tspg_trident::abi_of<IT, VT>(m->ncols, m->nrows, m->nnz, m->ptr_vec, m->idx_vec,
                                                m->val);
      converted_ = std::make_unique<tspg_trident::FreshOut<IT, VT>>();
      tspg_csr_out o = converted_->make(m->nrows, m->ncols);
      TSPG_TRIDENT_CHECK(tspg_transpose(tspg_trident::thread_ctx(), cudaStreamPerThread, &t, &o));
      mat = (mmio::CSX<IT, VT> *)std::calloc(1, sizeof(mmio::CSX<IT, VT>));
      mat->majordim = mmio::MajorDim::ROWS;
      mat->nrows = m->nrows;
      mat->ncols = m->ncols;
      mat->nnz = IT(o.nnz);
      mat->ptr_vec = converted_->dst->ptr;
      mat->idx_vec = converted_->dst->idx;
      mat->val = converted_->dst->val;
    } else {
      mat = m;
    }
  }
  explicit CusparseCSX(CsxBuffers<IT, VT> *b) : buffers(b), state(State::Buffs) {}
  CusparseCSX(const CusparseCSX &) = delete;
  CusparseCSX &operator=(const CusparseCSX &) = delete;

  ~CusparseCSX() {
    if (converted_) std::free(mat);  // the converted CSR's struct (arrays: converted_)
    if (state == State::Buffs) buffers->explicitFree();
    if (state == State::Both) {
      buffers->initialized = 0;  // aliases the LocalMatrix storage
      delete buffers;
    }
  }

  bool is_mat() const { return state == State::Mat || state == State::Both; }
  bool is_buffs() const { return state == State::Buffs || state == State::Both; }
  bool is_null() const { return state == State::Null; }

  IT nrows() const { return is_mat() ? mat->nrows : is_buffs() ? IT(buffers->ptr_dim - 1) : 0; }
  IT ncols() const { return is_mat() ? mat->ncols : is_buffs() ? IT(buffers->other_dim) : 0; }
  IT nnz() const { return is_mat() ? mat->nnz : is_buffs() ? IT(buffers->nnz) : 0; }

  tspg_csr abi() const {
    if (is_buffs()) return buffers->abi();
    return tspg_trident::abi_of<IT, VT>(mat->nrows, mat->ncols, mat->nnz, mat->ptr_vec, mat->idx_vec,
                                        mat->val);
  }

  // Buffs -> Mat: the tile copied into one contiguous device buffer
  // [val | idx | ptr] (CSX_create_contig_device), buffers released
  // (cusparse_helpers.cuh:248-277).
  void to_mat() {
    if (state != State::Buffs) return;
    const IT m = nrows(), n = ncols(), z = nnz();
    const size_t bytes = mmio::CSX_buf_size<IT, VT>(m, n, z, mmio::MajorDim::ROWS);
    mat = (mmio::CSX<IT, VT> *)std::calloc(1, sizeof(mmio::CSX<IT, VT>));
    mat->majordim = mmio::MajorDim::ROWS;
    mat->nrows = m;
    mat->ncols = n;
    mat->nnz = z;
    mat->contig = true;
    mat->buf_size = bytes;
    TSPG_TRIDENT_CUDA(cudaMalloc(&mat->buf, bytes));
    mmio::CSX_get_ptrs<IT, VT>(m, n, z, mat->buf, &mat->ptr_vec, &mat->idx_vec, &mat->val);
    cudaStream_t s = buffers->s();
    TSPG_TRIDENT_CUDA(cudaMemcpyAsync(mat->val, buffers->d_node_vals, sizeof(VT) * size_t(z),
                                      cudaMemcpyDeviceToDevice, s));
    TSPG_TRIDENT_CUDA(cudaMemcpyAsync(mat->idx_vec, buffers->d_node_colinds, sizeof(IT) * size_t(z),
                                      cudaMemcpyDeviceToDevice, s));
    TSPG_TRIDENT_CUDA(cudaMemcpyAsync(mat->ptr_vec, buffers->d_node_rowptrs, sizeof(IT) * (size_t(m) + 1),
                                      cudaMemcpyDeviceToDevice, s));
    TSPG_TRIDENT_CUDA(cudaStreamSynchronize(s));
    buffers->explicitFree();
    state = State::Mat;
  }

 private:
  std::unique_ptr<tspg_trident::FreshOut<IT, VT>> converted_;
};

// cusparse_spgeam (cusparse_helpers.cuh:799-905): C_accum = C_prod + C_local,
// union pattern; C_accum's buffers grow to the result.
template <typename IT, typename VT>
void cusparse_spgeam(cusparseHandle_t *, CusparseCSX<IT, VT> *C_prod, CusparseCSX<IT, VT> *C_local,
                     CusparseCSX<IT, VT> *C_accum) {
  const tspg_csr p = C_prod->abi(), l = C_local->abi();
  CsxBuffers<IT, VT> *acc = C_accum->buffers;
  cudaStream_t s = C_local->buffers && C_local->buffers->stream ? *C_local->buffers->stream
                                                                 : cudaStreamPerThread;
  tspg_csr_out o = acc->out(C_prod->nrows(), C_prod->ncols());
  TSPG_TRIDENT_CHECK(tspg_spadd(tspg_trident::thread_ctx(), s, &p, &l, &o));
  acc->commit(o);
  TSPG_TRIDENT_CUDA(cudaStreamSynchronize(s));
}

// sp_mma_hybrid (cusparse_helpers.cuh:708-739): C_accum = C_local + A·B, then
// swap, skipping an empty product — the stage operation of sparse_summa.cu:99
// and hns_spgemm.cu:969.
template <typename IT, typename VT>
void sp_mma_hybrid(cusparseHandle_t *handle, const LocalMatrix<IT, IT, VT> &A,
                   const LocalMatrix<IT, IT, VT> &B, CusparseCSX<IT, VT> **C_local,
                   CusparseCSX<IT, VT> **C_accum, bool &did_first) {
  LocalMatrix<IT, IT, VT> C_prod = LocalMatrix<IT, IT, VT>::spgemm(A, B);
  if (C_prod.storage.nnz() == 0) return;
  CusparseCSX<IT, VT> C_prod_csx(C_prod);
  did_first = true;
  cusparse_spgeam(handle, &C_prod_csx, *C_local, *C_accum);
  std::free(C_prod_csx.mat);
  std::swap(*C_local, *C_accum);
}

// cusparse_spmma (cusparse_helpers.cuh:744-796): C_prod = A·B into C_prod's
// buffers, then C_accum = C_local + C_prod and swap; returns 0 for an empty
// product.  `memefficient` picked between two cuSPARSE algorithms; the B200
// path has one.
template <typename IT, typename VT>
int cusparse_spmma(cusparseHandle_t *handle, CusparseCSX<IT, VT> *A, CusparseCSX<IT, VT> *B,
                   CusparseCSX<IT, VT> **C_prod, CusparseCSX<IT, VT> **C_accum,
                   CusparseCSX<IT, VT> **C_local, bool memefficient = true) {
  (void)memefficient;
  const tspg_csr a = A->abi(), b = B->abi();
  int64_t mults = 0, upper = 0;
  cudaStream_t s = (*C_prod)->buffers && (*C_prod)->buffers->stream ? *(*C_prod)->buffers->stream
                                                                     : cudaStreamPerThread;
  TSPG_TRIDENT_CHECK(tspg_spgemm_count(tspg_trident::thread_ctx(), s, &a, &b, &mults, &upper));
  if (mults == 0) return 0;
  tspg_csr_out o = (*C_prod)->buffers->out(A->nrows(), B->ncols());
  TSPG_TRIDENT_CHECK(tspg_spgemm(tspg_trident::thread_ctx(), s, &a, &b, &o, TSPG_F_NONE));
  (*C_prod)->buffers->commit(o);
  cusparse_spgeam(handle, *C_prod, *C_local, *C_accum);
  std::swap(*C_local, *C_accum);
  return 1;
}

// COO -> compressed tile on the device: coo_to_row_csx_contig /
// coo_to_col_csx_contig (cusparse_helpers.cuh:17-131) and coo_to_row_csx /
// coo_to_col_csx (kokkos_helpers.cuh:125-184, 280-352).  The reference sorts
// the host triples by the major index and copies the result to the device;
// here the triples are copied as they are and sorted on the device
// (tspg_coo_to_csx): same pointer array and entries per segment, repeated
// coordinates kept, order inside a segment (minor index, input position).
// The result is one contiguous [val | idx | ptr] device buffer (a CSX with
// contig = true; CSX_create_contig_device layout).
namespace tspg_trident {
template <typename IT, typename VT>
mmio::CSX<IT, VT> *coo_to_csx(const mmio::COO<IT, VT> *coo, mmio::MajorDim major) {
  const bool rows = major == mmio::MajorDim::ROWS;
  cudaStream_t s = cudaStreamPerThread;
  const size_t n = size_t(coo->nnz);
  IT *d_row = nullptr, *d_col = nullptr;
  VT *d_val = nullptr;
  TSPG_TRIDENT_CUDA(cudaMallocAsync((void **)&d_row, sizeof(IT) * (n ? n : 1), s));
  TSPG_TRIDENT_CUDA(cudaMallocAsync((void **)&d_col, sizeof(IT) * (n ? n : 1), s));
  TSPG_TRIDENT_CUDA(cudaMallocAsync((void **)&d_val, sizeof(VT) * (n ? n : 1), s));
  if (n) {
    TSPG_TRIDENT_CUDA(cudaMemcpyAsync(d_row, coo->row, sizeof(IT) * n, cudaMemcpyHostToDevice, s));
    TSPG_TRIDENT_CUDA(cudaMemcpyAsync(d_col, coo->col, sizeof(IT) * n, cudaMemcpyHostToDevice, s));
    TSPG_TRIDENT_CUDA(cudaMemcpyAsync(d_val, coo->val, sizeof(VT) * n, cudaMemcpyHostToDevice, s));
  }
  mmio::CSX<IT, VT> *csx = (mmio::CSX<IT, VT> *)std::calloc(1, sizeof(mmio::CSX<IT, VT>));
  csx->majordim = major;
  csx->nrows = coo->nrows;
  csx->ncols = coo->ncols;
  csx->nnz = coo->nnz;
  csx->contig = true;
  csx->buf_size = mmio::CSX_buf_size<IT, VT>(coo->nrows, coo->ncols, coo->nnz, major);
  TSPG_TRIDENT_CUDA(cudaMalloc(&csx->buf, csx->buf_size));
  mmio::CSX_get_ptrs<IT, VT>(coo->nrows, coo->ncols, coo->nnz, csx->buf, &csx->ptr_vec, &csx->idx_vec,
                             &csx->val);
  tspg_csr_out o{};
  o.nrows = rows ? coo->nrows : coo->ncols;
  o.ncols = rows ? coo->ncols : coo->nrows;
  o.rowptr = csx->ptr_vec;
  o.rowptr_bits = 32;
  o.val_bits = int32_t(sizeof(VT) * 8);
  o.col = csx->idx_vec;
  o.val = csx->val;
  o.capacity = int64_t(n);
  TSPG_TRIDENT_CHECK(tspg_coo_to_csx(thread_ctx(), s, coo->nrows, coo->ncols, coo->nnz, d_row, d_col, d_val,
                                     int(sizeof(VT) * 8), rows ? TSPG_ROWS : TSPG_COLS, &o));
  cudaFreeAsync(d_row, s);
  cudaFreeAsync(d_col, s);
  cudaFreeAsync(d_val, s);
  TSPG_TRIDENT_CUDA(cudaStreamSynchronize(s));
  return csx;
}
}  // namespace tspg_trident

template <typename IT, typename VT>
mmio::CSX<IT, VT> *coo_to_row_csx_contig(mmio::COO<IT, VT> *coo) {
  return tspg_trident::coo_to_csx(coo, mmio::MajorDim::ROWS);
}
template <typename IT, typename VT>
mmio::CSX<IT, VT> *coo_to_col_csx_contig(mmio::COO<IT, VT> *coo) {
  return tspg_trident::coo_to_csx(coo, mmio::MajorDim::COLS);
}
template <typename IT, typename VT>
mmio::CSX<IT, VT> *coo_to_row_csx(mmio::COO<IT, VT> *coo) {
  return tspg_trident::coo_to_csx(coo, mmio::MajorDim::ROWS);
}
template <typename IT, typename VT>
mmio::CSX<IT, VT> *coo_to_col_csx(mmio::COO<IT, VT> *coo) {
  return tspg_trident::coo_to_csx(coo, mmio::MajorDim::COLS);
}

// rownnz_to_rowptrs / rowptrs_to_rownnz (utils.cuh:412-448): in place on the
// device, synchronising `stream` as the reference does.
template <typename IT>
void rownnz_to_rowptrs(IT *d_rowptrs, const IT nrows, cudaStream_t stream = 0, void * = nullptr) {
  TSPG_TRIDENT_CHECK(tspg_rownnz_to_rowptrs(tspg_trident::thread_ctx(), stream, d_rowptrs,
                                            int(sizeof(IT) * 8), int64_t(nrows)));
  TSPG_TRIDENT_CUDA(cudaStreamSynchronize(stream));
}
template <typename IT>
void rowptrs_to_rownnz(IT *d_rowptrs, const IT nrows, cudaStream_t stream = 0, void * = nullptr) {
  TSPG_TRIDENT_CHECK(tspg_rowptrs_to_rownnz(tspg_trident::thread_ctx(), stream, d_rowptrs,
                                            int(sizeof(IT) * 8), int64_t(nrows)));
  TSPG_TRIDENT_CUDA(cudaStreamSynchronize(stream));
}

// ---------------------------------------------------------------------------
namespace SpaComm {

// gen_bitmask (spacomm.cuh:29-117): byte w bit b set iff segment 8w + b of
// ptr_d is non-empty; MASK_SIZE = 8.  The caller frees the result.
template <typename IT>
BMASK_TYPE *gen_bitmask(const IT *ptr_d, int n, int mask_size) {
  if (mask_size != 8) {
    std::fprintf(stderr, "libtspg: MASK_SIZE must be 8 (BMASK_TYPE uint8_t)\n");
    std::exit(EXIT_FAILURE);
  }
  BMASK_TYPE *out = nullptr;
  const size_t bytes = size_t((n + 7) / 8 > 0 ? (n + 7) / 8 : 1);
  TSPG_TRIDENT_CUDA(cudaMalloc(&out, bytes));
  TSPG_TRIDENT_CHECK(tspg_bitmask_gen(tspg_trident::thread_ctx(), cudaStreamPerThread, ptr_d,
                                      int(sizeof(IT) * 8), n, out));
  TSPG_TRIDENT_CUDA(cudaStreamSynchronize(cudaStreamPerThread));
  return out;
}

// intersect_bitmasks (spacomm.cuh:126-148): a & b over n elements; the caller
// frees the result.
template <typename T>
T *intersect_bitmasks(const T *a, const T *b, int n) {
  T *out = nullptr;
  TSPG_TRIDENT_CUDA(cudaMalloc(&out, sizeof(T) * (n > 0 ? n : 1)));
  TSPG_TRIDENT_CHECK(tspg_bitmask_and(tspg_trident::thread_ctx(), cudaStreamPerThread,
                                      (const uint8_t *)a, (const uint8_t *)b,
                                      int64_t(n) * int64_t(sizeof(T)), (uint8_t *)out));
  TSPG_TRIDENT_CUDA(cudaStreamSynchronize(cudaStreamPerThread));
  return out;
}

// SpaCommBuffers (spacomm.cuh:634-712): the send buffer of one packed tile,
// sized for the whole unpacked tile, with the [val | idx | ptr] pointers.
template <typename IT, typename VT>
struct SpaCommBuffers {
  bool initialized = false;
  VT *compressed_values = nullptr;
  IT *compressed_indices = nullptr;
  IT *compressed_pointers = nullptr;
  char *d_buf = nullptr;
  size_t d_buf_size = 0;

  explicit SpaCommBuffers(mmio::CSX<IT, VT> *to_compress) {
    initialized = true;
    d_buf_size = mmio::CSX_buf_size<IT, VT>(to_compress);
    TSPG_TRIDENT_CUDA(cudaMalloc(&d_buf, d_buf_size));
    set_ptrs(to_compress->nnz);
  }
  SpaCommBuffers(const SpaCommBuffers &) = delete;
  SpaCommBuffers &operator=(const SpaCommBuffers &) = delete;
  void set_ptrs(const IT nnz) {
    compressed_values = nnz > 0 ? (VT *)d_buf : nullptr;
    compressed_indices = nnz > 0 ? (IT *)(d_buf + size_t(nnz) * sizeof(VT)) : nullptr;
    compressed_pointers = (IT *)(d_buf + size_t(nnz) * (sizeof(VT) + sizeof(IT)));
  }
  void explicitFree() {
    if (d_buf) cudaFree(d_buf);
    d_buf = nullptr;
    initialized = false;
  }
  ~SpaCommBuffers() {
    if (initialized) explicitFree();
  }
};

// select_ptrs (spacomm.cuh:556-623): the pointer array of a packed tile in
// place — masked segments become empty, length unchanged.
template <typename IT>
IT *select_ptrs(IT *raw_ptr, int m, BMASK_TYPE *mask, cudaStream_t stream = 0, void * = nullptr) {
  TSPG_TRIDENT_CHECK(tspg_select_ptrs(tspg_trident::thread_ctx(), stream, raw_ptr, int(sizeof(IT) * 8),
                                      int64_t(m) - 1, mask));
  TSPG_TRIDENT_CUDA(cudaStreamSynchronize(stream));
  return raw_ptr;
}

// SpaCommHandler (spacomm.cuh:960-1120).  The reference builds the stage
// filters with an MPI exchange of bitmasks (spcomm_2D); on one GPU both tiles
// of a stage are local and the filters come from the fused flop-count pass
// (tspg_spgemm_count_mask), so the handler takes them ready-made: nfilters
// stages of mask_len bytes each, A column filters and B row filters, device
// memory the handler does not own.
template <typename IT, typename VT>
struct SpaCommHandler {
  BMASK_TYPE *A_column_filters = nullptr;
  BMASK_TYPE *B_rows_filters = nullptr;
  int nfilters = 0;
  IT mask_len = 0;
  IT sub_mask_len = 0;
  int node_size = 1, node_rank = 0;
  bool initialized = false;

  SpaCommHandler(BMASK_TYPE *a_column_filters, BMASK_TYPE *b_rows_filters, int n_filters, IT mlen,
                 int node_size_ = 1, int node_rank_ = 0)
      : A_column_filters(a_column_filters),
        B_rows_filters(b_rows_filters),
        nfilters(n_filters),
        mask_len(mlen),
        sub_mask_len(mlen / (node_size_ > 0 ? node_size_ : 1)),
        node_size(node_size_),
        node_rank(node_rank_),
        initialized(true) {}

  // Compress (spacomm.cuh:962-1091): the stage mask is sliced as the reference
  // slices it — B_rows_filters + mask_len * iteration + node_rank * sub_mask_len
  // for a CSR tile, A_column_filters + mask_len * iteration for a CSC tile —
  // and the kept entries, their indices and the pointer array land in
  // buffs->d_buf; the result is a contiguous CSX over that buffer (malloc'ed
  // struct, caller frees).
  mmio::CSX<IT, VT> *Compress(const mmio::CSX<IT, VT> *M, int iteration_number, SpaCommBuffers<IT, VT> *buffs,
                              cudaStream_t stream = 0, MPI_Comm comm = MPI_COMM_WORLD) {
    (void)comm;
    if (iteration_number < 0 || iteration_number >= nfilters) {
      std::fprintf(stderr, "ERROR: provided an invalid iteration number\n");
      std::exit(EXIT_FAILURE);
    }
    const bool rows = M->majordim == mmio::MajorDim::ROWS;
    const int64_t ptr_size = int64_t(rows ? M->nrows : M->ncols) + 1;
    BMASK_TYPE *mask = rows ? B_rows_filters + int64_t(mask_len) * iteration_number + int64_t(node_rank) * sub_mask_len
                            : A_column_filters + int64_t(mask_len) * iteration_number;
    const int64_t considered = rows ? sub_mask_len : mask_len;
    if (ptr_size - 1 != considered * MASK_SIZE) {
      std::fprintf(stderr, "ptr_size-1 must be equal to considered_mask_len*MASK_SIZE (%lld,%lld)\n",
                   (long long)(ptr_size - 1), (long long)(considered * MASK_SIZE));
      std::exit(EXIT_FAILURE);
    }
    tspg_csr m = tspg_trident::abi_of<IT, VT>(M->nrows, M->ncols, M->nnz, M->ptr_vec, M->idx_vec, M->val);
    int64_t kept = 0;
    TSPG_TRIDENT_CHECK(tspg_pack(tspg_trident::thread_ctx(), stream, &m, rows ? TSPG_ROWS : TSPG_COLS, mask,
                                 buffs->d_buf, buffs->d_buf_size, nullptr, &kept));
    buffs->set_ptrs(IT(kept));
    mmio::CSX<IT, VT> *out = (mmio::CSX<IT, VT> *)std::calloc(1, sizeof(mmio::CSX<IT, VT>));
    out->majordim = M->majordim;
    out->nnz = IT(kept);
    out->nrows = M->nrows;
    out->ncols = M->ncols;
    out->contig = true;
    out->buf_size = mmio::CSX_buf_size<IT, VT>(M->nrows, M->ncols, IT(kept), M->majordim);
    out->buf = buffs->d_buf;
    mmio::CSX_get_ptrs<IT, VT>(M->nrows, M->ncols, IT(kept), out->buf, &buffs->compressed_pointers,
                               &buffs->compressed_indices, &buffs->compressed_values);
    out->ptr_vec = buffs->compressed_pointers;
    out->idx_vec = buffs->compressed_indices;
    out->val = buffs->compressed_values;
    return out;
  }

  void explicitFree() { initialized = false; }
};

}  // namespace SpaComm
