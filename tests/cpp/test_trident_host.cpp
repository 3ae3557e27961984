// C++ GPU test of include/tspg_trident.hpp: the reference's own operator
// signatures over libtspg, driven by the reference's own call sequences.
//
//  * SpaComm known answers of test/test_compression.cu (gen_bitmask and
//    intersect_bitmasks :550-590; tmp_test1 :106-238 through
//    SpaCommHandler::Compress, with the production MASK_SIZE = 8), select_ptrs
//    and the rownnz <-> rowptrs round trip;
//  * the stage loop of src/sparse_summa.cu:63-99 on one GPU: for every output
//    tile C(i,j) of a q x q grid, per stage p the A(i,p) and B(p,j) tiles are
//    compressed with the stage filter (SpaCommHandler::Compress), wrapped as
//    CusparseCSX(&handle, csx, nullptr) (the CSC A tile converted to CSR),
//    viewed as LocalMatrix and accumulated with sp_mma_hybrid into
//    C_local / C_accum over CsxBuffers; C_local->to_mat() is then compared
//    with a dense host product — in FP64 and in the reference's FP32;
//  * LocalMatrix::sp_mma / ::spadd and cusparse_spmma on the same tiles;
//  * the COO builders (coo_to_row_csx_contig / coo_to_col_csx_contig).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "tspg_trident.hpp"

static int failures = 0;
#define EXPECT(cond, what)                                             \
  do {                                                                 \
    if (!(cond)) {                                                     \
      std::printf("FAIL %s (%s:%d)\n", what, __FILE__, __LINE__);      \
      ++failures;                                                      \
    }                                                                  \
  } while (0)

template <typename T>
static T *to_dev(const std::vector<T> &h) {
  T *d = nullptr;
  TSPG_TRIDENT_CUDA(cudaMalloc(&d, sizeof(T) * (h.empty() ? 1 : h.size())));
  if (!h.empty()) TSPG_TRIDENT_CUDA(cudaMemcpy(d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
  return d;
}

template <typename T>
static std::vector<T> to_host(const T *d, size_t n) {
  std::vector<T> h(n);
  if (n) TSPG_TRIDENT_CUDA(cudaMemcpy(h.data(), d, sizeof(T) * n, cudaMemcpyDeviceToHost));
  return h;
}

// host CSR / CSC of a dense tile
struct HostTile {
  int nrows, ncols;
  std::vector<double> d;  // row-major dense
};

template <typename VT>
static mmio::CSX<int32_t, VT> *device_tile(const HostTile &t, mmio::MajorDim major) {
  const bool rows = major == mmio::MajorDim::ROWS;
  const int len = rows ? t.nrows : t.ncols, other = rows ? t.ncols : t.nrows;
  std::vector<int32_t> ptr(len + 1, 0), idx;
  std::vector<VT> val;
  for (int a = 0; a < len; ++a) {
    for (int b = 0; b < other; ++b) {
      const double v = rows ? t.d[size_t(a) * t.ncols + b] : t.d[size_t(b) * t.ncols + a];
      if (v != 0.0) {
        idx.push_back(b);
        val.push_back(VT(v));
      }
    }
    ptr[a + 1] = int32_t(idx.size());
  }
  auto *c = (mmio::CSX<int32_t, VT> *)std::calloc(1, sizeof(mmio::CSX<int32_t, VT>));
  c->majordim = major;
  c->nrows = t.nrows;
  c->ncols = t.ncols;
  c->nnz = int32_t(idx.size());
  c->ptr_vec = to_dev(ptr);
  c->idx_vec = to_dev(idx);
  c->val = to_dev(val);
  return c;
}

template <typename VT>
static std::vector<double> dense_of(const mmio::CSX<int32_t, VT> *c) {
  auto rp = to_host(c->ptr_vec, size_t(c->nrows) + 1);
  auto ci = to_host(c->idx_vec, size_t(c->nnz));
  auto v = to_host(c->val, size_t(c->nnz));
  std::vector<double> d(size_t(c->nrows) * c->ncols, 0.0);
  for (int i = 0; i < c->nrows; ++i) {
    for (int p = rp[i]; p < rp[i + 1]; ++p) d[size_t(i) * c->ncols + ci[p]] += double(v[p]);
    for (int p = rp[i] + 1; p < rp[i + 1]; ++p)
      if (ci[p] <= ci[p - 1]) ++failures, std::printf("FAIL unsorted row %d\n", i);
  }
  return d;
}

static uint64_t lcg_state = 12345;
static double lcg() {
  lcg_state = lcg_state * 6364136223846793005ull + 1442695040888963407ull;
  return double(lcg_state >> 11) * (1.0 / 9007199254740992.0);
}

// the SUMMA loop of src/sparse_summa.cu:63-99 for one output tile
template <typename VT>
static std::vector<double> summa_tile(cusparseHandle_t &handle, const std::vector<std::vector<HostTile>> &T,
                                      int q, int i, int j, int tile) {
  cudaStream_t stream = cudaStreamPerThread;
  // stage filters: column mask of A(i,p) AND row mask of B(p,j), mask_len
  // bytes per stage, the same bytes for both operands (one GPU)
  const int mask_len = tile / MASK_SIZE;
  std::vector<mmio::CSX<int32_t, VT> *> Acsc(q), Bcsr(q);
  BMASK_TYPE *filters = nullptr;
  TSPG_TRIDENT_CUDA(cudaMalloc(&filters, size_t(q) * mask_len));
  for (int p = 0; p < q; ++p) {
    Acsc[p] = device_tile<VT>(T[i][p], mmio::MajorDim::COLS);
    Bcsr[p] = device_tile<VT>(T[p][j], mmio::MajorDim::ROWS);
    BMASK_TYPE *ca = SpaComm::gen_bitmask(Acsc[p]->ptr_vec, tile, MASK_SIZE);
    BMASK_TYPE *rb = SpaComm::gen_bitmask(Bcsr[p]->ptr_vec, tile, MASK_SIZE);
    BMASK_TYPE *f = SpaComm::intersect_bitmasks(ca, rb, mask_len);
    TSPG_TRIDENT_CUDA(cudaMemcpy(filters + size_t(p) * mask_len, f, mask_len, cudaMemcpyDeviceToDevice));
    cudaFree(ca);
    cudaFree(rb);
    cudaFree(f);
  }
  SpaComm::SpaCommHandler<int32_t, VT> handler(filters, filters, q, mask_len);
  CsxBuffers<int32_t, VT> *C_accum_buffs = new CsxBuffers<int32_t, VT>(64, tile + 1, tile, &stream, 1, true);
  CsxBuffers<int32_t, VT> *C_local_buffs = new CsxBuffers<int32_t, VT>(64, tile + 1, tile, &stream, 1, true);
  CusparseCSX<int32_t, VT> *C_accum = new CusparseCSX<int32_t, VT>(C_accum_buffs);
  CusparseCSX<int32_t, VT> *C_local = new CusparseCSX<int32_t, VT>(C_local_buffs);
  bool did_one_spgemm = false;
  for (int p = 0; p < q; ++p) {
    SpaComm::SpaCommBuffers<int32_t, VT> bufA(Acsc[p]), bufB(Bcsr[p]);
    mmio::CSX<int32_t, VT> *A_sent = handler.Compress(Acsc[p], p, &bufA, stream);
    mmio::CSX<int32_t, VT> *B_sent = handler.Compress(Bcsr[p], p, &bufB, stream);
    CusparseCSX<int32_t, VT> *A_remote = new CusparseCSX<int32_t, VT>(&handle, A_sent, nullptr);
    TSPG_TRIDENT_CUDA(cudaStreamSynchronize(stream));
    CusparseCSX<int32_t, VT> *B_remote = new CusparseCSX<int32_t, VT>(&handle, B_sent, nullptr);
    TSPG_TRIDENT_CUDA(cudaStreamSynchronize(stream));
    if (A_remote->nnz() > 0 && B_remote->nnz() > 0) {
      LocalMatrix<int32_t, int32_t, VT> A_p(A_remote->mat);
      LocalMatrix<int32_t, int32_t, VT> B_p(B_remote->mat);
      sp_mma_hybrid(&handle, A_p, B_p, &C_local, &C_accum, did_one_spgemm);
    }
    TSPG_TRIDENT_CUDA(cudaStreamSynchronize(stream));
    delete A_remote;
    delete B_remote;
    std::free(A_sent);
    std::free(B_sent);
  }
  EXPECT(did_one_spgemm, "summa did_one_spgemm");
  delete C_accum;
  C_local->to_mat();
  std::vector<double> out = dense_of(C_local->mat);
  cudaFree(C_local->mat->buf);
  std::free(C_local->mat);
  delete C_local;
  delete C_accum_buffs;
  delete C_local_buffs;
  for (int p = 0; p < q; ++p) {
    for (auto *c : {Acsc[p], Bcsr[p]}) {
      cudaFree(c->ptr_vec);
      cudaFree(c->idx_vec);
      cudaFree(c->val);
      std::free(c);
    }
  }
  cudaFree(filters);
  return out;
}

template <typename VT>
static void run_summa(const char *name, double tol) {
  const int q = 3, tile = 128, n = q * tile;
  lcg_state = 777;
  std::vector<double> M(size_t(n) * n, 0.0);
  for (int r = 0; r < n; ++r) {
    // rows of mixed length; a band of empty rows and columns so the masks drop entries
    if (r % 11 == 5) continue;
    const int k = 1 + int(lcg() * (r < 16 ? 60 : 12));
    for (int e = 0; e < k; ++e) {
      int c = int(lcg() * n);
      if (c % 13 == 7) c = (c + 1) % n;
      M[size_t(r) * n + c] = 2.0 * lcg() - 1.0;
    }
  }
  std::vector<std::vector<HostTile>> T(q, std::vector<HostTile>(q));
  for (int a = 0; a < q; ++a)
    for (int b = 0; b < q; ++b) {
      T[a][b] = {tile, tile, std::vector<double>(size_t(tile) * tile)};
      for (int r = 0; r < tile; ++r)
        for (int c = 0; c < tile; ++c) T[a][b].d[size_t(r) * tile + c] = M[size_t(a * tile + r) * n + b * tile + c];
    }
  cusparseHandle_t handle = nullptr;
  for (int i = 0; i < q; ++i)
    for (int j = 0; j < q; ++j) {
      std::vector<double> want(size_t(tile) * tile, 0.0), scale(size_t(tile) * tile, 0.0);
      for (int r = 0; r < tile; ++r)
        for (int c = 0; c < tile; ++c)
          for (int k = 0; k < n; ++k) {
            const double x = M[size_t(i * tile + r) * n + k] * M[size_t(k) * n + j * tile + c];
            want[size_t(r) * tile + c] += x;
            scale[size_t(r) * tile + c] += std::fabs(x);
          }
      std::vector<double> got = summa_tile<VT>(handle, T, q, i, j, tile);
      bool ok = got.size() == want.size();
      for (size_t e = 0; ok && e < want.size(); ++e)
        ok = std::fabs(got[e] - want[e]) <= tol * std::max(std::fabs(want[e]), scale[e]);
      if (!ok) std::printf("FAIL %s summa tile (%d,%d)\n", name, i, j), ++failures;
    }
  // LocalMatrix::sp_mma, ::spadd and cusparse_spmma on tile row 0 / column 0
  {
    LocalMatrix<int32_t, int32_t, VT> C, S;
    std::vector<double> want(size_t(tile) * tile, 0.0);
    CsxBuffers<int32_t, VT> acc_b(1, tile + 1, tile), loc_b(1, tile + 1, tile), prod_b(1, tile + 1, tile);
    CusparseCSX<int32_t, VT> *acc = new CusparseCSX<int32_t, VT>(&acc_b), *loc = new CusparseCSX<int32_t, VT>(&loc_b),
                             *prod = new CusparseCSX<int32_t, VT>(&prod_b);
    for (int p = 0; p < q; ++p) {
      mmio::CSX<int32_t, VT> *a = device_tile<VT>(T[0][p], mmio::MajorDim::ROWS);
      mmio::CSX<int32_t, VT> *b = device_tile<VT>(T[p][0], mmio::MajorDim::ROWS);
      LocalMatrix<int32_t, int32_t, VT> A(a), B(b);
      LocalMatrix<int32_t, int32_t, VT>::sp_mma(A, B, C);
      LocalMatrix<int32_t, int32_t, VT> P = LocalMatrix<int32_t, int32_t, VT>::spgemm(A, B);
      LocalMatrix<int32_t, int32_t, VT>::spadd(P, S);
      CusparseCSX<int32_t, VT> Ac(a), Bc(b);
      cusparse_spmma(&handle, &Ac, &Bc, &prod, &acc, &loc);
      for (int r = 0; r < tile; ++r)
        for (int c = 0; c < tile; ++c)
          for (int k = 0; k < tile; ++k)
            want[size_t(r) * tile + c] += T[0][p].d[size_t(r) * tile + k] * T[p][0].d[size_t(k) * tile + c];
      TSPG_TRIDENT_CUDA(cudaDeviceSynchronize());
      cudaFree(a->ptr_vec), cudaFree(a->idx_vec), cudaFree(a->val), std::free(a);
      cudaFree(b->ptr_vec), cudaFree(b->idx_vec), cudaFree(b->val), std::free(b);
    }
    auto check = [&](const std::vector<double> &got, const char *what) {
      bool ok = true;
      for (size_t e = 0; e < want.size(); ++e) ok = ok && std::fabs(got[e] - want[e]) <= tol * (1.0 + std::fabs(want[e])) * 8;
      if (!ok) std::printf("FAIL %s %s\n", name, what), ++failures;
    };
    mmio::CSX<int32_t, VT> *cx = C.get_csx(), *sx = S.get_csx(), *lx = loc->buffers->to_mmio_csx();
    check(dense_of(cx), "LocalMatrix::sp_mma");
    check(dense_of(sx), "LocalMatrix::spadd");
    check(dense_of(lx), "cusparse_spmma");
    std::free(cx), std::free(sx), std::free(lx);
    delete acc, delete loc, delete prod;
  }
}

int main() {
  TSPG_TRIDENT_CUDA(cudaSetDevice(0));
  // gen_bitmask / intersect_bitmasks known answers
  {
    const std::vector<std::vector<int32_t>> ptrs = {
        {0, 0, 1, 1, 3, 3, 6, 6}, {0, 1, 2, 2, 3, 4, 4, 5, 6}, {0, 0, 1, 2, 2, 3, 4, 4, 5}};
    const uint8_t want[3] = {0x2A, 0xDB, 0xB6};
    BMASK_TYPE *m[3];
    for (int i = 0; i < 3; ++i) {
      int32_t *d = to_dev(ptrs[i]);
      m[i] = SpaComm::gen_bitmask(d, int(ptrs[i].size()) - 1, MASK_SIZE);
      EXPECT(to_host(m[i], 1)[0] == want[i], "gen_bitmask");
      cudaFree(d);
    }
    BMASK_TYPE *x = SpaComm::intersect_bitmasks(m[1], m[2], 1);
    EXPECT(to_host(x, 1)[0] == 0x92, "intersect_bitmasks");
    cudaFree(x);
    for (auto p : m) cudaFree(p);
  }
  // tmp_test1 through SpaCommHandler::Compress (FP32, the reference's type):
  // B_rows_filters = {3}: rows 0 and 1 kept
  {
    std::vector<float> val;
    for (int i = 1; i <= 27; ++i) val.push_back(float(i));
    std::vector<int32_t> col = {0, 1, 3, 7, 0, 1, 4, 7, 8, 10, 0, 2, 4, 6,
                                8, 1, 3, 5, 7, 9, 2, 8, 1, 5, 7, 0, 10};
    std::vector<int32_t> row = {0, 1, 4, 10, 15, 20, 22, 25, 27};
    mmio::CSX<int32_t, float> M{};
    M.majordim = mmio::MajorDim::ROWS;
    M.nrows = 8;
    M.ncols = 11;
    M.nnz = 27;
    M.ptr_vec = to_dev(row);
    M.idx_vec = to_dev(col);
    M.val = to_dev(val);
    std::vector<uint8_t> hmask = {3, 9};
    BMASK_TYPE *filters = to_dev(hmask);
    SpaComm::SpaCommHandler<int32_t, float> h(filters, filters, 1, 1);
    SpaComm::SpaCommBuffers<int32_t, float> buffs(&M);
    mmio::CSX<int32_t, float> *P = h.Compress(&M, 0, &buffs, 0);
    EXPECT(P->nnz == 4 && P->contig, "Compress nnz");
    auto pc = to_host(P->idx_vec, 4);
    auto pv = to_host(P->val, 4);
    auto pp = to_host(P->ptr_vec, 9);
    const int32_t wc[4] = {0, 1, 3, 7};
    const int32_t wp[9] = {0, 1, 4, 4, 4, 4, 4, 4, 4};
    for (int i = 0; i < 4; ++i) EXPECT(pc[i] == wc[i] && pv[i] == float(i + 1), "Compress entries");
    for (int i = 0; i < 9; ++i) EXPECT(pp[i] == wp[i], "Compress ptr");
    EXPECT(P->buf == buffs.d_buf && P->ptr_vec == buffs.compressed_pointers, "Compress layout");
    // select_ptrs on its own: the same pointer array
    int32_t *rp = to_dev(row);
    SpaComm::select_ptrs(rp, 9, filters, 0);
    auto sp = to_host(rp, 9);
    for (int i = 0; i < 9; ++i) EXPECT(sp[i] == wp[i], "select_ptrs");
    // rowptrs -> rownnz -> rowptrs
    int32_t *rr = to_dev(row);
    rowptrs_to_rownnz(rr, 8, 0);
    auto cnt = to_host(rr, 9);
    for (int i = 0; i < 8; ++i) EXPECT(cnt[i + 1] == row[i + 1] - row[i], "rowptrs_to_rownnz");
    rownnz_to_rowptrs(rr, 8, 0);
    EXPECT(to_host(rr, 9) == row, "rownnz_to_rowptrs");
    std::free(P);
    cudaFree(rp), cudaFree(rr), cudaFree(filters);
    cudaFree(M.ptr_vec), cudaFree(M.idx_vec), cudaFree(M.val);
  }
  // the SUMMA stage loop, FP64 and FP32
  run_summa<double>("fp64", 1e-12);
  run_summa<float>("fp32", 2e-5);
  // COO -> CSR and CSC, a repeated coordinate kept
  {
    std::vector<int32_t> r = {2, 0, 2, 1, 0, 2}, c = {1, 3, 0, 2, 3, 1};
    std::vector<double> v = {1, 2, 3, 4, 5, 6};
    mmio::COO<int32_t, double> coo{3, 4, 6, r.data(), c.data(), v.data()};
    mmio::CSX<int32_t, double> *R = coo_to_row_csx_contig(&coo);
    EXPECT(R->nnz == 6 && R->contig, "coo_to_row_csx nnz");
    EXPECT((to_host(R->ptr_vec, 4) == std::vector<int32_t>{0, 2, 3, 6}), "coo_to_row_csx ptr");
    EXPECT((to_host(R->idx_vec, 6) == std::vector<int32_t>{3, 3, 2, 0, 1, 1}), "coo_to_row_csx idx");
    EXPECT((to_host(R->val, 6) == std::vector<double>{2, 5, 4, 3, 1, 6}), "coo_to_row_csx val");
    mmio::CSX<int32_t, double> *K = coo_to_col_csx_contig(&coo);
    EXPECT((to_host(K->ptr_vec, 5) == std::vector<int32_t>{0, 1, 3, 4, 6}), "coo_to_col_csx ptr");
    EXPECT((to_host(K->idx_vec, 6) == std::vector<int32_t>{2, 2, 2, 1, 0, 0}), "coo_to_col_csx idx");
    EXPECT((to_host(K->val, 6) == std::vector<double>{3, 1, 6, 4, 2, 5}), "coo_to_col_csx val");
    cudaFree(R->buf), cudaFree(K->buf), std::free(R), std::free(K);
  }
  std::printf(failures ? "FAILED %d\n" : "ALL OK\n", failures);
  return failures ? 1 : 0;
}
