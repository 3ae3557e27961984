// C++ host test of include/tspg_trident.hpp on a GPU: the known answers of the
// reference's test/test_compression.cu (gen_bitmask :550-590, tmp_test1
// :106-238 with the production MASK_SIZE = 8), a two-stage sp_mma /
// sp_mma_hybrid accumulation checked against a dense product, csc_to_csr and
// the COO builders.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "tspg_trident.hpp"

using namespace tspg_trident;

static int failures = 0;
#define EXPECT(cond, what)                                   \
  do {                                                       \
    if (!(cond)) {                                           \
      std::printf("FAIL %s (%s:%d)\n", what, __FILE__, __LINE__); \
      ++failures;                                            \
    }                                                        \
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

static Csx<int32_t, double> make_csr(int m, int n, std::vector<int32_t> rp, std::vector<int32_t> ci,
                                     std::vector<double> v) {
  Csx<int32_t, double> c;
  c.nrows = m;
  c.ncols = n;
  c.nnz = int32_t(ci.size());
  c.ptr_vec = to_dev(rp);
  c.idx_vec = to_dev(ci);
  c.val = to_dev(v);
  return c;
}

static std::vector<double> dense(const Csx<int32_t, double> &c) {
  auto rp = to_host(c.ptr_vec, c.nrows + 1);
  auto ci = to_host(c.idx_vec, c.nnz);
  auto v = to_host(c.val, c.nnz);
  std::vector<double> d(size_t(c.nrows) * c.ncols, 0.0);
  for (int i = 0; i < c.nrows; ++i)
    for (int p = rp[i]; p < rp[i + 1]; ++p) d[size_t(i) * c.ncols + ci[p]] += v[p];
  return d;
}

int main() {
  Context ctx(0);
  // gen_bitmask / intersect_bitmasks known answers
  {
    const std::vector<std::vector<int32_t>> ptrs = {
        {0, 0, 1, 1, 3, 3, 6, 6}, {0, 1, 2, 2, 3, 4, 4, 5, 6}, {0, 0, 1, 2, 2, 3, 4, 4, 5}};
    const uint8_t want[3] = {0x2A, 0xDB, 0xB6};
    uint8_t *m[3];
    for (int i = 0; i < 3; ++i) {
      int32_t *d = to_dev(ptrs[i]);
      m[i] = SpaComm::gen_bitmask(ctx, d, int(ptrs[i].size()) - 1, 8);
      EXPECT(to_host(m[i], 1)[0] == want[i], "gen_bitmask");
      cudaFree(d);
    }
    uint8_t *x = SpaComm::intersect_bitmasks(ctx, m[1], m[2], 1);
    EXPECT(to_host(x, 1)[0] == 0x92, "intersect_bitmasks");
    cudaFree(x);
    for (auto p : m) cudaFree(p);
  }
  // tmp_test1 through Compress (float values, the reference's FP32 twin)
  {
    std::vector<float> val;
    for (int i = 1; i <= 27; ++i) val.push_back(float(i));
    std::vector<int32_t> col = {0, 1, 3, 7, 0, 1, 4, 7, 8, 10, 0, 2, 4, 6,
                                8, 1, 3, 5, 7, 9, 2, 8, 1, 5, 7, 0, 10};
    std::vector<int32_t> row = {0, 1, 4, 10, 15, 20, 22, 25, 27};
    Csx<int32_t, float> M;
    M.nrows = 8;
    M.ncols = 11;
    M.nnz = 27;
    M.ptr_vec = to_dev(row);
    M.idx_vec = to_dev(col);
    M.val = to_dev(val);
    std::vector<uint8_t> hmask = {3, 9};
    uint8_t *mask = to_dev(hmask);
    const size_t cap = tspg_packed_bytes(27, 8, 32, 32);
    char *buf = nullptr;
    TSPG_TRIDENT_CUDA(cudaMalloc(&buf, cap));
    Csx<int32_t, float> P = SpaComm::Compress(ctx, M, mask, buf, cap);
    EXPECT(P.nnz == 4 && P.contig, "Compress nnz");
    auto pc = to_host(P.idx_vec, 4);
    auto pv = to_host(P.val, 4);
    auto pp = to_host(P.ptr_vec, 9);
    const int32_t wc[4] = {0, 1, 3, 7};
    const int32_t wp[9] = {0, 1, 4, 4, 4, 4, 4, 4, 4};
    for (int i = 0; i < 4; ++i) EXPECT(pc[i] == wc[i] && pv[i] == float(i + 1), "Compress entries");
    for (int i = 0; i < 9; ++i) EXPECT(pp[i] == wp[i], "Compress ptr");
    cudaFree(buf);
    cudaFree(mask);
  }
  // two SUMMA-like stages: C = A0 B0 + A1 B1 through sp_mma, and the same
  // through sp_mma_hybrid / cusparse_spgeam with CsxBuffers
  {
    auto A0 = make_csr(3, 4, {0, 2, 3, 4}, {0, 2, 1, 3}, {1.0, 2.0, 3.0, -1.0});
    auto B0 = make_csr(4, 3, {0, 1, 2, 4, 5}, {0, 2, 0, 1, 2}, {2.0, 1.0, -1.0, 4.0, 0.5});
    auto A1 = make_csr(3, 4, {0, 1, 2, 3}, {3, 0, 2}, {1.5, -2.0, 1.0});
    auto B1 = make_csr(4, 3, {0, 2, 2, 3, 4}, {0, 2, 1, 2}, {1.0, 1.0, 2.0, -3.0});
    std::vector<double> a0 = dense(A0), b0 = dense(B0), a1 = dense(A1), b1 = dense(B1), want(9, 0.0);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 4; ++k)
          want[i * 3 + j] += a0[i * 4 + k] * b0[k * 3 + j] + a1[i * 4 + k] * b1[k * 3 + j];
    LocalMatrix<int32_t, double> C;
    LocalMatrix<int32_t, double>::sp_mma(ctx, A0, B0, C);
    LocalMatrix<int32_t, double>::sp_mma(ctx, A1, B1, C);
    TSPG_TRIDENT_CUDA(cudaDeviceSynchronize());
    auto got = dense(C.get_csx());
    for (int i = 0; i < 9; ++i) EXPECT(std::fabs(got[i] - want[i]) < 1e-12, "sp_mma value");
    CsxBuffers<int32_t, double> b1buf(1, 4, 3), b2buf(1, 4, 3);
    CsxBuffers<int32_t, double> *loc = &b1buf, *accum = &b2buf;
    bool did_first = false;
    sp_mma_hybrid(ctx, A0, B0, &loc, &accum, did_first);
    sp_mma_hybrid(ctx, A1, B1, &loc, &accum, did_first);
    TSPG_TRIDENT_CUDA(cudaDeviceSynchronize());
    auto got2 = dense(loc->view());
    for (int i = 0; i < 9; ++i) EXPECT(std::fabs(got2[i] - want[i]) < 1e-12, "sp_mma_hybrid value");
    EXPECT(did_first, "sp_mma_hybrid did_first");
    // csc_to_csr round trip of A0
    LocalMatrix<int32_t, double> T, TT;
    Csx<int32_t, double> csc = A0;  // A0's arrays read as the CSC of A0^T
    csc.majordim = MajorDim::COLS;
    csc.nrows = 4;
    csc.ncols = 3;
    LocalMatrix<int32_t, double>::csc_to_csr(ctx, csc, T);
    auto t = dense(T.get_csx());
    for (int i = 0; i < 3; ++i)
      for (int k = 0; k < 4; ++k) EXPECT(t[k * 3 + i] == a0[i * 4 + k], "csc_to_csr");
    // COO -> CSR and CSC, with a repeated coordinate: both entries are kept
    // and come in input order
    {
      std::vector<int32_t> r = {2, 0, 2, 1, 0, 2}, c = {1, 3, 0, 2, 3, 1};
      std::vector<double> v = {1, 2, 3, 4, 5, 6};
      int32_t *dr = to_dev(r), *dc = to_dev(c);
      double *dv = to_dev(v);
      CsxBuffers<int32_t, double> R, K;
      coo_to_row_csx(ctx, 3, 4, 6, dr, dc, dv, R);
      auto rp = to_host(R.d_node_rowptrs, 4);
      auto ci = to_host(R.d_node_colinds, 6);
      auto rv = to_host(R.d_node_vals, 6);
      EXPECT(R.nnz == 6, "coo_to_row_csx nnz");
      EXPECT((rp == std::vector<int32_t>{0, 2, 3, 6}), "coo_to_row_csx ptr");
      EXPECT((ci == std::vector<int32_t>{3, 3, 2, 0, 1, 1}), "coo_to_row_csx idx");
      EXPECT((rv == std::vector<double>{2, 5, 4, 3, 1, 6}), "coo_to_row_csx val");
      coo_to_col_csx(ctx, 3, 4, 6, dr, dc, dv, K);
      auto kp = to_host(K.d_node_rowptrs, 5);
      auto ki = to_host(K.d_node_colinds, 6);
      auto kv = to_host(K.d_node_vals, 6);
      EXPECT((kp == std::vector<int32_t>{0, 1, 3, 4, 6}), "coo_to_col_csx ptr");
      EXPECT((ki == std::vector<int32_t>{2, 2, 2, 1, 0, 0}), "coo_to_col_csx idx");
      EXPECT((kv == std::vector<double>{3, 1, 6, 4, 2, 5}), "coo_to_col_csx val");
      cudaFree(dr);
      cudaFree(dc);
      cudaFree(dv);
    }
  }
  std::printf(failures ? "FAILED %d\n" : "ALL OK\n", failures);
  return failures ? 1 : 0;
}
