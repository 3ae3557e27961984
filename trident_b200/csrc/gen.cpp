// gen.cpp — seeded synthetic operands of the benchmark workloads, plus the
// .bmtx reader and a host transpose.  Host code (OpenMP); every random draw
// comes from a counter-based generator (splitmix64 of seed, stream, counter),
// so a matrix depends only on its parameters and seed, never on the thread
// count.  Values are uniform in [-1, 1], one per stored entry, drawn after
// duplicates are merged, indexed by the entry's CSR position.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "tspg_synth.h"

namespace {

inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
inline uint64_t rnd(uint64_t seed, uint64_t stream, uint64_t ctr) {
  return splitmix64(splitmix64(seed ^ splitmix64(stream * 0x632BE59BD9B4E019ull)) + ctr);
}
inline double u01(uint64_t r) { return double(r >> 11) * (1.0 / 9007199254740992.0); }

constexpr uint64_t kValueStream = 0xA5A5A5A5ull;

bool alloc_csr(tspg_host_csr *M, int64_t nrows, int64_t ncols, int64_t nnz) {
  M->nrows = nrows;
  M->ncols = ncols;
  M->nnz = nnz;
  M->rowptr = (int64_t *)std::malloc(sizeof(int64_t) * size_t(nrows + 1));
  M->col = (int32_t *)std::malloc(sizeof(int32_t) * size_t(nnz > 0 ? nnz : 1));
  M->val = (double *)std::malloc(sizeof(double) * size_t(nnz > 0 ? nnz : 1));
  return M->rowptr && M->col && M->val;
}

void fill_values(tspg_host_csr *M, uint64_t seed) {
  const int64_t nnz = M->nnz;
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < nnz; ++e)
    M->val[e] = 2.0 * u01(rnd(seed, kValueStream, uint64_t(e))) - 1.0;
}

// Build CSR from per-row column lists (already sorted and unique).
int from_rows(std::vector<std::vector<int32_t>> &rows, int64_t ncols,
              tspg_host_csr *out) {
  const int64_t n = (int64_t)rows.size();
  std::vector<int64_t> rp(n + 1, 0);
  for (int64_t i = 0; i < n; ++i) rp[i + 1] = rp[i] + (int64_t)rows[i].size();
  if (!alloc_csr(out, n, ncols, rp[n])) return TSPG_ENOMEM;
  std::memcpy(out->rowptr, rp.data(), sizeof(int64_t) * (n + 1));
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t i = 0; i < n; ++i)
    std::copy(rows[i].begin(), rows[i].end(), out->col + rp[i]);
  return TSPG_OK;
}

}  // namespace

extern "C" void tspg_host_free(tspg_host_csr *M) {
  if (!M) return;
  std::free(M->rowptr);
  std::free(M->col);
  std::free(M->val);
  M->rowptr = nullptr;
  M->col = nullptr;
  M->val = nullptr;
}

extern "C" int tspg_gen_uniform_rows(int64_t n, int k, int diag, uint64_t seed,
                                     tspg_host_csr *out) {
  if (!out || n <= 0 || k < 0 || k > n || n > INT32_MAX) return TSPG_EINVAL;
  std::vector<std::vector<int32_t>> rows(n);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < n; ++i) {
    std::vector<int32_t> &r = rows[i];
    r.reserve(k + 1);
    uint64_t ctr = 0;
    while ((int)r.size() < k) {
      const int32_t c = int32_t(rnd(seed, uint64_t(i), ctr++) % uint64_t(n));
      if (std::find(r.begin(), r.end(), c) == r.end()) r.push_back(c);
    }
    if (diag && std::find(r.begin(), r.end(), int32_t(i)) == r.end())
      r.push_back(int32_t(i));
    std::sort(r.begin(), r.end());
  }
  int st = from_rows(rows, n, out);
  if (st == TSPG_OK) fill_values(out, seed);
  return st;
}

extern "C" int tspg_gen_rmat(int scale, int edge_factor, double a, double b,
                             double c, uint64_t seed, tspg_host_csr *out) {
  if (!out || scale < 1 || scale > 30 || edge_factor < 1) return TSPG_EINVAL;
  const int64_t n = int64_t(1) << scale;
  const int64_t E = n * edge_factor;
  const double ab = a + b, abc = a + b + c;
  std::vector<int32_t> er(E), ec(E);
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < E; ++e) {
    int64_t r = 0, q = 0;
    for (int l = 0; l < scale; ++l) {
      const double u = u01(rnd(seed, uint64_t(e), uint64_t(l)));
      const int br = u >= ab;                    // c or d quadrant
      const int bc = (u >= a && u < ab) || u >= abc;  // b or d quadrant
      r = (r << 1) | br;
      q = (q << 1) | bc;
    }
    er[e] = int32_t(r);
    ec[e] = int32_t(q);
  }
  // counting sort by row, then sort + unique inside each row
  std::vector<int64_t> rp(n + 1, 0);
  for (int64_t e = 0; e < E; ++e) ++rp[er[e] + 1];
  for (int64_t i = 0; i < n; ++i) rp[i + 1] += rp[i];
  std::vector<int32_t> cols(E);
  {
    std::vector<int64_t> cur(rp.begin(), rp.end() - 1);
    for (int64_t e = 0; e < E; ++e) cols[cur[er[e]]++] = ec[e];
  }
  std::vector<int64_t> keep(n + 1, 0);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t i = 0; i < n; ++i) {
    int32_t *b0 = cols.data() + rp[i], *b1 = cols.data() + rp[i + 1];
    std::sort(b0, b1);
    keep[i + 1] = std::unique(b0, b1) - b0;
  }
  for (int64_t i = 0; i < n; ++i) keep[i + 1] += keep[i];
  if (!alloc_csr(out, n, n, keep[n])) return TSPG_ENOMEM;
  std::memcpy(out->rowptr, keep.data(), sizeof(int64_t) * (n + 1));
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t i = 0; i < n; ++i)
    std::copy(cols.data() + rp[i], cols.data() + rp[i] + (keep[i + 1] - keep[i]),
              out->col + keep[i]);
  fill_values(out, seed);
  return TSPG_OK;
}

extern "C" int tspg_gen_laplacian(int64_t nx, int64_t ny, int64_t nz, int pts,
                                  tspg_host_csr *out) {
  if (!out || nx < 1 || ny < 1 || nz < 1 || (pts != 7 && pts != 27)) return TSPG_EINVAL;
  const int64_t n = nx * ny * nz;
  if (n > INT32_MAX) return TSPG_EINVAL;
  const double diag = pts == 27 ? 26.0 : 6.0;
  std::vector<int64_t> rp(n + 1, 0);
  auto nbrs = [&](int64_t x, int64_t y, int64_t z, int32_t *cols, double *vals) {
    int cnt = 0;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int nzero = (dx != 0) + (dy != 0) + (dz != 0);
          if (pts == 7 && nzero > 1) continue;
          const int64_t xx = x + dx, yy = y + dy, zz = z + dz;
          if (xx < 0 || yy < 0 || zz < 0 || xx >= nx || yy >= ny || zz >= nz) continue;
          if (cols) {
            cols[cnt] = int32_t(xx + nx * (yy + ny * zz));
            vals[cnt] = nzero == 0 ? diag : -1.0;
          }
          ++cnt;
        }
    return cnt;
  };
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const int64_t x = i % nx, y = (i / nx) % ny, z = i / (nx * ny);
    rp[i + 1] = nbrs(x, y, z, nullptr, nullptr);
  }
  for (int64_t i = 0; i < n; ++i) rp[i + 1] += rp[i];
  if (!alloc_csr(out, n, n, rp[n])) return TSPG_ENOMEM;
  std::memcpy(out->rowptr, rp.data(), sizeof(int64_t) * (n + 1));
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const int64_t x = i % nx, y = (i / nx) % ny, z = i / (nx * ny);
    nbrs(x, y, z, out->col + rp[i], out->val + rp[i]);
  }
  return TSPG_OK;
}

// P = (I - omega D^-1 A) P_tent; row i of P collects, for every j in row i
// of A (column order), coef = [i == j] - (omega / D) A_ij on column agg(j).
extern "C" int tspg_gen_sa_prolongator(int64_t nx, int64_t ny, int64_t nz,
                                       int pts, int agg, double omega,
                                       tspg_host_csr *out) {
  if (!out || agg < 1) return TSPG_EINVAL;
  tspg_host_csr A{};
  int st = tspg_gen_laplacian(nx, ny, nz, pts, &A);
  if (st != TSPG_OK) return st;
  const int64_t n = A.nrows;
  const int64_t ax = (nx + agg - 1) / agg, ay = (ny + agg - 1) / agg,
                az = (nz + agg - 1) / agg;
  const int64_t nagg = ax * ay * az;
  const double D = pts == 27 ? 26.0 : 6.0;
  auto agg_of = [&](int64_t j) {
    const int64_t x = j % nx, y = (j / nx) % ny, z = j / (nx * ny);
    return int32_t((x / agg) + ax * ((y / agg) + ay * (z / agg)));
  };
  std::vector<int64_t> rp(n + 1, 0);
  auto row = [&](int64_t i, int32_t *cols, double *vals) {
    int32_t ka[32];
    double kv[32];
    int cnt = 0;
    for (int64_t p = A.rowptr[i]; p < A.rowptr[i + 1]; ++p) {
      const int64_t j = A.col[p];
      const double coef = (j == i ? 1.0 : 0.0) - (omega / D) * A.val[p];
      const int32_t g = agg_of(j);
      int q = 0;
      while (q < cnt && ka[q] != g) ++q;
      if (q == cnt) {
        ka[cnt] = g;
        kv[cnt] = coef;
        ++cnt;
      } else {
        kv[q] += coef;
      }
    }
    // sort by aggregate id (insertion sort, <= 8 entries)
    for (int x = 1; x < cnt; ++x)
      for (int y = x; y > 0 && ka[y - 1] > ka[y]; --y) {
        std::swap(ka[y - 1], ka[y]);
        std::swap(kv[y - 1], kv[y]);
      }
    if (cols)
      for (int q = 0; q < cnt; ++q) {
        cols[q] = ka[q];
        vals[q] = kv[q];
      }
    return cnt;
  };
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) rp[i + 1] = row(i, nullptr, nullptr);
  for (int64_t i = 0; i < n; ++i) rp[i + 1] += rp[i];
  if (!alloc_csr(out, n, nagg, rp[n])) {
    tspg_host_free(&A);
    return TSPG_ENOMEM;
  }
  std::memcpy(out->rowptr, rp.data(), sizeof(int64_t) * (n + 1));
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) row(i, out->col + rp[i], out->val + rp[i]);
  tspg_host_free(&A);
  return TSPG_OK;
}

extern "C" int tspg_host_transpose(const tspg_host_csr *M, tspg_host_csr *out) {
  if (!M || !out) return TSPG_EINVAL;
  const int64_t m = M->nrows, n = M->ncols, nnz = M->nnz;
  if (!alloc_csr(out, n, m, nnz)) return TSPG_ENOMEM;
  std::vector<int64_t> cnt(n + 1, 0);
  for (int64_t e = 0; e < nnz; ++e) ++cnt[M->col[e] + 1];
  for (int64_t j = 0; j < n; ++j) cnt[j + 1] += cnt[j];
  std::memcpy(out->rowptr, cnt.data(), sizeof(int64_t) * (n + 1));
  for (int64_t i = 0; i < m; ++i)
    for (int64_t p = M->rowptr[i]; p < M->rowptr[i + 1]; ++p) {
      const int64_t o = cnt[M->col[p]]++;
      out->col[o] = int32_t(i);
      out->val[o] = M->val[p];
    }
  return TSPG_OK;
}

extern "C" int tspg_gen_poisson_rows(int64_t rows, double lambda, uint64_t seed,
                                     tspg_host_csr *out) {
  if (!out || rows < 1 || rows > INT32_MAX || !(lambda > 0)) return TSPG_EINVAL;
  std::vector<int64_t> len(rows + 1, 0);
  const double e_l = std::exp(-lambda);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < rows; ++i) {
    // inversion of the Poisson CDF with one uniform
    const double u = u01(rnd(seed, uint64_t(i), 0));
    double pk = e_l, F = e_l;
    int64_t k = 0;
    while (u > F && k < 10 * int64_t(lambda) + 100) {
      ++k;
      pk *= lambda / double(k);
      F += pk;
    }
    len[i + 1] = k < rows ? k : rows;
  }
  for (int64_t i = 0; i < rows; ++i) len[i + 1] += len[i];
  if (!alloc_csr(out, rows, rows, len[rows])) return TSPG_ENOMEM;
  std::memcpy(out->rowptr, len.data(), sizeof(int64_t) * (rows + 1));
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t i = 0; i < rows; ++i) {
    int32_t *r = out->col + len[i];
    const int64_t L = len[i + 1] - len[i];
    int64_t have = 0;
    uint64_t ctr = 1;
    while (have < L) {
      const int32_t c = int32_t(rnd(seed, uint64_t(i), ctr++) % uint64_t(rows));
      bool dup = false;
      for (int64_t q = 0; q < have; ++q)
        if (r[q] == c) { dup = true; break; }
      if (!dup) r[have++] = c;
    }
    std::sort(r, r + L);
  }
  fill_values(out, seed);
  return TSPG_OK;
}

// .bmtx: line 1 "%%MatrixMarket matrix coordinate real general IB VB",
// line 2 "nrows ncols nnz", then nnz records (row: IB bytes, col: IB bytes,
// value: float32 when VB = 4 or float64 when VB = 8), little-endian, 0-based.
extern "C" int tspg_read_bmtx(const char *path, tspg_host_csr *out) {
  if (!path || !out) return TSPG_EINVAL;
  FILE *f = std::fopen(path, "rb");
  if (!f) return TSPG_EINVAL;
  char line[512];
  int ib = 0, vb = 0;
  long long nr = 0, nc = 0, nz = 0;
  int st = TSPG_EINVAL;
  if (std::fgets(line, sizeof line, f)) {
    std::string s(line);
    const size_t p = s.rfind("general");
    if (s.rfind("%%MatrixMarket", 0) == 0 && p != std::string::npos &&
        std::sscanf(s.c_str() + p + 7, "%d %d", &ib, &vb) == 2 &&
        std::fgets(line, sizeof line, f) &&
        std::sscanf(line, "%lld %lld %lld", &nr, &nc, &nz) == 3 && ib >= 1 &&
        ib <= 8 && (vb == 4 || vb == 8) && nr >= 0 && nc >= 0 && nz >= 0)
      st = TSPG_OK;
  }
  if (st != TSPG_OK) {
    std::fclose(f);
    return st;
  }
  const size_t rec = size_t(2 * ib + vb);
  std::vector<unsigned char> buf(rec * size_t(nz));
  if (std::fread(buf.data(), 1, buf.size(), f) != buf.size()) {
    std::fclose(f);
    return TSPG_EINVAL;
  }
  std::fclose(f);
  auto rd = [&](const unsigned char *p, int w) {
    uint64_t v = 0;
    for (int i = 0; i < w; ++i) v |= uint64_t(p[i]) << (8 * i);
    return int64_t(v);
  };
  std::vector<int64_t> r(nz), c(nz);
  std::vector<double> v(nz);
  for (long long e = 0; e < nz; ++e) {
    const unsigned char *p = buf.data() + rec * size_t(e);
    r[e] = rd(p, ib);
    c[e] = rd(p + ib, ib);
    if (vb == 4) {
      float x;
      std::memcpy(&x, p + 2 * ib, 4);
      v[e] = x;
    } else {
      std::memcpy(&v[e], p + 2 * ib, 8);
    }
    if (r[e] >= nr || c[e] >= nc) return TSPG_EINVAL;
  }
  if (!alloc_csr(out, nr, nc, nz)) return TSPG_ENOMEM;
  std::vector<int64_t> cnt(nr + 1, 0);
  for (long long e = 0; e < nz; ++e) ++cnt[r[e] + 1];
  for (long long i = 0; i < nr; ++i) cnt[i + 1] += cnt[i];
  std::memcpy(out->rowptr, cnt.data(), sizeof(int64_t) * size_t(nr + 1));
  for (long long e = 0; e < nz; ++e) {
    const int64_t o = cnt[r[e]]++;
    out->col[o] = int32_t(c[e]);
    out->val[o] = v[e];
  }
  return TSPG_OK;
}
