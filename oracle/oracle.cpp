// oracle.cpp — CPU restatement of Trident's on-node compute semantics.
//
// TEST INFRASTRUCTURE ONLY (see oracle.h): the checker for the CUDA path and
// the timed CPU baseline.  Never linked into or called by the product.
//
// Each function cites the reference code whose behaviour it restates.
// Parallelism: OpenMP over rows, dynamic schedule, one dense accumulator per
// thread (the usual Gustavson CPU layout); results do not depend on the
// thread count because every row is computed by one thread in a fixed order.
#include "oracle.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

extern "C" void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

// Work estimate per row: KokkosSparse::spgemm's internal count and
// cusparseSpGEMM_getNumProducts (include/cusparse_helpers.cuh:981-985).
extern "C" int64_t orc_row_mults(int64_t r0, int64_t r1, const int64_t *Ap,
                                 const int32_t *Aj, const int64_t *Bp,
                                 int64_t *row_mults) {
  int64_t total = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : total)
  for (int64_t i = r0; i < r1; ++i) {
    int64_t s = 0;
    for (int64_t p = Ap[i]; p < Ap[i + 1]; ++p) {
      int64_t k = Aj[p];
      s += Bp[k + 1] - Bp[k];
    }
    if (row_mults) row_mults[i - r0] = s;
    total += s;
  }
  return total;
}

// Structural row counts of C = A·B.  KokkosSparse::spgemm
// (include/KokkosWrap.hpp:375) and cusparseSpGEMM keep every (i,j) reached by
// some product, whatever its value; no drop tolerance is set anywhere in the
// reference.
extern "C" int64_t orc_spgemm_count(int64_t r0, int64_t r1, int64_t ncols,
                                    const int64_t *Ap, const int32_t *Aj,
                                    const int64_t *Bp, const int32_t *Bj,
                                    int64_t *cnt) {
  int64_t total = 0;
#pragma omp parallel reduction(+ : total)
  {
    std::vector<int64_t> mark((size_t)ncols, -1);
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = r0; i < r1; ++i) {
      int64_t c = 0;
      for (int64_t p = Ap[i]; p < Ap[i + 1]; ++p) {
        int64_t k = Aj[p];
        for (int64_t q = Bp[k]; q < Bp[k + 1]; ++q) {
          int32_t j = Bj[q];
          if (mark[j] != i) {
            mark[j] = i;
            ++c;
          }
        }
      }
      if (cnt) cnt[i - r0] = c;
      total += c;
    }
  }
  return total;
}

// Numeric C = A·B, rows sorted by column.  Accumulation order is fixed: A's
// row in stored order, and within it B's row k in stored order, all in FP64.
extern "C" int orc_spgemm_numeric(int64_t r0, int64_t r1, int64_t ncols,
                                  const int64_t *Ap, const int32_t *Aj,
                                  const double *Ax, const int64_t *Bp,
                                  const int32_t *Bj, const double *Bx,
                                  const int64_t *Cp, int32_t *Cj, double *Cx,
                                  double *Cabs) {
  const int64_t base = Cp[r0];
#pragma omp parallel
  {
    std::vector<int64_t> mark((size_t)ncols, -1);
    std::vector<double> acc((size_t)ncols, 0.0);
    std::vector<double> accabs(Cabs ? (size_t)ncols : 0, 0.0);
    std::vector<int32_t> cols;
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = r0; i < r1; ++i) {
      cols.clear();
      for (int64_t p = Ap[i]; p < Ap[i + 1]; ++p) {
        const int64_t k = Aj[p];
        const double a = Ax[p];
        for (int64_t q = Bp[k]; q < Bp[k + 1]; ++q) {
          const int32_t j = Bj[q];
          const double t = a * Bx[q];
          if (mark[j] != i) {
            mark[j] = i;
            cols.push_back(j);
            acc[j] = t;
            if (Cabs) accabs[j] = t < 0 ? -t : t;
          } else {
            acc[j] += t;
            if (Cabs) accabs[j] += t < 0 ? -t : t;
          }
        }
      }
      std::sort(cols.begin(), cols.end());
      int64_t o = Cp[i] - base;
      for (int32_t j : cols) {
        Cj[o] = j;
        Cx[o] = acc[j];
        if (Cabs) Cabs[o] = accabs[j];
        ++o;
      }
    }
  }
  return 0;
}

// Union merge of sorted rows: cusparseScsrgeam2 with alpha = beta = 1
// (include/cusparse_helpers.cuh:830-892) and KokkosSparse::spadd
// (include/KokkosWrap.hpp:420-425).  A column present in both gets a + b.
extern "C" int64_t orc_spadd_count(int64_t m, const int64_t *Ap,
                                   const int32_t *Aj, const int64_t *Bp,
                                   const int32_t *Bj, int64_t *cnt) {
  int64_t total = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : total)
  for (int64_t i = 0; i < m; ++i) {
    int64_t p = Ap[i], pe = Ap[i + 1], q = Bp[i], qe = Bp[i + 1], c = 0;
    while (p < pe && q < qe) {
      if (Aj[p] < Bj[q]) ++p;
      else if (Bj[q] < Aj[p]) ++q;
      else { ++p; ++q; }
      ++c;
    }
    c += (pe - p) + (qe - q);
    if (cnt) cnt[i] = c;
    total += c;
  }
  return total;
}

extern "C" int orc_spadd_numeric(int64_t m, const int64_t *Ap,
                                 const int32_t *Aj, const double *Ax,
                                 const int64_t *Bp, const int32_t *Bj,
                                 const double *Bx, const int64_t *Cp,
                                 int32_t *Cj, double *Cx) {
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < m; ++i) {
    int64_t p = Ap[i], pe = Ap[i + 1], q = Bp[i], qe = Bp[i + 1], o = Cp[i];
    while (p < pe || q < qe) {
      if (q >= qe || (p < pe && Aj[p] < Bj[q])) {
        Cj[o] = Aj[p]; Cx[o] = Ax[p]; ++p;
      } else if (p >= pe || Bj[q] < Aj[p]) {
        Cj[o] = Bj[q]; Cx[o] = Bx[q]; ++q;
      } else {
        Cj[o] = Aj[p]; Cx[o] = Ax[p] + Bx[q]; ++p; ++q;
      }
      ++o;
    }
  }
  return 0;
}

// SpaComm::gen_bitmask (include/spacomm.cuh:29-117): bit value
// 1 << (i % MASK_SIZE) when segment i is non-empty, summed over each group of
// MASK_SIZE = 8 segments into one uint8 (include/common.h:63-65).
extern "C" void orc_bitmask_gen(const int64_t *ptr, int64_t n, uint8_t *out) {
  const int64_t nbytes = (n + 7) / 8;
  for (int64_t w = 0; w < nbytes; ++w) {
    unsigned v = 0;
    for (int b = 0; b < 8; ++b) {
      const int64_t i = 8 * w + b;
      if (i < n && ptr[i] != ptr[i + 1]) v |= 1u << b;
    }
    out[w] = (uint8_t)v;
  }
}

// SpaComm::intersect_bitmasks (include/spacomm.cuh:126-148).
extern "C" void orc_bitmask_and(const uint8_t *a, const uint8_t *b,
                                int64_t nbytes, uint8_t *out) {
  for (int64_t i = 0; i < nbytes; ++i) out[i] = a[i] & b[i];
}

// One tile through SpaCommHandler::Compress (include/spacomm.cuh:962-1091):
//  - select_entries_cuda (:808-889): entry e is kept iff the mask bit of the
//    segment holding e is set, where the segment is the last r with
//    ptr[r] <= e (locate_segment_by_pos, :714-725); order is preserved;
//  - select_ptrs (:556-623): counts c_r = ptr[r+1]-ptr[r], zeroed for masked
//    segments, then ptr := [0, inclusive_scan(c)] at full length.
// A linear walk over the segments visits the same (segment, entry) pairs.
extern "C" int64_t orc_pack(const int64_t *ptr, int64_t len,
                            const int32_t *idx, const void *val,
                            int val_bytes, const uint8_t *mask,
                            int64_t *out_ptr, int32_t *out_idx,
                            void *out_val) {
  const char *vin = (const char *)val;
  char *vout = (char *)out_val;
  int64_t o = 0;
  out_ptr[0] = 0;
  for (int64_t r = 0; r < len; ++r) {
    const bool keep = (mask[r / 8] >> (r % 8)) & 1;
    if (keep) {
      for (int64_t e = ptr[r]; e < ptr[r + 1]; ++e) {
        out_idx[o] = idx[e];
        std::memcpy(vout + o * val_bytes, vin + e * val_bytes, val_bytes);
        ++o;
      }
    }
    out_ptr[r + 1] = o;
  }
  return o;
}
