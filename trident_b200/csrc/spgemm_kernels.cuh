// spgemm_kernels.cuh — device side of the two-phase row-wise SpGEMM.
//
// Layout in HBM.  Operands are plain CSR (row offsets int32 or int64, int32
// column indices, FP64 or FP32 values).  A launch covers one or many products
// ("prods"); rows of all products are numbered globally (row g of product p
// is g = base[p] + r) so that binning, scans and the persistent work queue
// see one flat row space.  Per global row the plan keeps:
//   rowf[g]  int64  products (a.k.a. mults / flops/2) of the row
//   rowc[g]  int32  distinct output columns (symbolic result)
//   cp[g]    int64  exclusive prefix of rowc over the flat row space
//   list[]   uint64 rows binned by class, entry = (p << 40) | r
//
// Row classes (the same five for both phases, heaviest first so that the
// persistent grid starts on the long rows):
//   DENSE  (three sub-classes by product count, heaviest first) one CTA per
//          row.  Symbolic: a bitmap of the whole column range in shared
//          memory.  Numeric: the same bitmap, then a CTA scan that writes the
//          sorted columns and keeps a rank base per 32 columns; every product
//          is then added into its output slot with a global FP64 reduction
//          (rows wider than the shared-memory bitmap use an FP64 window of
//          16384 columns swept with per-A-entry cursors instead).
//   G1024  one CTA per row, open-addressing hash in shared memory.
//   G256   256-thread groups, named barriers.
//   G128   128-thread groups.
//   G32    one warp per row.
// Hash rows are sorted after accumulation by an in-place compaction into the
// first half of the table and a stable LSD radix sort (bitonic below 65).
#pragma once

#include "internal.cuh"

namespace tspg {

constexpr int kThreads = 512;   // persistent CTA: 16 warps x 128 registers
// The symbolic CTA rows need no values (64 registers), so their persistent
// CTA runs 32 warps: more B-row loads and bitmap updates in flight per SM
// (R-MAT 20 symbolic phase: 58.4 ms at 16 warps, 49.4 at 24, 46.0 at 32).
constexpr int kSymThreads = 1024;
// The numeric DENSE rows of the rank form (k_dense_rank) likewise: their
// bitmap, scan and emission passes carry no values, and the value pass's
// 8 loads in flight fit 80 registers (8 bytes spilled with int32 offsets
// and FP64 values).  1024 threads (64 registers) measured the same.
constexpr int kRankThreads = 768;
constexpr int kTableSmem = 196608;              // hash tables / dense window
constexpr int kCountSmem = 16384;               // radix-sort digit counters
constexpr int kDynSmem = kTableSmem + kCountSmem;  // one CTA per SM
// The group-row kernel (k_groups): 24 warps x 80 registers over the same
// table space, so more rows are in flight per SM than the 16 warps of the
// persistent CTA-row kernel (group rows are latency-bound: shared-memory
// probes and the loads of short B rows); 1 KiB of digit counters per warp.
constexpr int kGroupThreads = 768;
constexpr int kGroupCountSmem = (kGroupThreads / 32) * 1024;
constexpr int kGroupDynSmem = kTableSmem + kGroupCountSmem;

// Row classes, heaviest first.  The first four are worked by the whole CTA
// (items fetched by one thread); G256 / G128 / G32 rows are fetched by each
// group on its own, so groups never wait for one another.
constexpr int NCLS = 8;
enum {
  CLS_DENSE0 = 0,  // DENSE rows with >= 2^20 products
  CLS_DENSE1 = 1,  // DENSE rows with >= 2^17 products
  CLS_DENSE2 = 2,  // other DENSE rows
  CLS_G1024 = 3,
  CLS_G256 = 4,
  CLS_G128 = 5,
  CLS_G32 = 6,
  CLS_ONEPASS = 7  // symbolic only: warp rows computed whole in the symbolic launch
};
constexpr int kCtaClasses = 4;  // classes [0, 4) are CTA-level
__host__ __device__ constexpr bool cls_dense(int c) { return c <= CLS_DENSE2; }

constexpr int kSymT32 = 1024, kSymT128 = 4096, kSymT256 = 8192,
              kSymT1024 = 32768;
constexpr int kNumT32 = 512, kNumT128 = 2048, kNumT256 = 4096,
              kNumT1024 = 16384;
constexpr int kDenseW = 16384;           // numeric dense window (columns)
constexpr int kDenseCurSmem = 8192;      // cursors kept in shared memory
constexpr int64_t kDenseBits = int64_t(kTableSmem + kCountSmem) * 8;  // whole-row bitmap
constexpr int kBitonicMax = 64;          // rows up to this size sort bitonic
// whole-row DENSE numeric form: per 32 columns a bitmap word (4 B) and a
// uint16 rank offset, per 1024 columns an int block base (196 B per block)
constexpr int64_t kRankMaxCols = int64_t(kDynSmem / 196) * 1024;
// numeric CTA-level rows: at most one heavy (DENSE0 / DENSE1) row per this
// many items; the period is also capped at 1 + light / heavy rows, so in
// practice the heavy rows spread evenly over the whole item sequence (R-MAT
// 20: 309.9 ms heaviest-first, 299.7 / 292.5 / 289.7 ms with periods 4 / 8 / 11)
constexpr int kHeavyPeriod = 64;

__host__ __device__ inline int dense_sub(int64_t f) {
  return f >= (int64_t(1) << 20) ? CLS_DENSE0 : f >= (int64_t(1) << 17) ? CLS_DENSE1 : CLS_DENSE2;
}
__host__ __device__ inline int sym_class(int64_t f, int64_t n, const Tune &t) {
  const int64_t fe = f < n ? f : n;
  if (f == 0) return -1;
  if (fe <= t.sym[0]) return CLS_G32;
  if (fe <= t.sym[1]) return CLS_G128;
  if (fe <= t.sym[2]) return CLS_G256;
  if (fe <= t.sym[3]) return CLS_G1024;
  return dense_sub(f);
}
// One-pass rows (plain products only, Sched::onepass set): rows of the
// symbolic warp, 128- and 256-thread classes are multiplied whole by a warp
// in the symbolic launch; their output waits in a scratch buffer for the
// numeric launch, which copies it into C.  A row whose output bound
// min(f, n) fits a 64-slot table is always finished there; a larger one is
// finished only when it has fewer than kCappedCols columns (its 64-slot
// attempt), else it is deferred to the two-pass path — so no row writes
// more than kCappedCols scratch entries, and the scratch stays dense.
constexpr int kCappedCols = 32;
__host__ __device__ inline bool onepass_row(int64_t f, int64_t n, const Tune &t) {
  const int64_t fe = f < n ? f : n;
  return f > 0 && fe <= t.sym[2];
}
// A one-pass row whose whole table fits 64 slots (else only its capped
// 64-slot attempt can finish it), and the scratch entries it may write.
__host__ __device__ inline bool onepass_full(int64_t f, int64_t n, const Tune &t) {
  const int64_t fe = f < n ? f : n;
  return int64_t(t.load) * fe <= 2 * kCappedCols;
}
__host__ __device__ inline int64_t onepass_bound(int64_t f, int64_t n, const Tune &t) {
  const int64_t fe = f < n ? f : n;
  return onepass_full(f, n, t) ? fe : kCappedCols;
}
__host__ __device__ inline int num_class(int64_t c, int64_t f, const Tune &t) {
  if (c == 0 || f < 0) return -1;  // f < 0: a one-pass row, already computed
  if (c <= t.num[0]) return CLS_G32;
  if (c <= t.num[1]) return CLS_G128;
  if (c <= t.num[2]) return CLS_G256;
  if (c <= t.num[3]) return CLS_G1024;
  return dense_sub(f);
}


template <typename PT, typename VT>
struct ProdDev {
  const PT *Ap;
  const int32_t *Aj;
  const VT *Ax;
  const PT *Bp;
  const int32_t *Bj;
  const VT *Bx;
  int64_t m, n;
  int32_t *Cj;
  VT *Cx;
  void *Cp;       // output rowptr (product-local), cp_bits wide
  int32_t cp_bits;
  int32_t b_sorted;
  // optional addend of C = E + A·B (tspg_spgemm_acc): E's row r joins row r's
  // products as entries with coefficient 1; Ej == nullptr when there is none
  const void *Ep;
  const int32_t *Ej;
  const VT *Ex;
  int32_t ep_bits;
};

template <typename PT, typename VT>
__device__ __forceinline__ void addend_row(const ProdDev<PT, VT> &P, int64_t r, int64_t &e0,
                                           int64_t &e1) {
  if (P.ep_bits == 32) {
    e0 = ((const int32_t *)P.Ep)[r];
    e1 = ((const int32_t *)P.Ep)[r + 1];
  } else {
    e0 = ((const int64_t *)P.Ep)[r];
    e1 = ((const int64_t *)P.Ep)[r + 1];
  }
}

// Work schedule of one phase: rows per class, their list offsets and the
// work-item prefix the persistent kernel decodes.
struct Sched {
  Tune tune;  // row binning of this run, set by k_set_tune after the reset
  int64_t cnt[NCLS];
  int64_t off[NCLS];
  int64_t cur[NCLS];
  unsigned long long next[NCLS];  // per-class row counters of the group-level classes
  unsigned long long work;        // item counter of the CTA-level classes
  int64_t total;      // sum of mults (symbolic) or of nnz (numeric)
  int64_t upper;      // sum of min(mults, ncols)
  int64_t max_a_row;  // longest A row (sizes the DENSE cursor scratch)
  int64_t nonempty;
  unsigned long long work2;  // row counter of the cluster kernel (column-window rows)
  int32_t onepass;  // symbolic record of a plain product: one-pass rows on
  int32_t pad32;
  int64_t cand[NCLS];           // one-pass candidates by the class they left
  unsigned long long ndefer;    // one-pass rows sent back to the two-pass path
  unsigned long long work3;     // row counter of the rank-form DENSE kernel
  int32_t rank_left;            // DENSE rows that kernel left to k_phase (0 / 1)
  int32_t pad32b;
};

__device__ __forceinline__ int find_prod(const int64_t *base, int nprod,
                                         int64_t g) {
  int lo = 0, hi = nprod;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (base[mid] <= g) lo = mid; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ uint32_t hash_slot(int32_t col, int logT) {
  return ((uint32_t)col * 2654435761u) >> (32 - logT);
}

__device__ __forceinline__ int ilog2_pow2(uint32_t x) { return 31 - __clz(x); }

__device__ __forceinline__ uint32_t pow2_at_least(int64_t x, uint32_t lo) {
  uint32_t t = lo;
  while ((int64_t)t < x) t <<= 1;
  return t;
}

// Sub-group width for the CTA rows' product loop (for_products_balanced):
// threads of a sub-group walk one B row together, sized to the row's average
// B row length f / na.
__device__ __forceinline__ int subgroup_width_avg(int64_t f, int64_t na, int G) {
  int64_t avg = na > 0 ? f / na : 0;
  int S = avg >= 24 ? 32 : avg >= 12 ? 16 : avg >= 6 ? 8 : avg >= 3 ? 4 : 2;
  return S > G ? G : S;
}

// ---------------------------------------------------------------------------
// Setup kernels

// Row binning of a run into its Sched records (after they were zeroed).
static __global__ void k_set_tune(Sched *S, int n, Tune t, int onepass = 0) {
  if (threadIdx.x < n) {
    S[threadIdx.x].tune = t;
    S[threadIdx.x].onepass = threadIdx.x == 0 ? onepass : 0;
  }
}

template <typename PT, typename VT>
__global__ void k_set_prod(ProdDev<PT, VT> *dst, ProdDev<PT, VT> v,
                           int64_t *base, int64_t m) {
  *dst = v;
  base[0] = 0;
  base[1] = m;
}

// int32 row offsets widened to int64 (operands of mixed offset widths).
static __global__ void k_widen(const int32_t *src, int64_t n, int64_t *dst) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[i];
}

// New operand arrays for a plan's numeric re-run; the sortedness found by the
// symbolic pass is kept.
template <typename PT, typename VT>
__global__ void k_set_operands(ProdDev<PT, VT> *dst, ProdDev<PT, VT> v) {
  const int32_t sorted = dst->b_sorted;
  const void *ep = dst->Ep;  // the addend stays the symbolic call's
  const int32_t *ej = dst->Ej;
  const VT *ex = dst->Ex;
  const int32_t eb = dst->ep_bits;
  *dst = v;
  dst->b_sorted = sorted;
  dst->Ep = ep;
  dst->Ej = ej;
  dst->Ex = ex;
  dst->ep_bits = eb;
}

template <typename PT, typename VT>
__global__ void k_set_out(ProdDev<PT, VT> *dst, int32_t *Cj, VT *Cx, void *Cp,
                          int cp_bits) {
  dst->Cj = Cj;
  dst->Cx = Cx;
  dst->Cp = Cp;
  dst->cp_bits = cp_bits;
}

// One warp per B row: set *flag = 0 if some row is not strictly increasing
// (the cursor sweep of the DENSE numeric class relies on sorted B rows).
template <typename PT>
__global__ void k_check_sorted_rows(const PT *Bp, const int32_t *Bj,
                                    int64_t nb, int32_t *flag) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  bool bad = false;
  for (int64_t r = warp; r < nb; r += nwarps) {
    const int64_t b0 = Bp[r], b1 = Bp[r + 1];
    for (int64_t q = b0 + lane; q + 1 < b1; q += 32)
      if (Bj[q] >= Bj[q + 1]) bad = true;
  }
  if (__any_sync(0xffffffffu, bad) && lane == 0) *flag = 0;
}

// ---------------------------------------------------------------------------
// Phase 0: mults per row and symbolic classes (one warp per row, shuffle
// reduction), block-aggregated class counts.
// Rows of at most this many A entries are walked by one lane in k_row_mults.
constexpr int kThreadRowMax = 64;
// A entries a one-pass candidate looks at for repeated columns.
constexpr int kHintEntries = 8;

// Products per row (rowf), the symbolic class counts, the product total, the
// sum of min(products, ncols) and the longest A row.  A warp takes 32 rows at
// a time: lane i walks row i's A entries itself (4 entries per step, so the
// loads of 32 rows are in flight together) when the row has at most
// kThreadRowMax entries, and the whole warp walks each longer row; class
// counts are aggregated per warp before the shared atomics (rows of one class
// would otherwise all hit one counter).  One warp per row, as first built,
// took 0.8 ms on the 2.1M rows of the Galerkin A·P (27 entries each): four
// dependent loads per row, one row per warp at a time.
template <typename PT, typename VT>
__global__ void __launch_bounds__(256) k_row_mults(
    const ProdDev<PT, VT> *prods, const int64_t *base, int nprod, int64_t R,
    int64_t *rowf, Sched *S, int32_t *obound = nullptr) {
  __shared__ unsigned long long s_cnt[NCLS], s_cand[NCLS];
  __shared__ unsigned long long s_tot, s_up, s_ne;
  __shared__ long long s_maxa;
  if (threadIdx.x < NCLS) s_cnt[threadIdx.x] = s_cand[threadIdx.x] = 0;
  if (threadIdx.x == 0) s_tot = s_up = s_ne = 0, s_maxa = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  const int64_t ntiles = (R + 31) / 32;
  unsigned long long tot = 0, up = 0, ne = 0;
  long long maxa = 0;
  for (int64_t tile = warp; tile < ntiles; tile += nwarps) {
    const int64_t g = tile * 32 + lane;
    const bool valid = g < R;
    int p = 0;
    int64_t r = 0, a0 = 0, a1 = 0;
    const int32_t *Aj = nullptr;
    const PT *Bp = nullptr;
    if (valid) {
      p = find_prod(base, nprod, g);
      r = g - base[p];
      const PT *Ap = prods[p].Ap;
      Aj = prods[p].Aj;
      Bp = prods[p].Bp;
      a0 = int64_t(Ap[r]);
      a1 = int64_t(Ap[r + 1]);
    }
    const int64_t len = a1 - a0;
    const bool mine = len <= kThreadRowMax;  // rows past R have len 0
    const int tmax = int(__reduce_max_sync(0xffffffffu, mine ? unsigned(len) : 0u));
    int64_t f = 0;
    for (int t = 0; t < tmax; t += 4) {
      int64_t k[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) k[u] = mine && t + u < len ? int64_t(__ldg(Aj + a0 + t + u)) : -1;
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (k[u] >= 0) f += int64_t(__ldg(Bp + k[u] + 1)) - int64_t(__ldg(Bp + k[u]));
    }
    for (unsigned lr = __ballot_sync(0xffffffffu, !mine); lr; lr &= lr - 1) {
      const int j = __ffs(lr) - 1;
      const int pj = __shfl_sync(0xffffffffu, p, j);
      const int64_t b0 = __shfl_sync(0xffffffffu, a0, j), b1 = __shfl_sync(0xffffffffu, a1, j);
      const int32_t *Ajj = prods[pj].Aj;
      const PT *Bpj = prods[pj].Bp;
      int64_t sum = 0;
      for (int64_t q = b0 + lane; q < b1; q += 32) {
        const int64_t k = __ldg(Ajj + q);
        sum += int64_t(__ldg(Bpj + k + 1)) - int64_t(__ldg(Bpj + k));
      }
      sum = warp_sum(sum);
      if (lane == j) f = sum;
    }
    // One-pass candidates too large for a warp's full table also need their
    // products to repeat columns: a row counts, over its first kHintEntries A
    // entries, those whose B row starts on the same column as the previous
    // entry's (0.5-0.6 of them on the Galerkin rows, 0.002 on uniform-random
    // rows); a few loads per such row.
    int same = 0, seen = 0;
    {
      const int64_t fe = f < (valid ? prods[p].n : 0) ? f : (valid ? prods[p].n : 0);
      const bool need = S->onepass && valid && fe > 0 && fe <= S->tune.sym[2] &&
                        int64_t(S->tune.load) * fe > 2 * kCappedCols;
      if (__any_sync(0xffffffffu, need)) {
        const int32_t *Bj = valid ? prods[p].Bj : nullptr;
        seen = need ? int(len < kHintEntries ? len : kHintEntries) : 0;
        int prev = -2;
        for (int t = 0; t < seen; ++t) {
          const int64_t k = __ldg(Aj + a0 + t);
          const int64_t q0 = int64_t(__ldg(Bp + k)), q1 = int64_t(__ldg(Bp + k + 1));
          const int first = q1 > q0 ? __ldg(Bj + q0) : -1;
          same += first >= 0 && first == prev;
          prev = first;
        }
      }
    }
    int c = -1, left = -1;
    if (valid) {
      if (prods[p].Ej) {  // the addend's entries count as products of the row
        int64_t e0, e1;
        addend_row(prods[p], r, e0, e1);
        f += e1 - e0;
      }
      rowf[g] = f;
      const int64_t n = prods[p].n;
      c = sym_class(f, n, S->tune);
      // one-pass rows: their scratch bound; the class they leave is kept
      // (cand) in case the product takes the two-pass path after all
      // candidates: rows whose bound fits a warp's full table, and larger
      // ones whose products look like repeating columns (their 64-slot
      // attempt is likely to hold the row)
      const bool one = S->onepass && onepass_row(f, n, S->tune) &&
                       (onepass_full(f, n, S->tune) || (seen > 1 && 4 * same >= seen - 1));
      if (one) {
        left = c;
        c = CLS_ONEPASS;
      }
      if (obound) obound[g] = one ? int32_t(onepass_bound(f, n, S->tune)) : 0;
      if (c >= 0) ne += 1;
      tot += f;
      up += f < n ? f : n;
      if (len > maxa) maxa = len;
    }
    // one shared atomic per class present in the warp
    for (unsigned todo = __ballot_sync(0xffffffffu, c >= 0); todo;) {
      const int cl = __shfl_sync(0xffffffffu, c, __ffs(todo) - 1);
      const unsigned m = __ballot_sync(0xffffffffu, c == cl);
      if (lane == __ffs(m) - 1) atomicAdd(&s_cnt[cl], (unsigned long long)__popc(m));
      todo &= ~m;
    }
    for (unsigned todo = __ballot_sync(0xffffffffu, left >= 0); todo;) {
      const int cl = __shfl_sync(0xffffffffu, left, __ffs(todo) - 1);
      const unsigned m = __ballot_sync(0xffffffffu, left == cl);
      if (lane == __ffs(m) - 1) atomicAdd(&s_cand[cl], (unsigned long long)__popc(m));
      todo &= ~m;
    }
  }
  tot = warp_sum(tot);
  up = warp_sum(up);
  ne = warp_sum(ne);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const long long other = __shfl_xor_sync(0xffffffffu, maxa, o);
    maxa = other > maxa ? other : maxa;
  }
  if (lane == 0) {
    atomicAdd(&s_tot, tot);
    atomicAdd(&s_up, up);
    atomicAdd(&s_ne, ne);
    atomicMax(&s_maxa, maxa);
  }
  __syncthreads();
  if (threadIdx.x < NCLS && s_cnt[threadIdx.x])
    atomicAdd((unsigned long long *)&S->cnt[threadIdx.x], s_cnt[threadIdx.x]);
  if (threadIdx.x < NCLS && s_cand[threadIdx.x])
    atomicAdd((unsigned long long *)&S->cand[threadIdx.x], s_cand[threadIdx.x]);
  if (threadIdx.x == 0) {
    atomicAdd((unsigned long long *)&S->total, s_tot);
    atomicAdd((unsigned long long *)&S->upper, s_up);
    atomicAdd((unsigned long long *)&S->nonempty, s_ne);
    atomicMax((long long *)&S->max_a_row, s_maxa);
  }
}

// The one-pass rows of a symbolic record go back to the classes they left
// (the product takes the two-pass path after all).
static __global__ void k_fold_onepass(Sched *S) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    for (int c = 0; c < NCLS; ++c) S->cnt[c] += S->cand[c];
    S->cnt[CLS_ONEPASS] = 0;
    S->onepass = 0;
  }
}

// The record of the one-pass rows sent back to the two-pass path (their
// list: the deferred rows), counted as 256-thread symbolic rows.
static __global__ void k_defer_setup(const Sched *S, Sched *D) {
  if (threadIdx.x == 0 && blockIdx.x == 0) D->cnt[CLS_G256] = int64_t(S->ndefer);
}

// Class offsets into the row list; resets the work counters.
static __global__ void k_sched_offsets(Sched *S) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    int64_t o = 0;
    for (int c = 0; c < NCLS; ++c) {
      S->off[c] = o;
      S->cur[c] = o;
      S->next[c] = 0;
      o += S->cnt[c];
    }
    S->work = 0;
    S->work2 = 0;
    S->work3 = 0;
    S->rank_left = 0;
  }
}

// Scatter rows into the class lists.  mode 0: symbolic (class from rowf);
// mode 1: numeric (class from rowc) which also writes the output row offsets
// of each product and the largest A row among DENSE rows.
template <typename PT, typename VT, int MODE>
__global__ void __launch_bounds__(256) k_scatter(
    ProdDev<PT, VT> *prods, const int64_t *base, int nprod, int64_t R,
    const int64_t *rowf, const int32_t *rowc, const int64_t *cp, Sched *S,
    uint64_t *list) {
  __shared__ unsigned long long s_cnt[NCLS], s_base[NCLS];
  if (threadIdx.x < NCLS) s_cnt[threadIdx.x] = 0;
  __syncthreads();
  const int64_t g = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  int c = -1, p = 0;
  int64_t r = 0;
  unsigned long long my = 0;
  if (g < R) {
    p = find_prod(base, nprod, g);
    r = g - base[p];
    if (MODE == 0) {
      c = sym_class(rowf[g], prods[p].n, S->tune);
      if (S->onepass && rowc[g] > 0) c = CLS_ONEPASS;  // the count pass's choice (bound > 0)
    } else {
      c = num_class(rowc[g], rowf[g], S->tune);
      const int64_t off = cp[g] - cp[base[p]];
      if (prods[p].cp_bits == 32)
        ((int32_t *)prods[p].Cp)[r] = (int32_t)off;
      else
        ((int64_t *)prods[p].Cp)[r] = off;
      if (r == prods[p].m - 1) {
        const int64_t end = cp[g + 1] - cp[base[p]];
        if (prods[p].cp_bits == 32)
          ((int32_t *)prods[p].Cp)[r + 1] = (int32_t)end;
        else
          ((int64_t *)prods[p].Cp)[r + 1] = end;
      }
    }
  }
  // each class present in the warp takes its slots with one shared atomic
  const int lane = threadIdx.x & 31;
  for (unsigned todo = __ballot_sync(0xffffffffu, c >= 0); todo;) {
    const int leader = __ffs(todo) - 1;
    const int cl = __shfl_sync(0xffffffffu, c, leader);
    const unsigned m = __ballot_sync(0xffffffffu, c == cl);
    unsigned long long b = 0;
    if (lane == leader) b = atomicAdd(&s_cnt[cl], (unsigned long long)__popc(m));
    b = __shfl_sync(0xffffffffu, b, leader);
    if (c == cl) my = b + __popc(m & ((1u << lane) - 1u));
    todo &= ~m;
  }
  __syncthreads();
  if (threadIdx.x < NCLS) {
    s_base[threadIdx.x] =
        s_cnt[threadIdx.x]
            ? atomicAdd((unsigned long long *)&S->cur[threadIdx.x],
                        s_cnt[threadIdx.x])
            : 0;
  }
  __syncthreads();
  if (c >= 0) list[s_base[c] + my] = (uint64_t(p) << 40) | uint64_t(r);
}

// Products whose A has zero rows still need rowptr[0] = 0.
template <typename PT, typename VT>
__global__ void k_zero_rowptr(ProdDev<PT, VT> *prods, int nprod) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < nprod && prods[p].m == 0) {
    if (prods[p].cp_bits == 32) ((int32_t *)prods[p].Cp)[0] = 0;
    else ((int64_t *)prods[p].Cp)[0] = 0;
  }
}

// ---------------------------------------------------------------------------
// Device-wide exclusive scan of int32 row counts into int64 offsets
// (reduce, scan of partials, final).  cp has R + 1 entries.
constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

static __global__ void __launch_bounds__(kScanThreads)
    k_scan_reduce(const int32_t *in, int64_t R, int64_t *partial) {
  __shared__ int64_t tmp[kScanThreads / 32 + 1];
  const int64_t t0 = int64_t(blockIdx.x) * kScanTile;
  int64_t s = 0;
  for (int i = 0; i < kScanItems; ++i) {
    const int64_t j = t0 + int64_t(i) * kScanThreads + threadIdx.x;
    if (j < R) s += in[j];
  }
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) tmp[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    int64_t v = threadIdx.x < kScanThreads / 32 ? tmp[threadIdx.x] : 0;
    v = warp_sum(v);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
  }
}

// Single block: exclusive scan of nb partials in place; partial[nb] = total.
static __global__ void __launch_bounds__(1024) k_scan_partials(int64_t *partial,
                                                        int64_t nb) {
  __shared__ int64_t tmp[33];
  __shared__ int64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t b0 = 0; b0 < nb; b0 += 1024) {
    const int64_t j = b0 + threadIdx.x;
    const int64_t v = j < nb ? partial[j] : 0;
    int64_t tot;
    const int64_t ex = group_excl_scan<1024, int64_t>(v, tmp, 0, &tot);
    if (j < nb) partial[j] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[nb] = carry;
}

// Also counts the numeric classes of the rows into *Snum.
static __global__ void __launch_bounds__(kScanThreads)
    k_scan_final(const int32_t *in, int64_t R, const int64_t *partial,
                 int64_t nb, int64_t *out, Sched *Snum, const int64_t *rowf) {
  __shared__ int64_t tmp[kScanThreads / 32 + 1];
  __shared__ unsigned long long s_cnt[NCLS];
  if (threadIdx.x < NCLS) s_cnt[threadIdx.x] = 0;
  __syncthreads();
  const int64_t t0 = int64_t(blockIdx.x) * kScanTile;
  // each thread owns kScanItems consecutive elements
  const int64_t j0 = t0 + int64_t(threadIdx.x) * kScanItems;
  int64_t v[kScanItems];
  int64_t s = 0;
  uint32_t packed = 0;  // 4-bit count per class (kScanItems <= 15)
  static_assert(kScanItems <= 15 && NCLS * 4 <= 32, "packed class counts");
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    v[i] = (j0 + i < R) ? in[j0 + i] : 0;
    s += v[i];
    if (rowf && v[i] > 0) {
      const int c = num_class(v[i], rowf[j0 + i], Snum->tune);
      if (c >= 0) packed += 1u << (4 * c);
    }
  }
  // class counts: a warp reduction per class, one shared atomic per warp
  // (rows of one class would otherwise all hit one counter)
  if (rowf) {
#pragma unroll
    for (int c = 0; c < NCLS; ++c) {
      const unsigned x = __reduce_add_sync(0xffffffffu, (packed >> (4 * c)) & 15u);
      if ((threadIdx.x & 31) == 0 && x) atomicAdd(&s_cnt[c], (unsigned long long)x);
    }
  }
  int64_t tot;
  int64_t ex = group_excl_scan<kScanThreads, int64_t>(s, tmp, 0, &tot);
  ex += partial[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (j0 + i < R) out[j0 + i] = ex;
    ex += v[i];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[R] = partial[nb];
  __syncthreads();
  if (threadIdx.x < NCLS && s_cnt[threadIdx.x])
    atomicAdd((unsigned long long *)&Snum->cnt[threadIdx.x], s_cnt[threadIdx.x]);
}

}  // namespace tspg
