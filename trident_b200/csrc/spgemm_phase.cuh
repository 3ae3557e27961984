// spgemm_phase.cuh — the persistent symbolic / numeric kernels.
//
// One 512-thread CTA per SM (208 KiB of dynamic shared memory, 128 registers
// per thread).  Work is taken in two stages:
//   1. CTA-level rows (DENSE0..2 heaviest first, then G1024): thread 0 takes
//      the next row index from a device counter, the whole CTA works on it.
//   2. When those run out, the CTA splits into two 256-thread groups that
//      take G256 rows from their own counter; a group that runs out splits
//      into two 128-thread groups (G128 rows), which split into warps (G32
//      rows).  Groups never wait for each other: their shared-memory slices
//      and digit counters nest (a 128-group's slice lies inside its 256-group's
//      slice, a warp's inside its 128-group's) and they use disjoint named
//      barriers.
#pragma once

#include <type_traits>

#include "spgemm_kernels.cuh"

namespace tspg {

// Walk B entries q0, q0 + step, ... below b1 calling fn(col, a*b), with U
// loads in flight per thread (all loads of a step are issued before the
// updates, so the L2/HBM latency is paid once per U entries).  IX is the
// position type: uint32_t when B's row offsets are 32-bit (positions below
// 2^31, so q + U * step stays below 2^32 for step <= 2^27), else int64_t.
template <bool NUM, typename IX, typename VT, typename F>
__device__ __forceinline__ void walk_row(const int32_t *__restrict__ Bj,
                                         const VT *__restrict__ Bx, IX q0, IX b1, int step,
                                         VT a, F &&fn) {
  constexpr int U = 8;
  for (IX q = q0; q < b1; q += IX(step) * U) {
    int32_t c[U];
    VT x[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const IX qq = q + IX(u) * IX(step);
      c[u] = qq < b1 ? __ldg(Bj + qq) : -1;
      if constexpr (NUM) x[u] = qq < b1 ? __ldg(Bx + qq) : VT(0);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (c[u] >= 0) {
        if constexpr (NUM) fn(c[u], a * x[u]);
        else fn(c[u], VT(0));
      }
    }
  }
}

// Balanced product loop for one row by a group of G threads.  Pass 1:
// sub-groups of S threads take A entries in turn and stride over the entry's
// B row, but an A entry whose B row is longer than the fair share of a
// sub-group (f / #sub-groups) is appended to `lst` (group-private shared
// memory, `cap` slots, count in *nl) instead; pass 2 walks each listed B row
// with all G threads, so a hub row of B never leaves the group waiting on
// one warp.  When the list is full the entry is done in pass 1.  With `ctr`
// (a group-private shared int) sub-groups take their next A entry from it as
// they finish instead of a fixed stride, so uneven B rows do not leave most of
// the group waiting at the pass's closing barrier.
template <int G, bool NUM, typename PT, typename VT, typename F>
__device__ __forceinline__ void for_products_balanced(
    const int32_t *__restrict__ Aj, const VT *__restrict__ Ax,
    const PT *__restrict__ Bp, const int32_t *__restrict__ Bj,
    const VT *__restrict__ Bx, int64_t a0, int64_t a1, int64_t f, int S,
    int lane, int gid, int *lst, int *nl, int cap, F &&fn, int *ctr = nullptr) {
  using IX = std::conditional_t<sizeof(PT) == 4, uint32_t, int64_t>;
  const int sub = lane / S, sl = lane - sub * S, nsub = G / S;
  const int64_t thr = nsub > 1 ? max(int64_t(4 * S), f / nsub) : INT64_MAX;
  const unsigned submask =
      S >= 32 ? 0xffffffffu : (((1u << S) - 1u) << (((lane & 31) / S) * S));
  if (lane == 0) {
    *nl = 0;
    if (ctr) *ctr = nsub;
  }
  group_sync<G>(gid);
  for (int64_t p = a0 + sub; p < a1;) {
    const int64_t pc = p;
    if (ctr) {  // the next entry for this sub-group (dynamic)
      int t = 0;
      if (sl == 0) t = atomicAdd(ctr, 1);
      p = a0 + __shfl_sync(submask, t, (lane & 31) - sl);
    } else {
      p += nsub;
    }
    const int64_t k = __ldg(Aj + pc);
    const IX b0 = IX(__ldg(Bp + k)), b1 = IX(__ldg(Bp + k + 1));
    if (int64_t(b1 - b0) > thr) {
      int slot = 0;
      if (sl == 0) slot = atomicAdd(nl, 1);
      slot = __shfl_sync(submask, slot, (lane & 31) - sl);
      if (slot < cap) {
        if (sl == 0) lst[slot] = int(pc - a0);
        continue;
      }
    }
    VT a = VT(0);
    if constexpr (NUM) a = __ldg(Ax + pc);
    walk_row<NUM, IX, VT>(Bj, Bx, b0 + IX(sl), b1, S, a, fn);
  }
  group_sync<G>(gid);
  const int n = min(*nl, cap);
  for (int i = 0; i < n; ++i) {
    const int64_t p = a0 + lst[i];
    const int64_t k = __ldg(Aj + p);
    VT a = VT(0);
    if constexpr (NUM) a = __ldg(Ax + p);
    walk_row<NUM, IX, VT>(Bj, Bx, IX(__ldg(Bp + k)) + IX(lane), IX(__ldg(Bp + k + 1)), G, a,
                          fn);
  }
}

// One chunk of at most 32 A entries of a warp row: lane j holds entry j's
// value a and B row bounds [b0, b0 + len) (len = 0 past the chunk's nc
// entries); fn(col, a*b) for every product.  A warp scan numbers the chunk's
// products and lanes take products lane, lane + 32, ... (U per step, loads in
// flight), each finding its entry by a 5-step shuffle search.  (Lane j
// walking entry j's B row itself, with no search, measured slower on the
// Galerkin A·P rows, 27 entries x ~4.5: symbolic 2.35 vs 1.81 ms, numeric
// 5.35 vs 3.72 ms — each load touches 32 B rows instead of a few, and lanes
// whose B rows list the same columns hit them in the same step.)
template <bool NUM, typename IX, typename VT, typename F>
__device__ __forceinline__ void warp_chunk(const int32_t *__restrict__ Bj,
                                           const VT *__restrict__ Bx, IX b0, IX len, VT a,
                                           int nc, int lane, F &&fn) {
  constexpr int U = 4;
  const IX inc = warp_scan_incl(len);
  const IX tot = __shfl_sync(0xffffffffu, inc, 31);
  const IX pre = inc - len;
  // the step loop is uniform across the warp (the search shuffles)
  for (IX pb = 0; pb < tot; pb += IX(32) * U) {
    int32_t cc[U];
    VT xv[U], av[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const IX p = pb + IX(u) * 32 + lane;
      int j = 0;
#pragma unroll
      for (int st = 16; st > 0; st >>= 1) {
        const IX v = __shfl_sync(0xffffffffu, pre, (j + st) & 31);
        if (j + st < nc && v <= p) j += st;
      }
      const IX pj = __shfl_sync(0xffffffffu, pre, j);
      const IX bj = __shfl_sync(0xffffffffu, b0, j);
      if constexpr (NUM) av[u] = __shfl_sync(0xffffffffu, a, j);
      const IX q = bj + (p - pj);
      cc[u] = p < tot ? __ldg(Bj + q) : -1;
      if constexpr (NUM) xv[u] = p < tot ? __ldg(Bx + q) : VT(0);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (cc[u] >= 0) {
        if constexpr (NUM) fn(cc[u], av[u] * xv[u]);
        else fn(cc[u], VT(0));
      }
    }
  }
}

// Flat product loop for group rows.  A entries are taken G at a time: lane j
// loads entry j's column, value and B row bounds, so a chunk's loads are all
// in flight together; a group scan of the B row lengths numbers the chunk's
// products and lanes take products lane, lane + G, ... (U per step, loads in
// flight), each finding its entry as the last one whose first product number
// is <= its own.  G = 32 keeps the per-entry data in registers (warp_chunk);
// larger groups stage it in `stage` (24 bytes per lane of shared memory).
template <int G, bool NUM, typename PT, typename VT, typename F>
__device__ __forceinline__ void for_products_flat(
    const int32_t *__restrict__ Aj, const VT *__restrict__ Ax,
    const PT *__restrict__ Bp, const int32_t *__restrict__ Bj,
    const VT *__restrict__ Bx, int64_t a0, int64_t a1, int lane, int gid,
    int64_t *tmp, unsigned char *stage, F &&fn) {
  constexpr int U = 4;
  int64_t *spre = (int64_t *)stage;
  int64_t *sb0 = spre + G;
  VT *sa = (VT *)(sb0 + G);
  // positions fit 32 bits when B's row offsets do (nnz(B) < 2^31): the warp
  // form then shuffles half the words
  using IX = std::conditional_t<G == 32 && sizeof(PT) == 4, int32_t, int64_t>;
  for (int64_t c0 = a0; c0 < a1; c0 += G) {
    const int nc = int(min(int64_t(G), a1 - c0));
    IX len = 0, b0 = 0;
    VT a = VT(0);
    if (lane < nc) {
      const int64_t k = __ldg(Aj + c0 + lane);
      if constexpr (NUM) a = __ldg(Ax + c0 + lane);
      b0 = IX(__ldg(Bp + k));
      len = IX(__ldg(Bp + k + 1)) - b0;
    }
    if constexpr (G == 32) {
      warp_chunk<NUM, IX, VT>(Bj, Bx, b0, len, a, nc, lane, fn);
      continue;  // no staging to guard
    } else {
      IX tot;
      const IX pre = group_excl_scan<G, int64_t>(len, tmp, gid, &tot);
      if (lane < nc) {
        spre[lane] = pre;
        sb0[lane] = b0;
        sa[lane] = a;
      }
      group_sync<G>(gid);
      // the step loop is uniform across the group
      for (IX pb = 0; pb < tot; pb += IX(G) * U) {
        int32_t cc[U];
        VT xv[U], av[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const IX p = pb + IX(u) * G + lane;
          int j = 0;
          for (int st = G / 2; st > 0; st >>= 1)
            if (j + st < nc && spre[j + st] <= p) j += st;
          const IX q = IX(sb0[j]) + (p - IX(spre[j]));
          if constexpr (NUM) av[u] = sa[j];
          cc[u] = p < tot ? __ldg(Bj + q) : -1;
          if constexpr (NUM) xv[u] = p < tot ? __ldg(Bx + q) : VT(0);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (cc[u] >= 0) {
            if constexpr (NUM) fn(cc[u], av[u] * xv[u]);
            else fn(cc[u], VT(0));
          }
        }
      }
      group_sync<G>(gid);  // the next chunk reuses the staging
    }
  }
}

// The addend row of C = E + A·B (ProdDev::Ej; nothing when there is none):
// fn(col, value) for E's row r, lanes lane, lane + G, ...
template <bool NUM, typename PT, typename VT, typename F>
__device__ __forceinline__ void for_addend(const ProdDev<PT, VT> &P, int64_t r, int lane,
                                           int G, F &&fn) {
  if (!P.Ej) return;
  int64_t e0, e1;
  addend_row(P, r, e0, e1);
  for (int64_t q = e0 + lane; q < e1; q += G) {
    if constexpr (NUM) fn(__ldg(P.Ej + q), __ldg(P.Ex + q));
    else fn(__ldg(P.Ej + q), VT(0));
  }
}

// Probe bound: tables are sized T >= 2 * (distinct keys), so a probe never
// runs T steps; the bound only turns a broken invariant into an error flag.
__device__ __forceinline__ int sym_insert(int *keys, int32_t col, int logT,
                                          uint32_t mask, int64_t *err) {
  uint32_t h = hash_slot(col, logT);
  for (uint32_t it = 0; it <= mask; ++it) {
    const int k = ((volatile int *)keys)[h];
    if (k == col) return 0;
    if (k == -1) {
      const int old = atomicCAS(keys + h, -1, col);
      if (old == -1) return 1;
      if (old == col) return 0;
    }
    h = (h + 1) & mask;
  }
  set_error(err, 101);
  return 0;
}

__device__ __forceinline__ uint32_t num_insert(int *keys, int32_t col,
                                               int logT, uint32_t mask,
                                               int64_t *err) {
  uint32_t h = hash_slot(col, logT);
  for (uint32_t it = 0; it <= mask; ++it) {
    const int k = ((volatile int *)keys)[h];
    if (k == col) return h;
    if (k == -1) {
      const int old = atomicCAS(keys + h, -1, col);
      if (old == -1 || old == col) return h;
    }
    h = (h + 1) & mask;
  }
  set_error(err, 102);
  return 0;
}

// Insert for a table that admits at most about `cap` columns: ocnt[0] counts
// the columns that took a slot, and once it reaches cap ocnt[1] is set and no
// further column takes one (kRefused; the caller redoes the row with a full
// table).  Columns already in the table are still found.  At most one column
// per lane in flight gets in past the count, so a table of T = 2 cap slots
// never fills (at most 2 cap - 1 columns) and every probe ends.
constexpr uint32_t kRefused = 0xffffffffu;
__device__ __forceinline__ uint32_t num_insert_capped(int *keys, int32_t col, int logT,
                                                      uint32_t mask, int *ocnt, uint32_t cap) {
  uint32_t h = hash_slot(col, logT);
  for (uint32_t it = 0; it <= mask; ++it) {
    const int k = ((volatile int *)keys)[h];
    if (k == col) return h;
    if (k == -1) {
      if (((volatile int *)ocnt)[1]) return kRefused;
      const int old = atomicCAS(keys + h, -1, col);
      if (old == -1) {
        if (uint32_t(atomicAdd(ocnt, 1)) + 1 >= cap) ocnt[1] = 1;
        return h;
      }
      if (old == col) return h;
    }
    h = (h + 1) & mask;
  }
  ocnt[1] = 1;  // not reached: the table never fills
  return kRefused;
}

struct PhaseArgs {
  const int64_t *base;
  Sched *S;
  const uint64_t *list;
  int64_t *rowf;
  int32_t *rowc;
  const int64_t *cp;
  int32_t *curbuf;     // per-CTA cursor scratch for DENSE rows with long A rows:
                       // 2 x cur_stride entries per CTA (cursor, column at it)
  int64_t cur_stride;  // entries per CTA in curbuf
  int64_t *err;
  unsigned long long *prof;  // optional: [class] cycles, [NCLS + class] rows
  int32_t *oj = nullptr;     // one-pass rows: scratch columns and values
  void *ox = nullptr;
  uint64_t *defer = nullptr;  // one-pass rows sent back to the two-pass path
};

// Optional per-class accounting (SM cycles spent in each row class), and
// sub-phase cycles of the DENSE numeric rows at [kProfSub + i].
constexpr int kProfSub = 2 * NCLS;
constexpr int kProfPerPhase = 32;
__device__ __forceinline__ void prof_add(const PhaseArgs &A, int cls, long long t0,
                                         bool leader) {
  if (A.prof && leader) {
    atomicAdd(A.prof + cls, (unsigned long long)(clock64() - t0));
    atomicAdd(A.prof + NCLS + cls, 1ull);
  }
}
__device__ __forceinline__ void prof_sub_g(const PhaseArgs &A, int i, long long &t,
                                           bool leader) {
  if (A.prof && leader) {
    const long long now = clock64();
    atomicAdd(A.prof + kProfSub + i, (unsigned long long)(now - t));
    t = now;
  }
}
__device__ __forceinline__ void prof_sub(const PhaseArgs &A, int i, long long &t) {
  if (A.prof && threadIdx.x == 0) {
    const long long now = clock64();
    atomicAdd(A.prof + kProfSub + i, (unsigned long long)(now - t));
    t = now;
  }
}

struct RowRef {
  int p;
  int64_t r, g;
};

__device__ __forceinline__ RowRef decode_row(const PhaseArgs &A, int64_t idx) {
  const uint64_t e = A.list[idx];
  RowRef rr;
  rr.p = int(e >> 40);
  rr.r = int64_t(e & ((uint64_t(1) << 40) - 1));
  rr.g = A.base[rr.p] + rr.r;
  return rr;
}

// What a group row function needs before its first product: the product, the
// local and flat row, its product count f, output count c and output offset
// inside the product (numeric phase only), and its A row bounds.  A chain of
// three dependent global loads, so warps fetch a whole chunk of rows' metadata
// at once (one row per lane) and pass it on by shuffles.
struct RowMeta {
  int p;
  int64_t r, g, f, c, off, a0, a1;
};

template <bool NUM, typename PT, typename VT>
__device__ __forceinline__ RowMeta load_meta(const ProdDev<PT, VT> *prods, const PhaseArgs &A,
                                             int64_t idx) {
  const uint64_t e = A.list[idx];
  RowMeta m;
  m.p = int(e >> 40);
  m.r = int64_t(e & ((uint64_t(1) << 40) - 1));
  const int64_t b = A.base[m.p];
  const PT *Ap = prods[m.p].Ap;
  m.g = b + m.r;
  m.a0 = int64_t(Ap[m.r]);
  m.a1 = int64_t(Ap[m.r + 1]);
  m.f = A.rowf[m.g];
  m.c = NUM ? int64_t(A.rowc[m.g]) : 0;
  m.off = NUM ? A.cp[m.g] - A.cp[b] : 0;
  return m;
}

__device__ __forceinline__ RowMeta shfl_meta(const RowMeta &m, int src) {
  RowMeta o;
  o.p = __shfl_sync(0xffffffffu, m.p, src);
  o.r = __shfl_sync(0xffffffffu, m.r, src);
  o.g = __shfl_sync(0xffffffffu, m.g, src);
  o.f = __shfl_sync(0xffffffffu, m.f, src);
  o.c = __shfl_sync(0xffffffffu, m.c, src);
  o.off = __shfl_sync(0xffffffffu, m.off, src);
  o.a0 = __shfl_sync(0xffffffffu, m.a0, src);
  o.a1 = __shfl_sync(0xffffffffu, m.a1, src);
  return o;
}

// Group-private shared scratch handed to the row functions.
struct GroupMem {
  int64_t *tmp;   // scan scratch (33 words)
  int *itmp;      // min/max scratch
  int *lst;       // deferred long B rows
  int *nl;        // their count
  int cap;        // list capacity
  uint16_t *cnt;  // radix digit counters
  unsigned char *stage;  // flat product loop staging (G = 128 / 256), 24 B per lane
};

// Hash table clears with 16-byte shared stores (T is a power of two >= 32 and
// every table starts on a 16-byte boundary of its slice).
template <int G>
__device__ __forceinline__ void clear_keys(int *keys, uint32_t T, int lane) {
  int4 *k4 = reinterpret_cast<int4 *>(keys);
  for (uint32_t s = lane; s < T / 4; s += G) k4[s] = make_int4(-1, -1, -1, -1);
}
template <int G, typename VT>
__device__ __forceinline__ void clear_vals(VT *vals, uint32_t T, int lane) {
  uint4 *v4 = reinterpret_cast<uint4 *>(vals);
  for (uint32_t s = lane; s < T * uint32_t(sizeof(VT)) / 16; s += G) v4[s] = make_uint4(0, 0, 0, 0);
}

// ---------------------------------------------------------------- symbolic

template <int G, int TMAX, typename PT, typename VT>
__device__ void sym_hash_row(const ProdDev<PT, VT> *prods, const PhaseArgs &A,
                             const RowMeta &m, int *keys, const GroupMem &gm, int gid,
                             int lane) {
  long long tp = clock64();
  const ProdDev<PT, VT> &P = prods[m.p];
  const int64_t f = m.f;
  const int64_t n = P.n;
  const int64_t fe = f < n ? f : n;
  uint32_t T = pow2_at_least(A.S->tune.load * fe, 32);
  if (T > TMAX) T = TMAX;
  const int logT = ilog2_pow2(T);
  const uint32_t mask = T - 1;
  clear_keys<G>(keys, T, lane);
  group_sync<G>(gid);
  const int64_t a0 = m.a0, a1 = m.a1;
  prof_sub_g(A, 9, tp, lane == 0);
  int cnt = 0;
  auto ins = [&](int32_t col, VT) { cnt += sym_insert(keys, col, logT, mask, A.err); };
  if constexpr (G <= 256) {
    for_products_flat<G, false, PT, VT>(P.Aj, P.Ax, P.Bp, P.Bj, P.Bx, a0, a1, lane, gid,
                                        gm.tmp, gm.stage, ins);
  } else {
    const int S = subgroup_width_avg(f, a1 - a0, G);
    for_products_balanced<G, false, PT, VT>(P.Aj, P.Ax, P.Bp, P.Bj, P.Bx, a0, a1, f, S, lane,
                                            gid, gm.lst, gm.nl, gm.cap, ins);
  }
  for_addend<false>(P, m.r, lane, G, ins);
  group_sync<G>(gid);
  prof_sub_g(A, 10, tp, lane == 0);
  int64_t total;
  if constexpr (G == 32)
    total = int64_t(__reduce_add_sync(0xffffffffu, unsigned(cnt)));  // cnt <= T <= 2^15
  else
    total = group_sum<G, int64_t>(int64_t(cnt), gm.tmp, gid);
  if (lane == 0) A.rowc[m.g] = int32_t(total);
  group_sync<G>(gid);
  prof_sub_g(A, 11, tp, lane == 0);
}

template <int NT, typename PT, typename VT>
__device__ void sym_dense_row(const ProdDev<PT, VT> *prods, const PhaseArgs &A,
                              int64_t idx, unsigned char *smem, const GroupMem &gm) {
  int64_t *scan_tmp = gm.tmp;
  const int tid = threadIdx.x;
  uint32_t *bm = (uint32_t *)smem;
  const RowRef rr = decode_row(A, idx);
  const ProdDev<PT, VT> &P = prods[rr.p];
  const int64_t n = P.n;
  const int64_t a0 = P.Ap[rr.r], a1 = P.Ap[rr.r + 1];
  const int S = subgroup_width_avg(A.rowf[rr.g], a1 - a0, 32);
  const int64_t W = n < kDenseBits ? n : kDenseBits;
  int64_t total = 0;
  for (int64_t w0 = 0; w0 < n; w0 += W) {
    const int64_t w1 = (w0 + W < n) ? w0 + W : n;
    const int64_t nw = (w1 - w0 + 31) >> 5;
    for (int64_t i = tid; i < nw; i += NT) bm[i] = 0u;
    __syncthreads();
    // columns are below 2^31: one unsigned compare tests w0 <= col < w1
    const uint32_t uw0 = uint32_t(w0), uW = uint32_t(w1 - w0);
    auto mark = [&](int32_t col, VT) {
      const uint32_t o = uint32_t(col) - uw0;
      if (o < uW) {
        const uint32_t bit = 1u << (o & 31);
        if (!(((volatile uint32_t *)bm)[o >> 5] & bit)) atomicOr(bm + (o >> 5), bit);
      }
    };
    for_products_balanced<NT, false, PT, VT>(P.Aj, P.Ax, P.Bp, P.Bj, P.Bx, a0, a1,
                                             A.rowf[rr.g], S, tid, 0, gm.lst, gm.nl, gm.cap,
                                             mark, gm.nl - 1);
    for_addend<false>(P, rr.r, tid, NT, mark);
    __syncthreads();
    int64_t local = 0;
    for (int64_t i = tid; i < nw; i += NT) local += __popc(bm[i]);
    total += group_sum<NT, int64_t>(local, scan_tmp, 0);
  }
  if (tid == 0) A.rowc[rr.g] = int32_t(total);
}

// ---------------------------------------------------------------- numeric

// Bitonic sort of P (pow2) pairs by key, in place.
template <int G, typename VT>
__device__ __forceinline__ void bitonic_pairs(int *keys, VT *vals, uint32_t P,
                                              int gid, int lane) {
  for (uint32_t k = 2; k <= P; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t t = lane; t < (P >> 1); t += G) {
        const uint32_t i = 2 * t - (t & (j - 1));
        const uint32_t l = i + j;
        const bool up = (i & k) == 0;
        const int ki = keys[i], kl = keys[l];
        if ((ki > kl) == up) {
          keys[i] = kl;
          keys[l] = ki;
          const VT vi = vals[i];
          vals[i] = vals[l];
          vals[l] = vi;
        }
      }
      group_sync<G>(gid);
    }
  }
}

// Bitonic sort of one (key, value) pair per lane across a warp, ascending by
// key, in registers: lanes i < l = i ^ j compare-exchange, the lower lane
// keeping the smaller key in ascending blocks ((i & k) == 0).  Equal keys stay
// put, so duplicates survive as adjacent pairs.
template <typename VT>
__device__ __forceinline__ void warp_bitonic32(int &key, VT &val, int lane) {
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      const int pk = __shfl_xor_sync(0xffffffffu, key, j);
      const VT pv = __shfl_xor_sync(0xffffffffu, val, j);
      const bool keep_min = ((lane & j) == 0) == ((lane & k) == 0);
      if (keep_min ? pk < key : pk > key) {
        key = pk;
        val = pv;
      }
    }
  }
}

// Stable LSD radix sort of n <= ITEMS*G (key, value) pairs with RB-bit digits
// (RAD * ITEMS = 512: fewer items per thread buy wider digits, so fewer
// passes, in the same 1 KiB of counters per warp).  Element e sits at item
// e / G of thread e % G; within a warp, equal digits are ranked with
// __match_any_sync.  cnt holds RAD digits x ITEMS x G/32 warps uint16
// counters laid out (digit, item, warp), so one exclusive scan over cnt
// yields every element's output base in stable order.  (ka, va) and (kb, vb)
// alternate as source and destination; returns 1 when the sorted pairs end in
// (kb, vb).
template <int G, int ITEMS, int RB, typename VT>
__device__ int radix_pairs(int *ka, VT *va, int *kb, VT *vb, int n, int bits,
                           uint16_t *cnt, int64_t *tmp, int gid, int lane) {
  constexpr int NW = G / 32, RAD = 1 << RB;
  static_assert(RAD * ITEMS == 512, "1 KiB of counters per warp");
  constexpr int E = RAD * ITEMS * NW, PER = E / G;
  static_assert(PER * G == E, "counter layout");
  const int w = lane >> 5;
  const unsigned below = (1u << (lane & 31)) - 1u;
  int src = 0;
  for (int shift = 0; shift < bits; shift += RB) {
    const int *ks = src ? kb : ka;
    const VT *vs = src ? vb : va;
    int *kd = src ? ka : kb;
    VT *vd = src ? va : vb;
    for (int i = lane; i < E; i += G) cnt[i] = 0;
    group_sync<G>(gid);
    int dig[ITEMS], rk[ITEMS];
#pragma unroll
    for (int it = 0; it < ITEMS; ++it) {
      dig[it] = RAD;
      rk[it] = 0;
      if (it * G < n) {  // uniform across the group
        const int e = it * G + lane;
        const int d = e < n ? ((ks[e] >> shift) & (RAD - 1)) : RAD;
        const unsigned m = __match_any_sync(0xffffffffu, d);
        rk[it] = __popc(m & below);
        dig[it] = d;
        if (d < RAD && rk[it] == 0) cnt[(d * ITEMS + it) * NW + w] = uint16_t(__popc(m));
      }
    }
    group_sync<G>(gid);
    int s = 0;
#pragma unroll
    for (int j = 0; j < PER; ++j) s += cnt[lane * PER + j];
    int64_t tot;
    int run = int(group_excl_scan<G, int64_t>(int64_t(s), tmp, gid, &tot));
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      const int v = cnt[lane * PER + j];
      cnt[lane * PER + j] = uint16_t(run);
      run += v;
    }
    group_sync<G>(gid);
#pragma unroll
    for (int it = 0; it < ITEMS; ++it) {
      const int e = it * G + lane;
      if (e < n) {
        const int pos = int(cnt[(dig[it] * ITEMS + it) * NW + w]) + rk[it];
        kd[pos] = ks[e];
        vd[pos] = vs[e];
      }
    }
    group_sync<G>(gid);
    src ^= 1;
  }
  return src;
}

// Output of a warp row whose table has at most 64 slots (so c <= 32): slot
// s = lane + 32 h is compacted by ballots into a list of the row's columns
// behind the table (keys + 64), and every column's output position is its
// rank in that list (the columns are distinct), counted with broadcast reads;
// no sort.  With CS > 0 the values are spread over NC copies CS apart.  The
// row goes to oj / ox; c is the count the symbolic phase found (checked), or
// -1 when none did (one-pass rows).  Returns the row's count.
template <int NC, typename VT>
__device__ __forceinline__ int warp_lean_output(const PhaseArgs &A, int *keys, const VT *vals,
                                                uint32_t T, uint32_t CS, int64_t c,
                                                int32_t *__restrict__ oj, VT *__restrict__ ox,
                                                int lane) {
  const unsigned lt = (1u << lane) - 1u;
  const int k0 = keys[lane];
  const int k1 = T > 32 ? keys[lane + 32] : -1;
  VT v0 = vals[lane];
  VT v1 = T > 32 ? vals[lane + 32] : VT(0);
  if (CS > 0) {
#pragma unroll
    for (int k = 1; k < NC; ++k) {
      v0 += vals[k * CS + lane];
      if (T > 32) v1 += vals[k * CS + lane + 32];
    }
  }
  const unsigned m0 = __ballot_sync(0xffffffffu, k0 != -1);
  const unsigned m1 = __ballot_sync(0xffffffffu, k1 != -1);
  const int n0 = __popc(m0), nt = n0 + __popc(m1);
  int *lk = keys + 64;  // behind the table (the key array has >= 128 slots)
  if (k0 != -1) lk[__popc(m0 & lt)] = k0;
  if (k1 != -1) lk[n0 + __popc(m1 & lt)] = k1;
  __syncwarp();
  int r0 = 0, r1 = 0;
  for (int j = 0; j < nt; ++j) {
    const int kj = lk[j];
    r0 += kj < k0;
    r1 += kj < k1;
  }
  if (c < 0) c = nt;
  else if (lane == 0 && nt != c) set_error(A.err, 103);
  if (k0 != -1 && r0 < c) {
    oj[r0] = k0;
    ox[r0] = v0;
  }
  if (k1 != -1 && r1 < c) {
    oj[r1] = k1;
    ox[r1] = v1;
  }
  __syncwarp();  // the next row clears the table
  return nt;
}

// ONEPASS (rows of a plain product taken by a warp in the symbolic launch):
// m.off is the row's scratch offset; the row is written to the scratch
// (A.oj / A.ox) with the count found here, which goes to rowc, and rowf
// becomes -1 - offset (the numeric launch copies the row into C and skips it
// otherwise).  A row whose bound min(products, ncols) needs more than 64
// slots and which holds kCappedCols columns or more is instead listed in
// A.defer for the two-pass path (its symbolic count follows in the same
// launch sequence).
template <int G, int TMAX, typename PT, typename VT, bool ONEPASS = false>
__device__ void num_hash_row(const ProdDev<PT, VT> *prods, const PhaseArgs &A,
                             const RowMeta &m, unsigned char *slice, const GroupMem &gm,
                             int gid, int lane) {
  int64_t *tmp = gm.tmp;
  int *itmp = gm.itmp;
  uint16_t *cnt = gm.cnt;
  constexpr int KEEP = TMAX / (2 * G);  // first-half slots held per thread
  static_assert(KEEP >= 1 && KEEP <= 16 && KEEP * 2 * G == TMAX, "compaction layout");
  VT *vals = (VT *)slice;
  int *keys = (int *)(slice + TMAX * 8);
  long long tp = clock64();
  const ProdDev<PT, VT> &P = prods[m.p];
  // one-pass rows: the output bound until the compaction counts the row
  int64_t c = ONEPASS ? (m.f < P.n ? m.f : P.n) : m.c;
  const int64_t off = m.off;
  int32_t *const oj = ONEPASS ? A.oj + off : P.Cj + off;
  VT *const ox = ONEPASS ? (VT *)A.ox + off : P.Cx + off;
  uint32_t Tfull = pow2_at_least(A.S->tune.load * c, 32);
  if (Tfull > TMAX) Tfull = TMAX;
  // Warp rows of at most 64 slots spread their values over NC copies of the
  // value table (lane & (NC - 1) picks one; copies 16 bytes apart in banks):
  // the FP64 shared atomics of lanes that hit one column in one step contend
  // (products of neighbouring B rows share columns: Galerkin A·P numeric
  // phase 3.72 ms with one table, 3.45 ms with 4 copies).
  constexpr int NC = G == 32 ? 4 : 1;
  static_assert(NC * (64 + 4) * 8 <= TMAX * 8, "value copies");
  // A one-pass row whose bound needs more than 64 slots tries 64 (its count
  // is unknown; the Galerkin A·P rows bound ~119 and hold ~12): once 32
  // columns are in (a counter in the warp's list slot) no new column gets a
  // slot, and a refused column sends the row to the two-pass path.
  bool capped = ONEPASS && G == 32 && Tfull > 64;
  int *ocnt = gm.lst;  // warp rows: [0] admitted columns, [1] refused
  uint32_t T = Tfull;
  int logT = 0;
  uint32_t mask = 0;
  const int64_t a0 = m.a0, a1 = m.a1;
  {  // the table, the products and (tables of at most 64 slots) the output
    T = capped ? 64 : Tfull;
    logT = ilog2_pow2(T);
    mask = T - 1;
    const bool copies = NC > 1 && T <= 64;
    const uint32_t CS = T + 16 / uint32_t(sizeof(VT));  // copy stride
    clear_keys<G>(keys, T, lane);
    clear_vals<G, VT>(vals, copies ? NC * CS : T, lane);
    if (capped && lane == 0) ocnt[0] = ocnt[1] = 0;
    group_sync<G>(gid);
    prof_sub_g(A, 9, tp, lane == 0);
    VT *myv = copies ? vals + (lane & (NC - 1)) * CS : vals;
    auto ins = [&](int32_t col, VT v) {
      uint32_t h;
      if (capped) {
        h = num_insert_capped(keys, col, logT, mask, ocnt, T / 2);
        if (h == kRefused) return;
      } else {
        h = num_insert(keys, col, logT, mask, A.err);
      }
      atomicAdd(myv + h, v);
    };
    if constexpr (G <= 256) {
      for_products_flat<G, true, PT, VT>(P.Aj, P.Ax, P.Bp, P.Bj, P.Bx, a0, a1, lane, gid,
                                         gm.tmp, gm.stage, ins);
    } else {
      const int S = subgroup_width_avg(m.f, a1 - a0, G);
      for_products_balanced<G, true, PT, VT>(P.Aj, P.Ax, P.Bp, P.Bj, P.Bx, a0, a1, m.f, S,
                                             lane, gid, gm.lst, gm.nl, gm.cap, ins);
    }
    for_addend<true>(P, m.r, lane, G, ins);
    group_sync<G>(gid);
    prof_sub_g(A, 10, tp, lane == 0);
    if (capped) {
      const bool refused = ((volatile int *)ocnt)[1] != 0;
      __syncwarp();
      if (refused) {  // 32 columns or more: the two-pass path
        if (lane == 0) {
          const unsigned long long i = atomicAdd(&A.S->ndefer, 1ull);
          A.defer[i] = (uint64_t(m.p) << 40) | uint64_t(m.r);
        }
        __syncwarp();
        return;
      }
    }
    if constexpr (G == 32) {
      if (T <= 64) {
        const int nt = warp_lean_output<NC>(A, keys, vals, T, copies ? CS : 0,
                                            ONEPASS ? -1 : c, oj, ox, lane);
        if (ONEPASS && lane == 0) {
          A.rowc[m.g] = nt;
          A.rowf[m.g] = -1 - off;
        }
        prof_sub_g(A, 13, tp, lane == 0);
        return;
      }
    }
  }
  // In-place compaction into [0, c): targets lie in the first half (c <= T/2),
  // so first-half slots are held in registers across the group barrier inside
  // group_minmax; second-half slots are never overwritten.
  const uint32_t H = T >> 1;
  int rk[KEEP];
  VT rv[KEEP];
  int mine = 0, mn = INT32_MAX, mx = -1;
#pragma unroll
  for (int i = 0; i < KEEP; ++i) {
    const uint32_t s = lane + i * G;
    rk[i] = -1;
    rv[i] = VT(0);
    if (s < H) {
      rk[i] = keys[s];
      rv[i] = vals[s];
    }
    if (rk[i] != -1) {
      ++mine;
      mn = min(mn, rk[i]);
      mx = max(mx, rk[i]);
    }
  }
  for (uint32_t s = H + lane; s < T; s += G) {
    const int k = keys[s];
    if (k != -1) {
      ++mine;
      mn = min(mn, k);
      mx = max(mx, k);
    }
  }
  group_minmax<G>(mn, mx, itmp, gid);
  int64_t tot;
  int64_t pos = group_excl_scan<G, int64_t>(int64_t(mine), tmp, gid, &tot);
  group_sync<G>(gid);
  if (ONEPASS) c = tot;
  else if (lane == 0 && tot != c) set_error(A.err, 103);
  if (ONEPASS && lane == 0) {
    A.rowc[m.g] = int32_t(c);
    A.rowf[m.g] = -1 - off;
  }
  const bool radix = c > kBitonicMax;
  const int bias = radix ? mn : 0;
#pragma unroll
  for (int i = 0; i < KEEP; ++i) {
    if (rk[i] != -1) {
      keys[pos] = rk[i] - bias;
      vals[pos] = rv[i];
      ++pos;
    }
  }
  for (uint32_t s = H + lane; s < T; s += G) {
    const int k = keys[s];
    if (k != -1) {
      const VT v = vals[s];
      keys[pos] = k - bias;
      vals[pos] = v;
      ++pos;
    }
  }
  group_sync<G>(gid);
  prof_sub_g(A, 11, tp, lane == 0);
  if constexpr (G == 32) {
    if (c <= 32) {  // warp rows of up to 32 outputs sort in registers
      int k = lane < c ? keys[lane] : INT32_MAX;
      VT v = lane < c ? vals[lane] : VT(0);
      warp_bitonic32<VT>(k, v, lane);
      prof_sub_g(A, 12, tp, lane == 0);
      if (lane < c) {
        oj[lane] = k;
        ox[lane] = v;
      }
      __syncwarp();
      prof_sub_g(A, 13, tp, lane == 0);
      return;
    }
  }
  int src = 0;
  if (!radix) {
    const uint32_t Pw = pow2_at_least(c, 2);
    for (uint32_t s = uint32_t(c) + lane; s < Pw; s += G) keys[s] = INT32_MAX;
    group_sync<G>(gid);
    bitonic_pairs<G, VT>(keys, vals, Pw, gid, lane);
  } else {
    const int bits = 32 - __clz(mx - mn);
    // widest digits whose item count still holds the row
    if (KEEP >= 4 && c <= 4 * G)
      src = radix_pairs<G, (KEEP < 4 ? KEEP : 4), (KEEP < 4 ? 5 : 7), VT>(
          keys, vals, keys + H, vals + H, int(c), bits, cnt, tmp, gid, lane);
    else if (KEEP >= 8 && c <= 8 * G)
      src = radix_pairs<G, (KEEP < 8 ? KEEP : 8), (KEEP < 8 ? 5 : 6), VT>(
          keys, vals, keys + H, vals + H, int(c), bits, cnt, tmp, gid, lane);
    else
      src = radix_pairs<G, 16, 5, VT>(keys, vals, keys + H, vals + H, int(c), bits, cnt, tmp,
                                      gid, lane);
  }
  prof_sub_g(A, 12, tp, lane == 0);
  const int *ko = src ? keys + H : keys;
  const VT *vo = src ? vals + H : vals;
  for (int64_t s = lane; s < c; s += G) {
    oj[s] = ko[s] + bias;
    ox[s] = vo[s];
  }
  group_sync<G>(gid);
  prof_sub_g(A, 13, tp, lane == 0);
}

// Numeric group row by expand-sort-compress, for rows with at most TMAX / 2
// products of which few repeat a column (the uniform-random rows of batched
// products): the products (and the addend row) are written to the slice in
// product order, sorted by column (the row radix sort), and runs of equal
// columns are summed as they are written out.  No hash table to clear, probe
// or compact; the sort sees f <= 2 c entries instead of c.
template <int G, int TMAX, typename PT, typename VT>
__device__ void num_esc_row(const ProdDev<PT, VT> *prods, const PhaseArgs &A, const RowMeta &m,
                            unsigned char *slice, const GroupMem &gm, int gid, int lane) {
  constexpr int U = 4, FMAX = TMAX / 2, KEEP = TMAX / (2 * G);
  VT *vals = (VT *)slice;  // [0, FMAX) and [FMAX, TMAX): the sort's two buffers
  int *keys = (int *)(slice + TMAX * 8);
  int64_t *spre = (int64_t *)gm.stage;  // G > 32: the chunk's entries
  int64_t *sb0 = spre + G;
  VT *sa = (VT *)(sb0 + G);
  long long tp = clock64();
  const ProdDev<PT, VT> &P = prods[m.p];
  const int64_t c = m.c;
  const int f = int(m.f);  // <= FMAX by the caller's test
  const int64_t off = m.off;
  const int64_t a0 = m.a0, a1 = m.a1;
  prof_sub_g(A, 9, tp, lane == 0);
  // expand: every product at its flat index
  int fb = 0;
  for (int64_t c0 = a0; c0 < a1; c0 += G) {
    const int nc = int(min(int64_t(G), a1 - c0));
    int64_t len = 0, b0 = 0;
    VT a = VT(0);
    if (lane < nc) {
      const int64_t k = __ldg(P.Aj + c0 + lane);
      a = __ldg(P.Ax + c0 + lane);
      b0 = int64_t(__ldg(P.Bp + k));
      len = int64_t(__ldg(P.Bp + k + 1)) - b0;
    }
    int64_t tot, pre;
    if constexpr (G == 32) {
      const int64_t inc = warp_scan_incl(len);
      tot = __shfl_sync(0xffffffffu, inc, 31);
      pre = inc - len;
    } else {
      pre = group_excl_scan<G, int64_t>(len, gm.tmp, gid, &tot);
      if (lane < nc) {
        spre[lane] = pre;
        sb0[lane] = b0;
        sa[lane] = a;
      }
      group_sync<G>(gid);
    }
    for (int64_t pb = 0; pb < tot; pb += int64_t(G) * U) {
      int32_t cc[U];
      VT xv[U], av[U];
      int64_t at[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int64_t p = pb + int64_t(u) * G + lane;
        int j = 0;
        int64_t pj, bj;
        if constexpr (G == 32) {
#pragma unroll
          for (int st = 16; st > 0; st >>= 1) {
            const int64_t v = __shfl_sync(0xffffffffu, pre, (j + st) & 31);
            if (j + st < nc && v <= p) j += st;
          }
          pj = __shfl_sync(0xffffffffu, pre, j);
          bj = __shfl_sync(0xffffffffu, b0, j);
          av[u] = __shfl_sync(0xffffffffu, a, j);
        } else {
          for (int st = G / 2; st > 0; st >>= 1)
            if (j + st < nc && spre[j + st] <= p) j += st;
          pj = spre[j];
          bj = sb0[j];
          av[u] = sa[j];
        }
        const int64_t q = bj + (p - pj);
        at[u] = p < tot ? fb + p : -1;
        cc[u] = p < tot ? __ldg(P.Bj + q) : 0;
        xv[u] = p < tot ? __ldg(P.Bx + q) : VT(0);
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (at[u] >= 0 && at[u] < FMAX) {
          keys[at[u]] = cc[u];
          vals[at[u]] = av[u] * xv[u];
        }
      }
    }
    fb += int(tot);
    group_sync<G>(gid);  // the next chunk reuses the staging
  }
  if (P.Ej) {
    int64_t e0, e1;
    addend_row(P, m.r, e0, e1);
    for (int64_t q = e0 + lane; q < e1; q += G) {
      const int64_t at = fb + (q - e0);
      if (at < FMAX) {
        keys[at] = __ldg(P.Ej + q);
        vals[at] = __ldg(P.Ex + q);
      }
    }
    fb += int(e1 - e0);
  }
  group_sync<G>(gid);
  if (lane == 0 && fb != f) set_error(A.err, 107);
  prof_sub_g(A, 10, tp, lane == 0);
  if constexpr (G == 32) {
    if (f <= 32) {  // up to 32 products: sort and compress in registers
      int k = lane < f ? keys[lane] : INT32_MAX;
      VT v = lane < f ? vals[lane] : VT(0);
      prof_sub_g(A, 11, tp, lane == 0);
      warp_bitonic32<VT>(k, v, lane);
      prof_sub_g(A, 12, tp, lane == 0);
      // sum each run of equal columns into its first lane (suffix sums inside
      // runs; keys are sorted, so equal keys are contiguous, and no column
      // equals the INT32_MAX padding)
      const int kprev = __shfl_up_sync(0xffffffffu, k, 1);
      const bool head = lane < f && (lane == 0 || kprev != k);
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int nk = __shfl_down_sync(0xffffffffu, k, o);
        const VT nv = __shfl_down_sync(0xffffffffu, v, o);
        if (lane + o < 32 && nk == k) v += nv;
      }
      const unsigned hm = __ballot_sync(0xffffffffu, head);
      const int pos = __popc(hm & ((1u << lane) - 1u));
      if (head && pos < c) {
        P.Cj[off + pos] = k;
        P.Cx[off + pos] = v;
      }
      if (lane == 0 && __popc(hm) != c) set_error(A.err, 108);
      __syncwarp();
      prof_sub_g(A, 13, tp, lane == 0);
      return;
    }
  }
  int mn = INT32_MAX, mx = -1;
  for (int e = lane; e < f; e += G) {
    mn = min(mn, keys[e]);
    mx = max(mx, keys[e]);
  }
  group_minmax<G>(mn, mx, gm.itmp, gid);
  int src = 0, bias = 0;
  if (f <= kBitonicMax) {
    const uint32_t Pw = pow2_at_least(f, 2);
    for (uint32_t e = uint32_t(f) + lane; e < Pw; e += G) keys[e] = INT32_MAX;
    group_sync<G>(gid);
    prof_sub_g(A, 11, tp, lane == 0);
    bitonic_pairs<G, VT>(keys, vals, Pw, gid, lane);
  } else {
    bias = mn;
    for (int e = lane; e < f; e += G) keys[e] -= bias;
    group_sync<G>(gid);
    prof_sub_g(A, 11, tp, lane == 0);
    const int bits = mx > mn ? 32 - __clz(mx - mn) : 1;
    if (KEEP >= 4 && f <= 4 * G)
      src = radix_pairs<G, (KEEP < 4 ? KEEP : 4), (KEEP < 4 ? 5 : 7), VT>(
          keys, vals, keys + FMAX, vals + FMAX, f, bits, gm.cnt, gm.tmp, gid, lane);
    else if (KEEP >= 8 && f <= 8 * G)
      src = radix_pairs<G, (KEEP < 8 ? KEEP : 8), (KEEP < 8 ? 5 : 6), VT>(
          keys, vals, keys + FMAX, vals + FMAX, f, bits, gm.cnt, gm.tmp, gid, lane);
    else
      src = radix_pairs<G, 16, 5, VT>(keys, vals, keys + FMAX, vals + FMAX, f, bits, gm.cnt,
                                      gm.tmp, gid, lane);
  }
  prof_sub_g(A, 12, tp, lane == 0);
  // compress: the first entry of every run of equal columns sums its run
  const int *ko = src ? keys + FMAX : keys;
  const VT *vo = src ? vals + FMAX : vals;
  int32_t *__restrict__ Cj = P.Cj + off;
  VT *__restrict__ Cx = P.Cx + off;
  int64_t running = 0;
  for (int e0 = 0; e0 < f; e0 += G) {
    const int e = e0 + lane;
    const int key = e < f ? ko[e] : 0;
    const bool head = e < f && (e == 0 || ko[e - 1] != key);
    int64_t ctot;
    const int64_t pos = running + group_excl_scan<G, int64_t>(head ? 1 : 0, gm.tmp, gid, &ctot);
    if (head) {
      VT v = vo[e];
      for (int k = e + 1; k < f && ko[k] == key; ++k) v += vo[k];
      if (pos < c) {
        Cj[pos] = key + bias;
        Cx[pos] = v;
      }
    }
    running += ctot;
  }
  if (lane == 0 && running != c) set_error(A.err, 108);
  group_sync<G>(gid);
  prof_sub_g(A, 13, tp, lane == 0);
}

// DENSE numeric row, whole-row form (ncols <= kRankMaxCols).  Pass 1 sets the
// row's column bitmap; a CTA scan of the bitmap gives every word's rank base
// (block base + uint16 offset inside the block); the row's values are zeroed
// (coalesced) and its sorted column indices written with the work balanced
// by entries, not by words (R-MAT bitmaps are far denser at the hub columns);
// pass 2 adds every product into its output slot, found as base + popc of the
// bits below, with a fire-and-forget global FP64 reduction.  No sort.
template <int NT, typename PT, typename VT>
__device__ void num_dense_rank_row(const ProdDev<PT, VT> *prods, const PhaseArgs &A,
                                   int64_t idx, unsigned char *smem, const GroupMem &gm) {
  const int tid = threadIdx.x;
  const RowRef rr = decode_row(A, idx);
  const ProdDev<PT, VT> &P = prods[rr.p];
  const int64_t n = P.n;
  const int nw = int((n + 31) >> 5);
  const int nb = (nw + 31) >> 5;
  // Bitmap word w lives at slot w ^ ((w >> 6) & 31): a bijection inside each
  // 32-word block that spreads threads walking words ~64 apart over all banks.
  uint32_t *bm = (uint32_t *)smem;
  uint16_t *wp = (uint16_t *)(smem + size_t(nb) * 128);
  int *bbase = (int *)(smem + size_t(nb) * 192);
  auto bmw = [&](int w) -> uint32_t & { return bm[w ^ ((w >> 6) & 31)]; };
  const int64_t a0 = P.Ap[rr.r], a1 = P.Ap[rr.r + 1], na = a1 - a0;
  const int64_t f = A.rowf[rr.g];
  const int64_t c = A.rowc[rr.g];
  const int32_t *__restrict__ Aj = P.Aj;
  const VT *__restrict__ Ax = P.Ax;
  const PT *__restrict__ Bp = P.Bp;
  const int32_t *__restrict__ Bj = P.Bj;
  const VT *__restrict__ Bx = P.Bx;
  const int S1 = subgroup_width_avg(f, na, 32);
  long long tp = clock64();
  for (int i = tid; i < nb * 32; i += NT) bm[i] = 0u;
  __syncthreads();
  auto mark = [&](int32_t col, VT) {
    const uint32_t bit = 1u << (col & 31);
    uint32_t &x = bmw(col >> 5);
    if (!(*(volatile uint32_t *)&x & bit)) atomicOr(&x, bit);
  };
  for_products_balanced<NT, false, PT, VT>(Aj, Ax, Bp, Bj, Bx, a0, a1, f, S1, tid, 0,
                                                 gm.lst, gm.nl, gm.cap, mark, gm.nl - 1);
  for_addend<false>(P, rr.r, tid, NT, mark);
  __syncthreads();
  prof_sub(A, 0, tp);
  // Block scan: block b = words [32b, 32b + 32), lane l of a warp takes word
  // 32b + l (no bank conflicts).  wp[w] = rank of word w's first bit within
  // its block (< 1024), bbase[b] = rank of block b's first bit.
  {
    const int warp = tid >> 5, lane = tid & 31;
    // four blocks per step: their scans are independent, so their shuffle
    // latencies overlap
    constexpr int NW = NT / 32, UB = 4;
    for (int b0 = warp; b0 < nb; b0 += NW * UB) {
      int pc[UB], inc[UB];
#pragma unroll
      for (int u = 0; u < UB; ++u) {
        const int w = ((b0 + u * NW) << 5) + lane;
        pc[u] = (b0 + u * NW < nb && w < nw) ? __popc(bmw(w)) : 0;
      }
#pragma unroll
      for (int u = 0; u < UB; ++u) inc[u] = warp_scan_incl(pc[u]);
#pragma unroll
      for (int u = 0; u < UB; ++u) {
        const int b = b0 + u * NW, w = (b << 5) + lane;
        if (b < nb) {
          if (w < nw) wp[w] = uint16_t(inc[u] - pc[u]);
          if (lane == 31) bbase[b] = inc[u];
        }
      }
    }
  }
  __syncthreads();
  {
    constexpr int BPT = 3;  // blocks per thread: nb <= kRankMaxCols / 1024 < 3 * NT
    int v[BPT], sum = 0;
#pragma unroll
    for (int k = 0; k < BPT; ++k) {
      const int b = tid * BPT + k;
      v[k] = b < nb ? bbase[b] : 0;
      sum += v[k];
    }
    int64_t tot;
    // the scan ends on a barrier, so every read of bbase above is done
    int run = int(group_excl_scan<NT, int64_t>(int64_t(sum), gm.tmp, 0, &tot));
#pragma unroll
    for (int k = 0; k < BPT; ++k) {
      const int b = tid * BPT + k;
      if (b < nb) bbase[b] = run;
      run += v[k];
    }
    if (tid == 0 && tot != c) set_error(A.err, 104);
  }
  __syncthreads();
  prof_sub(A, 1, tp);
  const int64_t off = A.cp[rr.g] - A.cp[A.base[rr.p]];
  int32_t *__restrict__ Cj = P.Cj + off;
  VT *__restrict__ Cx = P.Cx + off;
  // zeroed values: a contiguous range, coalesced
  // the values stay in L2 for the reductions, the indices may leave first
  const uint64_t keep = policy_evict_last(), pass = policy_evict_first();
  {
    // 16-byte stores from the first 16-byte boundary, scalar head and tail
    const int64_t bytes = c * int64_t(sizeof(VT));
    const int64_t head = min(bytes, int64_t((16 - (reinterpret_cast<uintptr_t>(Cx) & 15)) & 15));
    const int64_t hn = head / int64_t(sizeof(VT));
    const int64_t nv = (bytes - head) >> 4;
    const int64_t t0 = hn + nv * int64_t(16 / sizeof(VT));
    unsigned char *const zb = reinterpret_cast<unsigned char *>(Cx) + head;
    for (int64_t e = tid; e < hn; e += NT) store_hint(Cx + e, VT(0), keep);
    for (int64_t v = tid; v < nv; v += NT) store_zero16(zb + (v << 4), keep);
    for (int64_t e = t0 + tid; e < c; e += NT) store_hint(Cx + e, VT(0), keep);
  }
  prof_sub(A, 2, tp);
  // Column indices.  The bitmap walk is a merge of two sequences, the words
  // and the set bits (nw + c steps: every bit, then a step to the next word);
  // thread t takes steps [d_t, d_t+1), d_t = t * (nw + c) / NT (merge-
  // path split), so threads get equal work however the bits cluster, and the
  // loop below takes exactly one step per iteration, so the lanes of a warp
  // stay in step.  A split point is found by searching w + rank(w) over the
  // block bases, then over the word offsets of one block.
  {
    const int64_t steps = int64_t(nw) + c;
    const int64_t d0 = steps * tid / NT, d1 = steps * (tid + 1) / NT;
    int lo = 0, hi = nb - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (int64_t(mid) * 32 + bbase[mid] <= d0) lo = mid; else hi = mid - 1;
    }
    int w = lo << 5, wh = min(nw, (lo + 1) << 5) - 1;
    while (w < wh) {
      const int mid = (w + wh + 1) >> 1;
      if (int64_t(mid) + bbase[lo] + wp[mid] <= d0) w = mid; else wh = mid - 1;
    }
    int e = int(d0 - w);  // first rank of this thread
    uint32_t word = bmw(w);
    // the lowest e - rank(w) set bits of this word belong to earlier threads
    for (int k = e - bbase[w >> 5] - int(wp[w]); k > 0; --k) word &= word - 1u;
    // the next four words are loaded ahead, so runs of empty words do not
    // wait on one shared-memory load per step
    uint32_t n0 = w + 1 < nw ? bmw(w + 1) : 0u, n1 = w + 2 < nw ? bmw(w + 2) : 0u;
    uint32_t n2 = w + 3 < nw ? bmw(w + 3) : 0u, n3 = w + 4 < nw ? bmw(w + 4) : 0u;
    for (int64_t d = d0; d < d1; ++d) {
      if (word != 0u) {
        if (e < c)  // e < c unless rank sums broke
          store_hint(Cj + e, int32_t(w * 32 + (__ffs(word) - 1)), pass);
        ++e;
        word &= word - 1u;
      } else {
        ++w;
        word = n0;
        n0 = n1;
        n1 = n2;
        n2 = n3;
        n3 = w + 4 < nw ? bmw(w + 4) : 0u;
      }
    }
  }
  __syncthreads();
  prof_sub(A, 3, tp);
  auto rank_of = [&](int32_t col) {
    const int w = col >> 5;
    return bbase[w >> 5] + int(wp[w]) + __popc(bmw(w) & ((1u << (col & 31)) - 1u));
  };
  auto put = [&](int32_t col, VT v) { red_add_hint(Cx + rank_of(col), v, keep); };
  for_products_balanced<NT, true, PT, VT>(Aj, Ax, Bp, Bj, Bx, a0, a1, f, S1, tid, 0,
                                                gm.lst, gm.nl, gm.cap, put, gm.nl - 1);
  for_addend<true>(P, rr.r, tid, NT, put);
  __syncthreads();
  prof_sub(A, 4, tp);
}

// DENSE numeric row, column windows of kDenseW.  Each window accumulates in
// a dense shared FP64 array plus a presence bitmap (shared atomics, no global
// reductions) and is emitted in column order, so a heavy row's output is
// written once.  With sorted B every A entry keeps a cursor into its B row and
// the first column at the cursor: an entry with nothing in the window costs
// one shared load, and one thread walks an entry's window segment with U
// loads in flight (stopping at the first column past the window).  B rows
// longer than twice a thread's fair share are listed once per row and walked
// by one warp each, U x 32 entries per step, with the same stop rule.  With
// unsorted B every window rescans the rows.
template <typename PT, typename VT>
__device__ void num_dense_row(const ProdDev<PT, VT> *prods, const PhaseArgs &A,
                              int64_t idx, unsigned char *smem, const GroupMem &gm) {
  constexpr int kLongMark = INT32_MIN;
  constexpr int U = 8;
  const int tid = threadIdx.x;
  int64_t *scan_tmp = gm.tmp;
  VT *acc = (VT *)smem;
  uint32_t *bm = (uint32_t *)(smem + kDenseW * sizeof(VT));
  int32_t *cur_s = (int32_t *)(smem + kDenseW * sizeof(VT) + kDenseW / 8);
  int32_t *lcur = cur_s + 2 * kDenseCurSmem;  // cursor of listed entry i
  const RowRef rr = decode_row(A, idx);
  const ProdDev<PT, VT> &P = prods[rr.p];
  const int64_t n = P.n;
  const int64_t a0 = P.Ap[rr.r], a1 = P.Ap[rr.r + 1], na = a1 - a0;
  const int64_t f = A.rowf[rr.g];
  // cursor (offset into the B row) and the column at the cursor, per A entry
  int32_t *cur = na <= kDenseCurSmem ? cur_s : A.curbuf + 2 * blockIdx.x * A.cur_stride;
  int32_t *nxc = na <= kDenseCurSmem ? cur_s + kDenseCurSmem : cur + A.cur_stride;
  const bool sorted = P.b_sorted != 0;
  const int32_t *__restrict__ Aj = P.Aj;
  const VT *__restrict__ Ax = P.Ax;
  const PT *__restrict__ Bp = P.Bp;
  const int32_t *__restrict__ Bj = P.Bj;
  const VT *__restrict__ Bx = P.Bx;
  const int64_t thr = max(int64_t(4 * U), 2 * f / kThreads);
  long long tp = clock64();
  auto add = [&](int32_t o, VT v) {
    atomicAdd(acc + o, v);
    const uint32_t bit = 1u << (o & 31);
    if (!(((volatile uint32_t *)bm)[o >> 5] & bit)) atomicOr(bm + (o >> 5), bit);
  };
  if (tid == 0) *gm.nl = 0;
  for (int i = tid; i < kDenseW; i += kThreads) acc[i] = VT(0);
  for (int i = tid; i < kDenseW / 32; i += kThreads) bm[i] = 0u;
  __syncthreads();
  if (sorted) {
    for (int64_t j = tid; j < na; j += kThreads) {
      const int64_t k = __ldg(Aj + a0 + j);
      const int64_t b0 = __ldg(Bp + k), b1 = __ldg(Bp + k + 1);
      int32_t c0 = 0, nc = b1 > b0 ? __ldg(Bj + b0) : INT32_MAX;
      if (b1 - b0 > thr) {
        const int slot = atomicAdd(gm.nl, 1);
        if (slot < gm.cap) {
          gm.lst[slot] = int(j);
          lcur[slot] = 0;
          c0 = kLongMark;
          nc = INT32_MAX;
        }
      }
      cur[j] = c0;
      nxc[j] = nc;
    }
  }
  __syncthreads();
  const int nl = sorted ? min(*gm.nl, gm.cap) : 0;
  prof_sub(A, 5, tp);
  int64_t out = A.cp[rr.g] - A.cp[A.base[rr.p]];
  for (int64_t w0 = 0; w0 < n; w0 += kDenseW) {
    const int64_t w1 = (w0 + kDenseW < n) ? w0 + kDenseW : n;
    // short entries: one thread per entry
    for (int64_t j = tid; j < na; j += kThreads) {
      if (sorted && nxc[j] >= w1) continue;  // nothing in this window (or listed)
      const int64_t k = __ldg(Aj + a0 + j);
      const VT a = __ldg(Ax + a0 + j);
      const int64_t b0 = __ldg(Bp + k), b1 = __ldg(Bp + k + 1);
      if (sorted) {
        int64_t q = b0 + cur[j];
        int32_t ncol = INT32_MAX;
        while (q < b1) {
          int32_t cc[U];
          VT xv[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int64_t qq = q + u;
            cc[u] = qq < b1 ? __ldg(Bj + qq) : INT32_MAX;
            xv[u] = qq < b1 ? __ldg(Bx + qq) : VT(0);
          }
          int nin = 0;
#pragma unroll
          for (int u = 0; u < U; ++u) {
            if (cc[u] < w1) {
              add(int32_t(cc[u] - w0), a * xv[u]);
              ++nin;
            } else {
              ncol = min(ncol, cc[u]);
            }
          }
          q += nin;
          if (nin < U) break;
        }
        cur[j] = int32_t(q - b0);
        nxc[j] = ncol;
      } else {
        for (int64_t q = b0; q < b1; ++q) {
          const int32_t col = __ldg(Bj + q);
          if (col >= w0 && col < w1) add(int32_t(col - w0), a * __ldg(Bx + q));
        }
      }
    }
    // the addend row: every window scans it and takes its own columns
    for_addend<true>(P, rr.r, tid, kThreads, [&](int32_t col, VT v) {
      if (col >= w0 && col < w1) add(int32_t(col - w0), v);
    });
    if (A.prof) __syncthreads();  // profiling only: split short / long walks
    prof_sub(A, 6, tp);
    // long entries: warp w walks listed entries w, w + 16, ...; its lanes take
    // U x 32 entries per step and stop at the first column past the window
    for (int i = tid >> 5; i < nl; i += kThreads / 32) {
      const int lane = tid & 31;
      const int64_t p = a0 + gm.lst[i];
      const int64_t k = __ldg(Aj + p);
      const VT a = __ldg(Ax + p);
      const int64_t b0 = __ldg(Bp + k), b1 = __ldg(Bp + k + 1);
      int64_t q = b0 + lcur[i];
      while (q < b1) {
        int32_t cc[U];
        VT xv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int64_t qq = q + u * 32 + lane;
          cc[u] = qq < b1 ? __ldg(Bj + qq) : INT32_MAX;
          xv[u] = qq < b1 ? __ldg(Bx + qq) : VT(0);
        }
        int nin = 0;
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (cc[u] < w1) {
            add(int32_t(cc[u] - w0), a * xv[u]);
            ++nin;
          }
        }
        nin = __reduce_add_sync(0xffffffffu, nin);
        q += nin;
        if (nin < U * 32) break;
      }
      if (lane == 0) lcur[i] = int32_t(q - b0);
    }
    __syncthreads();
    prof_sub(A, 7, tp);
    uint32_t word = tid < kDenseW / 32 ? bm[tid] : 0u;
    int64_t tot;
    int64_t pos = group_excl_scan<kThreads, int64_t>(int64_t(__popc(word)),
                                                     scan_tmp, 0, &tot);
    int32_t *__restrict__ Cj = P.Cj + out;
    VT *__restrict__ Cx = P.Cx + out;
    while (word) {
      const int b = __ffs(word) - 1;
      word &= word - 1;
      const int o = tid * 32 + b;
      Cj[pos] = int32_t(w0 + o);
      Cx[pos] = acc[o];
      acc[o] = VT(0);
      ++pos;
    }
    if (tid < kDenseW / 32) bm[tid] = 0u;
    out += tot;
    __syncthreads();
    prof_sub(A, 8, tp);
  }
}

// DENSE numeric row, column-window form, for heavy rows with sorted B whose
// output fills at least 1/2^fill of the columns (tuning; default 1/16).  The row's columns are swept in
// windows of kWinCols; a window accumulates in a shared FP64 array indexed by
// column — one shared atomic per product, and no bitmap: a slot that still
// holds the bit pattern of -0.0 is empty, because every product is added as
// a*b + 0.0 (never -0.0 under round-to-nearest) and an IEEE sum is -0.0 only
// when all its terms are — then compacted in column order and written to C
// once, coalesced.  No global reductions, no zero fill of C, one pass over
// the products.  Every A entry keeps a cursor into its B row and the column
// at the cursor (an entry with nothing in the window costs one load).
// Pass 1: thread t takes entries t, t + 512, ... and walks U B entries from
// the cursor; an entry whose window segment goes on is queued, and pass 2
// walks each queued segment with a whole warp (U x 32 entries per step), so a
// hub row of B never holds up a warp of short entries (with one thread per
// whole segment, R-MAT rows kept 5 of 32 lanes busy).  Compaction: warp w owns
// 1/16 of the window, takes 32 slots per step, keeps the step ballots in
// registers (lane s holds step s), and a scan of the 16 warp counts places its
// entries.
// The rows the column-window form takes: heavy (>= 2^win products) DENSE rows
// with sorted B whose output fills >= 1/2^fill of the columns.
template <typename PT, typename VT>
__device__ __forceinline__ bool win_row(const ProdDev<PT, VT> &P, int64_t f, int64_t c, const Tune &t) {
  return P.b_sorted && t.win > 0 && f >= (int64_t(1) << t.win) && (c << t.fill) >= P.n;
}

// A product as the window forms add it: never -0.0, so that an accumulator
// slot still holding -0.0 is known to be empty.  Zeros and subnormals are
// added as +0.0 (float atomics flush subnormal operands to a zero of the same
// sign, so a negative subnormal could otherwise arrive as -0.0; the change is
// below the smallest normal number, 1.2e-38 in FP32, 2.2e-308 in FP64).
template <typename VT>
__device__ __forceinline__ VT win_value(VT v) {
  if constexpr (sizeof(VT) == 4) return fabsf(v) < 1.17549435e-38f ? 0.0f : v;
  else return fabs(v) < 2.2250738585072014e-308 ? 0.0 : v;
}

constexpr int kWinCols = 16384;   // columns per window (128 KiB of FP64)
constexpr int kWinQueue = 4096;   // queued long segments per window
static_assert(kWinCols * 8 + 2 * kDenseCurSmem * 4 + kWinQueue * 4 <= kDynSmem, "window smem");

template <typename PT, typename VT>
__device__ void num_dense_win_row(const ProdDev<PT, VT> *prods, const PhaseArgs &A,
                                  int64_t idx, unsigned char *smem, const GroupMem &gm) {
  using UT = std::conditional_t<sizeof(VT) == 8, unsigned long long, unsigned>;
  constexpr UT kEmpty = UT(1) << (sizeof(VT) * 8 - 1);  // -0.0
  constexpr int U = 8;
  constexpr int NWARP = kThreads / 32;
  constexpr int PER = kWinCols / NWARP;  // slots per warp
  constexpr int STEPS = PER / 32;
  static_assert(STEPS == 32, "one ballot per lane");
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  VT *acc = (VT *)smem;
  UT *accb = (UT *)smem;
  int32_t *cur_s = (int32_t *)(smem + kWinCols * sizeof(VT));
  int32_t *nxc_s = cur_s + kDenseCurSmem;
  int32_t *queue = nxc_s + kDenseCurSmem;
  const RowRef rr = decode_row(A, idx);
  const ProdDev<PT, VT> &P = prods[rr.p];
  const int64_t n = P.n;
  const int64_t a0 = P.Ap[rr.r], a1 = P.Ap[rr.r + 1], na = a1 - a0;
  const int64_t c = A.rowc[rr.g];
  int32_t *cur = na <= kDenseCurSmem ? cur_s : A.curbuf + 2 * blockIdx.x * A.cur_stride;
  int32_t *nxc = na <= kDenseCurSmem ? nxc_s : cur + A.cur_stride;
  const int32_t *__restrict__ Aj = P.Aj;
  const VT *__restrict__ Ax = P.Ax;
  const PT *__restrict__ Bp = P.Bp;
  const int32_t *__restrict__ Bj = P.Bj;
  const VT *__restrict__ Bx = P.Bx;
  int *nq = gm.nl;
  long long tp = clock64();
  for (int i = tid; i < kWinCols; i += kThreads) accb[i] = kEmpty;
  for (int64_t j = tid; j < na; j += kThreads) {
    const int64_t k = __ldg(Aj + a0 + j);
    const int64_t b0 = __ldg(Bp + k), b1 = __ldg(Bp + k + 1);
    cur[j] = 0;
    nxc[j] = b1 > b0 ? __ldg(Bj + b0) : INT32_MAX;
  }
  if (tid == 0) *nq = 0;
  __syncthreads();
  prof_sub(A, 5, tp);
  const uint64_t pass = policy_evict_first();
  int64_t out = A.cp[rr.g] - A.cp[A.base[rr.p]];
  int64_t emitted = 0;
  int32_t *__restrict__ Cj = P.Cj;
  VT *__restrict__ Cx = P.Cx;
  for (int64_t w0 = 0; w0 < n; w0 += kWinCols) {
    const int64_t w1 = (w0 + kWinCols < n) ? w0 + kWinCols : n;
    const int32_t w0i = int32_t(w0);  // columns are int32 (n <= INT32_MAX)
    const unsigned wlen = unsigned(w1 - w0);
    // pass 1: one thread per entry, U B entries from the cursor
    for (int64_t j = tid; j < na; j += kThreads) {
      if (nxc[j] >= w1) continue;  // nothing in this window
      const int64_t k = __ldg(Aj + a0 + j);
      const VT a = __ldg(Ax + a0 + j);
      const int64_t b0 = __ldg(Bp + k), b1 = __ldg(Bp + k + 1);
      int64_t q = b0 + cur[j];
      bool tried = false, queued = false;
      int32_t nextc = INT32_MAX;
      while (true) {
        int32_t cc[U];
        VT xv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int64_t qq = q + u;
          cc[u] = qq < b1 ? __ldg(Bj + qq) : INT32_MAX;
          xv[u] = qq < b1 ? __ldg(Bx + qq) : VT(0);
        }
        int nin = 0;
#pragma unroll
        for (int u = 0; u < U; ++u) {
          // in the window (one unsigned compare: a column below w0 — only
          // possible when B's rows are not sorted as promised — is skipped,
          // never written out of bounds)
          if (unsigned(cc[u] - w0i) < wlen) {
            atomicAdd(acc + (cc[u] - w0i), win_value(a * xv[u]));
            ++nin;
          }
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (u == nin) nextc = cc[u];  // the first column past the window (sorted B)
        q += nin;
        if (nin < U) break;
        if (q >= b1) {
          nextc = INT32_MAX;
          break;
        }
        if (!tried) {  // the segment goes on: hand it to a warp
          tried = true;
          const int slot = atomicAdd(nq, 1);
          if (slot < kWinQueue) {
            queue[slot] = int32_t(j);
            queued = true;
            break;
          }
        }
      }
      cur[j] = int32_t(q - b0);
      if (!queued) nxc[j] = nextc;
    }
    // the addend row of the accumulate form: every window takes its columns
    for_addend<true>(P, rr.r, tid, kThreads, [&](int32_t col, VT v) {
      if (col >= w0 && col < w1) atomicAdd(acc + (col - w0i), win_value(v));
    });
    __syncthreads();
    prof_sub(A, 6, tp);
    // pass 2: a warp per queued segment, U x 32 B entries per step
    const int nqueued = min(*nq, kWinQueue);
    for (int i = warp; i < nqueued; i += NWARP) {
      const int64_t j = queue[i];
      const int64_t k = __ldg(Aj + a0 + j);
      const VT a = __ldg(Ax + a0 + j);
      const int64_t b0 = __ldg(Bp + k), b1 = __ldg(Bp + k + 1);
      int64_t q = b0 + cur[j];
      while (q < b1) {
        int32_t cc[U];
        VT xv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int64_t qq = q + u * 32 + lane;
          cc[u] = qq < b1 ? __ldg(Bj + qq) : INT32_MAX;
          xv[u] = qq < b1 ? __ldg(Bx + qq) : VT(0);
        }
        int nin = 0;
#pragma unroll
        for (int u = 0; u < U; ++u) {
          // in the window (one unsigned compare: a column below w0 — only
          // possible when B's rows are not sorted as promised — is skipped,
          // never written out of bounds)
          if (unsigned(cc[u] - w0i) < wlen) {
            atomicAdd(acc + (cc[u] - w0i), win_value(a * xv[u]));
            ++nin;
          }
        }
        nin = __reduce_add_sync(0xffffffffu, nin);
        q += nin;  // sorted B: the entries below w1 are a prefix of the segment
        if (nin < U * 32) break;
      }
      if (lane == 0) {
        cur[j] = int32_t(q - b0);
        nxc[j] = q < b1 ? __ldg(Bj + q) : INT32_MAX;
      }
    }
    __syncthreads();
    if (tid == 0) *nq = 0;
    prof_sub(A, 7, tp);
    // compaction: ballots of the warp's 32 steps, one per lane
    unsigned mine = 0;
    int wcount = 0;
    const int sbase = warp * PER;
#pragma unroll 4
    for (int st = 0; st < STEPS; ++st) {
      const unsigned b = __ballot_sync(0xffffffffu, accb[sbase + st * 32 + lane] != kEmpty);
      if (lane == st) mine = b;
      wcount += __popc(b);
    }
    if (lane == 0) gm.tmp[warp] = wcount;
    __syncthreads();
    int64_t wbase = 0, total = 0;
#pragma unroll
    for (int w = 0; w < NWARP; ++w) {
      const int64_t v = gm.tmp[w];
      if (w < warp) wbase += v;
      total += v;
    }
    int64_t pos = out + wbase;
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll 4
    for (int st = 0; st < STEPS; ++st) {
      const unsigned b = __shfl_sync(0xffffffffu, mine, st);
      if ((b >> lane) & 1u) {
        const int s = sbase + st * 32 + lane;
        const int64_t e = pos + __popc(b & lt);
        if (emitted + (e - out) < c) {  // e < the row's end unless the counts broke
          store_hint(Cj + e, int32_t(w0 + s), pass);
          store_hint(Cx + e, acc[s], pass);
        }
        accb[s] = kEmpty;
      }
      pos += __popc(b);
    }
    out += total;
    emitted += total;
    __syncthreads();  // the slots are empty again and gm.tmp is free
    prof_sub(A, 8, tp);
  }
  if (tid == 0 && emitted != c) set_error(A.err, 109);
}

// ---------------------------------------------------------------- the kernel

struct PhaseShared {
  int64_t scan[16 * 33];      // group scan scratch: 256-groups 0-3, 128-groups 4-11
  int itmp[12 * 18];          // group min/max scratch, same slots
  unsigned long long slot[16];  // fetched row index per group; [15] = CTA
  int lst[1024];              // deferred long B rows: CTA 1024, 256-group g at 256g,
                              // 128-group g at 128g, warp w at 32w
  int nl[48];                 // list counts: 256-groups 0-3, 128-groups 4-11,
                              // warps 12-43, CTA 47; [46] the CTA's entry counter
  int64_t off[NCLS], cnt[NCLS];
};

// Group rows that take the expand-sort-compress form: at most fmax products
// (half the group's table), and at most 2 products per output (few repeated
// columns; measured equal to 4 and better than 1.5 on the Galerkin rows).
__device__ __forceinline__ bool esc_fits(const RowMeta &m, int64_t fmax) {
  return m.f <= fmax && m.f <= 2 * m.c;
}

// Group-level rows of class `cls`: the group leader fetches one row index at a
// time; the group exits when the class runs out.
template <int G, bool NUM, typename PT, typename VT, bool ONEPASS = false>
__device__ void group_rows(const ProdDev<PT, VT> *prods, const PhaseArgs &A,
                           int cls, unsigned char *smem, PhaseShared &sh) {
  static_assert(!ONEPASS || (G == 32 && NUM), "one-pass rows are warp rows");
  constexpr int NG = kGroupThreads / G;  // groups of this size per CTA
  // slices start on 16-byte boundaries (the tables are cleared with 16-byte stores)
  constexpr int SLICE = (NUM ? kTableSmem / NG : (kTableSmem * 2 / 3) / NG) & ~15;
  constexpr int TMAXS = G == 256 ? kSymT256 : G == 128 ? kSymT128 : kSymT32;
  constexpr int TMAXN = G == 256 ? kNumT256 : G == 128 ? kNumT128 : kNumT32;
  static_assert(!NUM || TMAXN * 12 <= SLICE, "numeric slice");
  static_assert(NUM || TMAXS * 4 <= SLICE, "symbolic slice");
  const int gid = threadIdx.x / G, lane = threadIdx.x % G;
  const int slot = G == 256 ? gid : G == 128 ? 4 + gid : 0;
  unsigned char *slice = smem + gid * SLICE;
  GroupMem gm;
  // digit counters nest like the slices: 1 KiB per warp, a group's counters
  // start at its first warp's (a warp's radix needs 32 digits x 16 items x 2 B)
  static_assert(32 * (TMAXN / (2 * G)) * (G / 32) * 2 <= (G / 32) * 1024, "counters");
  static_assert((kGroupThreads / 32) * 1024 <= kGroupCountSmem, "counter space");
  gm.cnt = (uint16_t *)(smem + kTableSmem + gid * (G / 32) * 1024);
  gm.tmp = sh.scan + slot * 33;
  gm.itmp = sh.itmp + slot * 18;
  gm.lst = sh.lst + gid * G;
  gm.nl = sh.nl + (G == 32 ? 12 + gid : slot);
  gm.cap = G;
  // flat-loop staging: the free part of the slice above the largest table
  static_assert(G == 32 || (NUM ? TMAXN * 12 : TMAXS * 4) + 24 * G <= SLICE, "staging");
  gm.stage = G == 32 ? nullptr : slice + (NUM ? TMAXN * 12 : TMAXS * 4);
  const int64_t base = sh.off[cls], count = sh.cnt[cls];
  // rows are taken in chunks (one counter atomic per chunk); the chunk shrinks
  // to one row as the class runs out so the tail stays balanced
  constexpr int64_t kChunk = G == 32 ? 16 : G == 128 ? 4 : 2;
  const int64_t groups = int64_t(gridDim.x) * NG;
  while (true) {
    int64_t i;
    if constexpr (G == 32) {
      unsigned long long v = 0;
      if (lane == 0) {
        const unsigned long long cur = *(volatile unsigned long long *)&A.S->next[cls];
        const int64_t left = count - int64_t(cur);
        const unsigned long long take =
            left > kChunk * groups * 2 ? kChunk : 1ull;
        v = atomicAdd(&A.S->next[cls], take) | (take << 48);
      }
      v = __shfl_sync(0xffffffffu, v, 0);
      i = int64_t(v & ((1ull << 48) - 1));
      const int64_t take = int64_t(v >> 48);
      if (i >= count) break;
      const int64_t e = min(count, i + take);
      // the chunk's metadata, one row per lane (take <= kChunk <= 32)
      RowMeta mine{};
      if (lane < e - i) mine = load_meta<NUM>(prods, A, base + i + lane);
      for (int t = 0; i < e; ++i, ++t) {
        const long long t0 = clock64();
        const RowMeta m = shfl_meta(mine, t);
        if constexpr (ONEPASS) {
          num_hash_row<G, TMAXN, PT, VT, true>(prods, A, m, slice, gm, gid, lane);
        } else if constexpr (NUM) {
          if (esc_fits(m, TMAXN / 2))
            num_esc_row<G, TMAXN, PT, VT>(prods, A, m, slice, gm, gid, lane);
          else
            num_hash_row<G, TMAXN, PT, VT>(prods, A, m, slice, gm, gid, lane);
        } else {
          sym_hash_row<G, TMAXS, PT, VT>(prods, A, m, (int *)slice, gm, gid, lane);
        }
        prof_add(A, cls, t0, lane == 0);
      }
    } else {
      if (lane == 0) {
        const unsigned long long cur = *(volatile unsigned long long *)&A.S->next[cls];
        const int64_t left = count - int64_t(cur);
        const unsigned long long take = left > kChunk * groups * 2 ? kChunk : 1ull;
        sh.slot[slot] = atomicAdd(&A.S->next[cls], take) | (take << 48);
      }
      group_sync<G>(gid);
      const unsigned long long v = sh.slot[slot];
      group_sync<G>(gid);
      i = int64_t(v & ((1ull << 48) - 1));
      if (i >= count) break;
      const int64_t e = min(count, i + int64_t(v >> 48));
      for (; i < e; ++i) {
        const long long t0 = clock64();
        const RowMeta m = load_meta<NUM>(prods, A, base + i);
        if constexpr (NUM) {
          if (esc_fits(m, TMAXN / 2))
            num_esc_row<G, TMAXN, PT, VT>(prods, A, m, slice, gm, gid, lane);
          else
            num_hash_row<G, TMAXN, PT, VT>(prods, A, m, slice, gm, gid, lane);
        } else
          sym_hash_row<G, TMAXS, PT, VT>(prods, A, m, (int *)slice, gm, gid, lane);
        prof_add(A, cls, t0, lane == 0);
      }
    }
  }
}

template <typename PT, typename VT, bool NUM>
__global__ void __launch_bounds__(NUM ? kThreads : kSymThreads, 1)
    k_phase(const ProdDev<PT, VT> *prods, PhaseArgs A) {
  constexpr int NT = NUM ? kThreads : kSymThreads;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ PhaseShared sh;
  __shared__ int64_t s_items[kCtaClasses + 1];
  const int tid = threadIdx.x;
  if (tid < NCLS) {
    sh.off[tid] = A.S->off[tid];
    sh.cnt[tid] = A.S->cnt[tid];
  }
  if (tid == 0) {
    int64_t it = 0;
    for (int c = 0; c < kCtaClasses; ++c) {
      s_items[c] = it;
      it += A.S->cnt[c];
    }
    s_items[kCtaClasses] = it;
  }
  __syncthreads();
  GroupMem gm;
  gm.cnt = (uint16_t *)(smem + kTableSmem);
  gm.tmp = sh.scan;
  gm.itmp = sh.itmp;
  gm.lst = sh.lst;
  gm.nl = sh.nl + 47;
  gm.cap = 1024;
  gm.stage = nullptr;
  // numeric: when k_dense_rank did every DENSE row, start past them
  const int64_t first = NUM && A.S->rank_left == 0 ? s_items[CLS_DENSE2 + 1] : 0;
  // stage 1: CTA-level rows, heaviest class first
  while (true) {
    if (tid == 0) sh.slot[15] = atomicAdd(&A.S->work, 1ull);
    __syncthreads();
    const int64_t item = first + (int64_t)sh.slot[15];
    __syncthreads();
    if (item >= s_items[kCtaClasses]) break;
    // numeric: the heavy DENSE0 / DENSE1 rows (heaviest first) are interleaved
    // with the lighter CTA rows, one in every K items, so fewer heavy rows are
    // in flight at once and their output segments (the targets of the global
    // reductions) stay in L2; symbolic: heaviest first
    int64_t pos = item;
    if (NUM && first == 0) {
      const int64_t H = s_items[2], L = s_items[kCtaClasses] - H;
      int64_t K = H > 0 ? min(int64_t(kHeavyPeriod), 1 + L / H) : 1;
      // (past the interleaved stretch the light rows follow in order: pos = item)
      if (K > 1 && item < K * H) pos = item % K == 0 ? item / K : H + (item - item / K - 1);
    }
    int c = 0;
    while (pos >= s_items[c + 1]) ++c;
    const int64_t idx = sh.off[c] + (pos - s_items[c]);
    const long long t0 = clock64();
    if (cls_dense(c)) {
      if constexpr (NUM) {
        const RowRef rr = decode_row(A, idx);
        const ProdDev<PT, VT> &P = prods[rr.p];
        // heavy rows whose output fills >= 1/2^fill of the columns: column
        // windows, in this CTA or (tune.cluster > 0) in the cluster kernel
        // that ran before this one
        if (win_row(P, A.rowf[rr.g], int64_t(A.rowc[rr.g]), A.S->tune)) {
          if (A.S->tune.cluster == 0) num_dense_win_row<PT, VT>(prods, A, idx, smem, gm);
        } else if (P.n > kRankMaxCols) {
          num_dense_row<PT, VT>(prods, A, idx, smem, gm);
        }  // else: a rank-form row, done by k_dense_rank before this kernel
      } else {
        sym_dense_row<NT, PT, VT>(prods, A, idx, smem, gm);
      }
    } else {
      if constexpr (NUM)
        num_hash_row<kThreads, kNumT1024, PT, VT>(prods, A, load_meta<true>(prods, A, idx), smem,
                                                  gm, 0, tid);
      else
        sym_hash_row<NT, kSymT1024, PT, VT>(prods, A, load_meta<false>(prods, A, idx),
                                            (int *)smem, gm, 0, tid);
    }
    prof_add(A, c, t0, tid == 0);
    __syncthreads();
  }
}

// The numeric DENSE rows of the rank form (at most kRankMaxCols columns, not
// taken by the column-window rule), persistent, before k_phase: 24 warps per
// SM, where k_phase's 16 warps keep the 128 registers of the hash rows'
// radix sort.  Heavy rows (DENSE0 / DENSE1) are spread over the DENSE2 rows
// as in k_phase, so few of their reduction targets are live at once.
template <typename PT, typename VT>
__global__ void __launch_bounds__(kRankThreads, 1)
    k_dense_rank(const ProdDev<PT, VT> *prods, PhaseArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ PhaseShared sh;
  __shared__ unsigned long long s_item;
  const int tid = threadIdx.x;
  const int64_t H = A.S->cnt[CLS_DENSE0] + A.S->cnt[CLS_DENSE1];
  const int64_t L = A.S->cnt[CLS_DENSE2];
  const int64_t c01 = A.S->cnt[CLS_DENSE0];
  const int64_t K = H > 0 ? min(int64_t(kHeavyPeriod), 1 + L / H) : 1;
  GroupMem gm;
  gm.cnt = nullptr;
  gm.tmp = sh.scan;
  gm.itmp = sh.itmp;
  gm.lst = sh.lst;
  gm.nl = sh.nl + 47;
  gm.cap = 1024;
  gm.stage = nullptr;
  while (true) {
    if (tid == 0) s_item = atomicAdd(&A.S->work3, 1ull);
    __syncthreads();
    const int64_t item = (int64_t)s_item;
    __syncthreads();
    if (item >= H + L) break;
    int64_t pos = item;
    if (K > 1 && item < K * H) pos = item % K == 0 ? item / K : H + (item - item / K - 1);
    // the DENSE classes' lists are contiguous: DENSE0, DENSE1, DENSE2
    const int c = pos < c01 ? CLS_DENSE0 : pos < H ? CLS_DENSE1 : CLS_DENSE2;
    const int64_t idx = A.S->off[CLS_DENSE0] + pos;
    const long long t0 = clock64();
    const RowRef rr = decode_row(A, idx);
    const ProdDev<PT, VT> &P = prods[rr.p];
    if (P.n <= kRankMaxCols && !win_row(P, A.rowf[rr.g], int64_t(A.rowc[rr.g]), A.S->tune)) {
      num_dense_rank_row<kRankThreads, PT, VT>(prods, A, idx, smem, gm);
      prof_add(A, c, t0, tid == 0);
    } else if (tid == 0) {
      A.S->rank_left = 1;  // read by k_phase, which runs after this kernel
    }
    __syncthreads();
  }
}

// The group classes (G256, G128, G32 rows), persistent: the CTA splits into
// 256-thread groups, then 128-thread groups, then warps; each fetches its
// rows on its own, and no CTA-wide barrier follows the set-up.
template <typename PT, typename VT, bool NUM>
__global__ void __launch_bounds__(kGroupThreads, 1)
    k_groups(const ProdDev<PT, VT> *prods, PhaseArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ PhaseShared sh;
  if (threadIdx.x < NCLS) {
    sh.off[threadIdx.x] = A.S->off[threadIdx.x];
    sh.cnt[threadIdx.x] = A.S->cnt[threadIdx.x];
  }
  __syncthreads();
  group_rows<256, NUM, PT, VT>(prods, A, CLS_G256, smem, sh);
  group_rows<128, NUM, PT, VT>(prods, A, CLS_G128, smem, sh);
  group_rows<32, NUM, PT, VT>(prods, A, CLS_G32, smem, sh);
}

// One-pass warp rows of a plain product (the symbolic record's CLS_ONEPASS
// list), after k_groups in the symbolic launch: each row is multiplied in
// full (the numeric warp-row form, its table sized by the output bound) into
// the scratch.  A warp row's symbolic pass (hash count) is then not needed:
// Galerkin A·P (27-point 128^3, ~119 products and ~12 outputs per row)
// paid 1.8 ms of symbolic and 3.5 ms of numeric launches for it.
template <typename PT, typename VT>
__global__ void __launch_bounds__(kGroupThreads, 1)
    k_onepass(const ProdDev<PT, VT> *prods, PhaseArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ PhaseShared sh;
  if (threadIdx.x < NCLS) {
    sh.off[threadIdx.x] = A.S->off[threadIdx.x];
    sh.cnt[threadIdx.x] = A.S->cnt[threadIdx.x];
  }
  __syncthreads();
  group_rows<32, true, PT, VT, true>(prods, A, CLS_ONEPASS, smem, sh);
}

// Numeric launch: the one-pass rows (rowf < 0) go from the scratch into C.  A
// warp takes 32 rows at a time (lane i loads row i's offsets and count, all
// together), numbers the tile's entries with a warp scan, and lanes copy
// entries lane, lane + 32, ... (4 per step, loads in flight), each finding
// its row by a 5-step shuffle search.  (A warp per row took 0.5 ms for the
// 2.1M rows of ~12 entries of the Galerkin A·P at 128^3: a chain of dependent
// loads per row.)
template <typename PT, typename VT>
__global__ void __launch_bounds__(256) k_onepass_copy(const ProdDev<PT, VT> *prods,
                                                      const int64_t *rowf, const int32_t *rowc,
                                                      const int64_t *cp, const int32_t *oj,
                                                      const VT *ox, int64_t R) {
  constexpr int U = 4;
  const int lane = threadIdx.x & 31;
  const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
  int32_t *Cj = prods[0].Cj;
  VT *Cx = prods[0].Cx;
  for (int64_t t0 = warp * 32; t0 < R; t0 += nwarps * 32) {
    const int64_t g = t0 + lane;
    int64_t src = 0, dst = 0;
    int len = 0;
    if (g < R) {
      const int64_t f = rowf[g];
      if (f < 0) {
        src = -1 - f;
        dst = cp[g];
        len = rowc[g];
      }
    }
    const int inc = warp_scan_incl(len);
    const int tot = __shfl_sync(0xffffffffu, inc, 31);
    const int pre = inc - len;
    for (int e0 = 0; e0 < tot; e0 += 32 * U) {
      int64_t from[U], to[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int e = e0 + u * 32 + lane;
        int j = 0;
#pragma unroll
        for (int st = 16; st > 0; st >>= 1) {
          const int v = __shfl_sync(0xffffffffu, pre, j + st);
          if (v <= e) j += st;
        }
        const int pj = __shfl_sync(0xffffffffu, pre, j);
        const int64_t sj = __shfl_sync(0xffffffffu, src, j), dj = __shfl_sync(0xffffffffu, dst, j);
        from[u] = e < tot ? sj + (e - pj) : -1;
        to[u] = dj + (e - pj);
      }
      int32_t cj[U];
      VT cx[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (from[u] >= 0) {
          cj[u] = __ldg(oj + from[u]);
          cx[u] = __ldg(ox + from[u]);
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (from[u] >= 0) {
          Cj[to[u]] = cj[u];
          Cx[to[u]] = cx[u];
        }
      }
    }
  }
}

}  // namespace tspg
