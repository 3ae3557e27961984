// spgemm_cluster.cuh — the column-window DENSE numeric form on a thread-block
// cluster: the heavy rows that take the window form (num_dense_win_row) are
// worked by K CTAs at once, the window spread over their shared memories, so
// one window spans K x kWinCols columns (K times fewer windows, so K times
// fewer cursor probes per A entry) and one heavy row is spread over K SMs.
//
// Per row: CTA rank r of the cluster takes A entries r, r + K, ... (cursors in
// its own shared memory, or its slice of the global cursor buffer); a product
// in column c of window [w0, w1) belongs to CTA (c - w0) / kWinCols, slot
// (c - w0) % kWinCols, and is added there with a distributed-shared-memory
// reduction (mapa + red.shared::cluster.add).  After a cluster barrier each
// CTA compacts its own slice (the -0.0 empty mark, as in the one-CTA form),
// publishes its count in the leader CTA's shared memory, and after a second
// barrier places its entries behind the counts of the lower ranks; a third
// barrier keeps the next window's reductions out of slices still being read.
// Every CTA of a cluster runs the same number of barriers (the row index is
// broadcast by the leader, the window loop depends only on the row), and no
// CTA touches another's shared memory after the last barrier, so no CTA exits
// while a peer can still reach it.
#pragma once

#include <cooperative_groups.h>

#include "spgemm_phase.cuh"

namespace tspg {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return uint32_t(__cvta_generic_to_shared(p));
}
// address of the same shared-memory location in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t cluster_map(uint32_t a, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
__device__ __forceinline__ void cluster_red_add(uint32_t a, double v) {
  asm volatile("red.relaxed.cluster.shared::cluster.add.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory");
}
__device__ __forceinline__ void cluster_red_add(uint32_t a, float v) {
  asm volatile("red.relaxed.cluster.shared::cluster.add.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}
__device__ __forceinline__ void cluster_st_s64(uint32_t a, long long v) {
  asm volatile("st.shared::cluster.s64 [%0], %1;" ::"r"(a), "l"(v) : "memory");
}
__device__ __forceinline__ long long cluster_ld_s64(uint32_t a) {
  long long v;
  asm volatile("ld.shared::cluster.s64 %0, [%1];" : "=l"(v) : "r"(a) : "memory");
  return v;
}

template <typename PT, typename VT>
__global__ void __launch_bounds__(kThreads, 1)
    k_dense_cluster(const ProdDev<PT, VT> *prods, PhaseArgs A) {
  namespace cg = cooperative_groups;
  using UT = std::conditional_t<sizeof(VT) == 8, unsigned long long, unsigned>;
  constexpr UT kEmpty = UT(1) << (sizeof(VT) * 8 - 1);  // -0.0
  constexpr int U = 8;
  constexpr int NWARP = kThreads / 32;
  constexpr int PER = kWinCols / NWARP;
  constexpr int STEPS = PER / 32;
  static_assert(STEPS == 32, "one ballot per lane");
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ long long s_row;      // row item broadcast by the leader (-1: done)
  __shared__ long long s_cnt[8];   // per-CTA window counts (used in the leader)
  __shared__ long long s_all[9];   // the counts as read by this CTA, [8] = total
  __shared__ long long s_wcnt[NWARP];
  __shared__ int s_nq;
  cg::cluster_group cl = cg::this_cluster();
  const unsigned K = cl.num_blocks(), rank = cl.block_rank();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  VT *acc = (VT *)smem;
  UT *accb = (UT *)smem;
  int32_t *cur_s = (int32_t *)(smem + kWinCols * sizeof(VT));
  int32_t *nxc_s = cur_s + kDenseCurSmem;
  int32_t *queue = nxc_s + kDenseCurSmem;
  const Tune t = A.S->tune;
  // every DENSE class (DENSE0, DENSE1, DENSE2: contiguous in the list); the
  // window rule, not the class, decides which rows are taken
  const int64_t n_items = A.S->cnt[CLS_DENSE0] + A.S->cnt[CLS_DENSE1] + A.S->cnt[CLS_DENSE2];
  const int64_t list0 = A.S->off[CLS_DENSE0];
  const uint32_t acc_u32 = smem_u32(acc);
  const uint64_t pass = policy_evict_first();
  for (int i = tid; i < kWinCols; i += kThreads) accb[i] = kEmpty;
  while (true) {
    // the leader takes the next window-form row and tells the cluster
    if (rank == 0 && tid == 0) {
      long long found = -1;
      while (true) {
        const unsigned long long i = atomicAdd(&A.S->work2, 1ull);
        if (int64_t(i) >= n_items) break;
        const int64_t idx = list0 + int64_t(i);
        const RowRef rr = decode_row(A, idx);
        if (win_row(prods[rr.p], A.rowf[rr.g], int64_t(A.rowc[rr.g]), t)) {
          found = idx;
          break;
        }
      }
      for (unsigned r = 0; r < K; ++r) cluster_st_s64(cluster_map(smem_u32(&s_row), r), found);
    }
    cl.sync();
    const long long idx = s_row;
    if (idx < 0) break;
    const RowRef rr = decode_row(A, idx);
    const ProdDev<PT, VT> &P = prods[rr.p];
    const int64_t n = P.n;
    const int64_t a0 = P.Ap[rr.r], a1 = P.Ap[rr.r + 1], na = a1 - a0;
    const int64_t c = A.rowc[rr.g];
    const int64_t nmine = na > int64_t(rank) ? (na - int64_t(rank) + K - 1) / K : 0;
    int32_t *cur = nmine <= kDenseCurSmem ? cur_s : A.curbuf + 2 * blockIdx.x * A.cur_stride;
    int32_t *nxc = nmine <= kDenseCurSmem ? nxc_s : cur + A.cur_stride;
    const int32_t *__restrict__ Aj = P.Aj;
    const VT *__restrict__ Ax = P.Ax;
    const PT *__restrict__ Bp = P.Bp;
    const int32_t *__restrict__ Bj = P.Bj;
    const VT *__restrict__ Bx = P.Bx;
    long long tp = clock64();
    for (int64_t jj = tid; jj < nmine; jj += kThreads) {
      const int64_t j = int64_t(rank) + jj * K;
      const int64_t k = __ldg(Aj + a0 + j);
      const int64_t b0 = __ldg(Bp + k), b1 = __ldg(Bp + k + 1);
      cur[jj] = 0;
      nxc[jj] = b1 > b0 ? __ldg(Bj + b0) : INT32_MAX;
    }
    if (tid == 0) s_nq = 0;
    __syncthreads();
    if (rank == 0) prof_sub(A, 5, tp);
    int64_t out = A.cp[rr.g] - A.cp[A.base[rr.p]];
    int64_t emitted = 0;
    const int64_t WC = int64_t(K) * kWinCols;
    for (int64_t w0 = 0; w0 < n; w0 += WC) {
      const int64_t w1 = (w0 + WC < n) ? w0 + WC : n;
      const int32_t w0i = int32_t(w0);
      const unsigned wlen = unsigned(w1 - w0);
      // a product in column col goes to CTA (col - w0) / kWinCols of the cluster
      auto add = [&](int32_t col, VT v) {
        const unsigned o = unsigned(col - w0i);
        cluster_red_add(cluster_map(acc_u32 + (o % kWinCols) * unsigned(sizeof(VT)), o / kWinCols), v);
      };
      // pass 1: one thread per entry, U B entries from the cursor
      for (int64_t jj = tid; jj < nmine; jj += kThreads) {
        if (nxc[jj] >= w1) continue;
        const int64_t j = int64_t(rank) + jj * K;
        const int64_t k = __ldg(Aj + a0 + j);
        const VT a = __ldg(Ax + a0 + j);
        const int64_t b0 = __ldg(Bp + k), b1 = __ldg(Bp + k + 1);
        int64_t q = b0 + cur[jj];
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
            if (unsigned(cc[u] - w0i) < wlen) {
              add(cc[u], win_value(a * xv[u]));
              ++nin;
            }
          }
#pragma unroll
          for (int u = 0; u < U; ++u)
            if (u == nin) nextc = cc[u];
          q += nin;
          if (nin < U) break;
          if (q >= b1) {
            nextc = INT32_MAX;
            break;
          }
          if (!tried) {
            tried = true;
            const int slot = atomicAdd(&s_nq, 1);
            if (slot < kWinQueue) {
              queue[slot] = int32_t(jj);
              queued = true;
              break;
            }
          }
        }
        cur[jj] = int32_t(q - b0);
        if (!queued) nxc[jj] = nextc;
      }
      // the addend row: this CTA takes entries rank, rank + K, ...
      if (P.Ej) {
        int64_t e0, e1;
        addend_row(P, rr.r, e0, e1);
        for (int64_t e = e0 + int64_t(rank) + int64_t(tid) * K; e < e1; e += int64_t(kThreads) * K) {
          const int32_t col = __ldg(P.Ej + e);
          if (col >= w0 && col < w1) add(col, win_value(__ldg(P.Ex + e)));
        }
      }
      __syncthreads();
      if (rank == 0) prof_sub(A, 6, tp);
      // pass 2: a warp per queued segment
      const int nqueued = min(s_nq, kWinQueue);
      for (int i = warp; i < nqueued; i += NWARP) {
        const int64_t jj = queue[i];
        const int64_t j = int64_t(rank) + jj * K;
        const int64_t k = __ldg(Aj + a0 + j);
        const VT a = __ldg(Ax + a0 + j);
        const int64_t b0 = __ldg(Bp + k), b1 = __ldg(Bp + k + 1);
        int64_t q = b0 + cur[jj];
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
            if (unsigned(cc[u] - w0i) < wlen) {
              add(cc[u], win_value(a * xv[u]));
              ++nin;
            }
          }
          nin = __reduce_add_sync(0xffffffffu, nin);
          q += nin;
          if (nin < U * 32) break;
        }
        if (lane == 0) {
          cur[jj] = int32_t(q - b0);
          nxc[jj] = q < b1 ? __ldg(Bj + q) : INT32_MAX;
        }
      }
      __syncthreads();
      if (tid == 0) s_nq = 0;
      cl.sync();  // every reduction of this window has landed in every slice
      if (rank == 0) prof_sub(A, 7, tp);
      // compaction of this CTA's slice: columns w0 + rank * kWinCols + s
      unsigned mine = 0;
      int wcount = 0;
      const int sbase = warp * PER;
#pragma unroll 4
      for (int st = 0; st < STEPS; ++st) {
        const unsigned b = __ballot_sync(0xffffffffu, accb[sbase + st * 32 + lane] != kEmpty);
        if (lane == st) mine = b;
        wcount += __popc(b);
      }
      if (lane == 0) s_wcnt[warp] = wcount;
      __syncthreads();
      if (tid == 0) {
        long long tot = 0;
        for (int w = 0; w < NWARP; ++w) tot += s_wcnt[w];
        cluster_st_s64(cluster_map(smem_u32(&s_cnt[rank]), 0), tot);
      }
      cl.sync();  // the counts of all CTAs are in the leader
      if (tid < int(K)) s_all[tid] = cluster_ld_s64(cluster_map(smem_u32(&s_cnt[tid]), 0));
      __syncthreads();
      int64_t before = 0, total = 0;
      for (unsigned r = 0; r < K; ++r) {
        if (r < rank) before += s_all[r];
        total += s_all[r];
      }
      int64_t wbase = 0;
#pragma unroll
      for (int w = 0; w < NWARP; ++w)
        if (w < warp) wbase += s_wcnt[w];
      int64_t pos = out + before + wbase;
      const unsigned lt = (1u << lane) - 1u;
      const int64_t colbase = w0 + int64_t(rank) * kWinCols;
#pragma unroll 4
      for (int st = 0; st < STEPS; ++st) {
        const unsigned b = __shfl_sync(0xffffffffu, mine, st);
        if ((b >> lane) & 1u) {
          const int s = sbase + st * 32 + lane;
          const int64_t e = pos + __popc(b & lt);
          if (emitted + (e - out) < c) {  // e < the row's end unless the counts broke
            store_hint(P.Cj + e, int32_t(colbase + s), pass);
            store_hint(P.Cx + e, acc[s], pass);
          }
          accb[s] = kEmpty;
        }
        pos += __popc(b);
      }
      out += total;
      emitted += total;
      __syncthreads();
      cl.sync();  // slices empty again before the next window's reductions; s_cnt free
      if (rank == 0) prof_sub(A, 8, tp);
    }
    if (rank == 0 && tid == 0 && emitted != c) set_error(A.err, 110);
    cl.sync();  // every CTA is done with this row (and with s_row) before the next fetch
  }
}

// Maximum co-resident clusters of K CTAs for the cluster kernel (0 when the
// device cannot run them), cached per device and K.
template <typename PT, typename VT>
int cluster_slots(int device, int K) {
  static int cache[64][4] = {};  // K = 2, 4, 8 -> index 1, 2, 3; value + 1
  const int ki = K == 2 ? 1 : K == 4 ? 2 : K == 8 ? 3 : 0;
  if (device < 0 || device >= 64 || ki == 0) return 0;
  if (cache[device][ki]) return cache[device][ki] - 1;
  if (cudaFuncSetAttribute(k_dense_cluster<PT, VT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           kDynSmem) != cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = unsigned(K);
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(unsigned(K));
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = kDynSmem;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k_dense_cluster<PT, VT>, &cfg) != cudaSuccess) {
    (void)cudaGetLastError();
    n = 0;
  }
  cache[device][ki] = n + 1;
  return n;
}

// Launch the cluster kernel over the column-window rows of a numeric phase
// (before k_phase, which then leaves those rows alone).  Returns the CUDA
// status of the launch; does nothing when the tuning asks for no cluster.
template <typename PT, typename VT>
cudaError_t launch_dense_cluster(tspg_ctx *ctx, cudaStream_t s, const ProdDev<PT, VT> *prods,
                                 const PhaseArgs &pa) {
  const int K = ctx->tune.cluster;
  if (K == 0) return cudaSuccess;
  const int slots = cluster_slots<PT, VT>(ctx->device, K);
  if (slots <= 0) return cudaErrorInvalidConfiguration;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = unsigned(K);
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(unsigned(slots * K));
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = kDynSmem;
  cfg.stream = s;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  ctx->launches += 1;
  return cudaLaunchKernelEx(&cfg, k_dense_cluster<PT, VT>, prods, pa);
}

}  // namespace tspg
