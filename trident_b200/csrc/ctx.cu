// ctx.cu — context lifetime and the resident workspace pool.
//
// Replaces the per-rank state Trident keeps around its local compute: the
// cusparseHandle_t, the grow-only temp buffers of CsxBuffers / cubTmpBuff
// (include/utils.cuh:320-410,527-784) and setup_mempool / teardown_mempool
// (include/mempool.cuh:9-30).  Instead of a grow-only malloc/free per call,
// every workspace block comes from a private cudaMemPool whose release
// threshold is UINT64_MAX, so freed blocks stay mapped and the next call on
// the stream reuses them without touching the driver.
#include <cstring>
#include <new>

#include "internal.cuh"

namespace tspg {

int ws_alloc(tspg_ctx *ctx, void **p, size_t bytes, cudaStream_t s) {
  bytes = (bytes + 255) & ~size_t(255);
  std::lock_guard<std::mutex> lk(ctx->live_mu);
  if (ctx->budget && ctx->in_use + bytes > ctx->budget) return TSPG_ENOMEM;
  cudaError_t e = cudaMallocFromPoolAsync(p, bytes, ctx->pool, s);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    ctx->last_cuda = (int)e;
    return e == cudaErrorMemoryAllocation ? TSPG_ENOMEM : TSPG_ECUDA;
  }
  ctx->live[*p] = bytes;
  ctx->in_use += bytes;
  if (ctx->in_use > ctx->high_water) ctx->high_water = ctx->in_use;
  return TSPG_OK;
}

void ws_free(tspg_ctx *ctx, void *p, cudaStream_t s) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(ctx->live_mu);
  auto it = ctx->live.find(p);
  if (it != ctx->live.end()) {
    ctx->in_use -= it->second;
    ctx->live.erase(it);
  }
  cudaFreeAsync(p, s);
}

}  // namespace tspg

using namespace tspg;

extern "C" int tspg_abi_version(void) { return TSPG_ABI_VERSION; }

extern "C" const char *tspg_strerror(int status) {
  switch (status) {
    case TSPG_OK: return "ok";
    case TSPG_EINVAL: return "invalid argument";
    case TSPG_ENOMEM: return "out of memory (context budget or output capacity)";
    case TSPG_EOVERFLOW: return "int32 row offsets cannot hold nnz";
    case TSPG_ETIMEOUT: return "bounded device wait timed out";
    case TSPG_ECUDA: return "CUDA runtime error";
    case TSPG_EUNSORTED: return "operand rows must be sorted";
    case TSPG_ESCRATCH: return "tile exceeds the static scratch of tspg_pack_noalloc";
    default: return "unknown status";
  }
}

extern "C" int tspg_last_cuda_error(const tspg_ctx *ctx) {
  return ctx ? ctx->last_cuda : 0;
}

extern "C" int tspg_ctx_create(int device, size_t pool_budget,
                               tspg_ctx **out) {
  if (!out) return TSPG_EINVAL;
  *out = nullptr;
  tspg_ctx *ctx = new (std::nothrow) tspg_ctx();
  if (!ctx) return TSPG_ENOMEM;
  ctx->device = device;
  ctx->budget = pool_budget;
  cudaError_t e = cudaSetDevice(device);
  int sms = 0, optin = 0;
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                               device);
  if (e == cudaSuccess) {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    e = cudaMemPoolCreate(&ctx->pool, &props);
  }
  if (e == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    e = cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold,
                                &thr);
  }
  if (e == cudaSuccess)
    e = cudaMallocHost((void **)&ctx->h_words, kHostWords * sizeof(int64_t));
  if (e == cudaSuccess)
    e = cudaMalloc((void **)&ctx->d_words, kDevWords * sizeof(int64_t));
  if (e == cudaSuccess)
    e = cudaMemset(ctx->d_words, 0, kDevWords * sizeof(int64_t));
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    if (ctx->h_words) cudaFreeHost(ctx->h_words);
    if (ctx->d_words) cudaFree(ctx->d_words);
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    delete ctx;
    return TSPG_ECUDA;
  }
  ctx->num_sms = sms;
  ctx->smem_optin = (size_t)optin;
  *out = ctx;
  return TSPG_OK;
}

extern "C" int tspg_ctx_destroy(tspg_ctx *ctx) {
  if (!ctx) return TSPG_EINVAL;
  cudaSetDevice(ctx->device);
  cudaDeviceSynchronize();
  for (auto &e : ctx->ev)
    if (e) cudaEventDestroy(e);
  if (ctx->d_prof) cudaFree(ctx->d_prof);
  for (auto &kv : ctx->live) cudaFree(kv.first);
  ctx->live.clear();
  if (ctx->h_words) cudaFreeHost(ctx->h_words);
  if (ctx->d_words) cudaFree(ctx->d_words);
  if (ctx->pool) {
    cudaMemPoolTrimTo(ctx->pool, 0);
    cudaMemPoolDestroy(ctx->pool);
  }
  delete ctx;
  return TSPG_OK;
}

extern "C" int tspg_ctx_mem(const tspg_ctx *ctx, size_t *in_use,
                            size_t *high_water) {
  if (!ctx) return TSPG_EINVAL;
  if (in_use) *in_use = ctx->in_use;
  if (high_water) *high_water = ctx->high_water;
  return TSPG_OK;
}

extern "C" int tspg_ctx_stats(const tspg_ctx *ctx, int64_t *launches) {
  if (!ctx) return TSPG_EINVAL;
  if (launches) *launches = ctx->launches;
  return TSPG_OK;
}

extern "C" int tspg_ctx_phase_timing(tspg_ctx *ctx, int enable) {
  if (!ctx) return TSPG_EINVAL;
  TSPG_CUDA(ctx, cudaSetDevice(ctx->device));
  if (enable && !ctx->ev[0])
    for (auto &e : ctx->ev) TSPG_CUDA(ctx, cudaEventCreate(&e));
  ctx->phase_timing = enable != 0;
  ctx->ev_sym = ctx->ev_num = false;
  return TSPG_OK;
}

extern "C" int tspg_ctx_phase_ms(tspg_ctx *ctx, float *symbolic_ms,
                                 float *numeric_ms) {
  if (!ctx || !ctx->ev[0]) return TSPG_EINVAL;
  float a = 0.f, b = 0.f;
  if (ctx->ev_sym) {
    TSPG_CUDA(ctx, cudaEventSynchronize(ctx->ev[1]));
    TSPG_CUDA(ctx, cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]));
  }
  if (ctx->ev_num) {
    TSPG_CUDA(ctx, cudaEventSynchronize(ctx->ev[3]));
    TSPG_CUDA(ctx, cudaEventElapsedTime(&b, ctx->ev[2], ctx->ev[3]));
  }
  if (symbolic_ms) *symbolic_ms = a;
  if (numeric_ms) *numeric_ms = b;
  return TSPG_OK;
}

extern "C" int tspg_ctx_set_tuning(tspg_ctx *ctx, const tspg_tuning *t) {
  if (!ctx || !t) return TSPG_EINVAL;
  Tune u{};
  for (int i = 0; i < 4; ++i) {
    u.sym[i] = t->sym_lim[i];
    u.num[i] = t->num_lim[i];
  }
  u.load = t->hash_load;
  u.win = t->dense_win_log2;
  u.fill = t->dense_win_fill_log2;
  u.cluster = t->dense_win_cluster;
  if (!tune_valid(u)) return TSPG_EINVAL;
  ctx->tune = u;
  return TSPG_OK;
}

extern "C" int tspg_ctx_get_tuning(const tspg_ctx *ctx, tspg_tuning *t) {
  if (!ctx || !t) return TSPG_EINVAL;
  for (int i = 0; i < 4; ++i) {
    t->sym_lim[i] = ctx->tune.sym[i];
    t->num_lim[i] = ctx->tune.num[i];
  }
  t->hash_load = ctx->tune.load;
  t->dense_win_log2 = ctx->tune.win;
  t->dense_win_fill_log2 = ctx->tune.fill;
  t->dense_win_cluster = ctx->tune.cluster;
  return TSPG_OK;
}

extern "C" int tspg_ctx_class_profile(tspg_ctx *ctx, int enable) {
  if (!ctx) return TSPG_EINVAL;
  TSPG_CUDA(ctx, cudaSetDevice(ctx->device));
  if (enable && !ctx->d_prof)
    TSPG_CUDA(ctx, cudaMalloc((void **)&ctx->d_prof, 64 * sizeof(unsigned long long)));
  if (enable) TSPG_CUDA(ctx, cudaMemset(ctx->d_prof, 0, 64 * sizeof(unsigned long long)));
  if (!enable && ctx->d_prof) {
    cudaFree(ctx->d_prof);
    ctx->d_prof = nullptr;
  }
  return TSPG_OK;
}

extern "C" int tspg_ctx_class_cycles(tspg_ctx *ctx, uint64_t *out64) {
  if (!ctx || !ctx->d_prof || !out64) return TSPG_EINVAL;
  TSPG_CUDA(ctx, cudaDeviceSynchronize());
  TSPG_CUDA(ctx, cudaMemcpy(out64, ctx->d_prof, 64 * sizeof(uint64_t), cudaMemcpyDeviceToHost));
  return TSPG_OK;
}
