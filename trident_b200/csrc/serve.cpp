// serve.cpp — continuous-batching server for A·B and Galerkin R·A·P requests.
//
// Requests arrive on any host thread (tspg_server_submit) with device-resident
// operands; submission does no device work.  A bounding thread (own context
// and stream) takes them in order and bounds their outputs with one batched
// flop-count pass per run of requests (sum_i min(mults_i, ncols), 12 bytes
// per entry plus row offsets) into the admission queue.  `lanes` worker
// threads, each with its own context, stream and tspg_batch objects, admit
// from the head of that queue, under the server lock and in submission order,
// the requests (up to max_batch) that fit the device-memory budget.  The admitted
// requests run as one batched product per stage: stage 1 = all A·B requests
// plus the A·P half of the R·A·P requests, stage 2 = R·(AP) for the R·A·P
// requests.  Lanes run concurrently on their own streams, so a batch that
// forms while others are on the device overlaps with them.  Results are not
// copied: a request's result is its view into the output slab of the batch
// that computed it, and the lane keeps that batch (a "group": the stage-1 and
// stage-2 batches of one admission) out of use until every request of the
// group is released; released groups go back to the lane for reuse.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "tspg.h"

#define TSPG_TRY_HOST(x)        \
  do {                          \
    const int st_ = (x);        \
    if (st_ != TSPG_OK) return st_; \
  } while (0)

namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// The two batches of one admitted group and how many of its requests still
// hold results in their slabs.
struct Group {
  tspg_batch *b1 = nullptr, *b2 = nullptr;
  int live = 0;
};

struct Req {
  int64_t ticket = 0;
  int kind = TSPG_REQ_AB;
  tspg_csr A{}, B{}, R{};
  size_t reserve = 0;  // output bound (bytes), reserved while admitted
  bool bounded = false;
  bool admitted = false;
  double t_submit = 0, t_start = 0, t_done = 0;
  int status = TSPG_OK;
  bool done = false;
  // result: a view into the output slab of its group's batch
  int lane = -1;
  Group *group = nullptr;
  int64_t nrows = 0, ncols = 0, nnz = 0;
  int64_t *rp = nullptr;
  int32_t *col = nullptr;
  void *val = nullptr;
};

}  // namespace

struct tspg_server {
  int device = 0;
  tspg_server_config cfg{};
  std::mutex mu;
  std::condition_variable cv_fresh, cv_work, cv_done;
  std::deque<Req *> fresh;  // submitted, output not bounded yet
  std::deque<Req *> queue;  // bounded, waiting for admission (submission order)
  std::unordered_map<int64_t, Req *> reqs;
  size_t reserved = 0;
  bool stop = false;
  int64_t next_ticket = 1;
  std::vector<std::thread> threads;
  tspg_ctx *bctx = nullptr;  // context and stream of the bounding thread
  cudaStream_t bstream = nullptr;
  std::vector<tspg_ctx *> lane_ctx;
  std::vector<cudaStream_t> lane_stream;
  // per lane: every group it made, and the released ones ready for reuse
  std::vector<std::vector<Group *>> lane_groups, lane_free;
  int64_t batches = 0, completed = 0, rejected = 0;
  int lane_error = TSPG_OK;
};

namespace {

// The operand checks of the product entry points, on the host.
bool csr_ok(const tspg_csr *M) {
  if (M->nrows < 0 || M->ncols < 0 || M->nnz < 0 || M->ncols > INT32_MAX) return false;
  if ((M->rowptr_bits != 32 && M->rowptr_bits != 64) || (M->val_bits != 32 && M->val_bits != 64))
    return false;
  if (M->rowptr_bits == 32 && M->nnz > INT32_MAX) return false;
  if (M->nnz > 0 && (!M->col || !M->val)) return false;
  return M->rowptr || M->nrows == 0;
}

size_t out_bytes(int64_t nnz_upper, int64_t rows, int vb) {
  return size_t(nnz_upper) * size_t(4 + vb) + size_t(rows + 1) * 8;
}

// Point request r at batch result i (a view into the batch's output slab).
int take_result(tspg_batch *b, int i, Req *r) {
  tspg_csr v{};
  int st = tspg_batch_result(b, i, &v);
  if (st != TSPG_OK) return st;
  r->nrows = v.nrows;
  r->ncols = v.ncols;
  r->nnz = v.nnz;
  r->rp = (int64_t *)v.rowptr;
  r->col = (int32_t *)v.col;
  r->val = (void *)v.val;
  return TSPG_OK;
}

// Output bounds (bytes) of the requests not bounded yet, one batched count
// pass: the A·B output, or A·P plus R·A·P (bounded by rows(R) x ncols(P)) for
// the Galerkin product.
int bound_requests(tspg_batch *bc, cudaStream_t s, const std::vector<Req *> &cand) {
  std::vector<Req *> todo;
  tspg_batch_clear(bc);
  for (Req *r : cand) {
    if (r->bounded) continue;
    int idx = 0;
    TSPG_TRY_HOST(tspg_batch_add(bc, &r->A, &r->B, &idx));
    todo.push_back(r);
  }
  if (todo.empty()) return TSPG_OK;
  std::vector<int64_t> mults(todo.size()), upper(todo.size());
  TSPG_TRY_HOST(tspg_batch_count(bc, s, mults.data(), upper.data()));
  for (size_t i = 0; i < todo.size(); ++i) {
    Req *r = todo[i];
    const int vb = r->A.val_bits / 8;
    size_t bytes = out_bytes(upper[i], r->A.nrows, vb);
    if (r->kind == TSPG_REQ_RAP) {
      const int64_t full = r->R.nrows * r->B.ncols;
      const int64_t up2 = std::min<int64_t>(
          full, upper[i] > 0 ? r->R.nnz * (upper[i] / std::max<int64_t>(1, r->A.nrows) + 1) : 0);
      bytes += out_bytes(up2, r->R.nrows, vb);
    }
    r->reserve = bytes;
    r->bounded = true;
  }
  return TSPG_OK;
}

// The bounding thread: takes the submitted requests in order (a run of one
// value width at a time), bounds their outputs with one batched count pass,
// and appends them to the admission queue (or completes them with
// TSPG_ENOMEM when the bound alone exceeds the budget).  Bounding ahead of
// the lanes keeps the count passes, which wait for SMs behind the lanes'
// persistent kernels, off the admission path.
void bound_main(tspg_server *S) {
  cudaSetDevice(S->device);
  tspg_batch *bc = nullptr;
  tspg_batch_create(S->bctx, &bc);
  std::vector<Req *> cand;
  while (true) {
    cand.clear();
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_fresh.wait(lk, [&] { return S->stop || !S->fresh.empty(); });
      if (S->stop) break;
      while (!S->fresh.empty() && cand.size() < 4096 &&
             (cand.empty() || S->fresh.front()->A.val_bits == cand[0]->A.val_bits)) {
        cand.push_back(S->fresh.front());
        S->fresh.pop_front();
      }
    }
    const int bst = bound_requests(bc, S->bstream, cand);
    bool rejected = false;
    {
      std::lock_guard<std::mutex> lk(S->mu);
      for (Req *r : cand) {
        if (bst != TSPG_OK || r->reserve > S->cfg.mem_budget) {
          r->status = bst != TSPG_OK ? bst : TSPG_ENOMEM;
          r->t_done = now_ms();
          r->done = true;
          S->rejected += 1;
          rejected = true;
        } else {
          S->queue.push_back(r);
        }
      }
      if (bst != TSPG_OK) S->lane_error = bst;
    }
    S->cv_work.notify_all();
    if (rejected) S->cv_done.notify_all();
  }
  tspg_batch_destroy(bc);
}

void lane_main(tspg_server *S, int lane) {
  cudaSetDevice(S->device);
  tspg_ctx *ctx = S->lane_ctx[lane];
  cudaStream_t s = S->lane_stream[lane];
  std::vector<Req *> take;
  while (true) {
    take.clear();
    Group *g = nullptr;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_work.wait(lk, [&] { return S->stop || !S->queue.empty(); });
      if (S->stop) break;  // requests still waiting for admission are dropped
      // FIFO admission by the memory budget, under the lock (no device work
      // here), so requests are admitted in submission order across lanes; the
      // head request is admitted whenever nothing else is reserved (its bound
      // fits the budget alone); one value width per batch
      while (!S->queue.empty() && (int)take.size() < S->cfg.max_batch) {
        Req *r = S->queue.front();
        if (!take.empty() && r->A.val_bits != take[0]->A.val_bits) break;
        if (S->reserved + r->reserve > S->cfg.mem_budget && !(S->reserved == 0 && take.empty()))
          break;
        S->queue.pop_front();
        S->reserved += r->reserve;
        r->admitted = true;
        take.push_back(r);
      }
      if (take.empty()) {
        // budget held by admitted requests: wait for a release
        S->cv_done.wait_for(lk, std::chrono::milliseconds(1));
        continue;
      }
      if (!S->lane_free[lane].empty()) {
        g = S->lane_free[lane].back();
        S->lane_free[lane].pop_back();
      }
    }
    if (!g) {  // a new group (its batches hold the results until released)
      g = new (std::nothrow) Group();
      int cst = g ? tspg_batch_create(ctx, &g->b1) : TSPG_ENOMEM;
      if (cst == TSPG_OK) cst = tspg_batch_create(ctx, &g->b2);
      if (cst != TSPG_OK && g) {  // a partial group is not kept
        if (g->b1) tspg_batch_destroy(g->b1);
        if (g->b2) tspg_batch_destroy(g->b2);
        delete g;
        g = nullptr;
      }
      std::lock_guard<std::mutex> lk(S->mu);
      if (cst != TSPG_OK) {
        for (Req *r : take) {
          r->status = cst;
          r->done = true;
          S->reserved -= r->reserve;
          r->admitted = false;
        }
        S->lane_error = cst;
        S->cv_done.notify_all();
        continue;
      }
      S->lane_groups[lane].push_back(g);
    }
    tspg_batch *b1 = g->b1, *b2 = g->b2;
    const double t0 = now_ms();
    for (Req *r : take) r->t_start = t0;
    int st = TSPG_OK;
    // stage 1: A·B and A·P
    tspg_batch_clear(b1);
    for (Req *r : take) {
      int idx = 0;
      if (st == TSPG_OK) st = tspg_batch_add(b1, &r->A, &r->B, &idx);
    }
    int64_t tot = 0;
    if (st == TSPG_OK) st = tspg_batch_run(b1, s, 0, &tot);
    // stage 2: R·(AP)
    std::vector<int> rap;
    if (st == TSPG_OK) {
      tspg_batch_clear(b2);
      for (int i = 0; i < (int)take.size() && st == TSPG_OK; ++i) {
        if (take[i]->kind != TSPG_REQ_RAP) continue;
        tspg_csr ap{};
        st = tspg_batch_result(b1, i, &ap);
        int idx = 0;
        if (st == TSPG_OK) st = tspg_batch_add(b2, &take[i]->R, &ap, &idx);
        rap.push_back(i);
      }
      if (st == TSPG_OK && !rap.empty()) st = tspg_batch_run(b2, s, 0, &tot);
    }
    if (st == TSPG_OK) {
      for (int i = 0, k = 0; i < (int)take.size() && st == TSPG_OK; ++i) {
        Req *r = take[i];
        if (r->kind == TSPG_REQ_RAP) st = take_result(b2, k++, r);
        else st = take_result(b1, i, r);
      }
    }
    if (cudaStreamSynchronize(s) != cudaSuccess && st == TSPG_OK) st = TSPG_ECUDA;
    const double t1 = now_ms();
    {
      std::lock_guard<std::mutex> lk(S->mu);
      for (Req *r : take) {
        r->status = st;
        r->t_done = t1;
        r->done = true;
        r->lane = lane;
        if (st != TSPG_OK) {
          S->reserved -= r->reserve;
          r->admitted = false;
        } else {
          r->group = g;
        }
      }
      if (st == TSPG_OK) g->live = int(take.size());
      else S->lane_free[lane].push_back(g);  // nothing refers to its slabs
      S->batches += 1;
      S->completed += int64_t(take.size());
      if (st != TSPG_OK) S->lane_error = st;
    }
    S->cv_done.notify_all();
  }
}

}  // namespace

extern "C" int tspg_server_create(tspg_ctx *ctx, const tspg_server_config *cfg,
                                  tspg_server **out) {
  if (!ctx || !cfg || !out || cfg->lanes < 1 || cfg->lanes > 16 || cfg->max_batch < 1 ||
      cfg->mem_budget == 0)
    return TSPG_EINVAL;
  *out = nullptr;
  tspg_server *S = new (std::nothrow) tspg_server();
  if (!S) return TSPG_ENOMEM;
  S->cfg = *cfg;
  S->lane_groups.resize(cfg->lanes);
  S->lane_free.resize(cfg->lanes);
  int dev = 0;
  cudaGetDevice(&dev);
  S->device = dev;
  tspg_tuning tune;  // lanes take the row binning of the parent context
  int st = tspg_ctx_get_tuning(ctx, &tune);
  for (int l = 0; l < cfg->lanes && st == TSPG_OK; ++l) {
    tspg_ctx *c = nullptr;
    cudaStream_t ls = nullptr;
    st = tspg_ctx_create(dev, 0, &c);
    if (st == TSPG_OK) st = tspg_ctx_set_tuning(c, &tune);
    if (st == TSPG_OK && cudaStreamCreateWithFlags(&ls, cudaStreamNonBlocking) != cudaSuccess)
      st = TSPG_ECUDA;
    S->lane_ctx.push_back(c);
    S->lane_stream.push_back(ls);
  }
  if (st == TSPG_OK) st = tspg_ctx_create(dev, 0, &S->bctx);
  if (st == TSPG_OK && cudaStreamCreateWithFlags(&S->bstream, cudaStreamNonBlocking) != cudaSuccess)
    st = TSPG_ECUDA;
  if (st != TSPG_OK) {
    tspg_server_destroy(S);
    return st;
  }
  for (int l = 0; l < cfg->lanes; ++l) S->threads.emplace_back(lane_main, S, l);
  S->threads.emplace_back(bound_main, S);
  *out = S;
  return TSPG_OK;
}

extern "C" int tspg_server_destroy(tspg_server *S) {
  if (!S) return TSPG_EINVAL;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_fresh.notify_all();
  S->cv_work.notify_all();
  for (auto &t : S->threads) t.join();
  cudaSetDevice(S->device);
  cudaDeviceSynchronize();
  for (auto &kv : S->reqs) delete kv.second;  // their results live in the groups' slabs
  for (auto &gs : S->lane_groups)
    for (Group *g : gs) {
      if (g->b1) tspg_batch_destroy(g->b1);
      if (g->b2) tspg_batch_destroy(g->b2);
      delete g;
    }
  // every request in fresh / queue is also in reqs (freed above)
  for (size_t l = 0; l < S->lane_ctx.size(); ++l) {
    if (S->lane_stream[l]) cudaStreamDestroy(S->lane_stream[l]);
    if (S->lane_ctx[l]) tspg_ctx_destroy(S->lane_ctx[l]);
  }
  if (S->bstream) cudaStreamDestroy(S->bstream);
  if (S->bctx) tspg_ctx_destroy(S->bctx);
  delete S;
  return TSPG_OK;
}

extern "C" int tspg_server_submit(tspg_server *S, int kind, const tspg_csr *A,
                                  const tspg_csr *B, const tspg_csr *R, int64_t *ticket) {
  if (!S || !A || !B || !ticket) return TSPG_EINVAL;
  if (kind != TSPG_REQ_AB && kind != TSPG_REQ_RAP) return TSPG_EINVAL;
  if (kind == TSPG_REQ_RAP && !R) return TSPG_EINVAL;
  if (!csr_ok(A) || !csr_ok(B) || A->ncols != B->nrows || A->val_bits != B->val_bits)
    return TSPG_EINVAL;
  if (kind == TSPG_REQ_RAP &&
      (!csr_ok(R) || R->ncols != A->nrows || R->val_bits != A->val_bits))
    return TSPG_EINVAL;
  Req *r = new (std::nothrow) Req();
  if (!r) return TSPG_ENOMEM;
  r->kind = kind;
  r->A = *A;
  r->B = *B;
  if (R) r->R = *R;
  r->t_submit = now_ms();
  std::lock_guard<std::mutex> lk(S->mu);
  r->ticket = S->next_ticket++;
  S->reqs[r->ticket] = r;
  S->fresh.push_back(r);
  *ticket = r->ticket;
  S->cv_fresh.notify_one();
  return TSPG_OK;
}

extern "C" int tspg_server_wait(tspg_server *S, int64_t ticket, int timeout_ms,
                                tspg_csr *result, double *latency_ms) {
  if (!S) return TSPG_EINVAL;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) return TSPG_EINVAL;
  Req *r = it->second;
  const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms);
  while (!r->done) {
    if (timeout_ms >= 0) {
      if (S->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && !r->done)
        return TSPG_ETIMEOUT;
    } else {
      S->cv_done.wait(lk);
    }
  }
  if (latency_ms) *latency_ms = r->t_done - r->t_submit;
  if (r->status != TSPG_OK) return r->status;
  if (result) {
    result->nrows = r->nrows;
    result->ncols = r->ncols;
    result->nnz = r->nnz;
    result->rowptr = r->rp;
    result->rowptr_bits = 64;
    result->val_bits = r->A.val_bits;
    result->col = r->col;
    result->val = r->val;
  }
  return TSPG_OK;
}

extern "C" int tspg_server_release(tspg_server *S, int64_t ticket) {
  if (!S) return TSPG_EINVAL;
  Req *r = nullptr;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end() || !it->second->done) return TSPG_EINVAL;
    r = it->second;
    S->reqs.erase(it);
    if (r->admitted) S->reserved -= r->reserve;
    // the last release of a group hands its batches back to the lane (the
    // lane's work on their slabs finished before the requests were done)
    if (r->group && --r->group->live == 0) S->lane_free[r->lane].push_back(r->group);
  }
  delete r;
  S->cv_work.notify_all();
  S->cv_done.notify_all();
  return TSPG_OK;
}

extern "C" int tspg_server_stats(tspg_server *S, int64_t *batches, int64_t *completed,
                                 int64_t *queued, size_t *reserved) {
  if (!S) return TSPG_EINVAL;
  std::lock_guard<std::mutex> lk(S->mu);
  if (batches) *batches = S->batches;
  if (completed) *completed = S->completed;
  if (queued) *queued = int64_t(S->queue.size() + S->fresh.size());
  if (reserved) *reserved = S->reserved;
  return S->lane_error;
}
