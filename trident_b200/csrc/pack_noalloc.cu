// pack_noalloc.cu — tspg_pack_noalloc: the bitmask tile pack without any
// allocation, for callers that cannot allocate device memory.
//
// Who needs it.  In Trident the pack runs on the communication side of a
// stage: a comm thread packs the next tile into its send buffer while the
// compute stream multiplies the current one and NCCL/MPI transfers are in
// flight.  cudaMalloc and cudaFree synchronise the whole device, so a pack
// that allocated would stall that overlap (and a stream-ordered pool would
// tie the pack to a context that the comm thread may not own).  This entry
// point takes no context, allocates nothing and synchronises nothing: its
// scratch is one file-scope device array.
//
// The scratch.  g_pack_scratch below is a static __device__ array of
// kNoallocScratchBytes (3 MiB + a few KiB), enough for tiles with up to
// TSPG_PACK_NOALLOC_MAX_SEGMENTS segments; every GPU that loads this library
// holds it until the process exits.  Larger tiles are rejected with
// TSPG_ESCRATCH.  Host code cannot use the array's name as a device address,
// so on the first call on each device (with that device current) the entry
// point asks the runtime for the address with cudaGetSymbolAddress and caches
// it, with the device's SM count; make that first call before any stream
// capture.  The device that is current on the calling thread must be the one
// that owns the stream and the buffers: a call whose output buffer lives on
// another device is rejected with TSPG_EINVAL.  All calls share the
// array and it keeps the previous call's contents: the kernels write every
// scratch word they read except the first pointer offset, which is cleared by
// a kernel at the start of each call.  Calls whose kernels overlap on the GPU
// (different streams, or different host threads) race on the scratch and must
// be serialised by the caller.
#include <mutex>

#include "pack_kernels.cuh"
#include "spgemm_kernels.cuh"

namespace tspg {
namespace {

constexpr int64_t kNoallocMaxSeg = TSPG_PACK_NOALLOC_MAX_SEGMENTS;
constexpr int64_t kNoallocMaxTiles = (kNoallocMaxSeg + kScanTile - 1) / kScanTile;
// layout: cnt int32[max] | newp int64[max + 1] | partial int64[tiles + 1] | Sched
constexpr size_t kOffNewp = ((size_t(kNoallocMaxSeg) * 4 + 255) / 256) * 256;
constexpr size_t kOffPartial = kOffNewp + ((size_t(kNoallocMaxSeg + 1) * 8 + 255) / 256) * 256;
constexpr size_t kOffSched = kOffPartial + ((size_t(kNoallocMaxTiles + 1) * 8 + 255) / 256) * 256;
constexpr size_t kNoallocScratchBytes = kOffSched + ((sizeof(Sched) + 255) / 256) * 256;

__device__ __align__(256) unsigned char g_pack_scratch[kNoallocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void *g_scratch_addr[kMaxDevices] = {};
int g_num_sms[kMaxDevices] = {};

// Device address of g_pack_scratch on the current device and that device's
// SM count (looked up once per device).  `probe` is a device buffer of the
// call: when it belongs to another device the call is rejected.
int scratch_for_current_device(const void *probe, void **out, int *num_sms) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    (void)cudaGetLastError();
    return TSPG_ECUDA;
  }
  cudaPointerAttributes pa{};
  if (cudaPointerGetAttributes(&pa, probe) != cudaSuccess) {
    (void)cudaGetLastError();
    return TSPG_EINVAL;
  }
  if (pa.type == cudaMemoryTypeDevice && pa.device != dev) return TSPG_EINVAL;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    int sms = 0;
    if (cudaGetSymbolAddress(&p, g_pack_scratch) != cudaSuccess || !p ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
      (void)cudaGetLastError();
      return TSPG_ECUDA;
    }
    g_num_sms[dev] = sms > 0 ? sms : 1;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  *num_sms = g_num_sms[dev];
  return TSPG_OK;
}

__global__ void k_clear_first(int64_t *newp) { newp[0] = 0; }

template <typename PT>
int pack_noalloc_impl(cudaStream_t s, const tspg_csr *M, int64_t len,
                      const uint8_t *mask, void *out_buf, int64_t *kept_dev,
                      unsigned char *scratch, int num_sms) {
  int32_t *cnt = (int32_t *)scratch;
  int64_t *newp = (int64_t *)(scratch + kOffNewp);
  int64_t *partial = (int64_t *)(scratch + kOffPartial);
  Sched *unused = (Sched *)(scratch + kOffSched);
  const PT *ptr = (const PT *)M->rowptr;
  const int64_t nb = (len + kScanTile - 1) / kScanTile;
  k_clear_first<<<1, 1, 0, s>>>(newp);
  if (len > 0) {
    k_pack_counts<PT><<<(unsigned)((len + 255) / 256), 256, 0, s>>>(ptr, len, mask, cnt);
    k_scan_reduce<<<(unsigned)nb, kScanThreads, 0, s>>>(cnt, len, partial);
    k_scan_partials<<<1, 1024, 0, s>>>(partial, nb);
    k_scan_final<<<(unsigned)nb, kScanThreads, 0, s>>>(cnt, len, partial, nb, newp, unused,
                                                       nullptr);
  }
  const int64_t work = (M->nnz + kPackItems - 1) / kPackItems;
  const int64_t w = work > len + 1 ? work : len + 1;
  const unsigned grid = (unsigned)std::min<int64_t>((w + 255) / 256, int64_t(num_sms) * 32);
  if (M->val_bits == 64)
    k_pack_copy<PT, 8><<<grid, 256, 0, s>>>(ptr, len, M->col, M->val, mask, newp,
                                            (char *)out_buf, kept_dev);
  else
    k_pack_copy<PT, 4><<<grid, 256, 0, s>>>(ptr, len, M->col, M->val, mask, newp,
                                            (char *)out_buf, kept_dev);
  if (cudaGetLastError() != cudaSuccess) return TSPG_ECUDA;
  return TSPG_OK;
}

}  // namespace
}  // namespace tspg

using namespace tspg;

extern "C" int tspg_pack_noalloc(void *stream, const tspg_csr *M, int major,
                                 const uint8_t *mask, void *out_buf, size_t cap,
                                 int64_t *nnz_kept_dev) {
  if (!out_buf) return TSPG_EINVAL;
  TSPG_TRY(check_csr(M));
  if (major != TSPG_ROWS && major != TSPG_COLS) return TSPG_EINVAL;
  const int64_t len = major == TSPG_ROWS ? M->nrows : M->ncols;
  if (len > kNoallocMaxSeg) return TSPG_ESCRATCH;
  // the pointer array has len + 1 entries: no segments means no entries, and
  // a non-empty pointer array must be given
  if ((len == 0 && M->nnz > 0) || (len > 0 && !M->rowptr)) return TSPG_EINVAL;
  if (len > 0 && !mask) return TSPG_EINVAL;
  if ((uintptr_t)out_buf & 7) return TSPG_EINVAL;
  if (cap < tspg_packed_bytes(M->nnz, len, M->val_bits, M->rowptr_bits)) return TSPG_ENOMEM;
  void *scratch = nullptr;
  int num_sms = 1;
  TSPG_TRY(scratch_for_current_device(out_buf, &scratch, &num_sms));
  cudaStream_t s = (cudaStream_t)stream;
  if (M->rowptr_bits == 32)
    return pack_noalloc_impl<int32_t>(s, M, len, mask, out_buf, nnz_kept_dev,
                                      (unsigned char *)scratch, num_sms);
  return pack_noalloc_impl<int64_t>(s, M, len, mask, out_buf, nnz_kept_dev,
                                    (unsigned char *)scratch, num_sms);
}
