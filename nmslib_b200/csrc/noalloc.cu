// nmsg_knn_batch_noalloc: the batch search for callers that must not allocate device memory.
//
// Some callers cannot call cudaMalloc at query time: real-time serving threads that may not
// enter the allocator (cudaMalloc can block on device-wide synchronisation and locks, so its
// latency is unbounded), hosts whose device memory is fully reserved up front by another
// framework's pool (a new allocation would fail or evict that pool's memory), and plug-ins
// running inside such an engine. For them this entry point runs the same persistent search kernel
// as nmsg_knn_batch with device pointers, but takes every piece of per-call scratch (work
// counter, status word, per-slot epochs, visited-set epoch bytes, SearchOld candidate heaps) from
// one file-scope device array of fixed size instead of the handle's grow-on-demand buffers.
//
// The array, kNoAllocScratchBytes (32 MiB), exists on every device that loads this library, for
// the life of the process. Its host-side name is only a stand-in for the device symbol: the
// device address is obtained once per device with cudaGetSymbolAddress (with that device
// current) on the first call that runs on the device, and passed to the kernel; that first call
// should come before any stream capture. One query slot needs round_up(n, 16) + 1 bytes (plus
// the SearchOld heaps when they run), so the array limits how many queries run at once: at
// n = 1M it holds 33 slots, i.e. 33 query warps in flight instead of the thousands the
// allocating entry point runs, and throughput drops accordingly.
//
// Calls share the array and it keeps the last call's contents. The epoch bytes stay valid across
// calls that use the same slot layout (each query takes the next epoch of its slot, as the
// reference's VisitedList does), so such a call clears only its work counter and status word; a
// call with a different layout (another index, or another ef / k that changes the slot count)
// clears every byte it uses first. Calls that overlap on the GPU race on the array.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "engine.h"
#include "handle.h"
#include "../../include/nmslib_b200.h"

namespace nmsg {
namespace {

constexpr size_t kNoAllocScratchBytes = 32u << 20;
constexpr int kMaxDevices = 64;
constexpr int kNoAllocMaxSmemPerBlock = 227 * 1024;

// Shared by every call on a device; keeps the previous call's contents (each call clears the
// part it uses before launching).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Slot layout of the last call on each device (host-side record): a call with the same layout
// keeps the epoch and visited bytes the previous one left, which are consistent by construction.
struct ScratchLayout {
  int64_t slots = -1, vpitch = -1, old_cap = -1;
  bool operator==(const ScratchLayout& o) const {
    return slots == o.slots && vpitch == o.vpitch && old_cap == o.old_cap;
  }
};
ScratchLayout g_last_layout[kMaxDevices];

// Device address of g_noalloc_scratch on `device` (which must be current), looked up once.
int scratch_address(int device, void** out) {
  if (device < 0 || device >= kMaxDevices) {
    set_last_error("device ordinal out of range for the no-alloc scratch");
    return NMSG_ERR_BAD_ARG;
  }
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_last_error(std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e));
      return NMSG_ERR_DEVICE;
    }
    g_scratch_addr[device] = p;
  }
  *out = g_scratch_addr[device];
  return NMSG_OK;
}

int cuda_error(cudaError_t e, const char* what) {
  set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
  return NMSG_ERR_DEVICE;
}

}  // namespace
}  // namespace nmsg

using namespace nmsg;

extern "C" NMSG_API int nmsg_knn_batch_noalloc(nmsg_index* h, const float* queries, int64_t nq, int32_t dim,
                                               int32_t k, int32_t kmax, int32_t* ids, float* dists,
                                               int32_t* counts, void* stream) {
  if (!h) {
    set_last_error("Must call createIndex or loadIndex before this method");
    return NMSG_ERR_BAD_ARG;
  }
  if (nq < 0 || k < 1 || kmax < k) {
    set_last_error("nq must be >= 0, k >= 1 and kmax >= k");
    return NMSG_ERR_BAD_ARG;
  }
  if (h->host.sift) {
    set_last_error("nmsg_knn_batch_noalloc takes float queries; l2sqr_sift indices are searched with nmsg_knn_batch_u8");
    return NMSG_ERR_BAD_ARG;
  }
  if (nq > 0 && (!queries || !ids || !dists || !counts)) {
    set_last_error("null buffer");
    return NMSG_ERR_BAD_ARG;
  }
  std::lock_guard<std::mutex> lk(h->mu);
  DeviceGuard guard(h->device);
  void* base = nullptr;
  int rc = scratch_address(h->device, &base);
  if (rc != NMSG_OK) return rc;
  if (nq == 0) return NMSG_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const DevIndex& d = h->dev;
  if (d.n == 0) {  // empty index: every query returns nothing
    cudaError_t e = cudaMemsetAsync(counts, 0, nq * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(ids, 0xff, nq * kmax * 4, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? NMSG_OK : cuda_error(e, "no-alloc search");
  }
  if (dim != d.dim) {
    set_last_error("query dimension " + std::to_string(dim) + " does not match the index dimension " +
                   std::to_string(d.dim));
    return NMSG_ERR_BAD_ARG;
  }
  const int ef = h->ef, algo = h->algo;
  const bool old = algo == NMSG_ALGO_OLD || (algo == NMSG_ALGO_HYBRID && ef >= 1000);

  SearchArgs a;
  a.ix = d;
  a.queries = queries;
  a.nq = nq;
  a.k_default = k;
  a.ef_default = ef;
  a.algo = algo;
  a.kmax = kmax;
  a.ids = ids;
  a.dists = dists;
  a.counts = counts;
  a.nbpad = ((std::max(d.maxM, d.maxM0) + 1 + 31) / 32) * 32;
  a.region_items = ((old ? ef + 1 + k : std::max(ef, k)) + 1) & ~1;
  a.hash_log2 = 0;
  a.stage_rows = 0;
  const int gather = (d.dist_type == kL1 || d.dist_type == kLInf) ? kLpGather : (d.pitch <= 256 ? 2 : 1);
  a.warp_smem = warp_smem_bytes(d, a.region_items, a.nbpad, 0, 0);
  int wpb = 4;
  while (wpb > 1 && wpb * a.warp_smem > kNoAllocMaxSmemPerBlock) wpb >>= 1;
  if (wpb * a.warp_smem > kNoAllocMaxSmemPerBlock) {
    set_last_error("max(ef, k) needs more shared memory per query than a block has");
    return NMSG_ERR_CAPACITY;
  }
  int bps = 0;
  rc = search_occupancy(false, gather, old, wpb, wpb * a.warp_smem, &bps);
  if (rc != 0 || bps < 1) {
    set_last_error("no resident block fits this configuration");
    return NMSG_ERR_DEVICE;
  }

  // Scratch layout: [0, 256) work counter and status word | epochs, one byte per slot |
  // visited epoch bytes, slots x vpitch | SearchOld candidate heaps, slots x old_cap x 8 bytes.
  const int64_t vpitch = ((d.n + 15) / 16) * 16;
  const int64_t old_cap = old ? std::min<int64_t>(d.n + 1, 1 << 17) : 0;
  const int64_t per_slot = vpitch + 1 + old_cap * 8;
  const int64_t avail = (int64_t)kNoAllocScratchBytes - 512;
  const int64_t fit = avail / per_slot;
  if (fit < 1) {
    set_last_error("the index is too large for nmsg_knn_batch_noalloc: one query slot needs " +
                   std::to_string(per_slot) + " bytes of scratch and the fixed scratch holds " +
                   std::to_string(kNoAllocScratchBytes) + " bytes");
    return NMSG_ERR_CAPACITY;
  }
  int64_t slots = std::min<int64_t>((int64_t)bps * h->num_sms * wpb, fit);
  if (slots < wpb) wpb = 1;
  const int blocks = (int)(slots / wpb);
  slots = (int64_t)blocks * wpb;
  char* p = static_cast<char*>(base);
  a.work_counter = reinterpret_cast<int32_t*>(p);
  a.status = reinterpret_cast<int32_t*>(p + 4);
  a.epochs = reinterpret_cast<uint8_t*>(p + 256);
  a.visited = reinterpret_cast<uint8_t*>(p + 256 + ((slots + 255) / 256) * 256);
  a.visited_pitch = vpitch;
  a.old_heap = reinterpret_cast<uint2*>(a.visited + slots * vpitch);
  a.old_heap_cap = old_cap;
  a.num_slots = (int)slots;
  const size_t used = (size_t)(reinterpret_cast<char*>(a.old_heap + slots * old_cap) - p);

  // the work counter and status word start at zero; epochs and visited bytes too unless the
  // previous call on this device used the same layout
  ScratchLayout layout;
  layout.slots = slots;
  layout.vpitch = vpitch;
  layout.old_cap = old_cap;
  bool same_layout;
  {
    std::lock_guard<std::mutex> lk2(g_scratch_mu);
    same_layout = g_last_layout[h->device] == layout;
    g_last_layout[h->device] = ScratchLayout();  // unknown until the clear below is queued
  }
  cudaError_t e = cudaMemsetAsync(base, 0, same_layout ? 256 : used, st);
  if (e != cudaSuccess) return cuda_error(e, "clear no-alloc scratch");
  {
    std::lock_guard<std::mutex> lk2(g_scratch_mu);
    g_last_layout[h->device] = layout;
  }
  rc = launch_search(a, false, gather, old, blocks, wpb, stream);
  if (rc != 0) return cuda_error((cudaError_t)rc, "no-alloc search kernel launch");
  int32_t status = 0;
  e = cudaMemcpyAsync(&status, a.status, 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_error(e, "no-alloc search");
  h->last_status = status;
  if (status != 0) {
    set_last_error("the search kernel reported a device-side error (status " + std::to_string(status) + ")");
    return status;
  }
  return NMSG_OK;
}
