// The index handle behind the C ABI (struct nmsg_index) and small device-memory helpers.
// Internal to the engine library.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "engine.h"
#include "host_stage.h"
#include "../../include/nmslib_b200.h"

namespace nmsg {

struct BruteForceState;  // bruteforce.cu
void destroy_bruteforce(BruteForceState* s);

// Sets the thread-local message returned by nmsg_last_error().
void set_last_error(const std::string& msg);

constexpr int kWarpsPerBlock = 4;
// Queries a persistent warp carries at once unless the launch configuration says otherwise.
constexpr int kDefaultQueriesPerWarp = 1;
// Rows wider than this many bytes are staged with one bulk copy each unless configured otherwise.
constexpr int kBulkRowMinBytes = 1024;
// Bytes of bulk row copies one staging round waits for on one mbarrier phase (plan_launch).
constexpr int kBulkRoundBytes = 32768;
constexpr int kMaxSmemPerBlock = 227 * 1024;

// Launch shape of one search launch (see plan_launch).
struct LaunchPlan {
  int gather = 1;         // 0: staged rows in shared memory; 1/2/4: register rows per 8-lane group; 3: L1 / LInf
  int stage_rows = 0;
  int hash_log2 = 0;
  int region = 0;         // shared-memory items per warp (beam array or SearchOld heaps)
  int nbpad = 32;
  int warp_smem = 0;
  int wpb = kWarpsPerBlock;
  int blocks_per_sm = 0;
  bool with_old = false;
  int ctx = 1;            // queries per persistent warp (> 1: search_multi_kernel)
  bool bulk_rows = false; // search_multi_kernel stages rows with bulk copies
  bool lean = false;      // search_lean_kernel
};

// Chooses gather mode, shared-memory sizes and warps per block for a launch whose largest query
// needs `region` items, honouring explicit settings in cfg; returns an nmsg_status.
int plan_launch(const DevIndex& d, const nmsg_launch_config& cfg, int region, bool with_old, bool plain,
                LaunchPlan* out, std::string* err);

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// A grow-only device buffer.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaError_t ensure(size_t want, bool zero) {
    if (want <= bytes) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) return e;
    bytes = want;
    if (zero) return cudaMemset(p, 0, want);
    return cudaSuccess;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <typename T>
  T* as() const {
    return reinterpret_cast<T*>(p);
  }
};

}  // namespace nmsg

struct nmsg_index {
  int device = 0;
  int space = 0;
  int ef = 20;
  int algo = NMSG_ALGO_HYBRID;
  int num_sms = 0;
  nmsg::HostIndex host;
  nmsg::DevIndex dev;
  nmsg::DevBuf vecs, norms, l0, up_off, up_links, ext_id;
  // search scratch (grown on demand)
  nmsg::DevBuf visited, epochs, locks, old_heap, counter, status, order, kq, efq;
  nmsg::DevBuf entry;       // split lean search: entry nodes, distances, counts, key range, order
  nmsg::DevBuf q_stage, ids_stage, dists_stage, counts_stage, stats_stage;
  nmsg::PinBuf pin_in, pin_out;  // page-locked staging of pageable host buffers
  int slots = 0;            // slots covered by visited/epochs/locks
  int64_t old_cap = 0;      // entries per slot in old_heap
  int64_t resident_bytes = 0;
  int last_status = NMSG_OK;
  int last_launches = 0;    // search kernels of the last batch call
  nmsg_launch_config cfg{0, 0, 0, 0, 0, 0, 0, 0, 0};
  nmsg::BruteForceState* bf = nullptr;  // brute-force data, built on first use
  cudaGraphExec_t graph_exec = nullptr;  // last captured device-pointer search (NMSG_CUDA_GRAPH)
  cudaStream_t capture_stream = nullptr;
  cudaStream_t copy_stream = nullptr;  // two-part query uploads of split searches
  cudaEvent_t part_ev[3] = {nullptr, nullptr, nullptr};  // first half copied, all copied, start
  nmsg::SearchArgs graph_args{};
  int graph_shape[5] = {0, 0, 0, 0, 0};
  std::mutex mu;
};
