// The index handle behind the C ABI (struct nmsg_index) and small device-memory helpers.
// Internal to the engine library.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "engine.h"
#include "../../include/nmslib_b200.h"

namespace nmsg {

// Sets the thread-local message returned by nmsg_last_error().
void set_last_error(const std::string& msg);

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
  nmsg::DevBuf vecs, l0, up_off, up_links, ext_id;
  // search scratch (grown on demand)
  nmsg::DevBuf visited, epochs, locks, old_heap, counter, status, order, kq, efq;
  nmsg::DevBuf q_stage, ids_stage, dists_stage, counts_stage, stats_stage;
  int slots = 0;            // slots covered by visited/epochs/locks
  int64_t old_cap = 0;      // entries per slot in old_heap
  int64_t resident_bytes = 0;
  int last_status = NMSG_OK;
  nmsg_launch_config cfg{0, 0, 0, 0};
  std::mutex mu;
};
