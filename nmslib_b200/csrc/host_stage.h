// Page-locked staging for batch calls on pageable host buffers. Internal to the engine library.
//
// A DMA from pageable memory goes through the CUDA driver's own bounce buffers, which one host
// thread fills. The batch entry points instead fill page-locked buffers with several host threads
// and copy those by DMA at the link's full rate. Results come back by DMA into page-locked memory,
// and the same threads spread them to the caller's arrays.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace nmsg {

// One copy: `bytes` from `src` to `dst` (host memory for the pool; one side device memory for
// upload_staged / download_staged, named there).
struct HostPiece {
  void* dst;
  const void* src;
  size_t bytes;
};

// Copies the pieces with the process-wide pool of host copy threads; the calling thread copies
// too. Returns when every byte is copied. Thread-safe (concurrent callers take turns).
void host_copy(const HostPiece* pieces, int n);

// Host threads the pool copies with, the calling thread included.
int host_copy_threads();

// Sleeping copy threads start polling again for a while, so that a host_copy soon after finds
// them running (waking a sleeping thread takes tens of microseconds).
void host_copy_wake();

// A grow-only page-locked host buffer. `done` marks the last copies queued on it; the next use
// (and release) waits for them, so a call that returned early with copies in flight cannot have
// them overwritten or freed under it. `ahead` marks, in download_staged, the work queued before
// the copies.
struct PinBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaEvent_t done = nullptr;
  cudaEvent_t ahead = nullptr;
  cudaError_t ensure(size_t want);
  cudaError_t wait();
  cudaError_t mark(cudaStream_t st);
  void release();
  template <typename T>
  T* as() const {
    return reinterpret_cast<T*>(p);
  }
};

// True when `p` points into page-locked memory the CUDA runtime knows (cudaHostAlloc,
// cudaMallocHost or cudaHostRegister), whose DMA needs no staging.
bool is_page_locked(const void* p);

// Batches whose host buffers total fewer bytes than this are copied directly.
constexpr size_t kStageMinBytes = 512 * 1024;

// Whether copies of these pieces go through staging in `pin`: `stage` allows it, they total
// kStageMinBytes or more, the first piece's host buffer (`host_src`: its source, else its
// destination) is pageable, and `pin` holds (or could grow to) room for them. When page-locked
// memory cannot be had, the copies go directly instead.
bool use_staging(PinBuf& pin, bool stage, const HostPiece* pieces, int n, bool host_src);

// upload_staged in two parts on `cs`: one fill of every piece, then the DMA of the first
// `first_bytes` of piece 0 followed by ready[0], then the DMAs of the rest followed by ready[1].
cudaError_t upload_staged_parts(PinBuf& pin, const HostPiece* pieces, int n, size_t first_bytes, cudaStream_t cs,
                                cudaEvent_t ready[2]);

// The copies of upload_staged_parts straight from the caller's buffers (page-locked ones, which
// need no staging): the first `first_bytes` of piece 0 followed by ready[0], then the rest followed
// by ready[1], on `cs`.
cudaError_t upload_parts_direct(const HostPiece* pieces, int n, size_t first_bytes, cudaStream_t cs,
                                cudaEvent_t ready[2]);

// True when the whole host range is page-locked memory (both of its ends, see is_page_locked).
bool host_range_page_locked(const void* p, size_t bytes);

// Queues on `st` the copies of a call's inputs (src: host memory, dst: device memory): through
// upload_staged when use_staging says so; otherwise directly.
cudaError_t copy_to_device(PinBuf& pin, bool stage, const HostPiece* pieces, int n, cudaStream_t st);

// Copies a call's results back (src: device memory, dst: host memory) and waits for `st`: through
// download_staged when use_staging says so, otherwise directly.
cudaError_t copy_to_host(PinBuf& pin, bool stage, const HostPiece* pieces, int n, cudaStream_t st);

// Queues on `st` the copies of every piece (src: host memory, dst: device memory) through `pin`:
// the pool fills `pin` with every piece, then one host-to-device copy per piece is queued. `pin`
// must not be touched again until `st` has passed these copies (PinBuf::wait).
cudaError_t upload_staged(PinBuf& pin, const HostPiece* pieces, int n, cudaStream_t st);

// Queues on `st` the copies of every piece (src: device memory, dst: host memory) into `pin`, waits
// for `st` (waking the pool when the work ahead of the copies ends), then spreads the bytes to
// their host destinations with the pool.
cudaError_t download_staged(PinBuf& pin, const HostPiece* pieces, int n, cudaStream_t st);

}  // namespace nmsg
