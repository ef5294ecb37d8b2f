// Page-locked staging and the host copy pool behind it (host_stage.h).
#include "host_stage.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

namespace nmsg {
namespace {

inline void cpu_relax() {
#if defined(__x86_64__) || defined(__i386__)
  __builtin_ia32_pause();
#elif defined(__aarch64__)
  asm volatile("yield");
#endif
}

constexpr size_t kBlock = 64 * 1024;  // bytes a thread claims at a time
constexpr size_t kPinAlign = 256;
constexpr int kMaxPieces = 8;
// A worker polls this long for the next job (after a job or a wake call) before it sleeps.
constexpr auto kSpin = std::chrono::microseconds(300);

// The job cursor packs a generation (24 bits), the job's block count (20 bits) and the next
// unclaimed block (20 bits) into one word, so a thread claims a block of the current job with one
// compare-and-swap and a thread still looking at an older job can never claim one.
constexpr int kGenShift = 40, kCountShift = 20;
constexpr uint64_t kField = (1ull << 20) - 1;

class CopyPool {
 public:
  explicit CopyPool(int workers) {
    for (int i = 0; i < workers; ++i) threads_.emplace_back([this] { worker(); });
  }

  int threads() const { return (int)threads_.size() + 1; }

  void copy(const HostPiece* p, int n) {
    std::lock_guard<std::mutex> call(call_mu_);
    size_t total = 0;
    for (int i = 0; i < n; ++i) total += p[i].bytes;
    if (total == 0) return;
    if (threads_.empty() || total < 2 * kBlock) {
      for (int i = 0; i < n; ++i)
        if (p[i].bytes) std::memcpy(p[i].dst, p[i].src, p[i].bytes);
      return;
    }
    job_.n = n;
    job_.start[0] = 0;
    for (int i = 0; i < n; ++i) {
      job_.pieces[i] = p[i];
      job_.start[i + 1] = job_.start[i] + p[i].bytes;
    }
    // blocks of at least kBlock bytes, at most 2^20 of them, 4 KB multiples
    size_t block = std::max(kBlock, (total + kField - 1) / kField);
    block = (block + 4095) & ~size_t(4095);
    job_.block = block;
    job_.total = total;
    const uint64_t nblocks = (total + block - 1) / block;
    done_.store(0, std::memory_order_relaxed);
    gen_ = (gen_ + 1) & ((1ull << (64 - kGenShift)) - 1);
    if (gen_ == 0) gen_ = 1;
    {
      std::lock_guard<std::mutex> lk(m_);
      cursor_.store(gen_ << kGenShift | nblocks << kCountShift, std::memory_order_release);
    }
    if (sleepers_.load(std::memory_order_relaxed)) wake_.notify_all();
    work(gen_);
    // every block is claimed; wait for the ones other threads are still copying
    while (done_.load(std::memory_order_acquire) < nblocks) cpu_relax();
  }

  // Sleeping workers start polling again (for kSpin), so that a job published soon after finds
  // them running.
  void wake() {
    if (threads_.empty() || !sleepers_.load(std::memory_order_relaxed)) return;
    {
      std::lock_guard<std::mutex> lk(m_);
      poke_.fetch_add(1, std::memory_order_relaxed);
    }
    wake_.notify_all();
  }

 private:
  struct Job {
    HostPiece pieces[kMaxPieces];
    size_t start[kMaxPieces + 1];
    int n = 0;
    size_t block = kBlock, total = 0;
  };

  // Claims and copies blocks of job `g` until none is left or a newer job is published.
  void work(uint64_t g) {
    uint64_t c = cursor_.load(std::memory_order_acquire);
    for (;;) {
      if ((c >> kGenShift) != g) return;
      const uint64_t count = (c >> kCountShift) & kField, next = c & kField;
      if (next >= count) return;
      if (cursor_.compare_exchange_weak(c, c + 1, std::memory_order_acq_rel, std::memory_order_acquire)) {
        // the caller waits for this block before it touches job_ again
        copy_block(next);
        done_.fetch_add(1, std::memory_order_release);
        c = cursor_.load(std::memory_order_acquire);
      }
    }
  }

  void copy_block(uint64_t b) {
    const size_t lo = b * job_.block, hi = std::min(job_.total, lo + job_.block);
    int i = 0;
    while (job_.start[i + 1] <= lo) ++i;
    for (size_t at = lo; at < hi; ++i) {
      const size_t end = std::min(hi, job_.start[i + 1]), off = at - job_.start[i];
      if (end > at)
        std::memcpy(static_cast<char*>(job_.pieces[i].dst) + off, static_cast<const char*>(job_.pieces[i].src) + off,
                    end - at);
      at = end;
    }
  }

  void worker() {
    uint64_t seen = 0, poked = 0;
    auto deadline = std::chrono::steady_clock::now() + kSpin;
    int it = 0;
    for (;;) {
      const uint64_t c = cursor_.load(std::memory_order_acquire);
      if ((c >> kGenShift) != seen) {
        seen = c >> kGenShift;
        work(seen);
        deadline = std::chrono::steady_clock::now() + kSpin;
        continue;
      }
      if (stop_.load(std::memory_order_relaxed)) return;
      if ((++it & 255) == 0 && std::chrono::steady_clock::now() > deadline) {
        std::unique_lock<std::mutex> lk(m_);
        sleepers_.fetch_add(1, std::memory_order_relaxed);
        wake_.wait(lk, [&] {
          return (cursor_.load(std::memory_order_acquire) >> kGenShift) != seen ||
                 poke_.load(std::memory_order_relaxed) != poked || stop_.load();
        });
        sleepers_.fetch_sub(1, std::memory_order_relaxed);
        poked = poke_.load(std::memory_order_relaxed);
        deadline = std::chrono::steady_clock::now() + kSpin;
      } else {
        cpu_relax();
      }
    }
  }

  std::vector<std::thread> threads_;
  std::mutex call_mu_;  // one job at a time
  std::mutex m_;        // sleeping workers
  std::condition_variable wake_;
  std::atomic<uint64_t> cursor_{0};
  std::atomic<uint64_t> done_{0};
  std::atomic<bool> stop_{false};
  std::atomic<int> sleepers_{0};
  std::atomic<uint64_t> poke_{0};
  uint64_t gen_ = 0;  // written by the caller holding call_mu_
  Job job_;
};

CopyPool& pool() {
  // Half the host's hardware threads, at most 8 with the caller. Never destroyed: its threads
  // sleep at process exit.
  static CopyPool* p = [] {
    const int hw = (int)std::thread::hardware_concurrency();
    return new CopyPool(std::max(0, std::min(7, hw / 2 - 1)));
  }();
  return *p;
}

inline size_t pin_round(size_t b) { return (b + kPinAlign - 1) & ~(kPinAlign - 1); }

}  // namespace

void host_copy(const HostPiece* pieces, int n) {
  for (int i = 0; i < n; i += kMaxPieces) pool().copy(pieces + i, std::min(kMaxPieces, n - i));
}

int host_copy_threads() { return pool().threads(); }

void host_copy_wake() { pool().wake(); }

cudaError_t PinBuf::wait() { return done ? cudaEventSynchronize(done) : cudaSuccess; }

cudaError_t PinBuf::mark(cudaStream_t st) {
  if (!done) {
    cudaError_t e = cudaEventCreateWithFlags(&done, cudaEventDisableTiming);
    if (e != cudaSuccess) {
      done = nullptr;
      return e;
    }
  }
  return cudaEventRecord(done, st);
}

cudaError_t PinBuf::ensure(size_t want) {
  cudaError_t e = wait();
  if (e != cudaSuccess) return e;
  if (want <= bytes) return cudaSuccess;
  if (p) cudaFreeHost(p);
  p = nullptr;
  bytes = 0;
  const size_t grow = (want + (2u << 20) - 1) & ~size_t((2u << 20) - 1);  // 2 MB steps
  e = cudaHostAlloc(&p, grow, cudaHostAllocDefault);
  if (e != cudaSuccess) {
    p = nullptr;
    return e;
  }
  bytes = grow;
  return cudaSuccess;
}

void PinBuf::release() {
  wait();
  if (p) cudaFreeHost(p);
  if (done) cudaEventDestroy(done);
  if (ahead) cudaEventDestroy(ahead);
  p = nullptr;
  done = ahead = nullptr;
  bytes = 0;
}

bool is_page_locked(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();  // clear the error it recorded
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

cudaError_t upload_staged(PinBuf& pin, const HostPiece* pieces, int n, cudaStream_t st) {
  size_t need = 0;
  for (int i = 0; i < n; ++i) need += pin_round(pieces[i].bytes);
  cudaError_t e = pin.ensure(need);
  if (e != cudaSuccess) return e;
  // One fill of every piece, then one DMA each: measured on a PCIe 5 host, chunked fills whose
  // DMAs overlap the next chunk's fill ended later than one fill followed by one DMA (5 MB: 1 MB
  // chunks 202 us, one fill 42 us + one DMA 103 us).
  std::vector<HostPiece> fill(n);
  size_t off = 0;
  for (int i = 0; i < n; ++i) {
    fill[i] = HostPiece{pin.as<char>() + off, pieces[i].src, pieces[i].bytes};
    off += pin_round(pieces[i].bytes);
  }
  host_copy(fill.data(), n);
  for (int i = 0; i < n; ++i) {
    if (!pieces[i].bytes) continue;
    e = cudaMemcpyAsync(pieces[i].dst, fill[i].dst, pieces[i].bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = pin.mark(st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t download_staged(PinBuf& pin, const HostPiece* pieces, int n, cudaStream_t st) {
  size_t need = 0;
  for (int i = 0; i < n; ++i) need += pin_round(pieces[i].bytes);
  cudaError_t e = pin.ensure(need);
  if (e != cudaSuccess) return e;
  if (!pin.ahead) {
    e = cudaEventCreateWithFlags(&pin.ahead, cudaEventDisableTiming);
    if (e != cudaSuccess) {
      pin.ahead = nullptr;
      return e;
    }
  }
  e = cudaEventRecord(pin.ahead, st);  // the work that produces the results
  if (e != cudaSuccess) return e;
  char* stage = pin.as<char>();
  std::vector<HostPiece> spread(n);
  size_t off = 0;
  for (int i = 0; i < n; ++i) {
    if (pieces[i].bytes) {
      e = cudaMemcpyAsync(stage + off, pieces[i].src, pieces[i].bytes, cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = pin.mark(st);
      if (e != cudaSuccess) return e;
    }
    spread[i] = HostPiece{pieces[i].dst, stage + off, pieces[i].bytes};
    off += pin_round(pieces[i].bytes);
  }
  // The copy threads have slept through the kernel; wake them once it ends, so they are polling
  // by the time the DMAs (tens of microseconds) land.
  e = cudaEventSynchronize(pin.ahead);
  if (e != cudaSuccess) return e;
  host_copy_wake();
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e;
  host_copy(spread.data(), n);
  return cudaSuccess;
}

namespace {

// Host buffers are pageable memory unless both ends are page-locked.
bool pageable(const void* p, size_t bytes) {
  return !(is_page_locked(p) && is_page_locked(static_cast<const char*>(p) + bytes - 1));
}

size_t total_bytes(const HostPiece* pieces, int n) {
  size_t t = 0;
  for (int i = 0; i < n; ++i) t += pieces[i].bytes;
  return t;
}

}  // namespace

bool use_staging(PinBuf& pin, bool stage, const HostPiece* pieces, int n, bool host_src) {
  if (!(stage && n > 0 && total_bytes(pieces, n) >= kStageMinBytes &&
        pageable(host_src ? pieces[0].src : pieces[0].dst, pieces[0].bytes)))
    return false;
  size_t need = 0;
  for (int i = 0; i < n; ++i) need += pin_round(pieces[i].bytes);
  if (pin.ensure(need) != cudaSuccess) {
    cudaGetLastError();  // no page-locked memory: copy directly
    return false;
  }
  return true;
}

cudaError_t upload_staged_parts(PinBuf& pin, const HostPiece* pieces, int n, size_t first_bytes, cudaStream_t cs,
                                cudaEvent_t ready[2]) {
  size_t need = 0;
  for (int i = 0; i < n; ++i) need += pin_round(pieces[i].bytes);
  cudaError_t e = pin.ensure(need);
  if (e != cudaSuccess) return e;
  std::vector<HostPiece> fill(n);
  size_t off = 0;
  for (int i = 0; i < n; ++i) {
    fill[i] = HostPiece{pin.as<char>() + off, pieces[i].src, pieces[i].bytes};
    off += pin_round(pieces[i].bytes);
  }
  host_copy(fill.data(), n);
  first_bytes = std::min(first_bytes, pieces[0].bytes);
  auto dma = [&](void* dst, const void* src, size_t bytes) {
    if (!bytes) return cudaSuccess;
    cudaError_t r = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, cs);
    return r == cudaSuccess ? pin.mark(cs) : r;
  };
  e = dma(pieces[0].dst, fill[0].dst, first_bytes);
  if (e == cudaSuccess) e = cudaEventRecord(ready[0], cs);
  if (e == cudaSuccess)
    e = dma(static_cast<char*>(pieces[0].dst) + first_bytes, static_cast<const char*>(fill[0].dst) + first_bytes,
            pieces[0].bytes - first_bytes);
  for (int i = 1; i < n && e == cudaSuccess; ++i) e = dma(pieces[i].dst, fill[i].dst, pieces[i].bytes);
  if (e == cudaSuccess) e = cudaEventRecord(ready[1], cs);
  return e;
}

cudaError_t upload_parts_direct(const HostPiece* pieces, int n, size_t first_bytes, cudaStream_t cs,
                                cudaEvent_t ready[2]) {
  first_bytes = std::min(first_bytes, pieces[0].bytes);
  auto dma = [&](void* dst, const void* src, size_t bytes) {
    return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, cs) : cudaSuccess;
  };
  cudaError_t e = dma(pieces[0].dst, pieces[0].src, first_bytes);
  if (e == cudaSuccess) e = cudaEventRecord(ready[0], cs);
  if (e == cudaSuccess)
    e = dma(static_cast<char*>(pieces[0].dst) + first_bytes, static_cast<const char*>(pieces[0].src) + first_bytes,
            pieces[0].bytes - first_bytes);
  for (int i = 1; i < n && e == cudaSuccess; ++i) e = dma(pieces[i].dst, pieces[i].src, pieces[i].bytes);
  if (e == cudaSuccess) e = cudaEventRecord(ready[1], cs);
  return e;
}

bool host_range_page_locked(const void* p, size_t bytes) { return bytes && !pageable(p, bytes); }

cudaError_t copy_to_device(PinBuf& pin, bool stage, const HostPiece* pieces, int n, cudaStream_t st) {
  if (use_staging(pin, stage, pieces, n, true)) return upload_staged(pin, pieces, n, st);
  for (int i = 0; i < n; ++i) {
    if (!pieces[i].bytes) continue;
    const cudaError_t e = cudaMemcpyAsync(pieces[i].dst, pieces[i].src, pieces[i].bytes, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t copy_to_host(PinBuf& pin, bool stage, const HostPiece* pieces, int n, cudaStream_t st) {
  if (use_staging(pin, stage, pieces, n, false)) return download_staged(pin, pieces, n, st);
  for (int i = 0; i < n; ++i) {
    if (!pieces[i].bytes) continue;
    const cudaError_t e = cudaMemcpyAsync(pieces[i].dst, pieces[i].src, pieces[i].bytes, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
  }
  return cudaStreamSynchronize(st);
}

}  // namespace nmsg
