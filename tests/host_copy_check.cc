// Checks the engine's host copy pool (nmslib_b200/csrc/host_stage.cc) without a GPU: random piece
// layouts, sizes around the pool's block and job limits, zero-length pieces, more pieces than one
// job carries, several threads calling at once, jobs spaced so the workers fall asleep in between,
// and wake calls with and without jobs. Prints "ok <jobs>" and exits 0, or names the first
// mismatch and exits 1.
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <random>
#include <thread>
#include <vector>

#include "host_stage.h"

using nmsg::HostPiece;

namespace {

std::atomic<int> failures{0};

// One job: n pieces of the given sizes, sources filled from `seed`, destinations poisoned.
bool run_job(std::mt19937_64& rng, const std::vector<size_t>& sizes) {
  const int n = (int)sizes.size();
  std::vector<std::vector<unsigned char>> src(n), dst(n);
  std::vector<HostPiece> pieces(n);
  for (int i = 0; i < n; ++i) {
    // odd offsets inside a larger buffer: the pool must not assume alignment
    const size_t pad = rng() % 13;
    src[i].resize(sizes[i] + pad + 1);
    dst[i].assign(sizes[i] + pad + 1, 0xA5);
    for (auto& b : src[i]) b = (unsigned char)rng();
    pieces[i] = HostPiece{dst[i].data() + pad, src[i].data() + pad, sizes[i]};
  }
  nmsg::host_copy(pieces.data(), n);
  for (int i = 0; i < n; ++i) {
    const unsigned char* d = static_cast<const unsigned char*>(pieces[i].dst);
    const unsigned char* s = static_cast<const unsigned char*>(pieces[i].src);
    if (sizes[i] && std::memcmp(d, s, sizes[i]) != 0) {
      std::printf("mismatch in piece %d of %d (%zu bytes)\n", i, n, sizes[i]);
      return false;
    }
    // bytes around the piece stay untouched
    const size_t pad = (size_t)(d - dst[i].data());
    for (size_t j = 0; j < pad; ++j)
      if (dst[i][j] != 0xA5) {
        std::printf("write before piece %d\n", i);
        return false;
      }
    if (dst[i][pad + sizes[i]] != 0xA5) {
      std::printf("write after piece %d\n", i);
      return false;
    }
  }
  return true;
}

size_t random_size(std::mt19937_64& rng) {
  switch (rng() % 6) {
    case 0: return 0;
    case 1: return rng() % 4096;
    case 2: return 64 * 1024 * (1 + rng() % 4) + (rng() % 3) - 1;  // around block multiples
    case 3: return rng() % (512 * 1024);
    case 4: return 1024 * 1024 + rng() % (1024 * 1024);
    default: return rng() % (3 * 1024 * 1024);
  }
}

void caller(int id, int jobs, int* done) {
  std::mt19937_64 rng(1234 + id);
  for (int j = 0; j < jobs && failures.load() == 0; ++j) {
    std::vector<size_t> sizes(1 + rng() % 12);  // up to 12 pieces: more than one job holds
    for (auto& s : sizes) s = random_size(rng);
    if (!run_job(rng, sizes)) {
      failures.fetch_add(1);
      return;
    }
    ++*done;
    if (j % 16 == 15) {
      std::this_thread::sleep_for(std::chrono::milliseconds(2));  // workers sleep
      if (j % 32 == 31) nmsg::host_copy_wake();                     // and are woken without a job
    }
  }
}

}  // namespace

int main() {
  std::mt19937_64 rng(7);
  int total = 0;
  // edge sizes, one piece each
  for (size_t s : {size_t(0), size_t(1), size_t(64 * 1024 - 1), size_t(64 * 1024), size_t(128 * 1024 - 1),
                   size_t(128 * 1024), size_t(128 * 1024 + 1), size_t(1 << 20), size_t(5 << 20) + 3}) {
    if (!run_job(rng, {s})) return 1;
    ++total;
  }
  // one caller, then four at once
  int done1 = 0;
  caller(0, 200, &done1);
  if (failures.load()) return 1;
  total += done1;
  std::vector<int> done(4, 0);
  std::vector<std::thread> ts;
  std::atomic<bool> stop_waking{false};
  std::thread waker([&] {  // wake calls racing with jobs
    while (!stop_waking.load()) {
      nmsg::host_copy_wake();
      std::this_thread::sleep_for(std::chrono::microseconds(700));
    }
  });
  for (int t = 0; t < 4; ++t) ts.emplace_back(caller, t + 1, 100, &done[t]);
  for (auto& t : ts) t.join();
  stop_waking.store(true);
  waker.join();
  if (failures.load()) return 1;
  for (int d : done) total += d;
  std::printf("ok %d threads %d\n", total, nmsg::host_copy_threads());
  return 0;
}
