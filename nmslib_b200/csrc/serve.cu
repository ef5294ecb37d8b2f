// Continuous-batching query server over a loaded index (the serving front of the HNSW query path).
//
// Requests (a batch of 1..max_batch queries with its own k and efSearch) are admitted as device
// memory frees up: each needs a run of search slots (a slot is one warp's visited-set epoch bytes,
// the memory that grows with the index) from a pool sized by the memory budget, one slot per
// query up to a block-rounded cap, and a lane (a CUDA stream with staging buffers; lanes are
// cheap). Admission is first come, first served: the oldest waiting request starts as soon as its
// slots and a lane are free. Every admitted request is one launch of the persistent search
// kernel on its lane's stream over its own slots, so requests that arrive while others run are
// searched concurrently on the device; nothing a request computes depends on the others, so its
// results are the same alone and in any mix. A worker thread admits requests and harvests
// finished lanes (event query); callers submit and wait without blocking the GPU.
//
// The reference has no server on this path (its Thrift front end, query_server/, is out of
// scope); per-request semantics are those of knnQueryBatch (python_bindings/nmslib.cc:142-168).
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.h"
#include "handle.h"
#include "../../include/nmslib_b200.h"

using namespace nmsg;

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
  int64_t id = 0;
  std::vector<float> q;
  int nq = 0, k = 0, ef = 0;
  double t_arrival = 0, t_done = 0;
  bool done = false;
  int status = NMSG_OK;
  std::vector<int32_t> ids, counts;
  std::vector<float> dists;
};

struct Lane {
  cudaStream_t st = nullptr;
  cudaEvent_t done = nullptr;
  DevBuf q, ids, dists, counts, counter, status;
  float* q_pin = nullptr;
  int32_t* ids_pin = nullptr;
  float* d_pin = nullptr;
  int32_t* c_pin = nullptr;
  int32_t* s_pin = nullptr;
  int64_t req = -1;
  int k = 0;
  int slot0 = 0, nslots = 0;  // the request's run of pool slots
};

}  // namespace

struct nmsg_server {
  nmsg_index* h = nullptr;
  int max_batch = 256, max_k = 100;
  int pool_slots = 0;        // search slots the memory budget holds
  int slot_cap = 0;          // most slots one request takes (its batch, rounded to whole blocks)
  std::vector<uint8_t> slot_used;  // per block of kWarpsPerBlock slots
  int64_t vpitch = 0;
  DevBuf visited, epochs;
  std::vector<Lane> lanes;
  std::mutex mu;
  std::condition_variable cv_done, cv_work;
  std::deque<int64_t> queue;
  std::unordered_map<int64_t, Request> reqs;
  int64_t next_id = 1;
  int in_flight = 0;
  bool stop = false;
  std::thread worker;
  std::string worker_error;

  ~nmsg_server() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stop = true;
    }
    cv_work.notify_all();
    if (worker.joinable()) worker.join();
    DeviceGuard g(h ? h->device : 0);
    for (Lane& l : lanes) {
      if (l.st) cudaStreamSynchronize(l.st);
      for (DevBuf* b : {&l.q, &l.ids, &l.dists, &l.counts, &l.counter, &l.status}) b->release();
      if (l.q_pin) cudaFreeHost(l.q_pin);
      if (l.ids_pin) cudaFreeHost(l.ids_pin);
      if (l.d_pin) cudaFreeHost(l.d_pin);
      if (l.c_pin) cudaFreeHost(l.c_pin);
      if (l.s_pin) cudaFreeHost(l.s_pin);
      if (l.done) cudaEventDestroy(l.done);
      if (l.st) cudaStreamDestroy(l.st);
    }
    visited.release();
    epochs.release();
  }

  // Launch request r on lane li (worker thread, mu held).
  int launch(int li, Request& r) {
    Lane& l = lanes[li];
    const DevIndex& d = h->dev;
    const int dim = d.dim;
    std::memcpy(l.q_pin, r.q.data(), (size_t)r.nq * dim * 4);
    cudaError_t e = cudaMemcpyAsync(l.q.p, l.q_pin, (size_t)r.nq * dim * 4, cudaMemcpyHostToDevice, l.st);
    if (e == cudaSuccess) e = cudaMemsetAsync(l.counter.p, 0, 4, l.st);
    if (e == cudaSuccess) e = cudaMemsetAsync(l.status.p, 0, 4, l.st);
    if (e != cudaSuccess) return NMSG_ERR_DEVICE;
    LaunchPlan plan;
    std::string err;
    nmsg_launch_config cfg = h->cfg;
    cfg.queries_per_warp = 1;  // a lane's slots are sized for one query per warp
    int rc = plan_launch(d, cfg, std::max(r.ef, r.k), false, false, &plan, &err);
    if (rc != NMSG_OK) return rc;
    SearchArgs a;
    a.ix = d;
    a.queries = l.q.as<float>();
    a.nq = r.nq;
    a.k_default = r.k;
    a.ef_default = r.ef;
    a.algo = NMSG_ALGO_V1MERGE;
    a.kmax = r.k;
    a.ids = l.ids.as<int32_t>();
    a.dists = l.dists.as<float>();
    a.counts = l.counts.as<int32_t>();
    a.visited = visited.as<uint8_t>() + (int64_t)l.slot0 * vpitch;
    a.visited_pitch = vpitch;
    a.epochs = epochs.as<uint8_t>() + l.slot0;
    a.work_counter = l.counter.as<int32_t>();
    a.status = l.status.as<int32_t>();
    a.region_items = plan.region;
    a.nbpad = plan.nbpad;
    a.hash_log2 = plan.hash_log2;
    a.stage_rows = plan.stage_rows;
    a.warp_smem = plan.warp_smem;
    a.lean = plan.lean ? 1 : 0;
    a.bulk_rows = plan.bulk_rows ? 1 : 0;
    const int wpb = plan.wpb;  // <= kWarpsPerBlock: the run holds whole blocks
    const int blocks = std::max(1, l.nslots / wpb);
    a.num_slots = blocks * wpb;
    rc = launch_search(a, false, plan.gather, false, blocks, wpb, l.st);
    if (rc != 0) return NMSG_ERR_DEVICE;
    const size_t ob = (size_t)r.nq * r.k * 4;
    e = cudaMemcpyAsync(l.ids_pin, a.ids, ob, cudaMemcpyDeviceToHost, l.st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(l.d_pin, a.dists, ob, cudaMemcpyDeviceToHost, l.st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(l.c_pin, a.counts, (size_t)r.nq * 4, cudaMemcpyDeviceToHost, l.st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(l.s_pin, a.status, 4, cudaMemcpyDeviceToHost, l.st);
    if (e == cudaSuccess) e = cudaEventRecord(l.done, l.st);
    if (e != cudaSuccess) return NMSG_ERR_DEVICE;
    l.req = r.id;
    l.k = r.k;
    return NMSG_OK;
  }

  // First run of `n` free slot blocks (mu held); its first block, or -1.
  int take_blocks(int n) {
    int run = 0;
    for (int b = 0; b < (int)slot_used.size(); ++b) {
      run = slot_used[b] ? 0 : run + 1;
      if (run == n) {
        for (int t = b - n + 1; t <= b; ++t) slot_used[t] = 1;
        return b - n + 1;
      }
    }
    return -1;
  }
  void give_blocks(int b0, int n) {
    for (int t = b0; t < b0 + n; ++t) slot_used[t] = 0;
  }

  void run() {
    cudaSetDevice(h->device);
    std::unique_lock<std::mutex> lk(mu);
    while (true) {
      bool progressed = false;
      // harvest finished lanes
      for (size_t li = 0; li < lanes.size(); ++li) {
        Lane& l = lanes[li];
        if (l.req < 0) continue;
        const cudaError_t q = cudaEventQuery(l.done);
        if (q == cudaErrorNotReady) continue;
        Request& r = reqs[l.req];
        r.t_done = now_s();
        r.status = (q == cudaSuccess) ? (*l.s_pin ? *l.s_pin : NMSG_OK) : NMSG_ERR_DEVICE;
        r.ids.assign(l.ids_pin, l.ids_pin + (size_t)r.nq * r.k);
        r.dists.assign(l.d_pin, l.d_pin + (size_t)r.nq * r.k);
        r.counts.assign(l.c_pin, l.c_pin + r.nq);
        r.q.clear();
        r.q.shrink_to_fit();
        r.done = true;
        l.req = -1;
        give_blocks(l.slot0 / kWarpsPerBlock, l.nslots / kWarpsPerBlock);
        --in_flight;
        progressed = true;
      }
      if (progressed) cv_done.notify_all();
      // admit waiting requests, oldest first, while a lane and a run of slots are free
      while (!queue.empty()) {
        int li = -1;
        for (size_t t = 0; t < lanes.size(); ++t)
          if (lanes[t].req < 0) {
            li = (int)t;
            break;
          }
        if (li < 0) break;
        Request& r = reqs[queue.front()];
        const int need_blocks = (std::min(r.nq, slot_cap) + kWarpsPerBlock - 1) / kWarpsPerBlock;
        const int b0 = take_blocks(need_blocks);
        if (b0 < 0) break;  // the oldest request waits for memory
        queue.pop_front();
        Lane& l = lanes[li];
        l.slot0 = b0 * kWarpsPerBlock;
        l.nslots = need_blocks * kWarpsPerBlock;
        ++in_flight;
        const int rc = launch(li, r);
        if (rc != NMSG_OK) {
          r.status = rc;
          r.done = true;
          r.t_done = now_s();
          --in_flight;
          l.req = -1;
          give_blocks(l.slot0 / kWarpsPerBlock, l.nslots / kWarpsPerBlock);
          cv_done.notify_all();
        }
        progressed = true;
      }
      if (stop && in_flight == 0) break;
      if (!progressed) {
        if (in_flight == 0 && queue.empty()) {
          cv_work.wait_for(lk, std::chrono::milliseconds(50));
        } else {
          // work on the device: poll again shortly without holding the lock (polling at once,
          // with a yield only, measured far worse: the worker took the lock back before the
          // threads submitting requests could, p50 1.74 -> 5.1 ms at 500K q/s offered)
          lk.unlock();
          std::this_thread::sleep_for(std::chrono::microseconds(5));
          lk.lock();
        }
      }
    }
  }
};

namespace {
int srv_fail(int code, const std::string& msg) {
  set_last_error(msg);
  return code;
}
}  // namespace

extern "C" {

NMSG_API int nmsg_server_create(nmsg_index* h, int64_t memory_budget_bytes, int32_t max_batch, int32_t max_k,
                                int32_t max_lanes, nmsg_server** out) {
  if (!h || !out) return srv_fail(NMSG_ERR_BAD_ARG, "null argument");
  if (max_batch < 1 || max_k < 1 || max_lanes < 1) return srv_fail(NMSG_ERR_BAD_ARG, "max_batch, max_k, max_lanes >= 1");
  *out = nullptr;
  const DevIndex& d = h->dev;
  if (d.n == 0) return srv_fail(NMSG_ERR_BAD_ARG, "the index is empty");
  if (h->host.sift) return srv_fail(NMSG_ERR_UNSUPPORTED, "serving l2sqr_sift indices is not supported");
  auto* s = new nmsg_server();
  s->h = h;
  s->max_batch = max_batch;
  s->max_k = max_k;
  s->vpitch = ((d.n + 15) / 16) * 16;
  // a request takes one slot per query up to its batch, in whole blocks; the lanes' staging comes
  // off the budget first, the slots share the rest
  s->slot_cap = ((max_batch + kWarpsPerBlock - 1) / kWarpsPerBlock) * kWarpsPerBlock;
  const int64_t per_lane = (int64_t)max_batch * (d.dim * 4 + max_k * 8 + 8);
  const int nlanes = max_lanes;
  const int64_t slot_bytes = memory_budget_bytes - (int64_t)nlanes * per_lane;
  const int64_t slots = slot_bytes > 0 ? slot_bytes / (s->vpitch + 1) : 0;
  s->pool_slots = (int)std::min<int64_t>(slots / kWarpsPerBlock * kWarpsPerBlock, 1 << 20);
  if (s->pool_slots < kWarpsPerBlock) {
    delete s;
    return srv_fail(NMSG_ERR_OOM, "the memory budget does not hold the lanes and one block of search slots (" +
                                      std::to_string((int64_t)nlanes * per_lane + kWarpsPerBlock * (s->vpitch + 1)) +
                                      " bytes)");
  }
  s->slot_cap = std::min(s->slot_cap, s->pool_slots);
  s->slot_used.assign(s->pool_slots / kWarpsPerBlock, 0);
  DeviceGuard g(h->device);
  int rc = NMSG_OK;
  if (s->visited.ensure((size_t)s->pool_slots * s->vpitch, true) != cudaSuccess ||
      s->epochs.ensure((size_t)s->pool_slots, true) != cudaSuccess)
    rc = NMSG_ERR_OOM;
  s->lanes.resize(nlanes);
  for (Lane& l : s->lanes) {
    if (rc != NMSG_OK) break;
    bool ok = cudaStreamCreateWithFlags(&l.st, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming) == cudaSuccess &&
              l.q.ensure((size_t)max_batch * d.dim * 4, false) == cudaSuccess &&
              l.ids.ensure((size_t)max_batch * max_k * 4, false) == cudaSuccess &&
              l.dists.ensure((size_t)max_batch * max_k * 4, false) == cudaSuccess &&
              l.counts.ensure((size_t)max_batch * 4, false) == cudaSuccess &&
              l.counter.ensure(4, true) == cudaSuccess && l.status.ensure(4, true) == cudaSuccess &&
              cudaMallocHost(&l.q_pin, (size_t)max_batch * d.dim * 4) == cudaSuccess &&
              cudaMallocHost(&l.ids_pin, (size_t)max_batch * max_k * 4) == cudaSuccess &&
              cudaMallocHost(&l.d_pin, (size_t)max_batch * max_k * 4) == cudaSuccess &&
              cudaMallocHost(&l.c_pin, (size_t)max_batch * 4) == cudaSuccess &&
              cudaMallocHost(&l.s_pin, 4) == cudaSuccess;
    if (!ok) rc = NMSG_ERR_OOM;
  }
  if (rc != NMSG_OK) {
    delete s;
    return srv_fail(rc, "allocating the server's lanes failed");
  }
  s->worker = std::thread([s]() { s->run(); });
  *out = s;
  return NMSG_OK;
}

NMSG_API int nmsg_server_lanes(const nmsg_server* s) { return s ? (int)s->lanes.size() : 0; }

NMSG_API int nmsg_server_submit(nmsg_server* s, const float* queries, int32_t nq, int32_t k, int32_t ef,
                                int64_t* request_id) {
  if (!s || !queries || !request_id) return srv_fail(NMSG_ERR_BAD_ARG, "null argument");
  if (nq < 1 || nq > s->max_batch) return srv_fail(NMSG_ERR_BAD_ARG, "batch size must be 1..max_batch");
  if (k < 1 || k > s->max_k) return srv_fail(NMSG_ERR_BAD_ARG, "k must be 1..max_k");
  if (ef < 0 || ef >= 1000)
    return srv_fail(NMSG_ERR_UNSUPPORTED, "the server runs V1Merge searches (efSearch < 1000)");
  const double t = now_s();
  std::lock_guard<std::mutex> lk(s->mu);
  Request r;
  r.id = s->next_id++;
  r.q.assign(queries, queries + (size_t)nq * s->h->dev.dim);
  r.nq = nq;
  r.k = k;
  r.ef = ef;
  r.t_arrival = t;
  *request_id = r.id;
  s->queue.push_back(r.id);
  s->reqs.emplace(r.id, std::move(r));
  s->cv_work.notify_one();
  return NMSG_OK;
}

// Blocks until the request finished; copies its results (row stride k) and removes it.
NMSG_API int nmsg_server_wait(nmsg_server* s, int64_t request_id, int32_t* ids, float* dists, int32_t* counts,
                              double* latency_s) {
  if (!s) return srv_fail(NMSG_ERR_BAD_ARG, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(request_id);
  if (it == s->reqs.end()) return srv_fail(NMSG_ERR_BAD_ARG, "unknown request id");
  s->cv_done.wait(lk, [&]() { return it->second.done; });
  Request& r = it->second;
  const int status = r.status;
  if (status == NMSG_OK) {
    if (ids) std::memcpy(ids, r.ids.data(), r.ids.size() * 4);
    if (dists) std::memcpy(dists, r.dists.data(), r.dists.size() * 4);
    if (counts) std::memcpy(counts, r.counts.data(), r.counts.size() * 4);
  }
  if (latency_s) *latency_s = r.t_done - r.t_arrival;
  s->reqs.erase(it);
  if (status != NMSG_OK) return srv_fail(status, "the request failed on the device");
  return NMSG_OK;
}

// Open-loop replay: request i arrives at arrival_s[i] seconds after the start (its queries are
// queries[q_offset[i] * dim ...], nq[i] rows), is submitted at that time whatever the server is
// doing, and its latency (completion minus arrival) goes to latency_s[i]. *wall_s gets the time
// from the first arrival to the last completion.
NMSG_API int nmsg_server_run_trace(nmsg_server* s, const float* queries, const int64_t* q_offset, const int32_t* nq,
                                   const int32_t* k, const int32_t* ef, const double* arrival_s, int64_t nreq,
                                   double* latency_s, double* wall_s) {
  if (!s || !queries || !q_offset || !nq || !k || !ef || !arrival_s || !latency_s)
    return srv_fail(NMSG_ERR_BAD_ARG, "null argument");
  const int dim = s->h->dev.dim;
  std::vector<int64_t> ids(nreq);
  const double t0 = now_s();
  for (int64_t i = 0; i < nreq; ++i) {
    const double due = t0 + arrival_s[i];
    while (now_s() < due) {
      const double left = due - now_s();
      if (left > 200e-6) std::this_thread::sleep_for(std::chrono::duration<double>(left - 100e-6));
    }
    const int rc = nmsg_server_submit(s, queries + q_offset[i] * dim, nq[i], k[i], ef[i], &ids[i]);
    if (rc != NMSG_OK) return rc;
    std::lock_guard<std::mutex> lk(s->mu);
    s->reqs[ids[i]].t_arrival = due;  // latency from the scheduled arrival
  }
  double last = t0;
  for (int64_t i = 0; i < nreq; ++i) {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ids[i]);
    s->cv_done.wait(lk, [&]() { return it->second.done; });
    latency_s[i] = it->second.t_done - it->second.t_arrival;
    last = std::max(last, it->second.t_done);
    const int st = it->second.status;
    s->reqs.erase(it);
    if (st != NMSG_OK) return srv_fail(st, "a request failed on the device");
  }
  if (wall_s) *wall_s = last - t0;
  return NMSG_OK;
}

NMSG_API void nmsg_server_free(nmsg_server* s) { delete s; }

}  // extern "C"
