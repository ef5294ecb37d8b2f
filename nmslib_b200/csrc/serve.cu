// Continuous-batching query server over a loaded index (the serving front of the HNSW query path).
//
// Requests (a batch of 1..max_batch queries with its own k and efSearch) are admitted into
// "lanes" as soon as one is free. A lane is a CUDA stream plus a fixed share of the search
// slots (per-warp visited-set epoch bytes) and its own staging buffers; the number of lanes is
// what the device-memory budget allows. Every admitted request is one launch of the persistent
// search kernel on its lane's stream, so requests that arrive while others run are searched
// concurrently on the device, each on its own slots; nothing a request computes depends on the
// others, so its results are the same alone and in any mix. A worker thread admits requests
// and harvests finished lanes (event query); callers submit and wait without blocking the GPU.
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
};

}  // namespace

struct nmsg_server {
  nmsg_index* h = nullptr;
  int max_batch = 256, max_k = 100;
  int lane_slots = 0;
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

  // Launch request r on lane li (worker thread, mu not held for the CUDA calls).
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
    a.visited = visited.as<uint8_t>() + (int64_t)li * lane_slots * vpitch;
    a.visited_pitch = vpitch;
    a.epochs = epochs.as<uint8_t>() + (int64_t)li * lane_slots;
    a.work_counter = l.counter.as<int32_t>();
    a.status = l.status.as<int32_t>();
    a.region_items = plan.region;
    a.nbpad = plan.nbpad;
    a.hash_log2 = plan.hash_log2;
    a.stage_rows = plan.stage_rows;
    a.warp_smem = plan.warp_smem;
    a.lean = plan.lean ? 1 : 0;
    const int wpb = plan.wpb;
    int blocks = std::min((r.nq + wpb - 1) / wpb, lane_slots / wpb);
    if (blocks < 1) blocks = 1;
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
        --in_flight;
        progressed = true;
      }
      if (progressed) cv_done.notify_all();
      // admit waiting requests into free lanes
      for (size_t li = 0; li < lanes.size() && !queue.empty(); ++li) {
        if (lanes[li].req >= 0) continue;
        Request& r = reqs[queue.front()];
        queue.pop_front();
        ++in_flight;
        const int rc = launch((int)li, r);
        if (rc != NMSG_OK) {
          r.status = rc;
          r.done = true;
          r.t_done = now_s();
          --in_flight;
          lanes[li].req = -1;
          cv_done.notify_all();
        }
        progressed = true;
      }
      if (stop && in_flight == 0) break;
      if (!progressed) {
        if (in_flight == 0 && queue.empty()) {
          cv_work.wait_for(lk, std::chrono::milliseconds(50));
        } else {
          // work on the device: poll again shortly without holding the lock
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
  // slots per lane: one warp per query of the largest batch, in whole blocks
  s->lane_slots = ((max_batch + kWarpsPerBlock - 1) / kWarpsPerBlock) * kWarpsPerBlock;
  const int64_t per_lane = (int64_t)s->lane_slots * (s->vpitch + 1) + (int64_t)max_batch * (d.dim * 4 + max_k * 8 + 8);
  int nlanes = (int)std::min<int64_t>(max_lanes, memory_budget_bytes / per_lane);
  if (nlanes < 1) {
    delete s;
    return srv_fail(NMSG_ERR_OOM, "the memory budget does not hold one lane (" + std::to_string(per_lane) + " bytes)");
  }
  DeviceGuard g(h->device);
  int rc = NMSG_OK;
  if (s->visited.ensure((size_t)nlanes * s->lane_slots * s->vpitch, true) != cudaSuccess ||
      s->epochs.ensure((size_t)nlanes * s->lane_slots, true) != cudaSuccess)
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
