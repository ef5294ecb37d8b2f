// Host-side HNSW index builder: writes NMSLIB's optimized index file so that large workloads can
// be indexed without the reference library. It follows the reference's construction algorithm
// (similarity_search/src/method/hnsw.cc:183-470 CreateIndex, :534-609 add, :611-708
// kSearchElementsWithAttemptsLevel; similarity_search/include/method/hnsw.h:129-169
// getNeighborsByHeuristic2 and :258-314 addFriendlevel/link) with the same defaults
// (maxM = M, maxM0 = 2M, mult = 1/ln M, delaunay_type 2, post 0) and the same packed layout
// (hnsw.cc:353-465). Like the reference's multi-threaded build, the graph depends on thread
// timing; node levels are a deterministic function of (seed, node).
//
// Construction distances are squared L2, 1 - dot on unit vectors (cosine) and -dot; the search
// path never uses them, so they need not follow the reference's FMA lane order.
#include <immintrin.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>
#include <queue>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "engine.h"
#include "handle.h"
#include "../../include/nmslib_b200.h"

namespace nmsg {
namespace {

thread_local std::string g_build_err;

__attribute__((target("avx2,fma"))) float dot_avx2(const float* a, const float* b, int d) {
  __m256 s0 = _mm256_setzero_ps(), s1 = _mm256_setzero_ps();
  int e = 0;
  for (; e + 16 <= d; e += 16) {
    s0 = _mm256_fmadd_ps(_mm256_loadu_ps(a + e), _mm256_loadu_ps(b + e), s0);
    s1 = _mm256_fmadd_ps(_mm256_loadu_ps(a + e + 8), _mm256_loadu_ps(b + e + 8), s1);
  }
  for (; e + 8 <= d; e += 8) s0 = _mm256_fmadd_ps(_mm256_loadu_ps(a + e), _mm256_loadu_ps(b + e), s0);
  s0 = _mm256_add_ps(s0, s1);
  alignas(32) float t[8];
  _mm256_store_ps(t, s0);
  float s = ((t[0] + t[1]) + (t[2] + t[3])) + ((t[4] + t[5]) + (t[6] + t[7]));
  for (; e < d; ++e) s += a[e] * b[e];
  return s;
}

__attribute__((target("avx2,fma"))) float l2_avx2(const float* a, const float* b, int d) {
  __m256 s0 = _mm256_setzero_ps(), s1 = _mm256_setzero_ps();
  int e = 0;
  for (; e + 16 <= d; e += 16) {
    __m256 x = _mm256_sub_ps(_mm256_loadu_ps(a + e), _mm256_loadu_ps(b + e));
    __m256 y = _mm256_sub_ps(_mm256_loadu_ps(a + e + 8), _mm256_loadu_ps(b + e + 8));
    s0 = _mm256_fmadd_ps(x, x, s0);
    s1 = _mm256_fmadd_ps(y, y, s1);
  }
  for (; e + 8 <= d; e += 8) {
    __m256 x = _mm256_sub_ps(_mm256_loadu_ps(a + e), _mm256_loadu_ps(b + e));
    s0 = _mm256_fmadd_ps(x, x, s0);
  }
  s0 = _mm256_add_ps(s0, s1);
  alignas(32) float t[8];
  _mm256_store_ps(t, s0);
  float s = ((t[0] + t[1]) + (t[2] + t[3])) + ((t[4] + t[5]) + (t[6] + t[7]));
  for (; e < d; ++e) {
    const float x = a[e] - b[e];
    s += x * x;
  }
  return s;
}

struct SpinLock {
  std::atomic<uint8_t> f{0};
  void lock() {
    while (f.exchange(1, std::memory_order_acquire)) {
      while (f.load(std::memory_order_relaxed)) _mm_pause();
    }
  }
  void unlock() { f.store(0, std::memory_order_release); }
};

struct Builder {
  const float* data = nullptr;  // n x dim (normalised copy for cosine)
  std::vector<float> normed;
  int64_t n = 0;
  int dim = 0, space = 0, M = 16, maxM = 16, maxM0 = 32, efc = 200;
  double mult = 0;
  uint64_t seed = 0;
  std::vector<int32_t> level;
  int l0_stride = 40;                      // round_up(maxM0 + 1, 8): the device's level-0 pitch
  std::vector<int32_t> l0;                 // n x l0_stride: cnt, ids
  std::vector<std::vector<int32_t>> up;    // per node: level x (maxM + 1)
  std::unique_ptr<SpinLock[]> locks;
  std::atomic<int32_t> enterpoint{0};
  std::atomic<int32_t> maxlevel{0};
  std::mutex maxlevel_guard;

  float dist(int64_t a, int64_t b) const { return dist_vec(data + a * dim, b); }
  float dist_vec(const float* q, int64_t b) const {
    const float* v = data + b * dim;
    if (space == NMSG_SPACE_L2) return l2_avx2(q, v, dim);
    const float d = dot_avx2(q, v, dim);
    return space == NMSG_SPACE_COSINE ? 1.0f - d : -d;
  }
  int32_t* list(int64_t node, int lev) {
    return lev == 0 ? l0.data() + node * l0_stride : up[node].data() + (maxM + 1) * (lev - 1);
  }
  int cap(int lev) const { return lev == 0 ? maxM0 : maxM; }

  int random_level(int64_t node) const {
    // splitmix64 of (seed, node) -> uniform in (0, 1]; level = floor(-ln(u) * mult)  (hnsw.h:478-483)
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (uint64_t)(node + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const double u = ((z >> 11) + 1) * (1.0 / 9007199254740992.0);
    return (int)(-std::log(u) * mult);
  }

  // getNeighborsByHeuristic2 (hnsw.h:129-169): candidates sorted ascending by distance to the
  // base point; keep a candidate unless a kept one is strictly closer to it than the base is.
  void heuristic(std::vector<std::pair<float, int32_t>>& cand, int nn) const {
    if ((int)cand.size() < nn) return;
    std::sort(cand.begin(), cand.end());
    std::vector<std::pair<float, int32_t>> keep;
    for (const auto& c : cand) {
      if ((int)keep.size() >= nn) break;
      bool good = true;
      for (const auto& k : keep) {
        if (dist(k.second, c.second) < c.first) {
          good = false;
          break;
        }
      }
      if (good) keep.push_back(c);
    }
    cand.swap(keep);
  }

  // addFriendlevel (hnsw.h:258-314): append; on overflow shrink with the heuristic to at most
  // size-1 and store the survivors farthest first, as the reference's max-heap pop order does.
  void add_friend(int64_t node, int lev, int32_t other) {
    std::lock_guard<SpinLock> g(locks[node]);
    int32_t* lst = list(node, lev);
    for (int j = 1; j <= lst[0]; ++j)
      if (lst[j] == other) return;
    if (lst[0] < cap(lev)) {
      lst[++lst[0]] = other;
      return;
    }
    std::vector<std::pair<float, int32_t>> c;
    c.reserve(lst[0] + 1);
    for (int j = 1; j <= lst[0]; ++j) c.push_back({dist(node, lst[j]), lst[j]});
    c.push_back({dist(node, other), other});
    heuristic(c, (int)c.size() - 1);
    std::sort(c.begin(), c.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    lst[0] = (int32_t)c.size();
    for (size_t j = 0; j < c.size(); ++j) lst[1 + j] = c[j].second;
  }

  // kSearchElementsWithAttemptsLevel (hnsw.cc:611-708)
  void search_layer(const float* q, int32_t ep, int lev, std::vector<uint32_t>& vis, uint32_t& epoch,
                    std::vector<std::pair<float, int32_t>>& out) {
    if (++epoch == 0) {
      std::fill(vis.begin(), vis.end(), 0);
      epoch = 1;
    }
    std::priority_queue<std::pair<float, int32_t>> result;                         // max-heap
    std::priority_queue<std::pair<float, int32_t>, std::vector<std::pair<float, int32_t>>,
                        std::greater<std::pair<float, int32_t>>> cand;             // min-heap
    const float d0 = dist_vec(q, ep);
    result.push({d0, ep});
    cand.push({d0, ep});
    vis[ep] = epoch;
    std::vector<int32_t> nb;
    while (!cand.empty()) {
      const auto cur = cand.top();
      if (cur.first > result.top().first) break;
      cand.pop();
      {
        std::lock_guard<SpinLock> g(locks[cur.second]);
        const int32_t* lst = list(cur.second, lev);
        nb.assign(lst + 1, lst + 1 + lst[0]);
      }
      for (int32_t id : nb) {
        if (vis[id] == epoch) continue;
        vis[id] = epoch;
        const float d = dist_vec(q, id);
        if ((int)result.size() < efc || result.top().first > d) {
          result.push({d, id});
          cand.push({d, id});
          if ((int)result.size() > efc) result.pop();
        }
      }
    }
    out.clear();
    while (!result.empty()) {
      out.push_back(result.top());
      result.pop();
    }
  }

  // add (hnsw.cc:534-609)
  void add(int64_t node, std::vector<uint32_t>& vis, uint32_t& epoch) {
    const int cur_level = level[node];
    std::unique_lock<std::mutex> top_lock;
    if (cur_level > maxlevel.load()) top_lock = std::unique_lock<std::mutex>(maxlevel_guard);
    const int maxl = maxlevel.load();
    int32_t ep = enterpoint.load();
    const float* q = data + node * dim;
    if (cur_level < maxl) {
      float curdist = dist_vec(q, ep);
      for (int lev = maxl; lev > cur_level; --lev) {
        bool changed = true;
        while (changed) {
          changed = false;
          std::vector<int32_t> nb;
          {
            std::lock_guard<SpinLock> g(locks[ep]);
            const int32_t* lst = list(ep, lev);
            nb.assign(lst + 1, lst + 1 + lst[0]);
          }
          for (int32_t id : nb) {
            const float d = dist_vec(q, id);
            if (d < curdist) {
              curdist = d;
              ep = id;
              changed = true;
            }
          }
        }
      }
    }
    std::vector<std::pair<float, int32_t>> res;
    for (int lev = std::min(cur_level, maxl); lev >= 0; --lev) {
      search_layer(q, ep, lev, vis, epoch, res);
      heuristic(res, M);
      // link farthest first; the closest becomes the entry for the next level
      std::sort(res.begin(), res.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
      for (const auto& r : res) {
        add_friend(r.second, lev, (int32_t)node);
        add_friend(node, lev, r.second);
      }
      if (!res.empty()) ep = res.back().second;
    }
    if (cur_level > maxlevel.load()) {
      enterpoint.store((int32_t)node);
      maxlevel.store(cur_level);
    }
  }
};

}  // namespace
}  // namespace nmsg

using namespace nmsg;

namespace nmsg {
namespace {

int check_build_args(const float* data, int64_t n, int32_t dim, int space, int M, int ef_construction,
                     const char* out_path) {
  if (space == NMSG_SPACE_L1 || space == NMSG_SPACE_LINF) {
    g_build_err = "the host builder supports l2, cosinesimil and negdotprod; build l1 / linf indices with the reference";
    return NMSG_ERR_UNSUPPORTED;
  }
  if (!data || n < 0 || dim <= 0 || !out_path || M < 2 || ef_construction < 1 || space < 0 || space > 2) {
    g_build_err = "invalid build arguments";
    return NMSG_ERR_BAD_ARG;
  }
  if (n > 0x7fffffffLL) {
    g_build_err = "too many elements for int32 ids";
    return NMSG_ERR_BAD_ARG;
  }
  return NMSG_OK;
}

// Parameters, levels, empty lists and (cosine) the unit-vector copy, as CreateIndex sets them up.
void setup_builder(Builder& b, const float* data, int64_t n, int32_t dim, int space, int M, int ef_construction,
                   uint64_t seed) {
  b.n = n;
  b.dim = dim;
  b.space = space;
  b.M = M;
  b.maxM = M;
  b.maxM0 = 2 * M;
  b.l0_stride = (b.maxM0 + 1 + 7) & ~7;
  b.efc = ef_construction;
  b.mult = 1.0 / std::log(1.0 * M);
  b.seed = seed;
  b.data = data;
  if (space == NMSG_SPACE_COSINE) {
    // the reference stores unit vectors for cosine (hnsw.cc:441-446, NormalizeVect hnsw.h:486-497)
    b.normed.assign(data, data + n * dim);
    for (int64_t i = 0; i < n; ++i) {
      float* v = b.normed.data() + i * dim;
      float sum = 0;
      for (int e = 0; e < dim; ++e) {
        volatile float sq = v[e] * v[e];  // unfused, as the reference computes it
        sum = sum + sq;
      }
      if (sum != 0.0f) {
        const float s = 1.0f / std::sqrt(sum);
        for (int e = 0; e < dim; ++e) v[e] *= s;
      }
    }
    b.data = b.normed.data();
  }
  b.level.resize(n);
  b.up.resize(n);
  for (int64_t i = 0; i < n; ++i) {
    b.level[i] = b.random_level(i);
    if (b.level[i] > 0) b.up[i].assign((size_t)b.level[i] * (b.maxM + 1), 0);
  }
  b.l0.assign((size_t)n * b.l0_stride, 0);
  b.locks.reset(new SpinLock[n]);
  b.enterpoint = 0;
  b.maxlevel = b.level[0];
}

// Inserts nodes[0..count) (all levels) with `nthreads` host threads, in list order.
void insert_on_host(Builder& b, const int32_t* nodes, int64_t count, int nthreads) {
  std::atomic<int64_t> next(0);
  auto worker = [&]() {
    std::vector<uint32_t> vis(b.n, 0);
    uint32_t epoch = 0;
    for (;;) {
      const int64_t i = next.fetch_add(1);
      if (i >= count) break;
      b.add(nodes[i], vis, epoch);
    }
  };
  std::vector<std::thread> th;
  for (int t = 0; t < nthreads; ++t) th.emplace_back(worker);
  for (auto& t : th) t.join();
}

// The optimized layout (hnsw.cc:353-465), written to out_path.
int pack_and_write(const Builder& b, const int32_t* ids, const char* out_path) {
  HostIndex out;
  std::string err;
  const int64_t n = b.n;
  const int dim = b.dim, space = b.space;
  out.n = (uint32_t)n;
  out.dim = dim;
  out.maxM = (uint64_t)b.maxM;
  out.maxM0 = (uint64_t)b.maxM0;
  out.off_data = 0;
  out.off_level0 = 16 + 4ull * dim;
  out.mem_per_obj = out.off_level0 + 4ull * (b.maxM0 + 1);
  out.maxlevel = b.maxlevel.load();
  out.enterpoint = (uint32_t)b.enterpoint.load();
  out.dist_type = space == NMSG_SPACE_L2 ? (dim % 16 == 0 ? kL2Sqr16Ext : kL2SqrExt)
                                         : (space == NMSG_SPACE_COSINE ? kNormCosine : kNegDot);
  out.search_method = 3;
  out.level0.assign(n * out.mem_per_obj, 1);  // padding bytes are 0x01, as memset(..., 1) leaves them
  out.link_bytes.assign(n, 0);
  out.up_off.assign(n, -1);
  out.level = b.level;
  for (int64_t i = 0; i < n; ++i) {
    char* row = out.level0.data() + i * out.mem_per_obj;
    const int32_t ext = ids ? ids[i] : (int32_t)i;
    const int32_t label = -1;
    const uint64_t dl = 4ull * dim;
    std::memcpy(row, &ext, 4);
    std::memcpy(row + 4, &label, 4);
    std::memcpy(row + 8, &dl, 8);
    std::memcpy(row + 16, b.data + i * dim, 4ull * dim);
    const int32_t* lst = b.l0.data() + i * b.l0_stride;
    std::memcpy(row + out.off_level0, lst, 4ull * (1 + lst[0]));
    if (b.level[i] > 0) {
      out.up_off[i] = (int64_t)out.up_links.size();
      out.link_bytes[i] = (uint32_t)(b.up[i].size() * 4);
      out.up_links.insert(out.up_links.end(), b.up[i].begin(), b.up[i].end());
    }
  }
  int rc = write_index_file(out_path, out, err);
  if (rc) g_build_err = err;
  return rc;
}

#define BUILD_CUDA(call, what)                                                                    \
  do {                                                                                            \
    const cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) {                                                                      \
      g_build_err = std::string(what) + ": " + cudaGetErrorString(e_);                            \
      return e_ == cudaErrorMemoryAllocation ? NMSG_ERR_OOM : NMSG_ERR_DEVICE;                    \
    }                                                                                             \
  } while (0)

// Level-0 insertion of nodes[0..count) (level-0-only nodes) in batches. Each batch's
// efConstruction-wide searches run on the device with the engine's search kernel (greedy descent
// through the finished upper levels, then the level-0 beam with ef = efConstruction, k =
// efConstruction) over the graph as it stands before the batch; then each node's neighbours are
// kept with heuristic 2 and the reverse links added as `add` does (hnsw.cc:576-600,
// hnsw.h:258-314) — on the device (build_gpu.cu, the level-0 graph stays there for the whole
// phase) for l2 and cosine with maxM0 <= 64, else on the host with the lists uploaded again per
// batch. Nodes of one batch do not see one
// another while they search (they are linked afterwards); a batch is an eighth of the graph so far.
int insert_level0_on_device(Builder& b, const int32_t* nodes, int64_t count, int device, int nthreads) {
  if (count == 0) return NMSG_OK;
  DeviceGuard guard(device);
  int sms = 0;
  BUILD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "device query");
  const int64_t n = b.n;
  const int dim = b.dim;
  DevIndex d;
  d.n = n;
  d.dim = dim;
  d.pitch = (dim + 31) & ~31;
  d.n16 = dim & ~15;
  d.n4 = dim & ~3;
  d.row_bytes = 4 * dim;
  d.maxM = b.maxM;
  d.maxM0 = b.maxM0;
  d.l0_pitch = b.l0_stride;
  d.maxlevel = b.maxlevel.load();
  d.enterpoint = b.enterpoint.load();
  d.dist_type = b.space == NMSG_SPACE_L2 ? (dim % 16 == 0 ? kL2Sqr16Ext : kL2SqrExt)
                                         : (b.space == NMSG_SPACE_COSINE ? kNormCosine : kNegDot);
  // vectors in the search kernels' permuted layout, upper levels as CSR, identity ids (the kernel
  // then reports internal node numbers)
  std::vector<float> vec((size_t)n * d.pitch, 0.0f);
  std::vector<int64_t> up_off(n, -1);
  std::vector<int32_t> up_links;
  std::vector<int32_t> ident(n);
  for (int64_t i = 0; i < n; ++i) {
    const float* src = b.data + i * dim;
    float* dst = vec.data() + i * d.pitch;
    for (int e = 0; e < dim; ++e) dst[permuted_pos(e, dim)] = src[e];
    if (b.level[i] > 0) {
      up_off[i] = (int64_t)up_links.size();
      up_links.insert(up_links.end(), b.up[i].begin(), b.up[i].end());
    }
    ident[i] = (int32_t)i;
  }
  if (up_links.empty()) up_links.push_back(0);
  DevBuf g_vec, g_l0, g_off, g_links, g_ext, g_q, g_ids, g_d, g_cnt, g_vis, g_ep, g_counter, g_status, g_nodes, g_pend,
      g_pend_cnt, g_touched, g_ntouched;
  struct Release {
    std::vector<DevBuf*> bufs;
    ~Release() {
      for (DevBuf* p : bufs) p->release();
    }
  } release{{&g_vec, &g_l0, &g_off, &g_links, &g_ext, &g_q, &g_ids, &g_d, &g_cnt, &g_vis, &g_ep, &g_counter, &g_status,
             &g_nodes, &g_pend, &g_pend_cnt, &g_touched, &g_ntouched}};
  // neighbour selection and links run on the device too when the lists fit its kernels, except
  // for negative dot product: there a few high-norm nodes are the nearest neighbours of nearly
  // every node and receive thousands of links per batch, more than the device's per-neighbour
  // queue keeps (the host path weighs each of them; measured recall@10 0.908 instead of 0.941)
  const bool link_on_device = b.maxM0 <= 64 && b.space != NMSG_SPACE_NEGDOT;
  BUILD_CUDA(g_vec.ensure(vec.size() * 4, false), "cudaMalloc(vectors)");
  BUILD_CUDA(g_l0.ensure(b.l0.size() * 4, false), "cudaMalloc(level-0 lists)");
  BUILD_CUDA(g_off.ensure(n * 8, false), "cudaMalloc(upper offsets)");
  BUILD_CUDA(g_links.ensure(up_links.size() * 4, false), "cudaMalloc(upper lists)");
  BUILD_CUDA(g_ext.ensure(n * 4, false), "cudaMalloc(ids)");
  BUILD_CUDA(cudaMemcpy(g_vec.p, vec.data(), vec.size() * 4, cudaMemcpyHostToDevice), "upload vectors");
  BUILD_CUDA(cudaMemcpy(g_off.p, up_off.data(), n * 8, cudaMemcpyHostToDevice), "upload offsets");
  BUILD_CUDA(cudaMemcpy(g_links.p, up_links.data(), up_links.size() * 4, cudaMemcpyHostToDevice), "upload links");
  BUILD_CUDA(cudaMemcpy(g_ext.p, ident.data(), n * 4, cudaMemcpyHostToDevice), "upload ids");
  vec.clear();
  vec.shrink_to_fit();
  d.vecs = g_vec.as<float>();
  d.l0 = g_l0.as<int32_t>();
  d.up_off = g_off.as<int64_t>();
  d.up_links = g_links.as<int32_t>();
  d.ext_id = g_ext.as<int32_t>();

  const int efc = b.efc;
  LaunchPlan plan;
  std::string perr;
  const nmsg_launch_config cfg{0, 0, 0, 0, 0, 1, 0, -1, 0};  // one construction search per warp, one pass
  int rc = plan_launch(d, cfg, efc, false, false, &plan, &perr);
  if (rc != NMSG_OK) {
    g_build_err = "device build: " + perr;
    return rc;
  }
  const int blocks = plan.blocks_per_sm * sms;
  const int slots = blocks * plan.wpb;
  const int64_t vpitch = ((n + 15) / 16) * 16;
  const int64_t max_batch = 65536;
  BUILD_CUDA(g_vis.ensure((size_t)slots * vpitch, true), "cudaMalloc(visited sets)");
  BUILD_CUDA(g_ep.ensure(slots, true), "cudaMalloc(epochs)");
  BUILD_CUDA(g_counter.ensure(4, true), "cudaMalloc(counter)");
  BUILD_CUDA(g_status.ensure(4, true), "cudaMalloc(status)");
  BUILD_CUDA(g_q.ensure((size_t)max_batch * dim * 4, false), "cudaMalloc(queries)");
  BUILD_CUDA(g_ids.ensure((size_t)max_batch * efc * 4, false), "cudaMalloc(results)");
  BUILD_CUDA(g_d.ensure((size_t)max_batch * efc * 4, false), "cudaMalloc(results)");
  BUILD_CUDA(g_cnt.ensure((size_t)max_batch * 4, false), "cudaMalloc(results)");
  if (link_on_device) {
    BUILD_CUDA(g_nodes.ensure((size_t)max_batch * 4, false), "cudaMalloc(batch)");
    BUILD_CUDA(g_pend.ensure((size_t)n * 32 * 4, false), "cudaMalloc(queued links)");
    BUILD_CUDA(g_pend_cnt.ensure((size_t)n * 4, true), "cudaMalloc(queued links)");
    BUILD_CUDA(g_touched.ensure((size_t)max_batch * b.M * 4, false), "cudaMalloc(queued links)");
    BUILD_CUDA(g_ntouched.ensure(4, true), "cudaMalloc(queued links)");
    BUILD_CUDA(cudaMemcpy(g_l0.p, b.l0.data(), b.l0.size() * 4, cudaMemcpyHostToDevice), "upload lists");
  }

  SearchArgs a;
  std::memset(&a, 0, sizeof(a));
  a.ix = d;
  a.k_default = efc;
  a.ef_default = efc;
  a.algo = NMSG_ALGO_V1MERGE;
  a.kmax = efc;
  a.queries = g_q.as<float>();
  a.ids = g_ids.as<int32_t>();
  a.dists = g_d.as<float>();
  a.counts = g_cnt.as<int32_t>();
  a.visited = g_vis.as<uint8_t>();
  a.visited_pitch = vpitch;
  a.epochs = g_ep.as<uint8_t>();
  a.num_slots = slots;
  a.work_counter = g_counter.as<int32_t>();
  a.status = g_status.as<int32_t>();
  a.region_items = plan.region;
  a.nbpad = plan.nbpad;
  a.hash_log2 = plan.hash_log2;
  a.stage_rows = plan.stage_rows;
  a.warp_smem = plan.warp_smem;
  a.lean = plan.lean ? 1 : 0;
  a.bulk_rows = plan.bulk_rows ? 1 : 0;

  std::vector<float> hq((size_t)max_batch * dim);
  std::vector<int32_t> hids((size_t)max_batch * efc), hcnt(max_batch);
  std::vector<float> hd((size_t)max_batch * efc);
  int64_t inserted = n - count, done = 0;
  while (done < count) {
    const int64_t bsz = std::min<int64_t>({count - done, max_batch, std::max<int64_t>(1024, inserted / 8)});
    const int32_t* batch = nodes + done;
    for (int64_t j = 0; j < bsz; ++j) std::memcpy(hq.data() + j * dim, b.data + (int64_t)batch[j] * dim, 4ull * dim);
    if (!link_on_device)
      BUILD_CUDA(cudaMemcpy(g_l0.p, b.l0.data(), b.l0.size() * 4, cudaMemcpyHostToDevice), "upload lists");
    BUILD_CUDA(cudaMemcpy(g_q.p, hq.data(), (size_t)bsz * dim * 4, cudaMemcpyHostToDevice), "upload queries");
    a.nq = bsz;
    BUILD_CUDA(cudaMemset(g_counter.p, 0, 4), "reset counter");
    BUILD_CUDA(cudaMemset(g_status.p, 0, 4), "reset status");
    const int lrc = launch_search(a, false, plan.gather, false, blocks, plan.wpb, nullptr);
    if (lrc != 0) {
      g_build_err = std::string("device build search launch: ") + cudaGetErrorString((cudaError_t)lrc);
      return NMSG_ERR_DEVICE;
    }
    if (link_on_device) {
      BUILD_CUDA(cudaMemcpy(g_nodes.p, batch, (size_t)bsz * 4, cudaMemcpyHostToDevice), "upload batch");
      const int lrc2 = level0_select_and_link(d, b.space, b.M, efc, bsz, g_nodes.as<int32_t>(), g_ids.as<int32_t>(),
                                              g_d.as<float>(), g_cnt.as<int32_t>(), g_l0.as<int32_t>(),
                                              g_pend.as<int32_t>(), g_pend_cnt.as<int32_t>(),
                                              g_touched.as<int32_t>(), g_ntouched.as<int32_t>(), nullptr);
      if (lrc2 != 0) {
        g_build_err = std::string("device build linking: ") + cudaGetErrorString((cudaError_t)lrc2);
        return NMSG_ERR_DEVICE;
      }
      int32_t status = 0;
      BUILD_CUDA(cudaMemcpy(&status, g_status.p, 4, cudaMemcpyDeviceToHost), "copy status");
      if (status != 0) {
        g_build_err = "device build: the search kernel reported status " + std::to_string(status);
        return status;
      }
      done += bsz;
      inserted += bsz;
      continue;
    }
    BUILD_CUDA(cudaMemcpy(hids.data(), g_ids.p, (size_t)bsz * efc * 4, cudaMemcpyDeviceToHost), "copy results");
    BUILD_CUDA(cudaMemcpy(hd.data(), g_d.p, (size_t)bsz * efc * 4, cudaMemcpyDeviceToHost), "copy results");
    BUILD_CUDA(cudaMemcpy(hcnt.data(), g_cnt.p, (size_t)bsz * 4, cudaMemcpyDeviceToHost), "copy results");
    int32_t status = 0;
    BUILD_CUDA(cudaMemcpy(&status, g_status.p, 4, cudaMemcpyDeviceToHost), "copy status");
    if (status != 0) {
      g_build_err = "device build: the search kernel reported status " + std::to_string(status);
      return status;
    }
    // neighbour selection and links, as in `add` at level 0
    std::atomic<int64_t> next(0);
    auto worker = [&]() {
      std::vector<std::pair<float, int32_t>> res;
      for (;;) {
        const int64_t j = next.fetch_add(1);
        if (j >= bsz) break;
        const int32_t node = batch[j];
        res.clear();
        for (int t = 0; t < hcnt[j]; ++t) res.push_back({hd[j * efc + t], hids[j * efc + t]});
        b.heuristic(res, b.M);
        std::sort(res.begin(), res.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
        for (const auto& r : res) {
          b.add_friend(r.second, 0, node);
          b.add_friend(node, 0, r.second);
        }
      }
    };
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; ++t) th.emplace_back(worker);
    for (auto& t : th) t.join();
    done += bsz;
    inserted += bsz;
  }
  if (link_on_device)
    BUILD_CUDA(cudaMemcpy(b.l0.data(), g_l0.p, b.l0.size() * 4, cudaMemcpyDeviceToHost), "download lists");
  return NMSG_OK;
}

int write_empty(const char* out_path) {
  HostIndex out;
  std::string err;
  out.empty_regular = true;
  int rc = write_index_file(out_path, out, err);
  if (rc) g_build_err = err;
  return rc;
}

}  // namespace
}  // namespace nmsg

using namespace nmsg;

extern "C" NMSG_API int nmsg_build_index(const float* data, int64_t n, int32_t dim, const int32_t* ids,
                                         int space, int M, int ef_construction, int nthreads, uint64_t seed,
                                         const char* out_path) {
  int rc = check_build_args(data, n, dim, space, M, ef_construction, out_path);
  if (rc != NMSG_OK) return rc;
  if (n == 0) return write_empty(out_path);
  Builder b;
  setup_builder(b, data, n, dim, space, M, ef_construction, seed);
  if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  std::vector<int32_t> order(n - 1);
  for (int64_t i = 1; i < n; ++i) order[i - 1] = (int32_t)i;  // node 0 is the initial entry point
  insert_on_host(b, order.data(), n - 1, nthreads);
  return pack_and_write(b, ids, out_path);
}

extern "C" NMSG_API int nmsg_build_index_device(const float* data, int64_t n, int32_t dim, const int32_t* ids,
                                                int space, int M, int ef_construction, int nthreads, uint64_t seed,
                                                int device, const char* out_path) {
  int rc = check_build_args(data, n, dim, space, M, ef_construction, out_path);
  if (rc != NMSG_OK) return rc;
  if (n == 0) return write_empty(out_path);
  Builder b;
  setup_builder(b, data, n, dim, space, M, ef_construction, seed);
  if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  // on the host: every node with an upper level and the first nodes, in node order; the rest
  // (level 0 only) in device-searched batches
  const int64_t head = std::min<int64_t>(n, 4096);
  std::vector<int32_t> host_nodes, dev_nodes;
  for (int64_t i = 1; i < n; ++i) (i < head || b.level[i] > 0 ? host_nodes : dev_nodes).push_back((int32_t)i);
  insert_on_host(b, host_nodes.data(), (int64_t)host_nodes.size(), nthreads);
  rc = insert_level0_on_device(b, dev_nodes.data(), (int64_t)dev_nodes.size(), device, nthreads);
  if (rc != NMSG_OK) return rc;
  return pack_and_write(b, ids, out_path);
}

extern "C" NMSG_API const char* nmsg_build_last_error(void) { return g_build_err.c_str(); }
