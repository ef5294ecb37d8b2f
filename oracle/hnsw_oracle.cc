// ORACLE — test infrastructure only. Nothing in the product (nmslib_b200/) links, loads or
// calls this file; only tests/, the smoke check and the CPU-baseline leg of bench.py do, and
// only as a checker.
//
// A plain C++ restatement of NMSLIB's optimized-HNSW query path, written from the reference's
// behaviour (file:line citations are relative to the reference project root):
//   * index file reader        — similarity_search/src/method/hnsw.cc:1025-1074 (LoadOptimizedIndex)
//                                 and the writer it mirrors, hnsw.cc:774-806
//   * distance kernels          — similarity_search/include/method/hnsw_distfunc_opt_impl_inline.h:42-173
//                                 (AVX L2Sqr16Ext / L2SqrExt / ScalarProduct, FMA-contracted lane order)
//                                 and the wrappers at src/method/hnsw.cc:70-102; L1 / LInf
//                                 (dist codes 5 / 6) from similarity_search/src/distcomp_lp.cc:77-251
//   * query normalisation       — similarity_search/include/method/hnsw.h:486-497 (NormalizeVect)
//   * greedy upper-level descent — src/method/hnsw_distfunc_opt.cc:62-92 and :168-198
//   * level-0 beam, V1Merge     — src/method/hnsw_distfunc_opt.cc:200-283 with the sorted-array
//                                 container of similarity_search/include/sort_arr_bi.h:30-216
//   * level-0 beam, SearchOld   — src/method/hnsw_distfunc_opt.cc:94-149
//   * dispatch (hybrid at ef>=1000) — src/method/hnsw.cc:717-746
//   * k-bounded result queue    — similarity_search/include/knnqueue.h:55-64,
//                                 src/knnquery.cc:67-75, python_bindings/nmslib.cc:170-184
//
// Arithmetic is pinned with explicit fmaf() in the reference's lane order; the file is
// compiled with -ffp-contract=off so that nothing else is fused. Tie order follows the
// reference by using the same libstdc++ algorithms it uses (std::sort for the neighbour
// buffer, std::priority_queue for SearchOld and for the result queue). The reference breaks
// result-queue ties by Object* address; Objects are allocated in node order by
// LoadOptimizedIndex, so this restatement breaks those ties by internal node index.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <climits>
#include <cstring>
#include <fstream>
#include <memory>
#include <queue>
#include <string>
#include <thread>
#include <vector>

namespace {

enum DistType { kL2Sqr16Ext = 1, kL2SqrExt = 2, kNormCosine = 3, kNegDot = 4, kL1 = 5, kLInf = 6 };

struct OracleIndex {
  uint32_t n = 0;
  uint64_t mem_per_obj = 0, off_level0 = 0, off_data = 0;
  int32_t maxlevel = 0;
  uint32_t enterpoint = 0;
  uint64_t maxM = 0, maxM0 = 0;
  int32_t dist_type = 0;
  uint64_t search_method = 0;
  int dim = 0;
  std::vector<char> level0;                   // N * mem_per_obj bytes, verbatim from the file
  std::vector<std::vector<int32_t>> links;    // per node: level*(maxM+1) ints, verbatim
  std::string err;

  const float* vec(int64_t i) const {
    return reinterpret_cast<const float*>(level0.data() + i * mem_per_obj + off_data + 16);
  }
  const int32_t* l0(int64_t i) const {
    return reinterpret_cast<const int32_t*>(level0.data() + i * mem_per_obj + off_level0);
  }
  int32_t ext_id(int64_t i) const {
    return *reinterpret_cast<const int32_t*>(level0.data() + i * mem_per_obj + off_data);
  }
  const int32_t* upper(int64_t i, int level) const {
    return links[i].data() + (maxM + 1) * (level - 1);
  }
  float distance(const float* q, int64_t i) const;
  int64_t row_bytes() const { return 4LL * dim; }
};

// ---------------------------------------------------------------- distances
// 8 accumulators over 8-wide blocks, acc[j] = fma(d, d, acc[j]) (impl_inline.h:42-70), summed
// left to right.
float l2sqr16(const float* a, const float* b, int dim) {
  float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int n16 = (dim >> 4) << 4;
  for (int e = 0; e < n16; ++e) {
    float d = a[e] - b[e];
    acc[e & 7] = fmaf(d, d, acc[e & 7]);
  }
  float s = acc[0];
  for (int j = 1; j < 8; ++j) s = s + acc[j];
  return s;
}

// impl_inline.h:72-122: 8 lanes over 16-blocks, fold to 4 lanes, 4-wide tail, sum of 4 lanes
// left to right, scalar FMA tail.
float l2sqr_any(const float* a, const float* b, int dim) {
  float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int n16 = (dim >> 4) << 4, n4 = (dim >> 2) << 2;
  for (int e = 0; e < n16; ++e) {
    float d = a[e] - b[e];
    acc[e & 7] = fmaf(d, d, acc[e & 7]);
  }
  float s4[4];
  for (int j = 0; j < 4; ++j) s4[j] = acc[j] + acc[j + 4];
  for (int e = n16; e < n4; ++e) {
    float d = a[e] - b[e];
    s4[e & 3] = fmaf(d, d, s4[e & 3]);
  }
  float s = ((s4[0] + s4[1]) + s4[2]) + s4[3];
  for (int e = n4; e < dim; ++e) {
    float d = a[e] - b[e];
    s = fmaf(d, d, s);
  }
  return s;
}

// impl_inline.h:124-173 (same lane structure as l2sqr_any, products instead of squared diffs).
float dot_avx(const float* a, const float* b, int dim) {
  float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int n16 = (dim >> 4) << 4, n4 = (dim >> 2) << 2;
  for (int e = 0; e < n16; ++e) acc[e & 7] = fmaf(a[e], b[e], acc[e & 7]);
  float s4[4];
  for (int j = 0; j < 4; ++j) s4[j] = acc[j] + acc[j + 4];
  for (int e = n16; e < n4; ++e) s4[e & 3] = fmaf(a[e], b[e], s4[e & 3]);
  float s = ((s4[0] + s4[1]) + s4[2]) + s4[3];
  for (int e = n4; e < dim; ++e) s = fmaf(a[e], b[e], s);
  return s;
}

// distcomp_lp.cc:191-251 (L1NormSIMD, SSE path): 4 float lanes over the first dim/4*4
// elements, lane j summing |a_e - b_e| for e == j (mod 4) in element order, unfused adds; the
// lanes are summed left to right in float, and the remaining elements are added in double.
float l1_sse(const float* a, const float* b, int dim) {
  float acc[4] = {0, 0, 0, 0};
  const int n4 = (dim >> 2) << 2;
  for (int e = 0; e < n4; ++e) acc[e & 3] = acc[e & 3] + std::fabs(a[e] - b[e]);
  double res = ((acc[0] + acc[1]) + acc[2]) + acc[3];
  for (int e = n4; e < dim; ++e) res += std::fabs(a[e] - b[e]);
  return (float)res;
}

// distcomp_lp.cc:77-136 (LInfNormSIMD): the largest |a_e - b_e|; a maximum of non-negative
// values, so the lane structure does not change the result.
float linf_sse(const float* a, const float* b, int dim) {
  float res = 0.0f;
  for (int e = 0; e < dim; ++e) res = std::max(res, std::fabs(a[e] - b[e]));
  return res;
}

float dist(int type, const float* q, const float* v, int dim) {
  switch (type) {
    case kL2Sqr16Ext: return l2sqr16(q, v, dim);
    case kL2SqrExt: return l2sqr_any(q, v, dim);
    case kNormCosine: {  // hnsw.cc:78-81
      float d = dot_avx(q, v, dim);
      return std::max(0.0f, 1 - std::max(-1.0f, std::min(1.0f, d)));
    }
    case kNegDot: return -dot_avx(q, v, dim);  // hnsw.cc:70-73
    case kL1: return l1_sse(q, v, dim);          // hnsw.cc:83-85
    case kLInf: return linf_sse(q, v, dim);      // hnsw.cc:87-89
  }
  return NAN;
}

// hnsw.h:486-497. Checked bit for bit against the normalised base vectors the reference stores
// in cosine index files: the sum of squares is accumulated sequentially WITHOUT fusing
// (round(v*v) then round(sum + .)), and the scale is the float 1.0f / sqrtf(sum).
// use_double selects the double-precision sqrt reading, kept only so a test can show that it
// does not match.
float OracleIndex::distance(const float* q, int64_t i) const { return dist(dist_type, q, vec(i), dim); }

// ---------------------------------------------------------------- l2sqr_sift (regular index)
// The objects of space l2sqr_sift: 128 uint8 values and the int sum of their squares
// (space_l2sqr_sift.cc:137-150); the distance is l2SqrSIFTPrecomp's |a|^2 + |b|^2 - 2 a.b in int
// (distcomp_l2sqr_sift.cc:40-50; its SSE / AVX forms add the same integers). Every value is at
// most 128 * 255^2 < 2^24, so the float key the searches carry holds it exactly.
constexpr int kSiftDim = 128;

struct SiftQuery {
  const uint8_t* v;
  int32_t norm;
};

struct SiftIndex {
  uint32_t n = 0;
  int32_t maxlevel = 0;  // the entry point's level: the generic search starts there (hnsw.cc:1183)
  uint32_t enterpoint = 0;
  uint64_t M = 0, maxM = 0, maxM0 = 0;
  std::vector<uint8_t> vecs;  // n x 128
  std::vector<int32_t> norms, obj_ids;
  size_t cap0 = 0, capu = 0;
  std::vector<int32_t> l0s;                 // n x (cap0 + 1): count, then ids
  std::vector<std::vector<int32_t>> links;  // per node: level x (capu + 1)

  const int32_t* l0(int64_t i) const { return l0s.data() + i * (cap0 + 1); }
  const int32_t* upper(int64_t i, int level) const { return links[i].data() + (capu + 1) * (level - 1); }
  float distance(const SiftQuery& q, int64_t i) const {
    const uint8_t* x = vecs.data() + i * kSiftDim;
    int32_t dot = 0;
    for (int e = 0; e < kSiftDim; ++e) dot += int32_t(q.v[e]) * int32_t(x[e]);
    return (float)(q.norm + norms[i] - 2 * dot);
  }
  int64_t row_bytes() const { return kSiftDim + 4; }
};

int32_t sift_norm(const uint8_t* v) {
  int32_t s = 0;
  for (int e = 0; e < kSiftDim; ++e) s += int32_t(v[e]) * int32_t(v[e]);
  return s;
}

void normalize(float* v, int dim, int use_double) {
  float sum = 0;
  for (int i = 0; i < dim; ++i) sum = sum + v[i] * v[i];  // -ffp-contract=off: not fused
  if (sum != 0.0f) {
    float s = use_double ? (float)(1.0 / std::sqrt((double)sum)) : 1.0f / sqrtf(sum);
    for (int i = 0; i < dim; ++i) v[i] *= s;
  }
}

// ---------------------------------------------------------------- per-query scratch
struct Stats {
  int64_t n_dist = 0;        // distance evaluations, upper levels included
  int64_t n_expand = 0;      // level-0 nodes whose neighbour list was scanned
  int64_t n_greedy = 0;      // upper-level list scans
  int64_t bytes = 0;         // algorithmic bytes: rows + neighbour lists read
};

struct Visited {  // epoch array, one byte per node (hnsw.h:568-590)
  std::vector<uint8_t> mass;
  uint8_t cur = 0;
  explicit Visited(size_t n) : mass(n + 1, 0) {}
  void reset() {
    ++cur;
    if (cur == 0) {
      std::fill(mass.begin(), mass.end(), 0);
      ++cur;
    }
  }
};

struct Item {  // sort_arr_bi.h:33-46; ordering by key only
  float key;
  bool used;
  int data;
  bool operator<(const Item& o) const { return key < o.key; }
};

// The bounded sorted array of sort_arr_bi.h, restated.
struct SortedArray {
  std::vector<Item> v;
  size_t num = 0;
  explicit SortedArray(size_t cap) : v(cap) {}
  void push_unsorted_grow(float key, int data) {  // :61-67
    if (num + 1 >= v.size()) v.resize(num + 1);
    v[num].used = false;
    v[num].key = key;
    v[num].data = data;
    ++num;
  }
  float top_key() const { return v[num - 1].key; }
  // :159-199 — append/drop at the tail; otherwise exponential probe from the tail followed
  // by lower_bound inside the last probed interval; shift right (dropping the last item when
  // full); return the insertion index.
  size_t push_or_replace_exp(float key, int data) {
    size_t curr = num - 1;
    if (v[curr].key <= key) {
      if (num < v.size()) {
        v[num].used = false;
        v[num].key = key;
        v[num].data = data;
        return num++;
      }
      return num;
    }
    size_t prev = curr, d = 1;
    while (curr > 0 && v[curr].key > key) {
      prev = curr;
      curr -= d;
      d *= 2;
      if (d > curr) d = curr;
    }
    if (curr < prev) {
      Item probe;
      probe.key = key;
      curr = std::lower_bound(v.begin() + curr, v.begin() + prev, probe) - v.begin();
    }
    if (num < v.size()) ++num;
    if (num - (1 + curr) > 0) std::memmove(&v[curr + 1], &v[curr], (num - (1 + curr)) * sizeof(Item));
    v[curr].used = false;
    v[curr].key = key;
    v[curr].data = data;
    return curr;
  }
  // :123-155 — in-place stable merge of a sorted batch.
  size_t merge_sorted(Item* items, size_t qty) {
    if (!qty) return num;
    if (qty > v.size()) qty = v.size();
    const size_t left = v.size() - num;
    if (left >= qty) {
      std::memcpy(&v[num], items, qty * sizeof(Item));
      std::inplace_merge(v.begin(), v.begin() + num, v.begin() + num + qty);
      num += qty;
    } else {
      size_t rem = 0;
      while (qty > left + rem && num > rem && items[left + rem].key < v[num - rem - 1].key) ++rem;
      std::memcpy(&v[num - rem], items, (left + rem) * sizeof(Item));
      std::inplace_merge(v.begin(), v.begin() + num - rem, v.end());
      num = v.size();
    }
    size_t r = 0;
    while (r < num && v[r].used) ++r;
    return r;
  }
};

// knnqueue.h:29-81 with (distance, node) pairs; node index stands in for the Object* address.
struct ResultQueue {
  std::priority_queue<std::pair<float, int64_t>> q;
  size_t k;
  explicit ResultQueue(size_t k_) : k(k_) {}
  void offer(float d, int64_t node) {  // knnquery.cc:67-75 + knnqueue.h:55-64
    if (q.size() < k) {
      q.push({d, node});
    } else if (q.top().first > d) {
      q.pop();
      q.push({d, node});
    }
  }
};

struct EvalNode {  // hnsw.h:410-431 — ordered by distance only
  float distance;
  int element;
  bool operator<(const EvalNode& o) const { return distance < o.distance; }
};

// hnsw_distfunc_opt.cc:62-92 / :168-198
// The searches below serve both index kinds: the optimized file (OracleIndex, float rows) and the
// regular file with l2sqr_sift objects (SiftIndex), whose generic search takes the same steps
// over node pointers (hnsw.cc:1078-1290 against hnsw_distfunc_opt.cc:48-283).
template <class Ix, class Q>
int greedy_descent(const Ix& ix, const Q& q, float* curdist_out, Stats& st) {
  int cur = (int)ix.enterpoint;
  float curdist = ix.distance(q, cur);
  st.n_dist += 1;
  st.bytes += ix.row_bytes();
  for (int lev = ix.maxlevel; lev > 0; --lev) {
    bool changed = true;
    while (changed) {
      changed = false;
      const int32_t* data = ix.upper(cur, lev);
      int size = data[0];
      st.n_greedy += 1;
      st.bytes += 4LL * (1 + size) + ix.row_bytes() * size;
      st.n_dist += size;
      for (int j = 1; j <= size; ++j) {
        int tnum = data[j];
        float d = ix.distance(q, tnum);
        if (d < curdist) {
          curdist = d;
          cur = tnum;
          changed = true;
        }
      }
    }
  }
  *curdist_out = curdist;
  return cur;
}

template <class Ix, class Q>
void search_v1merge(const Ix& ix, const Q& q, int k, int ef, Visited& vl, Stats& st,
                    std::vector<std::pair<float, int64_t>>& out) {
  vl.reset();
  float curdist;
  int cur = greedy_descent(ix, q, &curdist, st);
  SortedArray arr(std::max<size_t>(ef, k));
  arr.push_unsorted_grow(curdist, cur);
  size_t currElem = 0;
  std::vector<Item> buff(1 + std::max(ix.maxM, ix.maxM0));
  vl.mass[cur] = vl.cur;
  while (currElem < std::min(arr.num, (size_t)ef)) {
    Item& e = arr.v[currElem];
    e.used = true;
    cur = e.data;
    ++currElem;
    size_t qty = 0;
    float topKey = arr.top_key();
    const int32_t* data = ix.l0(cur);
    int size = data[0];
    st.n_expand += 1;
    st.bytes += 4LL * (1 + size);
    for (int j = 1; j <= size; ++j) {
      int tnum = data[j];
      if (vl.mass[tnum] != vl.cur) {
        vl.mass[tnum] = vl.cur;
        float d = ix.distance(q, tnum);
        st.n_dist += 1;
        st.bytes += ix.row_bytes();
        if (d < topKey || arr.num < (size_t)ef) {
          buff[qty].key = d;
          buff[qty].used = false;
          buff[qty].data = tnum;
          ++qty;
        }
      }
    }
    if (qty) {
      std::sort(buff.begin(), buff.begin() + qty);
      if (qty > 100) {
        size_t ins = arr.merge_sorted(&buff[0], qty);
        if (ins < currElem) currElem = ins;
      } else {
        for (size_t ii = 0; ii < qty; ++ii) {
          size_t ins = arr.push_or_replace_exp(buff[ii].key, buff[ii].data);
          if (ins < currElem) currElem = ins;
        }
      }
    }
    while (currElem < arr.num && arr.v[currElem].used) ++currElem;
  }
  ResultQueue rq(k);
  for (size_t i = 0; i < (size_t)k && i < arr.num; ++i) rq.offer(arr.v[i].key, arr.v[i].data);
  out.clear();
  while (!rq.q.empty()) {
    out.push_back(rq.q.top());
    rq.q.pop();
  }
  std::reverse(out.begin(), out.end());
}

template <class Ix, class Q>
void search_old(const Ix& ix, const Q& q, int k, int ef, Visited& vl, Stats& st,
                std::vector<std::pair<float, int64_t>>& out) {
  vl.reset();
  float curdist;
  int cur = greedy_descent(ix, q, &curdist, st);
  std::priority_queue<EvalNode> cand, closest;
  cand.push({-curdist, cur});
  closest.push({curdist, cur});
  ResultQueue rq(k);
  rq.offer(curdist, cur);
  vl.mass[cur] = vl.cur;
  while (!cand.empty()) {
    EvalNode ce = cand.top();
    float lb = closest.top().distance;
    if (-ce.distance > lb) break;
    cand.pop();
    cur = ce.element;
    const int32_t* data = ix.l0(cur);
    int size = data[0];
    st.n_expand += 1;
    st.bytes += 4LL * (1 + size);
    for (int j = 1; j <= size; ++j) {
      int tnum = data[j];
      if (vl.mass[tnum] != vl.cur) {
        vl.mass[tnum] = vl.cur;
        float d = ix.distance(q, tnum);
        st.n_dist += 1;
        st.bytes += ix.row_bytes();
        if (closest.top().distance > d || closest.size() < (size_t)ef) {
          cand.push({-d, tnum});
          rq.offer(d, tnum);
          closest.push({d, tnum});
          if (closest.size() > (size_t)ef) closest.pop();
        }
      }
    }
  }
  out.clear();
  while (!rq.q.empty()) {
    out.push_back(rq.q.top());
    rq.q.pop();
  }
  std::reverse(out.begin(), out.end());
}

thread_local std::string g_err;

}  // namespace

extern "C" {

const char* oracle_last_error() { return g_err.c_str(); }

// Reads the optimized index written by SaveOptimizedIndex (hnsw.cc:774-806).
void* oracle_load(const char* path) {
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    g_err = std::string("cannot open ") + path;
    return nullptr;
  }
  auto* ix = new OracleIndex();
  uint32_t flag = 0;
  bool ok = std::fread(&flag, 4, 1, f) == 1 && flag == 1;
  ok = ok && std::fread(&ix->n, 4, 1, f) == 1 && std::fread(&ix->mem_per_obj, 8, 1, f) == 1 &&
       std::fread(&ix->off_level0, 8, 1, f) == 1 && std::fread(&ix->off_data, 8, 1, f) == 1 &&
       std::fread(&ix->maxlevel, 4, 1, f) == 1 && std::fread(&ix->enterpoint, 4, 1, f) == 1 &&
       std::fread(&ix->maxM, 8, 1, f) == 1 && std::fread(&ix->maxM0, 8, 1, f) == 1 &&
       std::fread(&ix->dist_type, 4, 1, f) == 1 && std::fread(&ix->search_method, 8, 1, f) == 1;
  if (ok) {
    ix->level0.resize(ix->n * ix->mem_per_obj + 64);
    ok = std::fread(ix->level0.data(), 1, ix->n * ix->mem_per_obj, f) == ix->n * ix->mem_per_obj;
  }
  if (ok) {
    ix->links.resize(ix->n);
    for (uint32_t i = 0; ok && i < ix->n; ++i) {
      uint32_t sz = 0;
      ok = std::fread(&sz, 4, 1, f) == 1;
      if (ok && sz) {
        ix->links[i].resize(sz / 4);
        ok = std::fread(ix->links[i].data(), 1, sz, f) == sz;
      }
    }
  }
  std::fclose(f);
  if (!ok) {
    g_err = "truncated or non-optimized index file";
    delete ix;
    return nullptr;
  }
  ix->dim = ix->n ? (int)((ix->off_level0 - ix->off_data - 16) / 4) : 0;
  return ix;
}

void oracle_free(void* h) { delete static_cast<OracleIndex*>(h); }

// info: n, dim, maxlevel, enterpoint, maxM, maxM0, dist_type, mem_per_obj, off_level0
void oracle_info(void* h, int64_t* info) {
  auto* ix = static_cast<OracleIndex*>(h);
  info[0] = ix->n;
  info[1] = ix->dim;
  info[2] = ix->maxlevel;
  info[3] = ix->enterpoint;
  info[4] = (int64_t)ix->maxM;
  info[5] = (int64_t)ix->maxM0;
  info[6] = ix->dist_type;
  info[7] = (int64_t)ix->mem_per_obj;
  info[8] = (int64_t)ix->off_level0;
}

// Copies out the stored vectors (N x dim), external ids, level-0 lists (N x (maxM0+1)) and
// node levels, so tests can cross-check the product's own reader.
void oracle_export(void* h, float* vecs, int32_t* ext_ids, int32_t* l0, int32_t* levels) {
  auto* ix = static_cast<OracleIndex*>(h);
  for (int64_t i = 0; i < ix->n; ++i) {
    if (vecs) std::memcpy(vecs + i * ix->dim, ix->vec(i), 4 * ix->dim);
    if (ext_ids) ext_ids[i] = ix->ext_id(i);
    if (l0) std::memcpy(l0 + i * (ix->maxM0 + 1), ix->l0(i), 4 * (ix->maxM0 + 1));
    if (levels) levels[i] = (int32_t)(ix->links[i].size() / (ix->maxM + 1));
  }
}

float oracle_dist(int type, const float* a, const float* b, int dim) { return dist(type, a, b, dim); }

void oracle_normalize(float* v, int dim, int use_double) { normalize(v, dim, use_double); }

// Batch search. algo: 0 hybrid (old when ef >= 1000), 1 old, 2 v1merge (hnsw.cc:724).
// k_per_q / ef_per_q may be null. Outputs are row-major nq x kmax with -1 / +inf padding;
// stats is nq x 4 (n_dist, n_expand, n_greedy, bytes).
int oracle_search(void* h, const float* queries, int64_t nq, int dim, int k, const int32_t* k_per_q,
                  int ef, const int32_t* ef_per_q, int algo, int kmax, int32_t* ids, float* dists,
                  int32_t* counts, int64_t* stats, int nthreads) {
  auto* ix = static_cast<OracleIndex*>(h);
  if (dim != ix->dim && ix->n) {
    g_err = "dimension mismatch";
    return -1;
  }
  if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  std::atomic<int64_t> next(0);
  auto worker = [&]() {
    Visited vl(ix->n);
    std::vector<float> qv(dim);
    std::vector<std::pair<float, int64_t>> res;
    for (;;) {
      int64_t qi = next.fetch_add(1);
      if (qi >= nq) break;
      int kq = k_per_q ? k_per_q[qi] : k;
      int efq = ef_per_q ? ef_per_q[qi] : ef;
      Stats st;
      res.clear();
      if (ix->n) {
        std::memcpy(qv.data(), queries + qi * dim, 4 * dim);
        if (ix->dist_type == kNormCosine) normalize(qv.data(), dim, 0);
        bool use_old = algo == 1 || (algo == 0 && efq >= 1000);
        if (use_old)
          search_old(*ix, qv.data(), kq, efq, vl, st, res);
        else
          search_v1merge(*ix, qv.data(), kq, efq, vl, st, res);
      }
      int cnt = (int)std::min<size_t>(res.size(), (size_t)kmax);
      counts[qi] = cnt;
      for (int j = 0; j < kmax; ++j) {
        ids[qi * kmax + j] = j < cnt ? ix->ext_id(res[j].second) : -1;
        dists[qi * kmax + j] = j < cnt ? res[j].first : INFINITY;
      }
      if (stats) {
        stats[qi * 4 + 0] = st.n_dist;
        stats[qi * 4 + 1] = st.n_expand;
        stats[qi * 4 + 2] = st.n_greedy;
        stats[qi * 4 + 3] = st.bytes;
      }
    }
  };
  std::vector<std::thread> th;
  for (int t = 0; t < nthreads; ++t) th.emplace_back(worker);
  for (auto& t : th) t.join();
  return 0;
}

// Reads an l2sqr_sift index: the regular graph file written by SaveRegularIndexBin
// (hnsw.cc:810-842: u32 0 | u32 N | i32 maxlevel | u32 entry | u64 M | u64 maxM | u64 maxM0, then per
// node u32 level and, for each level 0..level, u32 count and the neighbour ids) and the objects
// file written by saveIndex(..., save_data=True) (python_bindings/nmslib.cc:115-125, space.cc:90-104:
// u64 count, then per object u64 length and the object: i32 id | i32 label | u64 datalength |
// 128 uint8 | i32 norm). Returns null with the reason in oracle_last_error().
void* oracle_sift_load(const char* graph_path, const char* data_path) {
  auto ix = std::make_unique<SiftIndex>();
  std::ifstream dat(data_path, std::ios::binary);
  if (!dat) {
    g_err = std::string("cannot open ") + data_path;
    return nullptr;
  }
  uint64_t qty = 0;
  dat.read(reinterpret_cast<char*>(&qty), 8);
  // every object takes 8 (length) + 16 (header) + 128 (vector) + 4 (norm) bytes: a count the
  // file cannot hold is rejected before anything is sized from it
  dat.seekg(0, std::ios::end);
  const uint64_t fsize = dat ? (uint64_t)dat.tellg() : 0;
  dat.seekg(8, std::ios::beg);
  if (!dat || fsize < 8 || qty > (fsize - 8) / (8 + 16 + kSiftDim + 4)) {
    g_err = "objects file: object count " + std::to_string(qty) + " does not fit the file";
    return nullptr;
  }
  ix->vecs.resize(qty * kSiftDim);
  ix->norms.resize(qty);
  ix->obj_ids.resize(qty);
  for (uint64_t i = 0; i < qty; ++i) {
    uint64_t len = 0, dlen = 0;
    int32_t id = 0, label = 0;
    dat.read(reinterpret_cast<char*>(&len), 8);
    dat.read(reinterpret_cast<char*>(&id), 4);
    dat.read(reinterpret_cast<char*>(&label), 4);
    dat.read(reinterpret_cast<char*>(&dlen), 8);
    if (!dat || dlen != kSiftDim + 4 || len != 16 + dlen) {
      g_err = "objects file: not a 128-byte l2sqr_sift object at position " + std::to_string(i);
      return nullptr;
    }
    dat.read(reinterpret_cast<char*>(ix->vecs.data() + i * kSiftDim), kSiftDim);
    dat.read(reinterpret_cast<char*>(&ix->norms[i]), 4);
    ix->obj_ids[i] = id;
  }
  if (!dat) {
    g_err = "objects file is truncated";
    return nullptr;
  }
  std::ifstream g(graph_path, std::ios::binary);
  uint32_t flag = 1, n = 0;
  g.read(reinterpret_cast<char*>(&flag), 4);
  g.read(reinterpret_cast<char*>(&n), 4);
  g.read(reinterpret_cast<char*>(&ix->maxlevel), 4);
  g.read(reinterpret_cast<char*>(&ix->enterpoint), 4);
  g.read(reinterpret_cast<char*>(&ix->M), 8);
  g.read(reinterpret_cast<char*>(&ix->maxM), 8);
  g.read(reinterpret_cast<char*>(&ix->maxM0), 8);
  if (!g || flag != 0 || n != qty || (n && ix->enterpoint >= n)) {
    g_err = "graph file: not a regular index over these objects";
    return nullptr;
  }
  ix->n = n;
  std::vector<std::vector<std::vector<int32_t>>> lists(n);
  size_t cap0 = ix->maxM0, capu = ix->maxM;
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t level = 0;
    g.read(reinterpret_cast<char*>(&level), 4);
    if (!g || level > 64) {
      g_err = "graph file: bad level at node " + std::to_string(i);
      return nullptr;
    }
    lists[i].resize(level + 1);
    for (uint32_t lev = 0; lev <= level; ++lev) {
      uint32_t cnt = 0;
      g.read(reinterpret_cast<char*>(&cnt), 4);
      if (!g || cnt > n) {
        g_err = "graph file: bad list at node " + std::to_string(i);
        return nullptr;
      }
      lists[i][lev].resize(cnt);
      g.read(reinterpret_cast<char*>(lists[i][lev].data()), 4LL * cnt);
      for (int32_t f : lists[i][lev])
        if (f < 0 || (uint32_t)f >= n) {
          g_err = "graph file: neighbour id out of range at node " + std::to_string(i);
          return nullptr;
        }
      (lev ? capu : cap0) = std::max<size_t>(lev ? capu : cap0, cnt);
    }
  }
  if (!g) {
    g_err = "graph file is truncated";
    return nullptr;
  }
  ix->cap0 = cap0;
  ix->capu = capu;
  ix->l0s.assign((size_t)n * (cap0 + 1), 0);
  ix->links.resize(n);
  for (uint32_t i = 0; i < n; ++i) {
    int32_t* d = ix->l0s.data() + (size_t)i * (cap0 + 1);
    d[0] = (int32_t)lists[i][0].size();
    std::copy(lists[i][0].begin(), lists[i][0].end(), d + 1);
    const size_t levels = lists[i].size() - 1;
    ix->links[i].assign(levels * (capu + 1), 0);
    for (size_t lev = 1; lev <= levels; ++lev) {
      int32_t* u = ix->links[i].data() + (lev - 1) * (capu + 1);
      u[0] = (int32_t)lists[i][lev].size();
      std::copy(lists[i][lev].begin(), lists[i][lev].end(), u + 1);
    }
  }
  if (n) ix->maxlevel = (int32_t)lists[ix->enterpoint].size() - 1;
  return ix.release();
}

void oracle_sift_free(void* h) { delete static_cast<SiftIndex*>(h); }

// info: n, maxlevel (the entry point's), entry point, M, maxM, maxM0
void oracle_sift_info(void* h, int64_t* info) {
  auto* ix = static_cast<SiftIndex*>(h);
  info[0] = ix->n;
  info[1] = ix->maxlevel;
  info[2] = ix->enterpoint;
  info[3] = (int64_t)ix->M;
  info[4] = (int64_t)ix->maxM;
  info[5] = (int64_t)ix->maxM0;
}

// Batch search over nq x 128 uint8 queries; algo as oracle_search. Outputs nq x kmax object ids
// and int distances, -1 / INT32_MAX padding; stats (optional) as oracle_search's, with 132 bytes
// (values and norm) per row.
int oracle_sift_search(void* h, const uint8_t* queries, int64_t nq, int k, int ef, int algo, int kmax, int32_t* ids,
                       int32_t* dists, int32_t* counts, int64_t* stats, int nthreads) {
  auto* ix = static_cast<SiftIndex*>(h);
  if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  std::atomic<int64_t> next(0);
  auto worker = [&]() {
    Visited vl(ix->n);
    std::vector<std::pair<float, int64_t>> res;
    for (;;) {
      const int64_t qi = next.fetch_add(1);
      if (qi >= nq) break;
      Stats st;
      res.clear();
      if (ix->n) {
        const SiftQuery q{queries + qi * kSiftDim, sift_norm(queries + qi * kSiftDim)};
        if (algo == 1 || (algo == 0 && ef >= 1000))
          search_old(*ix, q, k, ef, vl, st, res);
        else
          search_v1merge(*ix, q, k, ef, vl, st, res);
      }
      const int cnt = (int)std::min<size_t>(res.size(), (size_t)kmax);
      counts[qi] = cnt;
      for (int j = 0; j < kmax; ++j) {
        ids[qi * kmax + j] = j < cnt ? ix->obj_ids[res[j].second] : -1;
        dists[qi * kmax + j] = j < cnt ? (int32_t)res[j].first : INT32_MAX;
      }
      if (stats) {
        stats[qi * 4 + 0] = st.n_dist;
        stats[qi * 4 + 1] = st.n_expand;
        stats[qi * 4 + 2] = st.n_greedy;
        stats[qi * 4 + 3] = st.bytes;
      }
    }
  };
  std::vector<std::thread> th;
  for (int t = 0; t < nthreads; ++t) th.emplace_back(worker);
  for (auto& t : th) t.join();
  return 0;
}

// libstdc++ std::sort on (key, payload) pairs compared by key only — the order the reference
// gives its neighbour buffer (hnsw_distfunc_opt.cc:251). Used to check the product's device
// restatement of that order.
void oracle_std_sort_items(float* keys, int32_t* payload, int n) {
  std::vector<Item> v(n);
  for (int i = 0; i < n; ++i) v[i] = {keys[i], false, payload[i]};
  std::sort(v.begin(), v.end());
  for (int i = 0; i < n; ++i) {
    keys[i] = v[i].key;
    payload[i] = v[i].data;
  }
}

}  // extern "C"
