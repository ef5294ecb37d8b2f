// HNSW query kernels for sm_100a: upper-level greedy descent, level-0 beam search with the
// reference's SearchV1Merge and SearchOld semantics, and the warp-cooperative distances they use.
//
// One warp owns one query at a time. Everything the reference keeps per query — the query
// vector, the sorted candidate array (SortArrBI), the neighbour buffer, SearchOld's heaps —
// lives in the warp's slice of shared memory; the visited set is a per-warp epoch byte array in
// HBM (the reference's VisitedList, similarity_search/include/method/hnsw.h:568-590), and
// SearchOld's unbounded candidate heap spills to a per-warp HBM area.
//
// Arithmetic matches the reference bit for bit:
//  * distances follow the AVX kernels of similarity_search/include/method/hnsw_distfunc_opt_impl_inline.h:42-173
//    (8 accumulators fed by FMAs in element order, left-to-right lane sums, a 4-wide fused
//    remainder and a scalar fused tail), computed by 8 lanes, lane j owning accumulator j;
//  * the cosine query is normalised as in hnsw.h:486-497 (unfused sum of squares, 1/sqrtf);
//  * every rounding step is an explicit __f*_rn intrinsic, so nvcc's contraction cannot
//    change the result.
// Tie order matches too: neighbour batches are ordered exactly as libstdc++ std::sort orders
// them (stable rank sort where that is provably identical, a restatement of libstdc++'s
// introsort otherwise), and insertion follows push_or_replace_non_empty_exp
// (similarity_search/include/sort_arr_bi.h:159-199) including its exponential probe.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>
#include <set>
#include <utility>

#include "engine.h"
#include "search_device.cuh"
#include "sm100.cuh"
#include "../../include/nmslib_b200.h"

namespace nmsg {

namespace {

// ------------------------------------------------------------------ distances
// Row and query are in the permuted layout (engine.h). `acc` is lane j's accumulator of the
// 8-wide loop; the combine step reproduces the reference's reduction for each distance code.
template <int R>
struct RowAcc {
  float acc[R];
};

__device__ __forceinline__ float fma_term(int code, float a, float b, float acc) {
  if (code == kL2Sqr16Ext || code == kL2SqrExt) {
    const float d = __fsub_rn(a, b);
    return __fmaf_rn(d, d, acc);
  }
  return __fmaf_rn(a, b, acc);
}

// Reduce the 8 lane accumulators of one group into the reference's final value; every lane of
// the group returns the same value. `row` and `q` are needed for the remainder elements.
__device__ __forceinline__ float combine(const DevIndex& ix, float acc, const float* __restrict__ row,
                                         const float* __restrict__ q) {
  const int lane = lane_id();
  const int gb = lane & ~7, j = lane & 7;
  const int code = ix.dist_type;
  if (code == kL2Sqr16Ext) {
    // impl_inline.h:68-69: TmpRes[0] + ... + TmpRes[7], left to right
    float s = __shfl_sync(kFull, acc, gb);
#pragma unroll
    for (int t = 1; t < 8; ++t) s = __fadd_rn(s, __shfl_sync(kFull, acc, gb + t));
    return s;
  }
  // impl_inline.h:100,152: fold the 8 lanes to 4 (acc[j] + acc[j+4])
  float t4 = __fadd_rn(acc, __shfl_down_sync(kFull, acc, 4, 8));
  // 4-wide fused remainder over elements [n16, n4); lane j < 4 owns elements e == j (mod 4)
  if (j < 4) {
    for (int e = ix.n16 + j; e < ix.n4; e += 4) t4 = fma_term(code, q[e], row[e], t4);
  }
  float s = __fadd_rn(__shfl_sync(kFull, t4, gb), __shfl_sync(kFull, t4, gb + 1));
  s = __fadd_rn(s, __shfl_sync(kFull, t4, gb + 2));
  s = __fadd_rn(s, __shfl_sync(kFull, t4, gb + 3));
  // scalar fused tail over [n4, dim)
  for (int e = ix.n4; e < ix.dim; ++e) s = fma_term(code, q[e], row[e], s);
  if (code == kNormCosine) {
    // hnsw.cc:78-81: max(0, 1 - max(-1, min(1, dot))) with std::min/std::max operand order
    const float mn = (s < 1.0f) ? s : 1.0f;
    const float mx = (-1.0f < mn) ? mn : -1.0f;
    const float v = __fsub_rn(1.0f, mx);
    return (0.0f < v) ? v : 0.0f;
  }
  if (code == kNegDot) return -s;  // hnsw.cc:70-73
  return s;
}

// L1 (code 5) and LInf (code 6) of one row, by the 8 lanes of a group; every lane of the group
// returns the value. `row` is in global memory (GLOBAL) or in the warp's staging area.
//  * L1 restates distcomp_lp.cc:191-251: four float accumulators, accumulator a summing
//    |q_e - x_e| over e == a (mod 4) in element order with unfused adds, then
//    ((s0 + s1) + s2) + s3 in float, then the last dim % 4 elements added in double. In the
//    permuted layout lane j holds e == j (mod 8), so accumulator a (lane a < 4) takes lane a+4's
//    values by shuffle and interleaves them: a, a+4, a+8, a+12, ...
//  * LInf (distcomp_lp.cc:77-136) is the maximum of non-negative values: any order gives it.
template <bool GLOBAL>
__device__ __forceinline__ float4 ld_row4(const float* p) {
  if (GLOBAL) return __ldg(reinterpret_cast<const float4*>(p));
  return *reinterpret_cast<const float4*>(p);
}
template <bool GLOBAL>
__device__ __forceinline__ float2 ld_row2(const float* p) {
  if (GLOBAL) return __ldg(reinterpret_cast<const float2*>(p));
  return *reinterpret_cast<const float2*>(p);
}
template <bool GLOBAL>
__device__ __forceinline__ float ld_row1(const float* p) {
  if (GLOBAL) return __ldg(p);
  return *p;
}

template <bool GLOBAL>
__device__ float lp_group_dist(const DevIndex& ix, const float* __restrict__ q, const float* __restrict__ row,
                               bool act) {
  const int lane = lane_id();
  const int gb = lane & ~7, j = lane & 7;
  const int nfull = ix.n16 >> 5;
  const bool half = (ix.n16 & 31) != 0;
  const bool l1 = ix.dist_type == kL1;
  float s = 0.0f;  // L1: accumulator j of lanes j < 4; LInf: this lane's maximum
  for (int c = 0; c < nfull; ++c) {
    const float4 qv = reinterpret_cast<const float4*>(q + c * 32)[j];
    const float4 xv = act ? ld_row4<GLOBAL>(row + c * 32 + 4 * j) : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 d = make_float4(fabsf(__fsub_rn(qv.x, xv.x)), fabsf(__fsub_rn(qv.y, xv.y)),
                                 fabsf(__fsub_rn(qv.z, xv.z)), fabsf(__fsub_rn(qv.w, xv.w)));
    if (l1) {
      const float4 e = make_float4(__shfl_down_sync(kFull, d.x, 4, 8), __shfl_down_sync(kFull, d.y, 4, 8),
                                   __shfl_down_sync(kFull, d.z, 4, 8), __shfl_down_sync(kFull, d.w, 4, 8));
      s = __fadd_rn(s, d.x);
      s = __fadd_rn(s, e.x);
      s = __fadd_rn(s, d.y);
      s = __fadd_rn(s, e.y);
      s = __fadd_rn(s, d.z);
      s = __fadd_rn(s, e.z);
      s = __fadd_rn(s, d.w);
      s = __fadd_rn(s, e.w);
    } else {
      s = fmaxf(fmaxf(fmaxf(s, d.x), fmaxf(d.y, d.z)), d.w);
    }
  }
  if (half) {
    const float2 qv = reinterpret_cast<const float2*>(q + nfull * 32)[j];
    const float2 xv = act ? ld_row2<GLOBAL>(row + nfull * 32 + 2 * j) : make_float2(0.f, 0.f);
    const float2 d = make_float2(fabsf(__fsub_rn(qv.x, xv.x)), fabsf(__fsub_rn(qv.y, xv.y)));
    if (l1) {
      const float2 e = make_float2(__shfl_down_sync(kFull, d.x, 4, 8), __shfl_down_sync(kFull, d.y, 4, 8));
      s = __fadd_rn(s, d.x);
      s = __fadd_rn(s, e.x);
      s = __fadd_rn(s, d.y);
      s = __fadd_rn(s, e.y);
    } else {
      s = fmaxf(s, fmaxf(d.x, d.y));
    }
  }
  const int n4 = (ix.dim >> 2) << 2;
  if (l1) {
    // [n16, n4): accumulator j continues in natural order
    if (act && j < 4)
      for (int e = ix.n16 + j; e < n4; e += 4) s = __fadd_rn(s, fabsf(__fsub_rn(q[e], ld_row1<GLOBAL>(row + e))));
    float t = __fadd_rn(__shfl_sync(kFull, s, gb), __shfl_sync(kFull, s, gb + 1));
    t = __fadd_rn(t, __shfl_sync(kFull, s, gb + 2));
    t = __fadd_rn(t, __shfl_sync(kFull, s, gb + 3));
    double r = (double)t;
    if (act)
      for (int e = n4; e < ix.dim; ++e) r = __dadd_rn(r, (double)fabsf(__fsub_rn(q[e], ld_row1<GLOBAL>(row + e))));
    return __double2float_rn(r);
  }
  if (act)
    for (int e = ix.n16 + j; e < ix.dim; e += 8) s = fmaxf(s, fabsf(__fsub_rn(q[e], ld_row1<GLOBAL>(row + e))));
  s = fmaxf(s, __shfl_xor_sync(kFull, s, 4, 8));
  s = fmaxf(s, __shfl_xor_sync(kFull, s, 2, 8));
  s = fmaxf(s, __shfl_xor_sync(kFull, s, 1, 8));
  return s;
}

// Distances from the query (shared memory, permuted) to rows ids[0..n), written to out[0..n).
// Four 8-lane groups per warp, R rows per group in flight.
template <int R>
__device__ void compute_dists(const DevIndex& ix, const float* __restrict__ q, const int* __restrict__ ids, int n,
                              float* __restrict__ out) {
  const int lane = lane_id();
  const int g = lane >> 3, j = lane & 7;
  const int nfull = ix.n16 >> 5;
  const bool half = (ix.n16 & 31) != 0;
  const int code = ix.dist_type;
  if constexpr (R == kSiftGather) {
    // l2sqr_sift: eight 4-lane groups, one 128-byte row per group; lane j of a group takes bytes
    // [32j, 32j + 32) of the row and of the query (shared memory: 128 values, then the query's
    // norm). The reference's distance |q|^2 + |x|^2 - 2 q.x in int (distcomp_l2sqr_sift.cc:40-50)
    // is exact whatever the order of the products and sums, so byte dot products (dp4a) and a
    // butterfly over the group give the same integer; it is below 2^24, so the float key is exact.
    const int g4 = lane >> 2, j4 = lane & 3;
    const uint4* qv = reinterpret_cast<const uint4*>(q) + 2 * j4;
    const uint4 qa = qv[0], qb = qv[1];
    const int qn = reinterpret_cast<const int*>(q)[kSiftDim / 4];
    for (int base = 0; base < n; base += 8) {
      const int idx = base + g4;
      const bool act = idx < n;
      const int id = act ? ids[idx] : 0;
      uint4 xa = make_uint4(0u, 0u, 0u, 0u), xb = xa;
      if (act) {
        const uint4* row = reinterpret_cast<const uint4*>(ix.vecs_u8 + (int64_t)id * kSiftDim) + 2 * j4;
        xa = __ldg(row);
        xb = __ldg(row + 1);
      }
      unsigned dot = __dp4a(xa.x, qa.x, 0u);
      dot = __dp4a(xa.y, qa.y, dot);
      dot = __dp4a(xa.z, qa.z, dot);
      dot = __dp4a(xa.w, qa.w, dot);
      dot = __dp4a(xb.x, qb.x, dot);
      dot = __dp4a(xb.y, qb.y, dot);
      dot = __dp4a(xb.z, qb.z, dot);
      dot = __dp4a(xb.w, qb.w, dot);
      unsigned xx = __dp4a(xa.x, xa.x, 0u);
      xx = __dp4a(xa.y, xa.y, xx);
      xx = __dp4a(xa.z, xa.z, xx);
      xx = __dp4a(xa.w, xa.w, xx);
      xx = __dp4a(xb.x, xb.x, xx);
      xx = __dp4a(xb.y, xb.y, xx);
      xx = __dp4a(xb.z, xb.z, xx);
      xx = __dp4a(xb.w, xb.w, xx);
      dot += __shfl_xor_sync(kFull, dot, 1);
      xx += __shfl_xor_sync(kFull, xx, 1);
      dot += __shfl_xor_sync(kFull, dot, 2);
      xx += __shfl_xor_sync(kFull, xx, 2);
      if (act && j4 == 0) {
        const int xn = ix.norms ? __ldg(ix.norms + id) : (int)xx;
        out[idx] = __int2float_rn(qn + xn - 2 * (int)dot);
      }
    }
    __syncwarp();
  } else if constexpr (R == kLpGather) {  // L1 / LInf indices run kernels of their own (gather code 3)
    for (int base = 0; base < n; base += 4) {
      const int idx = base + g;
      const bool act = idx < n;
      const float* row = ix.vecs + (int64_t)(act ? ids[idx] : 0) * ix.pitch;
      const float d = lp_group_dist<true>(ix, q, row, act);
      if (act && j == 0) out[idx] = d;
    }
    __syncwarp();
  } else {
    for (int base = 0; base < n; base += 4 * R) {
      const float* rows[R];
      bool act[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int idx = base + g + 4 * r;
        act[r] = idx < n;
        rows[r] = ix.vecs + (int64_t)(act[r] ? ids[idx] : 0) * ix.pitch;
      }
      float acc[R];
#pragma unroll
      for (int r = 0; r < R; ++r) acc[r] = 0.0f;
#pragma unroll 4
      for (int c = 0; c < nfull; ++c) {
        const float4 qv = reinterpret_cast<const float4*>(q + c * 32)[j];
        float4 x[R];
#pragma unroll
        for (int r = 0; r < R; ++r)
          x[r] = act[r] ? __ldg(reinterpret_cast<const float4*>(rows[r] + c * 32) + j) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          acc[r] = fma_term(code, qv.x, x[r].x, acc[r]);
          acc[r] = fma_term(code, qv.y, x[r].y, acc[r]);
          acc[r] = fma_term(code, qv.z, x[r].z, acc[r]);
          acc[r] = fma_term(code, qv.w, x[r].w, acc[r]);
        }
      }
      if (half) {
        const float2 qv = reinterpret_cast<const float2*>(q + nfull * 32)[j];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const float2 x = act[r] ? __ldg(reinterpret_cast<const float2*>(rows[r] + nfull * 32) + j) : make_float2(0.f, 0.f);
          acc[r] = fma_term(code, qv.x, x.x, acc[r]);
          acc[r] = fma_term(code, qv.y, x.y, acc[r]);
        }
      }
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const float d = combine(ix, acc[r], rows[r], q);
        if (act[r] && j == 0) out[base + g + 4 * r] = d;
      }
    }
    __syncwarp();
  }
}

// Distances to rows ids[0..n) through the warp's staging area: each round copies up to
// `stage_rows` rows into shared memory with asynchronous 16-byte copies (every row of the round
// in flight at once, no registers held), then the four 8-lane groups reduce them.
// With `bar` set, each row is one bulk copy (TMA unit) issued by one lane and completing on that
// mbarrier (phase in *phase); a copy that does not complete within the wait bound sets *failed.
__device__ void compute_dists_staged(const DevIndex& ix, const float* __restrict__ q, const int* __restrict__ ids,
                                     int n, float* __restrict__ out, float* __restrict__ stage, int stage_rows,
                                     uint64_t* bar, uint32_t* phase, bool* failed) {
  const int lane = lane_id();
  const int g = lane >> 3, j = lane & 7;
  const int nf4 = (ix.dim + 3) >> 2;  // 16-byte chunks covering elements [0, dim)
  const int nfull = ix.n16 >> 5;
  const bool half = (ix.n16 & 31) != 0;
  const int code = ix.dist_type;
  const uint32_t row_bytes = (uint32_t)bulk_row_bytes(ix);
  for (int base = 0; base < n; base += stage_rows) {
    const int cnt = min(stage_rows, n - base);
    if (bar) {
      if (lane == 0) sm100::mbar_arrive_expect_tx(bar, (uint32_t)cnt * row_bytes);
      __syncwarp();
      for (int r = lane; r < cnt; r += 32) {
        sm100::fence_proxy_async_smem();
        sm100::bulk_copy_g2s(stage + r * ix.pitch, ix.vecs + (int64_t)ids[base + r] * ix.pitch, row_bytes, bar);
      }
      if (!sm100::mbar_wait(bar, *phase)) {
        sm100::mbar_wait(bar, *phase);  // bounded: no copy may be left writing the staging rows
        *failed = true;
      }
      *phase ^= 1;
    } else {
      for (int r = 0; r < cnt; ++r) {
        const float* src = ix.vecs + (int64_t)ids[base + r] * ix.pitch;
        float* dst = stage + r * ix.pitch;
        for (int c = lane; c < nf4; c += 32) cp_async16(dst + 4 * c, src + 4 * c);
      }
      cp_async_wait_all();
    }
    __syncwarp();
    for (int r0 = 0; r0 < cnt; r0 += 4) {
      const int r = r0 + g;
      const bool act = r < cnt;
      const float* row = stage + (act ? r : 0) * ix.pitch;
      float acc = 0.0f;
#pragma unroll 4
      for (int c = 0; c < nfull; ++c) {
        const float4 qv = reinterpret_cast<const float4*>(q + c * 32)[j];
        const float4 x = reinterpret_cast<const float4*>(row + c * 32)[j];
        acc = fma_term(code, qv.x, x.x, acc);
        acc = fma_term(code, qv.y, x.y, acc);
        acc = fma_term(code, qv.z, x.z, acc);
        acc = fma_term(code, qv.w, x.w, acc);
      }
      if (half) {
        const float2 qv = reinterpret_cast<const float2*>(q + nfull * 32)[j];
        const float2 x = reinterpret_cast<const float2*>(row + nfull * 32)[j];
        acc = fma_term(code, qv.x, x.x, acc);
        acc = fma_term(code, qv.y, x.y, acc);
      }
      const float d = combine(ix, acc, row, q);
      if (act && j == 0) out[base + r] = d;
    }
    __syncwarp();
  }
}

// ------------------------------------------------------------------ binary heaps (SearchOld)
// std::priority_queue<EvaluatedMSWNodeInt> semantics (hnsw.h:410-431: ordered by distance only)
// with libstdc++'s push_heap / pop_heap. Single-lane code.
__device__ void heap_push(uint2* h, int& size, float key, int id) {
  int hole = size++;
  int parent = (hole - 1) / 2;
  while (hole > 0 && key_of(h[parent]) < key) {
    h[hole] = h[parent];
    hole = parent;
    parent = (hole - 1) / 2;
  }
  h[hole] = make_uint2(__float_as_uint(key), (uint32_t)id);
}

__device__ void heap_pop(uint2* h, int& size) {
  if (size > 1) {
    const int len = size - 1;
    const uint2 value = h[len];
    h[len] = h[0];
    int hole = 0, child = 0;
    while (child < (len - 1) / 2) {
      child = 2 * (child + 1);
      if (key_of(h[child]) < key_of(h[child - 1])) child--;
      h[hole] = h[child];
      hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
      child = 2 * (child + 1);
      h[hole] = h[child - 1];
      hole = child - 1;
    }
    int parent = (hole - 1) / 2;
    while (hole > 0 && key_of(h[parent]) < key_of(value)) {
      h[hole] = h[parent];
      hole = parent;
      parent = (hole - 1) / 2;
    }
    h[hole] = value;
  }
  --size;
}

// The k-bounded result queue (knnqueue.h:55-64 + knnquery.cc:67-75) kept as an array sorted by
// (distance, node); node index stands in for the reference's Object* order. Single lane.
__device__ void result_offer(uint2* res, int& size, int k, float d, int node) {
  if (size >= k) {
    if (!(key_of(res[size - 1]) > d)) return;
    --size;  // pop the largest (distance, node) pair
  }
  int pos = size;
  while (pos > 0) {
    const float pk = key_of(res[pos - 1]);
    const int pn = (int)res[pos - 1].y;
    if (pk < d || (pk == d && pn < node)) break;
    res[pos] = res[pos - 1];
    --pos;
  }
  res[pos] = make_uint2(__float_as_uint(d), (uint32_t)node);
  ++size;
}

// ------------------------------------------------------------------ per-query driver
struct WarpCtx {
  float* q;      // [pitch]
  uint2* items;  // shared region (V1Merge array, or SearchOld closest heap + result set)
  int* nb_id;    // [nbpad]
  float* nb_d;   // [nbpad]
  float* sk;     // [nbpad]
  int* sv;       // [nbpad]
  float* stage;  // staged-gather rows (stage_rows x pitch), or null
  uint64_t* bar; // bulk row copies: the warp's mbarrier (after the staging rows), or null
  uint32_t phase;
  bool failed;   // a bulk copy did not complete within the wait bound
  int* htab;     // shared-memory visited table (open addressing, -1 = empty), or null
  uint8_t* vis;  // HBM epoch bytes of this warp's slot
  uint8_t epoch;
  int hshift;    // 32 - log2(table size)
  int hmask;     // table size - 1
  int hcount;    // ids in the table
  int hlimit;    // entries allowed before the query spills to the HBM epoch bytes
  bool spilled;
  int st_dist, st_expand, st_greedy;
  int64_t st_bytes;
};

// ------------------------------------------------------------------ visited set
// Exact membership: the shared-memory table holds the first hlimit visited ids of a query;
// after that the query "spills" and new ids go to the slot's HBM epoch bytes (the reference's
// VisitedList scheme, hnsw.h:568-590). An id is visited iff it is in the table or, once
// spilled, its epoch byte equals the query's epoch.
__device__ __forceinline__ uint32_t hslot(const WarpCtx& w, int id) {
  return ((uint32_t)id * 2654435761u) >> w.hshift;
}

// Inserts id; true if it was absent. The table always keeps a free slot (hcount <= hlimit <
// size), so the probe ends.
__device__ __forceinline__ bool hash_insert(const WarpCtx& w, int id) {
  uint32_t h = hslot(w, id);
  while (true) {
    const int old = atomicCAS(w.htab + h, -1, id);
    if (old == -1) return true;
    if (old == id) return false;
    h = (h + 1) & w.hmask;
  }
}

__device__ __forceinline__ bool hash_contains(const WarpCtx& w, int id) {
  uint32_t h = hslot(w, id);
  while (true) {
    const int v = w.htab[h];
    if (v == id) return true;
    if (v == -1) return false;
    h = (h + 1) & w.hmask;
  }
}

// Marks one id visited (lane 0 only); used for the level-0 entry point.
__device__ void visit_one(WarpCtx& w, int id) {
  if (w.htab) {
    if (lane_id() == 0) hash_insert(w, id);
    w.hcount += 1;
  } else if (lane_id() == 0) {
    w.vis[id] = w.epoch;
  }
  __syncwarp();
}

__device__ void load_query(const SearchArgs& a, float* qdst, int64_t qi) {
  const DevIndex& ix = a.ix;
  const int lane = lane_id();
  if (ix.dist_type == kSiftL2) {
    // 128 uint8 values, then their int sum of squares (the query object's norm,
    // space_l2sqr_sift.cc:137-150): exact in any order
    const uint32_t word = reinterpret_cast<const uint32_t*>(a.queries_u8 + qi * kSiftDim)[lane];
    reinterpret_cast<uint32_t*>(qdst)[lane] = word;
    int s = (int)__dp4a(word, word, 0u);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    if (lane == 0) reinterpret_cast<int*>(qdst)[kSiftDim / 4] = s;
    __syncwarp();
    return;
  }
  const float* src = a.queries + qi * ix.dim;
  // zero padding first (the permuted chunks read whole float4 / float2 groups)
  for (int e = lane; e < ix.pitch; e += 32) qdst[e] = 0.0f;
  __syncwarp();
  float s = 1.0f;
  bool scale = false;
  if (ix.dist_type == kNormCosine) {
    // hnsw.h:486-497, sequential and unfused
    if (lane == 0) {
      float sum = 0.0f;
      for (int e = 0; e < ix.dim; ++e) {
        const float v = src[e];
        sum = __fadd_rn(sum, __fmul_rn(v, v));
      }
      if (sum != 0.0f) {
        s = __fdiv_rn(1.0f, __fsqrt_rn(sum));
        scale = true;
      }
    }
    s = __shfl_sync(kFull, s, 0);
    scale = __shfl_sync(kFull, scale, 0);
  }
  for (int e = lane; e < ix.dim; e += 32) {
    float v = src[e];
    if (scale) v = __fmul_rn(v, s);
    qdst[permuted_pos(e, ix.dim)] = v;
  }
  __syncwarp();
}

// Reads a level-0 list (count and ids in one round of independent loads), marks its unvisited
// neighbours and gathers them, in list order, into w.nb_id. Returns how many were new; *cnt_out
// gets the list length. Duplicate ids inside one list count once (the first occurrence), as the
// reference's sequential visited check does (hnsw_distfunc_opt.cc:233-236).
__device__ int expand_list(WarpCtx& w, const int32_t* lst, int maxcnt, int* cnt_out) {
  const int lane = lane_id();
  int v[4];  // maxM0 <= 100 (validated at load) -> at most 4 chunks of 32
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int j = 32 * c + lane;
    v[c] = (j < maxcnt) ? __ldg(lst + 1 + j) : -1;
  }
  const int cnt = __ldg(lst);
  *cnt_out = cnt;
  int nnew = 0;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    if (32 * c >= cnt) break;
    const int j = 32 * c + lane;
    const int id = (j < cnt) ? v[c] : -1;
    const unsigned same = __match_any_sync(kFull, id);
    const bool cand = j < cnt && (__ffs(same) - 1) == lane;
    bool isnew = false;
    if (w.htab && !w.spilled) {
      if (w.hcount + __popc(__ballot_sync(kFull, cand)) > w.hlimit) w.spilled = true;
    }
    if (!w.htab) {
      if (cand) {
        isnew = w.vis[id] != w.epoch;
        if (isnew) w.vis[id] = w.epoch;
      }
    } else if (!w.spilled) {
      if (cand) isnew = hash_insert(w, id);
      w.hcount += __popc(__ballot_sync(kFull, isnew));
    } else if (cand && !hash_contains(w, id)) {
      isnew = w.vis[id] != w.epoch;
      if (isnew) w.vis[id] = w.epoch;
    }
    const unsigned m = __ballot_sync(kFull, isnew);
    if (isnew) w.nb_id[nnew + __popc(m & lanemask_lt())] = id;
    nnew += __popc(m);
    __syncwarp();
  }
  return nnew;
}

template <int G>
__device__ __forceinline__ void dists(const SearchArgs& a, WarpCtx& w, const int* ids, int n, float* out) {
  if (G == 0)
    compute_dists_staged(a.ix, w.q, ids, n, out, w.stage, a.stage_rows, w.bar, &w.phase, &w.failed);
  else
    compute_dists<(G > 0 ? G : 1)>(a.ix, w.q, ids, n, out);
}


template <int R>
__device__ void greedy_descent(const SearchArgs& a, WarpCtx& w, int& cur_out, float& dist_out) {
  const DevIndex& ix = a.ix;
  const int lane = lane_id();
  int cur = ix.enterpoint;
  if (lane == 0) w.nb_id[0] = cur;
  __syncwarp();
  compute_dists<(R == kLpGather || R == kSiftGather ? R : 1)>(ix, w.q, w.nb_id, 1, w.nb_d);
  float curdist = w.nb_d[0];
  w.st_dist += 1;
  w.st_bytes += ix.row_bytes;
  __syncwarp();
  for (int lev = ix.maxlevel; lev > 0; --lev) {
    bool changed = true;
    while (changed) {
      changed = false;
      const int32_t* lst = ix.up_links + ix.up_off[cur] + (int64_t)(ix.maxM + 1) * (lev - 1);
      const int cnt = __ldg(lst);
      for (int t = lane; t < cnt; t += 32) w.nb_id[t] = __ldg(lst + 1 + t);
      __syncwarp();
      dists<R>(a, w, w.nb_id, cnt, w.nb_d);
      w.st_greedy += 1;
      w.st_dist += cnt;
      w.st_bytes += 4LL * (1 + cnt) + (int64_t)ix.row_bytes * cnt;
      // sequential scan with strict improvement == earliest position of the minimum below curdist
      float best = curdist;
      int bpos = 0x7fffffff;
      for (int t = lane; t < cnt; t += 32) {
        const float d = w.nb_d[t];
        if (d < best || (d == best && d < curdist && t < bpos)) {
          best = d;
          bpos = t;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const float ob = __shfl_xor_sync(kFull, best, o);
        const int op = __shfl_xor_sync(kFull, bpos, o);
        if (ob < best || (ob == best && op < bpos)) {
          best = ob;
          bpos = op;
        }
      }
      if (bpos != 0x7fffffff && best < curdist) {
        cur = w.nb_id[bpos];
        curdist = best;
        changed = true;
      }
      __syncwarp();
    }
  }
  cur_out = cur;
  dist_out = curdist;
}


template <int R>
__device__ void search_v1merge(const SearchArgs& a, WarpCtx& w, int64_t qi, int k, int ef, int cur,
                               float curdist) {
  const DevIndex& ix = a.ix;
  const int lane = lane_id();
  const int cap = max(ef, k);
  uint2* items = w.items;
  int num = 1;
  if (lane == 0) items[0] = make_item(curdist, cur, false);
  visit_one(w, cur);
  int curr = 0;
  while (curr < min(num, ef)) {
    const uint2 e = items[curr];
    const int node = (int)(e.y & kIdMask);
    __syncwarp();
    if (lane == 0) items[curr].y = e.y | kUsedBit;
    __syncwarp();
    ++curr;
    const float top_key = key_of(items[num - 1]);
    const int size_now = num;
    // the next candidate in line is usually expanded next: start pulling its list into L2
    if (lane < 2 && curr < num) {
      const int nxt = (int)(items[curr].y & kIdMask);
      const int32_t* p = ix.l0 + (int64_t)nxt * ix.l0_pitch + 32 * lane;
      if (32 * lane < ix.l0_pitch) prefetch_l2(p);
    }
    const int32_t* lst = ix.l0 + (int64_t)node * ix.l0_pitch;
    int cnt;
    const int nnew = expand_list(w, lst, ix.maxM0, &cnt);
    w.st_expand += 1;
    w.st_bytes += 4LL * (1 + cnt);
    dists<R>(a, w, w.nb_id, nnew, w.nb_d);
    w.st_dist += nnew;
    w.st_bytes += (int64_t)ix.row_bytes * nnew;
    // keep d < topKey || size < ef, preserving list order
    int qty = 0;
    for (int base = 0; base < nnew; base += 32) {
      const int t = base + lane;
      bool keep = false;
      float d = 0.0f;
      int id = 0;
      if (t < nnew) {
        d = w.nb_d[t];
        id = w.nb_id[t];
        keep = (d < top_key) || (size_now < ef);
      }
      const unsigned m = __ballot_sync(kFull, keep);
      if (keep) {
        const int p = qty + __popc(m & lanemask_lt());
        w.sk[p] = d;
        w.sv[p] = id;
      }
      qty += __popc(m);
    }
    __syncwarp();
    if (qty) {
      int p0;
      if (merge_unsorted_batch(items, num, cap, w.sk, w.sv, qty, w.nb_d, w.nb_id, &p0)) {
        if (p0 < curr) curr = p0;
      } else {
        sort_like_std(w.sk, w.sv, qty, w.nb_d, w.nb_id);
        for (int i = 0; i < qty; ++i) {
          const int ins = sorted_insert(items, num, cap, w.sk[i], w.sv[i]);
          if (ins < curr) curr = ins;
        }
      }
    }
    // advance to the first unused item
    while (curr < num) {
      const int t = curr + lane;
      const bool unused = t < num && !(items[t].y & kUsedBit);
      const unsigned m = __ballot_sync(kFull, unused);
      if (m) {
        curr += __ffs(m) - 1;
        break;
      }
      curr += 32;
      if (curr > num) curr = num;
    }
    __syncwarp();
  }
  const int cnt = min(k, num);
  write_result_row(a, qi, items, cnt, false);
}

template <int R>
__device__ bool search_old(const SearchArgs& a, WarpCtx& w, int64_t qi, int k, int ef, int cur, float curdist,
                           uint2* cand) {
  const DevIndex& ix = a.ix;
  const int lane = lane_id();
  uint2* closest = w.items;               // ef + 1 entries
  uint2* res = w.items + (ef + 1);        // k entries
  int csize = 0, rsize = 0, qsize = 0;    // closest, result, candidate sizes (lane 0's copy)
  bool overflow = false;
  if (lane == 0) {
    heap_push(cand, qsize, -curdist, cur);
    heap_push(closest, csize, curdist, cur);
    result_offer(res, rsize, k, curdist, cur);
  }
  visit_one(w, cur);
  while (true) {
    int node = -1;
    if (lane == 0 && qsize > 0) {
      const uint2 top = cand[0];
      const float lb = key_of(closest[0]);
      if (!(-key_of(top) > lb)) {
        heap_pop(cand, qsize);
        node = (int)top.y;
      }
    }
    node = __shfl_sync(kFull, node, 0);
    if (node < 0) break;
    const int32_t* lst = ix.l0 + (int64_t)node * ix.l0_pitch;
    int cnt;
    const int nnew = expand_list(w, lst, ix.maxM0, &cnt);
    w.st_expand += 1;
    w.st_bytes += 4LL * (1 + cnt);
    dists<R>(a, w, w.nb_id, nnew, w.nb_d);
    w.st_dist += nnew;
    w.st_bytes += (int64_t)ix.row_bytes * nnew;
    if (lane == 0) {
      for (int t = 0; t < nnew; ++t) {
        const float d = w.nb_d[t];
        const int id = w.nb_id[t];
        if (key_of(closest[0]) > d || csize < ef) {
          if (qsize >= a.old_heap_cap) {
            overflow = true;
            break;
          }
          heap_push(cand, qsize, -d, id);
          result_offer(res, rsize, k, d, id);
          heap_push(closest, csize, d, id);
          if (csize > ef) heap_pop(closest, csize);
        }
      }
    }
    overflow = __shfl_sync(kFull, overflow, 0);
    __syncwarp();
    if (overflow) break;
  }
  rsize = __shfl_sync(kFull, rsize, 0);
  if (overflow) {
    set_status(a.status, NMSG_ERR_CAPACITY);
    rsize = 0;
  }
  write_result_row(a, qi, res, rsize, true);
  return !overflow;
}

// bar_phase: the warp's bulk-copy mbarrier phase, kept across its queries; kBarUninit before the
// warp's first query, which initialises the mbarrier (once per warp: it is never re-initialised
// while the warp runs).
constexpr uint32_t kBarUninit = 2;

template <int R, bool OLD>
__device__ void run_query(const SearchArgs& a, char* wsmem, int slot, int64_t qi, uint32_t& bar_phase) {
  const DevIndex& ix = a.ix;
  const int lane = lane_id();
  WarpCtx w;
  w.q = reinterpret_cast<float*>(wsmem);
  w.items = reinterpret_cast<uint2*>(w.q + ix.pitch);
  w.nb_id = reinterpret_cast<int*>(w.items + a.region_items);
  w.nb_d = reinterpret_cast<float*>(w.nb_id + a.nbpad);
  w.sk = w.nb_d + a.nbpad;
  w.sv = reinterpret_cast<int*>(w.sk + a.nbpad);
  w.vis = a.visited + (int64_t)slot * a.visited_pitch;
  w.st_dist = w.st_expand = w.st_greedy = 0;
  w.st_bytes = 0;
  w.htab = nullptr;
  w.hcount = 0;
  w.spilled = false;
  char* tail = reinterpret_cast<char*>(w.sv + a.nbpad);
  if (a.hash_log2 > 0) {
    const int size = 1 << a.hash_log2;
    w.htab = reinterpret_cast<int*>(tail);
    tail += 4 * size;
    w.hshift = 32 - a.hash_log2;
    w.hmask = size - 1;
    w.hlimit = size - size / 4 - 32;
    for (int t = lane; t < size; t += 32) w.htab[t] = -1;
    __syncwarp();
  }
  w.stage = reinterpret_cast<float*>(tail);
  w.bar = nullptr;
  w.phase = 0;
  w.failed = false;
  if (a.bulk_rows && a.stage_rows > 0) {
    w.bar = reinterpret_cast<uint64_t*>(w.stage + (size_t)a.stage_rows * ix.pitch);
    if (bar_phase == kBarUninit) {
      if (lane == 0) {
        sm100::mbar_init(w.bar, 1);
        sm100::fence_barrier_init();
      }
      __syncwarp();
      bar_phase = 0;
    }
    w.phase = bar_phase;
  }

  // next epoch of this slot's visited array; clear it when the byte wraps (hnsw.h:582-589). The
  // descent pass of a split search touches no visited set.
  int ep = 0;
  if (a.split != 1) {
    if (lane == 0) ep = a.epochs[slot] + 1;
    ep = __shfl_sync(kFull, ep, 0);
    if (ep == 256) {
      uint4* p = reinterpret_cast<uint4*>(w.vis);
      const int64_t n16 = a.visited_pitch / 16;
      for (int64_t t = lane; t < n16; t += 32) p[t] = make_uint4(0, 0, 0, 0);
      ep = 1;
      __syncwarp();
    }
    if (lane == 0) a.epochs[slot] = (uint8_t)ep;
  }
  w.epoch = (uint8_t)ep;

  const int k = a.k_per_q ? a.k_per_q[qi] : a.k_default;
  const int ef = a.ef_per_q ? a.ef_per_q[qi] : a.ef_default;
  load_query(a, w.q, qi);
  int cur;
  float curdist;
  bool search = true;
  if (a.split == 2) {  // level 0 from where the descent pass ended, with its counts
    cur = __ldg(a.entry_node + qi);
    curdist = __ldg(a.entry_dist + qi);
    w.st_dist = __ldg(a.entry_stats + 3 * qi + 0);
    w.st_greedy = __ldg(a.entry_stats + 3 * qi + 1);
    w.st_bytes = __ldg(a.entry_stats + 3 * qi + 2);
    if (cur < 0 || cur >= ix.n) {  // the descent pass gave up on this query
      search = false;
      w.failed = true;
    }
  } else {
    greedy_descent<R>(a, w, cur, curdist);
    if (a.split == 1) {  // the descent pass: where level 0 starts and the key it is ordered by
      if (lane == 0 && !w.failed) {
        a.entry_node[qi] = cur;
        a.entry_dist[qi] = curdist;
        a.entry_stats[3 * qi + 0] = w.st_dist;
        a.entry_stats[3 * qi + 1] = w.st_greedy;
        a.entry_stats[3 * qi + 2] = (int32_t)w.st_bytes;
        const uint32_t key = ordered_key(curdist);
        atomicMin(a.entry_range + 0, key);
        atomicMax(a.entry_range + 1, key);
      }
      search = false;
    }
  }
  if (search) {
    const bool use_old = a.algo == NMSG_ALGO_OLD || (a.algo == NMSG_ALGO_HYBRID && ef >= 1000);
    if (OLD && use_old) {
      search_old<R>(a, w, qi, k, ef, cur, curdist, a.old_heap + (int64_t)slot * a.old_heap_cap);
    } else {
      search_v1merge<R>(a, w, qi, k, ef, cur, curdist);
    }
  }
  bar_phase = w.phase;
  if (w.failed && lane == 0) {  // a row copy gave up: the query's results are not trusted
    set_status(a.status, NMSG_ERR_TIMEOUT);
    a.counts[qi] = 0;
  }
  if (a.stats && lane == 0 && a.split != 1) {
    a.stats[qi * 4 + 0] = w.st_dist;
    a.stats[qi * 4 + 1] = w.st_expand;
    a.stats[qi * 4 + 2] = w.st_greedy;
    a.stats[qi * 4 + 3] = w.st_bytes;
  }
  __syncwarp();
}

// Persistent kernel: each warp owns one slot and pulls queries from a work counter.
template <int R, bool OLD>
__global__ void __launch_bounds__(128, 8) search_batched_kernel(SearchArgs a) {
  extern __shared__ __align__(16) char smem[];
  const int warp = threadIdx.x >> 5;
  const int lane = lane_id();
  char* wsmem = smem + warp * a.warp_smem;
  const int slot = blockIdx.x * (blockDim.x >> 5) + warp;
  if (slot >= a.num_slots) return;
  uint32_t bar_phase = kBarUninit;
  while (true) {
    int item = 0;
    if (lane == 0) item = atomicAdd(a.work_counter, 1);
    item = __shfl_sync(kFull, item, 0);
    if (item >= a.nq) break;
    const int64_t qi = a.order ? a.order[item] : item;
    run_query<R, OLD>(a, wsmem, slot, qi, bar_phase);
  }
}

// One query per block of one warp; a free slot is taken from the slot locks for the duration.
template <int R, bool OLD>
__global__ void __launch_bounds__(32, 32) search_plain_kernel(SearchArgs a) {
  extern __shared__ __align__(16) char smem[];
  const int lane = lane_id();
  const int64_t qi = blockIdx.x;
  int slot = -1;
  if (lane == 0) {
    // at most num_slots blocks are resident, so one pass over the locks finds a free slot
    for (int t = 0; t < 2 * a.num_slots && slot < 0; ++t) {
      const int s = (int)((blockIdx.x + t) % a.num_slots);
      if (atomicCAS(a.slot_locks + s, 0, 1) == 0) slot = s;
    }
    __threadfence();
  }
  slot = __shfl_sync(kFull, slot, 0);
  if (slot < 0) {
    if (lane == 0) {
      set_status(a.status, NMSG_ERR_TIMEOUT);
      a.counts[qi] = 0;
    }
    return;
  }
  uint32_t bar_phase = kBarUninit;
  run_query<R, OLD>(a, smem, slot, qi, bar_phase);
  __threadfence();
  if (lane == 0) atomicExch(a.slot_locks + slot, 0);
}

// ------------------------------------------------------------------ several queries per warp
// search_multi_kernel<C, NCH>: a persistent warp owns C query contexts (C visited slots) and moves
// every active one by one step per loop iteration. A step is exactly one step of the
// single-query code above: the entry point's distance, one greedy-descent list at one level, or
// one SearchV1Merge expansion (pop, list, visited check, distances, filter, merge, advance). Each
// context therefore takes the same steps in the same order as a warp that owned it alone, and
// its results and per-query counts are the same bit for bit. What changes is the overlap: the
// contexts' list reads, then their visited-byte reads, then all their new rows (one shared
// staging area, rounds of stage_rows asynchronous copies) are issued together, so C dependent
// chains are in flight per warp for about the registers of one, and a small batch fills the GPU
// in one wave. V1Merge only, float rows through shared memory, lists of up to 32 * NCH ids.

struct MultiCtx {  // lane-uniform state of one context (shared memory; lane 0 writes)
  int64_t qi;
  int mode;        // kIdle, kEntry, kGreedy, kBeam
  int k, ef;
  int level, cur;  // greedy descent
  float curdist;
  int curr, num;   // level-0 beam (SortArrBI state)
  float top_key;   // the expansion's topKey and size (hnsw_distfunc_opt.cc:216-222)
  int size_now;
  int cnt, nnew;
  int st_dist, st_expand, st_greedy, st_list_ints;
  int epoch;
  int steps;       // steps taken; bounded (see multi_step_bound)
};
static_assert(sizeof(MultiCtx) % 16 == 0, "context state keeps 16-byte alignment");
enum { kIdle = 0, kEntry = 1, kGreedy = 2, kBeam = 3 };

__host__ __device__ inline int multi_ctx_bytes(const DevIndex& ix, int region_items, int nbpad) {
  return ((ix.pitch * 4 + region_items * 8 + nbpad * 16 + (int)sizeof(MultiCtx)) + 15) & ~15;
}

// No query takes more steps than this: every level-0 expansion pops a node that was inserted
// once (at most n), and each level of the descent moves at most n times before it drops a level.
// A context past it has met a broken invariant; it stops with NMSG_ERR_TIMEOUT instead of looping.
__device__ __forceinline__ int64_t multi_step_bound(const DevIndex& ix) {
  return ix.n + (int64_t)(ix.maxlevel + 1) * (ix.n + 1) + 4;
}

struct MultiView {  // one context's shared-memory pieces
  float* q;
  uint2* items;
  int* nb_id;
  float* nb_d;
  float* sk;
  int* sv;
  MultiCtx* st;
};

__device__ __forceinline__ MultiView multi_view(const SearchArgs& a, char* base, int c) {
  MultiView v;
  char* p = base + (size_t)c * multi_ctx_bytes(a.ix, a.region_items, a.nbpad);
  v.q = reinterpret_cast<float*>(p);
  v.items = reinterpret_cast<uint2*>(v.q + a.ix.pitch);
  v.nb_id = reinterpret_cast<int*>(v.items + a.region_items);
  v.nb_d = reinterpret_cast<float*>(v.nb_id + a.nbpad);
  v.sk = v.nb_d + a.nbpad;
  v.sv = reinterpret_cast<int*>(v.sk + a.nbpad);
  v.st = reinterpret_cast<MultiCtx*>(v.sv + a.nbpad);
  return v;
}

// Distance from the query (shared memory, permuted) to one staged row, by the 8 lanes of a group
// (every lane of the warp takes part: combine shuffles across the whole warp).
__device__ __forceinline__ float staged_row_dist(const DevIndex& ix, const float* __restrict__ q,
                                                 const float* __restrict__ row) {
  const int j = lane_id() & 7;
  const int nfull = ix.n16 >> 5;
  const int code = ix.dist_type;
  float acc = 0.0f;
#pragma unroll 4
  for (int c = 0; c < nfull; ++c) {
    const float4 qv = reinterpret_cast<const float4*>(q + c * 32)[j];
    const float4 x = reinterpret_cast<const float4*>(row + c * 32)[j];
    acc = fma_term(code, qv.x, x.x, acc);
    acc = fma_term(code, qv.y, x.y, acc);
    acc = fma_term(code, qv.z, x.z, acc);
    acc = fma_term(code, qv.w, x.w, acc);
  }
  if (ix.n16 & 31) {
    const float2 qv = reinterpret_cast<const float2*>(q + nfull * 32)[j];
    const float2 x = reinterpret_cast<const float2*>(row + nfull * 32)[j];
    acc = fma_term(code, qv.x, x.x, acc);
    acc = fma_term(code, qv.y, x.y, acc);
  }
  return combine(ix, acc, row, q);
}

// Starts query `item` of the work list in a context: parameters, the slot's next epoch (the
// visited bytes are cleared when the byte wraps, hnsw.h:582-589) and the query vector.
__device__ void multi_start(const SearchArgs& a, const MultiView& v, int slot, int item) {
  const int lane = lane_id();
  const int64_t qi = a.order ? a.order[item] : item;
  int ep = 0;
  if (lane == 0) ep = a.epochs[slot] + 1;
  ep = __shfl_sync(kFull, ep, 0);
  if (ep == 256) {
    uint4* p = reinterpret_cast<uint4*>(a.visited + (int64_t)slot * a.visited_pitch);
    const int64_t n16 = a.visited_pitch / 16;
    for (int64_t t = lane; t < n16; t += 32) p[t] = make_uint4(0, 0, 0, 0);
    ep = 1;
  }
  load_query(a, v.q, qi);
  if (lane == 0) {
    a.epochs[slot] = (uint8_t)ep;
    MultiCtx& st = *v.st;
    st.qi = qi;
    st.mode = kEntry;
    st.k = a.k_per_q ? a.k_per_q[qi] : a.k_default;
    st.ef = a.ef_per_q ? a.ef_per_q[qi] : a.ef_default;
    st.epoch = ep;
    st.steps = 0;
    st.st_dist = st.st_expand = st.st_greedy = st.st_list_ints = 0;
  }
  __syncwarp();
}

// The context reached level 0: the beam starts from the descent's result (hnsw_distfunc_opt.cc:
// 200-214); a beam that has nothing to expand (efSearch 0) finishes at once.
__device__ void multi_beam_init(const SearchArgs& a, const MultiView& v, int slot) {
  MultiCtx& st = *v.st;
  if (lane_id() == 0) {
    v.items[0] = make_item(st.curdist, st.cur, false);
    a.visited[(int64_t)slot * a.visited_pitch + st.cur] = (uint8_t)st.epoch;
    st.num = 1;
    st.curr = 0;
    st.mode = kBeam;
  }
  __syncwarp();
}

__device__ void multi_finish(const SearchArgs& a, const MultiView& v, bool ok) {
  MultiCtx& st = *v.st;
  const int64_t qi = st.qi;
  write_result_row(a, qi, v.items, ok ? min(st.k, st.num) : 0, false);
  if (a.stats && lane_id() == 0) {
    a.stats[qi * 4 + 0] = st.st_dist;
    a.stats[qi * 4 + 1] = st.st_expand;
    a.stats[qi * 4 + 2] = st.st_greedy;
    a.stats[qi * 4 + 3] = (int64_t)a.ix.row_bytes * st.st_dist + 4LL * st.st_list_ints;
  }
  __syncwarp();
  if (lane_id() == 0) {
    if (!ok) set_status(a.status, NMSG_ERR_TIMEOUT);
    st.mode = kIdle;
  }
  __syncwarp();
}

template <int C, int NCH>
__global__ void __launch_bounds__(128, 8) search_multi_kernel(SearchArgs a) {
  extern __shared__ __align__(16) char smem[];
  const DevIndex& ix = a.ix;
  const int warp = threadIdx.x >> 5, lane = lane_id();
  const int g = lane >> 3;
  char* wbase = smem + warp * a.warp_smem;
  const int wslot = blockIdx.x * (blockDim.x >> 5) + warp;
  if ((wslot + 1) * C > a.num_slots) return;
  float* stage = reinterpret_cast<float*>(wbase + (size_t)C * multi_ctx_bytes(ix, a.region_items, a.nbpad));
  // bulk row copies complete on this warp's mbarrier (after the staging rows)
  uint64_t* row_bar = reinterpret_cast<uint64_t*>(stage + (size_t)a.stage_rows * ix.pitch);
  uint32_t row_phase = 0;
  const uint32_t row_bytes = (uint32_t)bulk_row_bytes(ix);
  if (a.bulk_rows) {
    if (lane == 0) {
      sm100::mbar_init(row_bar, 1);
      sm100::fence_barrier_init();
    }
    __syncwarp();
  }
  // a context's pieces are recomputed where they are used (a few integer operations) rather than
  // kept in registers for the whole loop
  auto V = [&](int c) { return multi_view(a, wbase, c); };
#pragma unroll
  for (int c = 0; c < C; ++c)
    if (lane == 0) V(c).st->mode = kIdle;
  __syncwarp();
  bool drained = false;
  const int nf4 = (ix.dim + 3) >> 2;  // 16-byte pieces of a row
  const int64_t step_bound = multi_step_bound(ix);
  while (true) {
    // ---- refill idle contexts from the work counter
    unsigned active = 0;
#pragma unroll
    for (int c = 0; c < C; ++c) {
      if (V(c).st->mode == kIdle && !drained) {
        int item = 0;
        if (lane == 0) item = atomicAdd(a.work_counter, 1);
        item = __shfl_sync(kFull, item, 0);
        if (item < a.nq)
          multi_start(a, V(c), wslot * C + c, item);
        else
          drained = true;
      }
      if (V(c).st->mode != kIdle) active |= 1u << c;
    }
    if (!active) break;

    // ---- lists: issue every context's list read before using any of them
    int lv[C][NCH], lcnt[C];
#pragma unroll
    for (int c = 0; c < C; ++c) {
      const MultiCtx& st = *V(c).st;
      const int mode = st.mode;
      const int32_t* lst = nullptr;
      int maxcnt = 0;
      if (mode == kGreedy) {
        lst = ix.up_links + __ldg(ix.up_off + st.cur) + (int64_t)(ix.maxM + 1) * (st.level - 1);
        maxcnt = ix.maxM;
      } else if (mode == kBeam) {
        const uint2 e = V(c).items[st.curr];
        const int node = (int)(e.y & kIdMask);
        lst = ix.l0 + (int64_t)node * ix.l0_pitch;
        maxcnt = ix.maxM0;
      }
#pragma unroll
      for (int h = 0; h < NCH; ++h) {
        const int t = 32 * h + lane;
        lv[c][h] = (lst && t < maxcnt) ? __ldg(lst + 1 + t) : -1;
      }
      lcnt[c] = lst ? __ldg(lst) : 0;
    }
    // beam contexts: mark the popped item used, note topKey and the size (hnsw_distfunc_opt.cc:
    // 212-222); the next candidate's list is pulled into L2 (it is usually expanded next)
#pragma unroll
    for (int c = 0; c < C; ++c) {
      MultiCtx& st = *V(c).st;
      if (st.mode == kBeam) {
        const int curr = st.curr;
        const int num = st.num;
        if (lane == 0) {
          V(c).items[curr].y |= kUsedBit;
          st.curr = curr + 1;
          st.top_key = key_of(V(c).items[num - 1]);
          st.size_now = num;
        }
        if (lane < 2 && curr + 1 < num) {
          const int nxt = (int)(V(c).items[curr + 1].y & kIdMask);
          const int32_t* p = ix.l0 + (int64_t)nxt * ix.l0_pitch + 32 * lane;
          if (32 * lane < ix.l0_pitch) prefetch_l2(p);
        }
      }
    }
    __syncwarp();
    // ---- new neighbours: greedy lists are taken whole; beam lists go through the visited set,
    // 32 entries at a time in list order (duplicates inside a list count once, as the reference's
    // sequential check does), every context's visited bytes read before any is marked
    int nnew[C];
#pragma unroll
    for (int c = 0; c < C; ++c) {
      nnew[c] = 0;
      const int mode = V(c).st->mode;
      if (mode == kEntry) {
        if (lane == 0) V(c).nb_id[0] = ix.enterpoint;
        nnew[c] = 1;
      } else if (mode == kGreedy) {
#pragma unroll
        for (int h = 0; h < NCH; ++h)
          if (32 * h + lane < lcnt[c]) V(c).nb_id[32 * h + lane] = lv[c][h];
        nnew[c] = lcnt[c];
      }
    }
#pragma unroll
    for (int h = 0; h < NCH; ++h) {
      uint8_t vb[C];
      bool cand[C];
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const MultiCtx& st = *V(c).st;
        cand[c] = false;
        vb[c] = 0;
        if (st.mode == kBeam && 32 * h < lcnt[c]) {
          const int t = 32 * h + lane;
          const int id = t < lcnt[c] ? lv[c][h] : -1;
          const unsigned same = __match_any_sync(kFull, id);
          cand[c] = t < lcnt[c] && (__ffs(same) - 1) == lane;
          if (cand[c]) vb[c] = a.visited[(int64_t)(wslot * C + c) * a.visited_pitch + id];
        }
      }
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const MultiCtx& st = *V(c).st;
        if (st.mode == kBeam && 32 * h < lcnt[c]) {
          const int id = lv[c][h];
          const bool isnew = cand[c] && vb[c] != (uint8_t)st.epoch;
          if (isnew) a.visited[(int64_t)(wslot * C + c) * a.visited_pitch + id] = (uint8_t)st.epoch;
          const unsigned m = __ballot_sync(kFull, isnew);
          if (isnew) V(c).nb_id[nnew[c] + __popc(m & lanemask_lt())] = id;
          nnew[c] += __popc(m);
        }
      }
      __syncwarp();  // this chunk's marks are seen by the next chunk's reads (an id listed twice)
    }
    // ---- distances: every context's new rows through the staging area
    int off[C + 1];
    off[0] = 0;
#pragma unroll
    for (int c = 0; c < C; ++c) off[c + 1] = off[c] + nnew[c];
    const int total = off[C];
    for (int base = 0; base < total; base += a.stage_rows) {
      const int cnt = min(a.stage_rows, total - base);
      // lane r < cnt finds row r's vector, then the warp copies the rows one after another
      const float* src_mine = ix.vecs;
      if (lane < cnt) {
        const int gr = base + lane;
        int id = 0;
#pragma unroll
        for (int c = 0; c < C; ++c)
          if (gr >= off[c] && gr < off[c + 1]) id = V(c).nb_id[gr - off[c]];
        src_mine = ix.vecs + (int64_t)id * ix.pitch;
      }
      if (a.bulk_rows) {
        // one bulk copy per row, issued by the lane that looked the row up; the staging rows' last
        // reads (the previous round) are ordered before the copies that overwrite them
        if (lane == 0) sm100::mbar_arrive_expect_tx(row_bar, (uint32_t)cnt * row_bytes);
        __syncwarp();
        if (lane < cnt) {
          sm100::fence_proxy_async_smem();
          sm100::bulk_copy_g2s(stage + lane * ix.pitch, src_mine, row_bytes, row_bar);
        }
        const bool ok = sm100::mbar_wait(row_bar, row_phase);
        row_phase ^= 1;
        if (!ok) {
          // the copies did not complete within the bound: report it and end this warp's work
          // after waiting (bounded) once more, so no copy is left writing shared memory
          if (lane == 0) set_status(a.status, NMSG_ERR_TIMEOUT);
          sm100::mbar_wait(row_bar, row_phase ^ 1);
          return;
        }
      } else {
        for (int r = 0; r < cnt; ++r) {
          const float* src = reinterpret_cast<const float*>(
              __shfl_sync(kFull, reinterpret_cast<unsigned long long>(src_mine), r));
          float* dst = stage + r * ix.pitch;
          for (int f = lane; f < nf4; f += 32) cp_async16(dst + 4 * f, src + 4 * f);
        }
        cp_async_wait_all();
      }
      __syncwarp();
      for (int r0 = 0; r0 < cnt; r0 += 4) {
        const int r = r0 + g;
        const bool act = r < cnt;
        const int gr = base + (act ? r : 0);
        int cc = 0;
#pragma unroll
        for (int c = 1; c < C; ++c)
          if (gr >= off[c]) cc = c;
        const float* q = V(0).q;
        float* out = V(0).nb_d;
#pragma unroll
        for (int c = 1; c < C; ++c)
          if (cc == c) {
            q = V(c).q;
            out = V(c).nb_d;
          }
        const float d = staged_row_dist(ix, q, stage + (act ? r : 0) * ix.pitch);
        if (act && (lane & 7) == 0) out[gr - off[cc]] = d;
      }
      __syncwarp();
    }
    // ---- per context: what the step's distances mean
#pragma unroll
    for (int c = 0; c < C; ++c) {
      MultiCtx& st = *V(c).st;
      const int mode = st.mode;
      if (mode == kEntry) {
        const float d0 = V(c).nb_d[0];
        __syncwarp();
        if (lane == 0) {
          st.cur = ix.enterpoint;
          st.curdist = d0;
          st.st_dist += 1;
          st.level = ix.maxlevel;
          st.mode = kGreedy;
        }
        __syncwarp();
        if (ix.maxlevel == 0) multi_beam_init(a, V(c), wslot * C + c);
      } else if (mode == kGreedy) {
        // hnsw_distfunc_opt.cc:168-198: the earliest strictly smaller distance of the list wins
        const int cnt = lcnt[c];
        const float curdist = st.curdist;
        float best = curdist;
        int bpos = 0x7fffffff;
        for (int t = lane; t < cnt; t += 32) {
          const float d = V(c).nb_d[t];
          if (d < best || (d == best && d < curdist && t < bpos)) {
            best = d;
            bpos = t;
          }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const float ob = __shfl_xor_sync(kFull, best, o);
          const int op = __shfl_xor_sync(kFull, bpos, o);
          if (ob < best || (ob == best && op < bpos)) {
            best = ob;
            bpos = op;
          }
        }
        const bool moved = bpos != 0x7fffffff && best < curdist;
        const int next = moved ? V(c).nb_id[bpos] : 0;
        __syncwarp();
        if (lane == 0) {
          st.st_greedy += 1;
          st.st_dist += cnt;
          st.st_list_ints += 1 + cnt;
          if (moved) {
            st.cur = next;
            st.curdist = best;
          } else {
            st.level -= 1;
          }
        }
        __syncwarp();
        if (!moved && st.level == 0) multi_beam_init(a, V(c), wslot * C + c);
      } else if (mode == kBeam) {
        const float top_key = st.top_key;
        const int size_now = st.size_now, ef = st.ef, k = st.k;
        const int n_new = nnew[c];
        // keep d < topKey || size < ef, preserving list order (hnsw_distfunc_opt.cc:237-247)
        int qty = 0;
        for (int b0 = 0; b0 < n_new; b0 += 32) {
          const int t = b0 + lane;
          bool keep = false;
          float d = 0.0f;
          int id = 0;
          if (t < n_new) {
            d = V(c).nb_d[t];
            id = V(c).nb_id[t];
            keep = (d < top_key) || (size_now < ef);
          }
          const unsigned m = __ballot_sync(kFull, keep);
          if (keep) {
            const int p = qty + __popc(m & lanemask_lt());
            V(c).sk[p] = d;
            V(c).sv[p] = id;
          }
          qty += __popc(m);
        }
        __syncwarp();
        int num = st.num, curr = st.curr;
        const int cap = max(ef, k);
        if (qty) {
          int p0;
          if (merge_unsorted_batch(V(c).items, num, cap, V(c).sk, V(c).sv, qty, V(c).nb_d, V(c).nb_id, &p0)) {
            if (p0 < curr) curr = p0;
          } else {
            sort_like_std(V(c).sk, V(c).sv, qty, V(c).nb_d, V(c).nb_id);
            for (int i = 0; i < qty; ++i) {
              const int ins = sorted_insert(V(c).items, num, cap, V(c).sk[i], V(c).sv[i]);
              if (ins < curr) curr = ins;
            }
          }
        }
        // advance to the first unused item
        while (curr < num) {
          const int t = curr + lane;
          const bool unused = t < num && !(V(c).items[t].y & kUsedBit);
          const unsigned m = __ballot_sync(kFull, unused);
          if (m) {
            curr += __ffs(m) - 1;
            break;
          }
          curr += 32;
          if (curr > num) curr = num;
        }
        __syncwarp();
        if (lane == 0) {
          st.st_expand += 1;
          st.st_dist += n_new;
          st.st_list_ints += 1 + lcnt[c];
          st.num = num;
          st.curr = curr;
        }
        __syncwarp();
      }
      if (mode != kIdle) {
        if (lane == 0) st.steps += 1;
        __syncwarp();
        if (st.mode == kBeam && !(st.curr < min(st.num, st.ef)))
          multi_finish(a, V(c), true);
        else if (st.mode != kIdle && st.steps > step_bound)
          multi_finish(a, V(c), false);
      }
    }
  }
}

// ------------------------------------------------------------------ exact scan on CUDA cores
// Exact k-NN (SeqSearch semantics, similarity_search/src/method/seqsearch.cc:143-177) for what the
// tensor-core brute force does not take: L1 / LInf and rows wider than 256. A block owns kTileQ
// queries and one chunk of base rows; every distance is computed with the query path's own
// arithmetic (so it is the value the HNSW search reports), each warp keeps a best-k list by
// (distance, row) per query, and scan_merge_kernel merges the lists.

__device__ __forceinline__ bool scan_better(float da, int ia, float db, int ib) {
  return da < db || (da == db && ia < ib);
}

// Offers (d, row) to the warp's sorted list (lane i < k holds the i-th best); warp-uniform inputs.
__device__ __forceinline__ void scan_offer(float& bd, int& bi, int k, float d, int row) {
  const int lane = lane_id();
  const float kd = __shfl_sync(kFull, bd, k - 1);
  const int ki = __shfl_sync(kFull, bi, k - 1);
  if (!scan_better(d, row, kd, ki)) return;
  const int pos = __popc(__ballot_sync(kFull, lane < k && scan_better(bd, bi, d, row)));
  const float ud = __shfl_up_sync(kFull, bd, 1);
  const int ui = __shfl_up_sync(kFull, bi, 1);
  if (lane > pos && lane < k) {
    bd = ud;
    bi = ui;
  } else if (lane == pos) {
    bd = d;
    bi = row;
  }
}

// One warp writes query qi (zeros when !valid) into q[pitch] in the permuted layout, normalised
// for cosine as the search normalises it.
__device__ void scan_load_query(const DevIndex& ix, const float* __restrict__ queries, int64_t qi, bool valid,
                                float* q) {
  const int lane = lane_id();
  for (int e = lane; e < ix.pitch; e += 32) q[e] = 0.0f;
  __syncwarp();
  if (valid) {
    const float* src = queries + qi * ix.dim;
    float s = 1.0f;
    bool scale = false;
    if (ix.dist_type == kNormCosine) {
      if (lane == 0) {
        float sum = 0.0f;
        for (int e = 0; e < ix.dim; ++e) sum = __fadd_rn(sum, __fmul_rn(src[e], src[e]));
        if (sum != 0.0f) {
          s = __fdiv_rn(1.0f, __fsqrt_rn(sum));
          scale = true;
        }
      }
      s = __shfl_sync(kFull, s, 0);
      scale = __shfl_sync(kFull, scale, 0);
    }
    for (int e = lane; e < ix.dim; e += 32) {
      float v = src[e];
      if (scale) v = __fmul_rn(v, s);
      q[permuted_pos(e, ix.dim)] = v;
    }
  }
  __syncwarp();
}

struct ScanArgs {
  DevIndex ix;
  const float* queries;  // [nq][dim]
  int64_t nq;
  int k;                 // <= 32
  int64_t chunk_rows;
  int n_chunks;
  float* part_d;         // [nq][n_chunks * kTileWarps][k]
  int32_t* part_id;
};

// The fused-multiply-add codes (squared L2, cosine, negative dot), register tiled: a block holds kTileQ queries in shared memory and its warps split the chunk's rows, each
// 8-lane group taking kTileR rows at a time, streamed through a per-warp ring of asynchronous
// 16-byte copies kTileStages blocks deep (each lane copies exactly the pieces it reads, so a lane
// waits only for its own copies). Lane j of a group keeps
// one accumulator per (row, query) pair and adds the same elements in the same order as the
// search's lane j (elements 4j..4j+3 of every 32-element block, then 2j..2j+1 of the 16-element
// block), and combine() finishes each pair as the search does, so every distance is the search's
// value bit for bit. A pass costs 12 shared-memory 16-byte loads and 4 asynchronous copies per
// 128 FMAs, against 2 loads per 4 FMAs when a warp owns one query. Each warp keeps its own best-k list per query in
// shared memory (offers are rare once the list fills; the k-th sits in a register).
constexpr int kTileQ = 8;
constexpr int kTileR = 4;
constexpr int kTileWarps = 8;
static_assert(kTileQ == kTileWarps, "one warp loads each query");
static_assert(kTileQ <= 32, "one lane holds each query's k-th");
constexpr int kTileStages = 3;                       // blocks of rows in flight per warp
constexpr int kTileStage = 4 * kTileR * 32;          // floats per stage: the warp's 16 rows x 32
constexpr int kTileRing = kTileStages * kTileStage > kTileR * kTileQ * 32 ? kTileStages * kTileStage
                                                                          : kTileR * kTileQ * 32;
constexpr int kTileWarpSmem = kTileRing + 2 * kTileQ * 32;  // floats per warp

template <bool kSub>
__device__ __forceinline__ float tile_term(float a, float b, float acc) {
  if constexpr (kSub) {
    const float d = __fsub_rn(a, b);
    return __fmaf_rn(d, d, acc);
  } else {
    return __fmaf_rn(a, b, acc);
  }
}

template <bool kSub>
__global__ void __launch_bounds__(32 * kTileWarps, 2) exact_scan_tiled_kernel(ScanArgs a) {
  extern __shared__ __align__(16) float scan_smem[];
  const DevIndex& ix = a.ix;
  const int warp = threadIdx.x >> 5, lane = lane_id(), g = lane >> 3, j = lane & 7;
  const int64_t q0 = (int64_t)blockIdx.x * kTileQ;
  const int nq_here = (int)min((int64_t)kTileQ, a.nq - q0);
  scan_load_query(ix, a.queries, q0 + warp, warp < nq_here, scan_smem + (size_t)warp * ix.pitch);
  __syncthreads();
  const float* qs = scan_smem;  // [kTileQ][pitch]
  // per warp: the row ring [kTileStages][16 rows][32], which also holds the pass's parked lane
  // partials [kTileR * kTileQ][32] once it has drained, then its best-k lists [kTileQ][32]
  float* part = scan_smem + (size_t)kTileQ * ix.pitch + (size_t)warp * kTileWarpSmem;
  float* list_d = part + kTileRing;
  int* list_i = reinterpret_cast<int*>(list_d + kTileQ * 32);
  for (int i = lane; i < kTileQ * 32; i += 32) {
    list_d[i] = INFINITY;
    list_i[i] = 0x7fffffff;
  }
  // lane qq < kTileQ holds query qq's current k-th (distance, row)
  float kth_d = INFINITY;
  int kth_i = 0x7fffffff;
  const int nfull = ix.n16 >> 5;
  const bool half = (ix.n16 & 31) != 0;
  constexpr int kWarpRows = 4 * kTileR;  // rows a warp takes per pass
  const int64_t r0 = (int64_t)blockIdx.y * a.chunk_rows, r1 = min(ix.n, r0 + a.chunk_rows);
  for (int64_t wb = r0 + (int64_t)warp * kWarpRows; wb < r1; wb += (int64_t)kTileWarps * kWarpRows) {
    // rows past the chunk's end read its last row and are never offered
    const float* rp[kTileR];
#pragma unroll
    for (int r = 0; r < kTileR; ++r) rp[r] = ix.vecs + min(wb + g * kTileR + r, r1 - 1) * ix.pitch;
    float acc[kTileR][kTileQ];
#pragma unroll
    for (int r = 0; r < kTileR; ++r)
#pragma unroll
      for (int qq = 0; qq < kTileQ; ++qq) acc[r][qq] = 0.0f;
    // a ring of kTileStages 32-element blocks of the lane's own 4 rows (the ring shares its space
    // with the parked partials; each lane reads only what its own copies wrote)
    float* ring = part + (g * kTileR) * 32 + 4 * j;
#pragma unroll
    for (int sb = 0; sb < kTileStages - 1; ++sb) {
      if (sb < nfull) {
#pragma unroll
        for (int r = 0; r < kTileR; ++r) cp_async16(ring + sb * kTileStage + r * 32, rp[r] + sb * 32 + 4 * j);
      }
      cp_async_commit();
    }
    for (int c = 0; c < nfull; ++c) {
      const int cb = c + kTileStages - 1;
      if (cb < nfull) {
        const int slot = cb % kTileStages;
#pragma unroll
        for (int r = 0; r < kTileR; ++r) cp_async16(ring + slot * kTileStage + r * 32, rp[r] + cb * 32 + 4 * j);
      }
      cp_async_commit();
      cp_async_wait_keep<kTileStages - 1>();
      const float* src = ring + (c % kTileStages) * kTileStage;
      float4 x[kTileR];
#pragma unroll
      for (int r = 0; r < kTileR; ++r) x[r] = *reinterpret_cast<const float4*>(src + r * 32);
#pragma unroll
      for (int qq = 0; qq < kTileQ; ++qq) {
        const float4 qv = reinterpret_cast<const float4*>(qs + (size_t)qq * ix.pitch + c * 32)[j];
#pragma unroll
        for (int r = 0; r < kTileR; ++r) {
          acc[r][qq] = tile_term<kSub>(qv.x, x[r].x, acc[r][qq]);
          acc[r][qq] = tile_term<kSub>(qv.y, x[r].y, acc[r][qq]);
          acc[r][qq] = tile_term<kSub>(qv.z, x[r].z, acc[r][qq]);
          acc[r][qq] = tile_term<kSub>(qv.w, x[r].w, acc[r][qq]);
        }
      }
    }
    cp_async_wait_keep<0>();
    __syncwarp();  // every lane is done with the ring before the partials are parked over it
    if (half) {
      float2 xv[kTileR];
#pragma unroll
      for (int r = 0; r < kTileR; ++r) xv[r] = __ldg(reinterpret_cast<const float2*>(rp[r] + nfull * 32) + j);
#pragma unroll
      for (int qq = 0; qq < kTileQ; ++qq) {
        const float2 qv = reinterpret_cast<const float2*>(qs + (size_t)qq * ix.pitch + nfull * 32)[j];
#pragma unroll
        for (int r = 0; r < kTileR; ++r) {
          acc[r][qq] = tile_term<kSub>(qv.x, xv[r].x, acc[r][qq]);
          acc[r][qq] = tile_term<kSub>(qv.y, xv[r].y, acc[r][qq]);
        }
      }
    }
    // park the partials, then finish one pair at a time (a rolled loop keeps the code small)
#pragma unroll
    for (int r = 0; r < kTileR; ++r)
#pragma unroll
      for (int qq = 0; qq < kTileQ; ++qq) part[(r * kTileQ + qq) * 32 + lane] = acc[r][qq];
    __syncwarp();
    for (int p = 0; p < kTileR * kTileQ; ++p) {
      const int r = p / kTileQ, qq = p - r * kTileQ;
      const int64_t row = wb + g * kTileR + r;
      const float d = combine(ix, part[p * 32 + lane], ix.vecs + min(row, r1 - 1) * ix.pitch, qs + (size_t)qq * ix.pitch);
      if (qq >= nq_here) continue;
      const float kd = __shfl_sync(kFull, kth_d, qq);
      const int ki = __shfl_sync(kFull, kth_i, qq);
      unsigned m = __ballot_sync(kFull, j == 0 && row < r1 && scan_better(d, (int)row, kd, ki));
      if (m) {
        float bd = list_d[qq * 32 + lane];
        int bi = list_i[qq * 32 + lane];
        while (m) {
          const int src = __ffs(m) - 1;
          m &= m - 1;
          const float dc = __shfl_sync(kFull, d, src);
          const int rc = __shfl_sync(kFull, (int)row, src);
          scan_offer(bd, bi, a.k, dc, rc);
        }
        list_d[qq * 32 + lane] = bd;
        list_i[qq * 32 + lane] = bi;
        const float nd = __shfl_sync(kFull, bd, a.k - 1);
        const int ni = __shfl_sync(kFull, bi, a.k - 1);
        if (lane == qq) {
          kth_d = nd;
          kth_i = ni;
        }
      }
    }
    __syncwarp();  // the next pass overwrites the partials
  }
  if (lane < a.k) {
    const int n_lists = a.n_chunks * kTileWarps;
    for (int qq = 0; qq < nq_here; ++qq) {
      const size_t o = ((size_t)(q0 + qq) * n_lists + (size_t)blockIdx.y * kTileWarps + warp) * a.k + lane;
      a.part_d[o] = list_d[qq * 32 + lane];
      a.part_id[o] = list_i[qq * 32 + lane];
    }
  }
}

// L1 / LInf, tiled the same way with 4-lane groups (8 per warp, kLpR rows each per pass). The
// reference's L1 keeps four float accumulators, accumulator a adding |q_e - x_e| over
// e == a (mod 4) in element order (distcomp_lp.cc:191-251). In the permuted layout the 16-byte
// piece at position a of a 32-element block holds elements a, a+8, a+16, a+24 and the piece at
// position a+4 holds a+4, a+12, a+20, a+28, so lane a of a group reads both (for the query and
// its rows) and adds in exactly that order: the same accumulators as lp_group_dist, without its
// shuffles. LInf is a maximum of non-negative values, which any order gives.
constexpr int kLpR = 2;

template <bool kL1>
__device__ __forceinline__ float lp_term(float s, float q, float x) {
  const float d = fabsf(__fsub_rn(q, x));
  if constexpr (kL1) {
    return __fadd_rn(s, d);
  } else {
    return fmaxf(s, d);
  }
}

// Finishes one (row, query) pair from the 4 lane accumulators of each 4-lane group: the tails
// past the 16-element blocks and the reference's final reduction. Every lane of the warp calls it.
template <bool kL1>
__device__ float lp_finish4(const DevIndex& ix, float s, const float* __restrict__ row, const float* __restrict__ q) {
  const int lane = lane_id();
  const int gb = lane & ~3, ac = lane & 3;
  if constexpr (kL1) {
    const int n4 = (ix.dim >> 2) << 2;
    for (int e = ix.n16 + ac; e < n4; e += 4) s = __fadd_rn(s, fabsf(__fsub_rn(q[e], __ldg(row + e))));
    float t = __fadd_rn(__shfl_sync(kFull, s, gb), __shfl_sync(kFull, s, gb + 1));
    t = __fadd_rn(t, __shfl_sync(kFull, s, gb + 2));
    t = __fadd_rn(t, __shfl_sync(kFull, s, gb + 3));
    double r = (double)t;
    for (int e = n4; e < ix.dim; ++e) r = __dadd_rn(r, (double)fabsf(__fsub_rn(q[e], __ldg(row + e))));
    return __double2float_rn(r);
  } else {
    for (int e = ix.n16 + ac; e < ix.dim; e += 4) s = fmaxf(s, fabsf(__fsub_rn(q[e], __ldg(row + e))));
    s = fmaxf(s, __shfl_xor_sync(kFull, s, 2, 4));
    s = fmaxf(s, __shfl_xor_sync(kFull, s, 1, 4));
    return s;
  }
}

template <bool kL1>
__global__ void __launch_bounds__(32 * kTileWarps, 2) exact_scan_lp_tiled_kernel(ScanArgs a) {
  extern __shared__ __align__(16) float scan_smem[];
  const DevIndex& ix = a.ix;
  const int warp = threadIdx.x >> 5, lane = lane_id(), G = lane >> 2, ac = lane & 3;
  const int64_t q0 = (int64_t)blockIdx.x * kTileQ;
  const int nq_here = (int)min((int64_t)kTileQ, a.nq - q0);
  scan_load_query(ix, a.queries, q0 + warp, warp < nq_here, scan_smem + (size_t)warp * ix.pitch);
  __syncthreads();
  const float* qs = scan_smem;  // [kTileQ][pitch]
  // per warp: the row ring (which also holds the parked partials once drained), then the lists
  float* part = scan_smem + (size_t)kTileQ * ix.pitch + (size_t)warp * kTileWarpSmem;
  float* list_d = part + kTileRing;
  int* list_i = reinterpret_cast<int*>(list_d + kTileQ * 32);
  for (int i = lane; i < kTileQ * 32; i += 32) {
    list_d[i] = INFINITY;
    list_i[i] = 0x7fffffff;
  }
  float kth_d = INFINITY;  // lane qq < kTileQ: query qq's current k-th (distance, row)
  int kth_i = 0x7fffffff;
  const int nfull = ix.n16 >> 5;
  const bool half = (ix.n16 & 31) != 0;
  constexpr int kWarpRows = 8 * kLpR;
  static_assert(kWarpRows * 32 <= kTileStage, "a stage holds the warp's rows of one block");
  static_assert(kLpR * kTileQ * 32 <= kTileRing, "the ring holds the parked partials");
  const int64_t r0 = (int64_t)blockIdx.y * a.chunk_rows, r1 = min(ix.n, r0 + a.chunk_rows);
  for (int64_t wb = r0 + (int64_t)warp * kWarpRows; wb < r1; wb += (int64_t)kTileWarps * kWarpRows) {
    // rows past the chunk's end read its last row and are never offered
    const float* rp[kLpR];
#pragma unroll
    for (int r = 0; r < kLpR; ++r) rp[r] = ix.vecs + min(wb + G * kLpR + r, r1 - 1) * ix.pitch;
    float acc[kLpR][kTileQ];
#pragma unroll
    for (int r = 0; r < kLpR; ++r)
#pragma unroll
      for (int qq = 0; qq < kTileQ; ++qq) acc[r][qq] = 0.0f;
    // lane ac copies (and later reads) pieces ac and ac + 4 of its group's rows
    float* ring = part + (G * kLpR) * 32 + 4 * ac;
#pragma unroll
    for (int sb = 0; sb < kTileStages - 1; ++sb) {
      if (sb < nfull) {
#pragma unroll
        for (int r = 0; r < kLpR; ++r) {
          cp_async16(ring + sb * kTileStage + r * 32, rp[r] + sb * 32 + 4 * ac);
          cp_async16(ring + sb * kTileStage + r * 32 + 16, rp[r] + sb * 32 + 16 + 4 * ac);
        }
      }
      cp_async_commit();
    }
    for (int c = 0; c < nfull; ++c) {
      const int cb = c + kTileStages - 1;
      if (cb < nfull) {
        const int slot = cb % kTileStages;
#pragma unroll
        for (int r = 0; r < kLpR; ++r) {
          cp_async16(ring + slot * kTileStage + r * 32, rp[r] + cb * 32 + 4 * ac);
          cp_async16(ring + slot * kTileStage + r * 32 + 16, rp[r] + cb * 32 + 16 + 4 * ac);
        }
      }
      cp_async_commit();
      cp_async_wait_keep<kTileStages - 1>();
      const float* src = ring + (c % kTileStages) * kTileStage;
      float4 x0[kLpR], x1[kLpR];
#pragma unroll
      for (int r = 0; r < kLpR; ++r) {
        x0[r] = *reinterpret_cast<const float4*>(src + r * 32);
        x1[r] = *reinterpret_cast<const float4*>(src + r * 32 + 16);
      }
#pragma unroll
      for (int qq = 0; qq < kTileQ; ++qq) {
        const float* qb = qs + (size_t)qq * ix.pitch + c * 32 + 4 * ac;
        const float4 p0 = *reinterpret_cast<const float4*>(qb);
        const float4 p1 = *reinterpret_cast<const float4*>(qb + 16);
#pragma unroll
        for (int r = 0; r < kLpR; ++r) {
          float t = acc[r][qq];
          t = lp_term<kL1>(t, p0.x, x0[r].x);
          t = lp_term<kL1>(t, p1.x, x1[r].x);
          t = lp_term<kL1>(t, p0.y, x0[r].y);
          t = lp_term<kL1>(t, p1.y, x1[r].y);
          t = lp_term<kL1>(t, p0.z, x0[r].z);
          t = lp_term<kL1>(t, p1.z, x1[r].z);
          t = lp_term<kL1>(t, p0.w, x0[r].w);
          acc[r][qq] = lp_term<kL1>(t, p1.w, x1[r].w);
        }
      }
    }
    cp_async_wait_keep<0>();
    __syncwarp();  // every lane is done with the ring before the partials are parked over it
    if (half) {
      // the 16-element block: pieces of 2 at positions ac (elements ac, ac+8) and ac+4 (ac+4, ac+12)
#pragma unroll
      for (int r = 0; r < kLpR; ++r) {
        const float2 y0 = __ldg(reinterpret_cast<const float2*>(rp[r] + nfull * 32) + ac);
        const float2 y1 = __ldg(reinterpret_cast<const float2*>(rp[r] + nfull * 32) + ac + 4);
#pragma unroll
        for (int qq = 0; qq < kTileQ; ++qq) {
          const float2 p0 = reinterpret_cast<const float2*>(qs + (size_t)qq * ix.pitch + nfull * 32)[ac];
          const float2 p1 = reinterpret_cast<const float2*>(qs + (size_t)qq * ix.pitch + nfull * 32)[ac + 4];
          float t = acc[r][qq];
          t = lp_term<kL1>(t, p0.x, y0.x);
          t = lp_term<kL1>(t, p1.x, y1.x);
          t = lp_term<kL1>(t, p0.y, y0.y);
          acc[r][qq] = lp_term<kL1>(t, p1.y, y1.y);
        }
      }
    }
#pragma unroll
    for (int r = 0; r < kLpR; ++r)
#pragma unroll
      for (int qq = 0; qq < kTileQ; ++qq) part[(r * kTileQ + qq) * 32 + lane] = acc[r][qq];
    __syncwarp();
    for (int p = 0; p < kLpR * kTileQ; ++p) {
      const int r = p / kTileQ, qq = p - r * kTileQ;
      const int64_t row = wb + G * kLpR + r;
      const float d = lp_finish4<kL1>(ix, part[p * 32 + lane], ix.vecs + min(row, r1 - 1) * ix.pitch,
                                      qs + (size_t)qq * ix.pitch);
      if (qq >= nq_here) continue;
      const float kd = __shfl_sync(kFull, kth_d, qq);
      const int ki = __shfl_sync(kFull, kth_i, qq);
      unsigned m = __ballot_sync(kFull, ac == 0 && row < r1 && scan_better(d, (int)row, kd, ki));
      if (m) {
        float bd = list_d[qq * 32 + lane];
        int bi = list_i[qq * 32 + lane];
        while (m) {
          const int src = __ffs(m) - 1;
          m &= m - 1;
          scan_offer(bd, bi, a.k, __shfl_sync(kFull, d, src), __shfl_sync(kFull, (int)row, src));
        }
        list_d[qq * 32 + lane] = bd;
        list_i[qq * 32 + lane] = bi;
        const float nd = __shfl_sync(kFull, bd, a.k - 1);
        const int ni = __shfl_sync(kFull, bi, a.k - 1);
        if (lane == qq) {
          kth_d = nd;
          kth_i = ni;
        }
      }
    }
    __syncwarp();  // the next pass overwrites the partials
  }
  if (lane < a.k) {
    const int n_lists = a.n_chunks * kTileWarps;
    for (int qq = 0; qq < nq_here; ++qq) {
      const size_t o = ((size_t)(q0 + qq) * n_lists + (size_t)blockIdx.y * kTileWarps + warp) * a.k + lane;
      a.part_d[o] = list_d[qq * 32 + lane];
      a.part_id[o] = list_i[qq * 32 + lane];
    }
  }
}

// One warp per query: the best k of its lists, then external ids. The query's lists are one run of
// n_lists * k entries (a list's unused tail holds the (inf, 0x7fffffff) sentinel); the warp reads
// 4 x 32 of them at a time, one per lane, and offers only those that beat its current k-th.
__global__ void scan_merge_kernel(const float* __restrict__ part_d, const int32_t* __restrict__ part_id, int64_t nq,
                                  int n_lists, int k, int kmax, const int32_t* __restrict__ ext_id,
                                  int32_t* __restrict__ ids, float* __restrict__ dists, int32_t* __restrict__ counts) {
  const int lane = lane_id();
  const int64_t qi = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (qi >= nq) return;
  float bd = INFINITY;
  int bi = 0x7fffffff;
  const int total = n_lists * k;
  const size_t base = (size_t)qi * total;
  constexpr int kBatch = 4;
  for (int t0 = 0; t0 < total; t0 += 32 * kBatch) {
    float d[kBatch];
    int r[kBatch];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int t = t0 + u * 32 + lane;
      d[u] = t < total ? __ldg(part_d + base + t) : INFINITY;
      r[u] = t < total ? __ldg(part_id + base + t) : 0x7fffffff;
    }
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const float kd = __shfl_sync(kFull, bd, k - 1);
      const int ki = __shfl_sync(kFull, bi, k - 1);
      unsigned m = __ballot_sync(kFull, r[u] != 0x7fffffff && scan_better(d[u], r[u], kd, ki));
      while (m) {
        const int src = __ffs(m) - 1;
        m &= m - 1;
        scan_offer(bd, bi, k, __shfl_sync(kFull, d[u], src), __shfl_sync(kFull, r[u], src));
      }
    }
  }
  const int have = __popc(__ballot_sync(kFull, lane < k && bi != 0x7fffffff));
  for (int i = lane; i < kmax; i += 32) {
    const bool ok = i < have;
    ids[qi * kmax + i] = ok ? __ldg(ext_id + bi) : -1;
    dists[qi * kmax + i] = ok ? bd : __int_as_float(0x7f800000);
  }
  if (lane == 0) counts[qi] = have;
}

}  // namespace

int exact_scan_lists(const DevIndex&) { return kTileWarps; }

int exact_scan_knn(const DevIndex& ix, const float* queries, int64_t nq, int k, int kmax, float* part_d,
                   int32_t* part_id, int n_chunks, int32_t* ids, float* dists, int32_t* counts, void* stream) {
  if (nq == 0) return 0;
  if (k < 1 || k > 32) return (int)cudaErrorInvalidValue;
  cudaStream_t st = (cudaStream_t)stream;
  const int code = ix.dist_type;
  void (*kern)(ScanArgs) = nullptr;
  if (code == kL2Sqr16Ext || code == kL2SqrExt) kern = exact_scan_tiled_kernel<true>;
  else if (code == kNormCosine || code == kNegDot) kern = exact_scan_tiled_kernel<false>;
  else if (code == kL1) kern = exact_scan_lp_tiled_kernel<true>;
  else if (code == kLInf) kern = exact_scan_lp_tiled_kernel<false>;
  else return (int)cudaErrorInvalidValue;
  const int smem = kTileQ * ix.pitch * 4 + kTileWarps * kTileWarpSmem * 4;
  if (smem > kMaxDynamicSmem) return (int)cudaErrorInvalidValue;
  const int rc = allow_max_smem((const void*)kern);
  if (rc != 0) return rc;
  ScanArgs a;
  a.ix = ix;
  a.queries = queries;
  a.nq = nq;
  a.k = k;
  a.n_chunks = n_chunks;
  a.chunk_rows = (ix.n + n_chunks - 1) / n_chunks;
  a.part_d = part_d;
  a.part_id = part_id;
  const dim3 grid((unsigned)((nq + kTileQ - 1) / kTileQ), (unsigned)n_chunks);
  kern<<<grid, 32 * kTileWarps, smem, st>>>(a);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  scan_merge_kernel<<<(unsigned)((nq + 7) / 8), 256, 0, st>>>(part_d, part_id, nq, n_chunks * kTileWarps, k, kmax,
                                                              ix.ext_id, ids, dists, counts);
  return (int)cudaGetLastError();
}

int multi_list_chunks(const DevIndex& ix) { return std::max(ix.maxM, ix.maxM0) <= 32 ? 1 : 2; }

int multi_warp_smem_bytes(const DevIndex& ix, int region_items, int nbpad, int stage_rows, int ctx) {
  return ctx * multi_ctx_bytes(ix, region_items, nbpad) + stage_rows * ix.pitch * 4 + 16;  // + the mbarrier
}

int warp_smem_bytes(const DevIndex& ix, int region_items, int nbpad, int hash_log2, int stage_rows) {
  int bytes = ix.pitch * 4 + region_items * 8 + nbpad * 16 + (hash_log2 > 0 ? (4 << hash_log2) : 0) +
              stage_rows * ix.pitch * 4 + (stage_rows > 0 ? 16 : 0);  // + the bulk-copy mbarrier
  return (bytes + 15) & ~15;
}

namespace {
using Kern = void (*)(SearchArgs);

template <bool OLD>
Kern pick(bool plain, int gather) {
  if (plain) {
    switch (gather) {
      case 0: return search_plain_kernel<0, OLD>;
      case 1: return search_plain_kernel<1, OLD>;
      case 2: return search_plain_kernel<2, OLD>;
      case kLpGather: return search_plain_kernel<kLpGather, OLD>;
      case kSiftGather: return search_plain_kernel<kSiftGather, OLD>;
      default: return search_plain_kernel<4, OLD>;
    }
  }
  switch (gather) {
    case 0: return search_batched_kernel<0, OLD>;
    case 1: return search_batched_kernel<1, OLD>;
    case 2: return search_batched_kernel<2, OLD>;
    case kLpGather: return search_batched_kernel<kLpGather, OLD>;
    case kSiftGather: return search_batched_kernel<kSiftGather, OLD>;
    default: return search_batched_kernel<4, OLD>;
  }
}

// The lean kernel for this index shape, or null when it has none.
Kern lean_kernel_for(const DevIndex& ix) {
  if (ix.dim % 16 != 0 || std::max(ix.maxM, ix.maxM0) > 64) return nullptr;
  switch (ix.dist_type) {
    case kL2Sqr16Ext: return reinterpret_cast<Kern>(lean_kernel_l2(ix));
    case kNormCosine: return reinterpret_cast<Kern>(lean_kernel_cos(ix));
    case kNegDot: return reinterpret_cast<Kern>(lean_kernel_negdot(ix));
  }
  return nullptr;
}

Kern kernel_for(bool plain, int gather, bool with_old, int ctx = 1, int nch = 1) {
  if (ctx > 1 && !plain && !with_old && gather == 0) {
    if (ctx == 2) return nch == 1 ? search_multi_kernel<2, 1> : search_multi_kernel<2, 2>;
    if (ctx == 3) return nch == 1 ? search_multi_kernel<3, 1> : search_multi_kernel<3, 2>;
    return nch == 1 ? search_multi_kernel<4, 1> : search_multi_kernel<4, 2>;
  }
  return with_old ? pick<true>(plain, gather) : pick<false>(plain, gather);
}
}  // namespace

int allow_max_smem(const void* kern) {
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({dev, kern})) return 0;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynamicSmem);
  if (e != cudaSuccess) return (int)e;
  done.insert({dev, kern});
  return 0;
}

namespace {

// The level-0 pass's work order: queries by their level-0 entry distance, largest first (the
// queries that enter level 0 far from their query tend to need the most expansions, and starting
// them first keeps the batch's end from waiting on a long query that started late). One block:
// kOrderBuckets buckets spread evenly over the range of the ordered keys, counted, scanned, and
// filled (the order inside a bucket is arbitrary; results do not depend on the order).
constexpr int kOrderBuckets = 2048;

// Bucket of a key, largest keys in bucket 0; scale = (kOrderBuckets - 1) / (hi - lo). The same
// float arithmetic in both passes over the keys, so a key lands in the same bucket each time.
__device__ __forceinline__ int order_bucket(float v, uint32_t lo, uint32_t hi, float scale) {
  const uint32_t k = min(max(ordered_key(v), lo), hi);
  const int b = min((int)(__uint2float_rz(k - lo) * scale), kOrderBuckets - 1);
  return kOrderBuckets - 1 - b;
}

__global__ void __launch_bounds__(1024) order_by_entry_kernel(const float* __restrict__ key, int64_t nq,
                                                             const uint32_t* __restrict__ range,
                                                             int32_t* __restrict__ order) {
  __shared__ int cnt[kOrderBuckets];
  for (int b = threadIdx.x; b < kOrderBuckets; b += blockDim.x) cnt[b] = 0;
  __syncthreads();
  const uint32_t lo = range[0], hi = range[1];
  const float scale = (float)(kOrderBuckets - 1) / __uint2float_ru(hi > lo ? hi - lo : 1u);
  for (int64_t i = threadIdx.x; i < nq; i += blockDim.x) atomicAdd(&cnt[order_bucket(key[i], lo, hi, scale)], 1);
  __syncthreads();
  if (threadIdx.x < 32) {  // exclusive scan: each lane a run of 64 buckets, then across the lanes
    constexpr int kRun = kOrderBuckets / 32;
    const int lane = threadIdx.x;
    int sum = 0;
    for (int b = 0; b < kRun; ++b) sum += cnt[lane * kRun + b];
    int pre = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(kFull, pre, o);
      if (lane >= o) pre += v;
    }
    int s = pre - sum;
    for (int b = 0; b < kRun; ++b) {
      const int c = cnt[lane * kRun + b];
      cnt[lane * kRun + b] = s;
      s += c;
    }
  }
  __syncthreads();
  for (int64_t i = threadIdx.x; i < nq; i += blockDim.x)
    order[atomicAdd(&cnt[order_bucket(key[i], lo, hi, scale)], 1)] = (int32_t)i;
}

}  // namespace

int launch_search(const SearchArgs& a, bool plain, int gather, bool with_old, int blocks, int warps_per_block,
                  void* stream, const QueryParts* parts) {
  Kern kern = a.lean ? lean_kernel_for(a.ix) : kernel_for(plain, gather, with_old, a.ctx_per_warp, multi_list_chunks(a.ix));
  if (!kern) return (int)cudaErrorInvalidDeviceFunction;
  const int smem = a.warp_smem * (plain ? 1 : warps_per_block);
  const int rc = allow_max_smem((const void*)kern);
  if (rc != 0) return rc;
  if (!plain && a.entry_node) {
    // split: the upper-level descent of every query, the order, then level 0 in that order
    cudaStream_t st = (cudaStream_t)stream;
    SearchArgs d = a;
    d.split = 1;
    d.order = nullptr;
    cudaError_t e = cudaMemsetAsync(a.entry_node, 0xff, (size_t)a.nq * 4, st);  // -1: no entry yet
    if (e == cudaSuccess) e = cudaMemsetAsync(a.entry_dist, 0, (size_t)a.nq * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.entry_range, 0xff, 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.entry_range + 1, 0, 4, st);
    if (e != cudaSuccess) return (int)e;
    if (parts && a.lean && parts->first > 0 && parts->first < a.nq) {
      // the first part's descents run while the rest of the queries are still being copied
      e = cudaStreamWaitEvent(st, parts->ready[0], 0);
      if (e != cudaSuccess) return (int)e;
      d.nq = parts->first;
      kern<<<blocks, 32 * warps_per_block, smem, st>>>(d);
      e = cudaMemsetAsync(a.work_counter, 0, 4, st);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(st, parts->ready[1], 0);
      if (e != cudaSuccess) return (int)e;
      d.q_base = parts->first;
      d.nq = a.nq - parts->first;
      kern<<<blocks, 32 * warps_per_block, smem, st>>>(d);
    } else {
      if (parts) {
        e = cudaStreamWaitEvent(st, parts->ready[1], 0);
        if (e != cudaSuccess) return (int)e;
      }
      kern<<<blocks, 32 * warps_per_block, smem, st>>>(d);
    }
    order_by_entry_kernel<<<1, 1024, 0, st>>>(a.entry_dist, a.nq, a.entry_range, a.entry_order);
    e = cudaMemsetAsync(a.work_counter, 0, 4, st);
    if (e != cudaSuccess) return (int)e;
    SearchArgs l = a;
    l.split = 2;
    l.order = a.entry_order;
    kern<<<blocks, 32 * warps_per_block, smem, st>>>(l);
    return (int)cudaGetLastError();
  }
  if (parts) {
    const cudaError_t e = cudaStreamWaitEvent((cudaStream_t)stream, parts->ready[1], 0);
    if (e != cudaSuccess) return (int)e;
  }
  if (plain)
    kern<<<(unsigned)a.nq, 32, smem, (cudaStream_t)stream>>>(a);
  else
    kern<<<blocks, 32 * warps_per_block, smem, (cudaStream_t)stream>>>(a);
  return (int)cudaGetLastError();
}

bool lean_supported(const DevIndex& ix) { return lean_kernel_for(ix) != nullptr; }

int lean_occupancy(const DevIndex& ix, int warps_per_block, int smem_per_block, int* blocks_per_sm) {
  Kern kern = lean_kernel_for(ix);
  if (!kern) return (int)cudaErrorInvalidDeviceFunction;
  const int rc = allow_max_smem((const void*)kern);
  if (rc != 0) return rc;
  return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kern, 32 * warps_per_block, smem_per_block);
}

int lean_smem_bytes(const DevIndex& ix, int region_items, int nbpad, int stage_rows) {
  return lean_warp_smem_bytes(ix.dim, region_items, nbpad, stage_rows);
}

int search_occupancy(bool plain, int gather, bool with_old, int warps_per_block, int smem_per_block,
                     int* blocks_per_sm, int ctx, int nch) {
  Kern kern = kernel_for(plain, gather, with_old, ctx, nch);
  const int rc = allow_max_smem((const void*)kern);
  if (rc != 0) return rc;
  return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kern, 32 * (plain ? 1 : warps_per_block),
                                                            smem_per_block);
}

}  // namespace nmsg
