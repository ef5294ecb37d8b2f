// Exact brute-force k-NN over the loaded index's vectors — the semantics of NMSLIB's sequential
// search (similarity_search/src/method/seqsearch.cc:143-177: every stored object is compared
// with the query and the k best are kept, knnquery.cc:67-75) — computed as:
//
//   pass A  a tcgen05 BF16 x BF16 -> FP32 GEMM of 128-query tiles against 256-row base tiles
//           (TMA-fed, accumulators double-buffered in TMEM) whose epilogue keeps, per query and
//           per chunk of the base, the C best BF16 scores;
//   rerank  exact scores of those candidates in double-float arithmetic (error-free products and
//           sums on FP32 units, about 2^-44 relative), top-k by (distance, id);
//   certify with a rigorous per-query bound eps on |BF16 score - exact score|: if every chunk's
//           C-th best BF16 score is below (exact k-th score - eps), no vector outside the
//           candidates can reach the top k;
//   pass B  for the queries that are not certified, the same GEMM again, now collecting every
//           vector whose BF16 score is >= exact k-th score - eps, then the exact rerank of
//           that set. Queries whose set overflows fall back to an exact scan on CUDA cores.
//
// So the returned ids are the exact top-k (ties by id), independent of BF16 rounding.
// Scores ("keys", larger is better): negdot and cosine use q.x (queries of the cosine space
// are normalised as NormalizeVect does, base vectors are stored normalised); l2 uses
// 2 q.x - |x|^2, so distance = |q|^2 - key is the squared L2 the HNSW path reports.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "engine.h"
#include "handle.h"
#include "sm100.cuh"
#include "../../include/nmslib_b200.h"

namespace nmsg {
namespace {

using namespace sm100;

constexpr int BM = 128;                 // queries per tile = TMEM lanes
constexpr int BN = 256;                 // base rows per tile = accumulator columns
constexpr int BK = 64;                  // bf16 elements per 128-byte swizzle row
constexpr int CAND = 32;                // candidates kept per query per list (pass A)
constexpr int KB_MAX = 4;               // padded dim <= 256
constexpr int Q_BLOCK_BYTES = BM * BK * 2;   // 16 KB
constexpr int X_STAGE_BYTES = BN * BK * 2;   // 32 KB
constexpr int EPI_WARPS = 8;            // two warps per TMEM lane quarter, one per column half
constexpr int HALVES = 2;
constexpr int kThreads = (EPI_WARPS + 2) * 32;  // + TMA warp + MMA warp
constexpr int LIST_STRIDE = CAND + 1;   // +1: rows of a list on different banks

struct GemmArgs {
  int kb;             // padded dim / 64
  int stages;         // base-tile pipeline depth (3 when kb <= 2, else 2)
  int n;              // base rows
  int nq;             // queries
  int n_tiles;        // ceil(n / BN)
  int chunk_tiles;    // base tiles per work item
  int n_chunks;
  int q_blocks;
  int mode;           // 0: top-CAND per (chunk, column half); 1: collect keys >= tau
  int key_l2;         // 1: key = 2 dot - |x|^2
  const float* xnorm2;  // padded to n_tiles * BN
  float* cand_key;    // [nq][n_chunks * HALVES][CAND]
  int32_t* cand_id;
  const float* tau;   // [nq]
  const uint8_t* q_active;  // [q_blocks * BM]
  int32_t* coll_id;   // [nq][coll_cap]
  float* coll_key;
  int32_t* coll_cnt;  // [nq]
  int coll_cap;
  int32_t* status;
};

// Shared memory: Q blocks | base stages | candidate lists | barriers (1024-aligned base).
struct SmemLayout {
  int q_off, x_off, key_off, id_off, bar_off, total;
  __host__ __device__ SmemLayout(int kb, int stages) {
    q_off = 0;
    x_off = q_off + kb * Q_BLOCK_BYTES;
    key_off = x_off + stages * X_STAGE_BYTES;
    id_off = key_off + HALVES * BM * LIST_STRIDE * 4;
    bar_off = (id_off + HALVES * BM * LIST_STRIDE * 4 + 7) & ~7;
    total = bar_off + 8 * (2 * 4 + 2 + 4) + 16;
  }
};

__device__ __forceinline__ bool item_active(const GemmArgs& a, int qb) {
  if (a.mode == 0) return true;
  const uint8_t* p = a.q_active + (size_t)qb * BM;
  for (int i = 0; i < BM; ++i)
    if (p[i]) return true;
  return false;
}

// A row's candidate list is a min-heap of CAND (key, column) pairs in shared memory: the root is
// the smallest kept key, i.e. the threshold a new key must beat. The first CAND offers fill it,
// then it is heapified once; later insertions replace the root and sift down (log2 CAND steps).
__device__ __forceinline__ void heap_sift_down(float* lk, int32_t* li, int pos) {
  const float key = lk[pos];
  const int32_t id = li[pos];
  while (true) {
    int child = 2 * pos + 1;
    if (child >= CAND) break;
    if (child + 1 < CAND && lk[child + 1] < lk[child]) ++child;
    if (!(lk[child] < key)) break;
    lk[pos] = lk[child];
    li[pos] = li[child];
    pos = child;
  }
  lk[pos] = key;
  li[pos] = id;
}

__device__ __forceinline__ void list_offer(float* lk, int32_t* li, int& nfill, float& thr, float key, int col) {
  if (nfill < CAND) {
    lk[nfill] = key;
    li[nfill] = col;
    if (++nfill == CAND) {
      for (int p = CAND / 2 - 1; p >= 0; --p) heap_sift_down(lk, li, p);
      thr = lk[0];
    }
    return;
  }
  if (!(key > thr)) return;
  lk[0] = key;
  li[0] = col;
  heap_sift_down(lk, li, 0);
  thr = lk[0];
}

__global__ void __launch_bounds__(kThreads, 1)
    bf16_scan_kernel(const __grid_constant__ CUtensorMap tmq, const __grid_constant__ CUtensorMap tmx, GemmArgs a) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const SmemLayout L(a.kb, a.stages);
  uint8_t* sq = base + L.q_off;
  uint8_t* sx = base + L.x_off;
  float* skey = reinterpret_cast<float*>(base + L.key_off);
  int32_t* sid = reinterpret_cast<int32_t*>(base + L.id_off);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + L.bar_off);
  uint64_t* x_full = bars;          // [4]
  uint64_t* x_empty = bars + 4;     // [4]
  uint64_t* q_full = bars + 8;
  uint64_t* q_empty = bars + 9;
  uint64_t* acc_full = bars + 10;   // [2]
  uint64_t* acc_empty = bars + 12;  // [2]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 14);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n_items = a.q_blocks * a.n_chunks;
  const int stages = a.stages;

  if (threadIdx.x == 0) {
    for (int i = 0; i < stages; ++i) {
      mbar_init(&x_full[i], 1);
      mbar_init(&x_empty[i], 1);
    }
    mbar_init(q_full, 1);
    mbar_init(q_empty, 1);
    for (int i = 0; i < 2; ++i) {
      mbar_init(&acc_full[i], 1);
      mbar_init(&acc_empty[i], EPI_WARPS);  // one arrival per epilogue warp
    }
    fence_barrier_init();
  }
  if (warp == 0) tmem_alloc(tmem_slot, 512);
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  bool ok = true;

  if (warp == EPI_WARPS) {
    // ------------------------------------------------ TMA producer
    if (lane == 0) {
      prefetch_tmap(&tmq);
      prefetch_tmap(&tmx);
      int stage = 0;
      uint32_t xphase = 0, qphase = 0;
      int done_items = 0;
      for (int item = blockIdx.x; item < n_items && ok; item += gridDim.x) {
        const int qb = item / a.n_chunks, chunk = item % a.n_chunks;
        if (!item_active(a, qb)) continue;
        if (done_items > 0) {
          ok = mbar_wait(q_empty, qphase);
          qphase ^= 1;
        }
        mbar_arrive_expect_tx(q_full, a.kb * Q_BLOCK_BYTES);
        for (int kb = 0; kb < a.kb; ++kb) tma_load_2d(sq + kb * Q_BLOCK_BYTES, &tmq, q_full, kb * BK, qb * BM);
        const int t0 = chunk * a.chunk_tiles, t1 = min(a.n_tiles, t0 + a.chunk_tiles);
        for (int t = t0; t < t1 && ok; ++t) {
          for (int kb = 0; kb < a.kb && ok; ++kb) {
            ok = mbar_wait(&x_empty[stage], xphase ^ 1);
            mbar_arrive_expect_tx(&x_full[stage], X_STAGE_BYTES);
            tma_load_2d(sx + stage * X_STAGE_BYTES, &tmx, &x_full[stage], kb * BK, t * BN);
            if (++stage == stages) {
              stage = 0;
              xphase ^= 1;
            }
          }
        }
        ++done_items;
      }
    }
  } else if (warp == EPI_WARPS + 1) {
    // ------------------------------------------------ MMA issuer
    if (lane == 0) {
      const uint32_t idesc = idesc_bf16_f32(BM, BN);
      int stage = 0;
      uint32_t xphase = 0, qphase = 0;
      uint32_t accphase[2] = {0, 0};
      int tcount = 0;
      for (int item = blockIdx.x; item < n_items && ok; item += gridDim.x) {
        const int qb = item / a.n_chunks, chunk = item % a.n_chunks;
        if (!item_active(a, qb)) continue;
        ok = mbar_wait(q_full, qphase);
        qphase ^= 1;
        tc_fence_after();
        const int t0 = chunk * a.chunk_tiles, t1 = min(a.n_tiles, t0 + a.chunk_tiles);
        for (int t = t0; t < t1 && ok; ++t, ++tcount) {
          const int buf = tcount & 1;
          ok = mbar_wait(&acc_empty[buf], accphase[buf] ^ 1);
          accphase[buf] ^= 1;
          tc_fence_after();
          const uint32_t dcol = tmem + buf * BN;
          for (int kb = 0; kb < a.kb && ok; ++kb) {
            ok = mbar_wait(&x_full[stage], xphase);
            tc_fence_after();
            const uint32_t qa = smem_u32(sq + kb * Q_BLOCK_BYTES), xa = smem_u32(sx + stage * X_STAGE_BYTES);
#pragma unroll
            for (int k = 0; k < BK / 16; ++k)
              umma_bf16(dcol, smem_desc_sw128(qa + 32 * k), smem_desc_sw128(xa + 32 * k), idesc, kb > 0 || k > 0);
            umma_commit(&x_empty[stage]);
            if (++stage == stages) {
              stage = 0;
              xphase ^= 1;
            }
          }
          umma_commit(&acc_full[buf]);
        }
        umma_commit(q_empty);
      }
    }
  } else {
    // ------------------------------------------------ epilogue: warps 0-7; thread = one query row
    // (TMEM lane) for one half of the tile's columns
    const int quarter = warp & 3, half = warp >> 2;
    const int row = quarter * 32 + lane;
    float* lk = skey + (half * BM + row) * LIST_STRIDE;
    int32_t* li = sid + (half * BM + row) * LIST_STRIDE;
    uint32_t accphase[2] = {0, 0};
    int tcount = 0;
    for (int item = blockIdx.x; item < n_items && ok; item += gridDim.x) {
      const int qb = item / a.n_chunks, chunk = item % a.n_chunks;
      if (!item_active(a, qb)) continue;
      const int q = qb * BM + row;
      const bool qvalid = q < a.nq;
      float thr = -INFINITY;  // mode 0: the list's smallest key once full; mode 1: tau
      int nfill = 0;
      if (a.mode == 1) thr = (qvalid && a.q_active[q]) ? a.tau[q] : INFINITY;
      const int t0 = chunk * a.chunk_tiles, t1 = min(a.n_tiles, t0 + a.chunk_tiles);
      // |x|^2 of this half's 128 columns, 4 per lane, loaded one tile ahead and handed to the
      // other lanes by shuffles
      const float4* xn4 = reinterpret_cast<const float4*>(a.xnorm2) + half * (BN / HALVES / 4) + lane;
      float4 nrm_next = make_float4(0.f, 0.f, 0.f, 0.f);
      if (a.key_l2 && t0 < t1) nrm_next = __ldg(xn4 + (size_t)t0 * (BN / 4));
      for (int t = t0; t < t1 && ok; ++t, ++tcount) {
        const int buf = tcount & 1;
        const float4 nrm = nrm_next;
        if (a.key_l2 && t + 1 < t1) nrm_next = __ldg(xn4 + (size_t)(t + 1) * (BN / 4));
        ok = mbar_wait(&acc_full[buf], accphase[buf]);
        accphase[buf] ^= 1;
        tc_fence_after();
#pragma unroll 1
        for (int c = 0; c < BN / 32 / HALVES; ++c) {
          const int ccol = half * (BN / HALVES) + c * 32;  // column inside the tile
          float v[32];
          tmem_ld32(tmem + ((uint32_t)(quarter * 32) << 16) + buf * BN + ccol, v);
          const int col0 = t * BN + ccol;
          // keys of all 32 columns without branches (independent, so they overlap), then one
          // test of their maximum against the threshold; the per-column path runs only if it passes
          if (a.key_l2) {
#pragma unroll
            for (int i = 0; i < 32; ++i) {
              const float comp = (i & 3) == 0 ? nrm.x : (i & 3) == 1 ? nrm.y : (i & 3) == 2 ? nrm.z : nrm.w;
              const float xn = __shfl_sync(0xffffffffu, comp, c * 8 + (i >> 2));
              v[i] = __fsub_rn(__fmul_rn(2.0f, v[i]), xn);
            }
          }
          if (col0 + 32 > a.n) {
#pragma unroll
            for (int i = 0; i < 32; ++i)
              if (col0 + i >= a.n) v[i] = -INFINITY;
          }
          float mx = v[0];
#pragma unroll
          for (int i = 1; i < 32; ++i) mx = fmaxf(mx, v[i]);
          if (a.mode == 0) {
            if (mx > thr || nfill < CAND) {
#pragma unroll
              for (int i = 0; i < 32; ++i)
                if (v[i] > thr || nfill < CAND) {
                  if (col0 + i < a.n) list_offer(lk, li, nfill, thr, v[i], col0 + i);
                }
            }
          } else if (mx >= thr) {
#pragma unroll
            for (int i = 0; i < 32; ++i)
              if (v[i] >= thr) {
                const int slot = atomicAdd(a.coll_cnt + q, 1);
                if (slot < a.coll_cap) {
                  a.coll_id[(size_t)q * a.coll_cap + slot] = col0 + i;
                  a.coll_key[(size_t)q * a.coll_cap + slot] = v[i];
                }
              }
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&acc_empty[buf]);
      }
      if (a.mode == 0 && qvalid) {
        const size_t list = (size_t)q * a.n_chunks * HALVES + chunk * HALVES + half;
        float* ok_out = a.cand_key + list * CAND;
        int32_t* oi_out = a.cand_id + list * CAND;
        for (int j = 0; j < CAND; ++j) {
          ok_out[j] = j < nfill ? lk[j] : -INFINITY;
          oi_out[j] = j < nfill ? li[j] : -1;
        }
      }
    }
  }
  if (!ok) atomicCAS(a.status, 0, NMSG_ERR_TIMEOUT);
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, 512);
}

// ------------------------------------------------------------------ exact scores
// Double-float (hi, lo) arithmetic on FP32 units: TwoProduct by FMA, TwoSum (Knuth).
struct DF {
  float hi, lo;
};
__device__ __forceinline__ DF df_add(DF a, float b) {
  const float s = __fadd_rn(a.hi, b);
  const float bb = __fsub_rn(s, a.hi);
  const float e = __fadd_rn(__fsub_rn(a.hi, __fsub_rn(s, bb)), __fsub_rn(b, bb));
  const float lo = __fadd_rn(a.lo, e);
  const float hi = __fadd_rn(s, lo);
  return DF{hi, __fsub_rn(lo, __fsub_rn(hi, s))};
}
__device__ __forceinline__ DF df_add_df(DF a, DF b) {
  DF r = df_add(a, b.hi);
  return df_add(r, b.lo);
}
__device__ __forceinline__ DF df_mul_ff(float a, float b) {
  const float p = __fmul_rn(a, b);
  return DF{p, __fmaf_rn(a, b, -p)};
}
__device__ __forceinline__ bool df_greater(DF a, DF b) { return a.hi > b.hi || (a.hi == b.hi && a.lo > b.lo); }

// Exact-ish key of one (query, row) pair, warp-cooperative over the dimension.
__device__ DF exact_key(const float* q, const float* x, int dim, bool l2, DF xnorm) {
  const int lane = threadIdx.x & 31;
  DF acc{0.0f, 0.0f};
  for (int e = lane; e < dim; e += 32) acc = df_add_df(acc, df_mul_ff(q[e], x[e]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    DF other{__shfl_xor_sync(0xffffffffu, acc.hi, o), __shfl_xor_sync(0xffffffffu, acc.lo, o)};
    acc = df_add_df(acc, other);
  }
  if (l2) {
    DF two{__fmul_rn(2.0f, acc.hi), __fmul_rn(2.0f, acc.lo)};
    DF neg{-xnorm.hi, -xnorm.lo};
    return df_add_df(two, neg);
  }
  return acc;
}

struct RerankArgs {
  const float* q;        // [nq][dim] (normalised for cosine)
  const float* x;        // [n][dim] natural order, fp32
  const float* xn_hi;    // l2: |x|^2 as double-float
  const float* xn_lo;
  int dim, n, nq, k, l2;
  int n_lists, list_len;       // pass A: candidate lists per query and their length
  const int32_t* ids;          // pass A: [nq][n_lists * list_len] (-1 = empty); pass B: [nq][coll_cap]
  const float* bf_keys;        // BF16 keys, same layout
  const int32_t* list_count;   // pass B: per-query count (null in pass A)
  const float* eps;            // [nq] bound on |BF16 key - exact key|
  int coll_cap;
  // outputs
  int32_t* out_ids;            // [nq][k] internal ids, best first
  DF* out_keys;                // [nq][k]
  int32_t* out_count;          // [nq]
  float* tau;                  // pass A: [nq] threshold for the second pass
  uint8_t* needs;              // pass A: 1 = not certified; pass B: 1 = collection overflowed
};

// (key, id) order of the result: larger key first, then smaller id.
__device__ __forceinline__ bool better(DF ka, int ia, DF kb, int ib) {
  return df_greater(ka, kb) || (ka.hi == kb.hi && ka.lo == kb.lo && ia < ib);
}

// Exact key of one (query, row) pair computed by a single lane (sequential over the dimension).
__device__ DF exact_key_lane(const float* __restrict__ q, const float* __restrict__ x, int dim, bool l2, DF xnorm) {
  DF acc{0.0f, 0.0f};
  for (int e = 0; e < dim; ++e) acc = df_add_df(acc, df_mul_ff(q[e], __ldg(x + e)));
  if (l2) return df_add_df(DF{__fmul_rn(2.0f, acc.hi), __fmul_rn(2.0f, acc.lo)}, DF{-xnorm.hi, -xnorm.lo});
  return acc;
}

// One warp per query:
//  1. B_k = the k-th largest BF16 key among the candidates (pairs (key, slot), k rounds of
//     warp max);
//  2. only candidates with BF16 key >= B_k - 2 eps can be in the exact top k (the k candidates
//     at or above B_k all have exact keys >= B_k - eps, anything below B_k - 2 eps has an exact
//     key < B_k - eps), so only they get exact keys, one candidate per lane;
//  3. the exact top k by (key desc, id asc), merged 32 candidates at a time;
//  4. pass A: the certificate and the second-pass threshold.
__global__ void rerank_kernel(RerankArgs a) {
  const int lane = threadIdx.x & 31;
  const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (q >= a.nq) return;
  const bool pass_b = a.list_count != nullptr;
  int total = pass_b ? min(a.list_count[q], a.coll_cap) : a.n_lists * a.list_len;
  const size_t base = pass_b ? (size_t)q * a.coll_cap : (size_t)q * a.n_lists * a.list_len;
  const int32_t* ids = a.ids + base;
  const float* bk = a.bf_keys + base;
  const float eps = a.eps[q];

  // pass A: every full list bounds the vectors it dropped by its smallest key
  float worst_bf_list = -INFINITY;
  if (!pass_b) {
    for (int c = 0; c < a.n_lists; ++c) {
      float mn = INFINITY;
      bool full = true;
      for (int j = lane; j < a.list_len; j += 32) {
        full &= ids[c * a.list_len + j] >= 0;
        mn = fminf(mn, bk[c * a.list_len + j]);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      if (__all_sync(0xffffffffu, full)) worst_bf_list = fmaxf(worst_bf_list, mn);
    }
  }

  // 1. k-th largest BF16 key (pairs ordered by key desc, slot asc)
  float prev_k = INFINITY;
  int prev_s = -1;
  int found = 0;
  for (int r = 0; r < a.k; ++r) {
    float bkey = -INFINITY;
    int bslot = 0x7fffffff;
    for (int t = lane; t < total; t += 32) {
      if (ids[t] < 0) continue;
      const float kv = bk[t];
      const bool below = kv < prev_k || (kv == prev_k && t > prev_s);  // after the previous pick
      if (below && (kv > bkey || (kv == bkey && t < bslot))) {
        bkey = kv;
        bslot = t;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const float ok = __shfl_xor_sync(0xffffffffu, bkey, o);
      const int os = __shfl_xor_sync(0xffffffffu, bslot, o);
      if (ok > bkey || (ok == bkey && os < bslot)) {
        bkey = ok;
        bslot = os;
      }
    }
    if (bslot == 0x7fffffff) break;
    prev_k = bkey;
    prev_s = bslot;
    ++found;
  }
  const float cut = found == a.k ? __fsub_rd(prev_k, __fmul_ru(2.0f, eps)) : -INFINITY;

  // 2-3. exact keys of the candidates at or above the cut, one per lane, merged into the top k
  const float* qv = a.q + (size_t)q * a.dim;
  DF top_k = DF{-INFINITY, 0.0f};  // lane j holds the j-th best so far (j < k)
  int top_i = 0x7fffffff;
  int have = 0;
  for (int t0 = 0; t0 < total; t0 += 32) {
    const int t = t0 + lane;
    int id = -1;
    if (t < total) {
      id = ids[t];
      if (id >= 0 && !(bk[t] >= cut)) id = -1;
    }
    if (__ballot_sync(0xffffffffu, id >= 0) == 0) continue;
    DF key{-INFINITY, 0.0f};
    if (id >= 0) {
      DF xn{0.0f, 0.0f};
      if (a.l2) xn = DF{a.xn_hi[id], a.xn_lo[id]};
      key = exact_key_lane(qv, a.x + (size_t)id * a.dim, a.dim, a.l2, xn);
    }
    // merge: the new top k = the k best of (old top k held by lanes < have) and the 32 new ones
    DF nk{-INFINITY, 0.0f};
    int ni = 0x7fffffff;
    bool my_old = lane < have, my_new = id >= 0;
    int taken = 0;
    for (int r = 0; r < a.k; ++r) {
      // candidate of this lane: its better remaining entry
      DF ck{-INFINITY, 0.0f};
      int ci = 0x7fffffff, cw = -1;  // which: 0 old, 1 new
      if (my_old && (!my_new || better(top_k, top_i, key, id))) {
        ck = top_k;
        ci = top_i;
        cw = 0;
      } else if (my_new) {
        ck = key;
        ci = id;
        cw = 1;
      }
      DF bkk = ck;
      int bi = ci, bl = cw >= 0 ? lane : 32;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const DF ok{__shfl_xor_sync(0xffffffffu, bkk.hi, o), __shfl_xor_sync(0xffffffffu, bkk.lo, o)};
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        const int ol = __shfl_xor_sync(0xffffffffu, bl, o);
        if (ol < 32 && (bl == 32 || better(ok, oi, bkk, bi))) {
          bkk = ok;
          bi = oi;
          bl = ol;
        }
      }
      if (bl == 32) break;
      if (lane == bl) {
        if (cw == 0)
          my_old = false;
        else
          my_new = false;
      }
      if (lane == r) {
        nk = bkk;
        ni = bi;
      }
      ++taken;
    }
    top_k = nk;
    top_i = ni;
    have = taken;
  }
  // 4. outputs
  const int kk = a.k;
  if (lane < kk) {
    a.out_ids[(size_t)q * kk + lane] = lane < have ? top_i : -1;
    a.out_keys[(size_t)q * kk + lane] = lane < have ? top_k : DF{-INFINITY, 0.0f};
  }
  const float kth = __shfl_sync(0xffffffffu, top_k.hi, kk - 1);
  if (lane == 0) {
    a.out_count[q] = have;
    if (!pass_b) {
      // every vector outside the lists has BF16 key <= worst_bf_list, so exact key <=
      // worst_bf_list + eps; certified when that is below the k-th exact key (less half an ulp)
      const float tau = have == kk ? __fsub_rd(__fsub_rd(kth, eps), fabsf(kth) * 1.1920929e-7f) : -INFINITY;
      const bool cert = have == a.n || (have == kk && worst_bf_list < tau);
      a.tau[q] = tau;
      a.needs[q] = cert ? 0 : 1;
    } else {
      a.needs[q] = a.list_count[q] > a.coll_cap ? 1 : 0;
    }
  }
}

}  // namespace
}  // namespace nmsg

// ====================================================================== host side
#include <cudaTypedefs.h>

namespace nmsg {

struct BruteForceState {
  int kp = 0;       // padded dim (multiple of 64, <= 256)
  float max_xn = 0; // largest |x|^2 over the base (l2 bound)
  DevBuf x16, x32, xn, xn_hi, xn_lo, xt_max, dx_max;
  DevBuf q32, q16, qn_hi, qn_lo, eps, cand_key, cand_id, tau, needs, qact, coll_id, coll_key, coll_cnt;
  DevBuf out_id, out_key, out_cnt, scr_id, scr_key, fin_id, fin_key, fin_cnt, status;
  DevBuf h_q, h_ids, h_dists, h_counts;
  CUtensorMap tmx;
};

void destroy_bruteforce(BruteForceState* s) {
  if (!s) return;
  for (DevBuf* b : {&s->x16, &s->x32, &s->xn, &s->xn_hi, &s->xn_lo, &s->xt_max, &s->dx_max, &s->q32, &s->q16, &s->qn_hi,
                    &s->qn_lo, &s->eps, &s->cand_key, &s->cand_id, &s->tau, &s->needs, &s->qact, &s->coll_id,
                    &s->coll_key, &s->coll_cnt, &s->out_id, &s->out_key, &s->out_cnt, &s->scr_id, &s->scr_key,
                    &s->fin_id, &s->fin_key, &s->fin_cnt, &s->status, &s->h_q, &s->h_ids, &s->h_dists, &s->h_counts})
    b->release();
  delete s;
}

namespace {

// bf16 copy of the base (row pitch kp, zero padded), |x|^2 in fp32 and double-float, and the
// per-dimension maxima of |bf16(x)| and |x - bf16(x)| (as float bits, non-negative, so integer
// max is float max). One warp per row.
__global__ void prep_base_kernel(const float* __restrict__ x, int64_t n, int dim, int kp, __nv_bfloat16* __restrict__ x16,
                                 float* __restrict__ xn, float* __restrict__ xn_hi, float* __restrict__ xn_lo,
                                 unsigned* __restrict__ xt_max, unsigned* __restrict__ dx_max) {
  const int lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (row >= n) return;
  const float* xr = x + row * dim;
  DF acc{0.0f, 0.0f};
  for (int e = lane; e < kp; e += 32) {
    const float v = e < dim ? xr[e] : 0.0f;
    const __nv_bfloat16 b = __float2bfloat16_rn(v);
    x16[row * kp + e] = b;
    if (e < dim) {
      const float bv = __bfloat162float(b);
      atomicMax(xt_max + e, __float_as_uint(fabsf(bv)));
      atomicMax(dx_max + e, __float_as_uint(fabsf(__fsub_rn(v, bv))));
      acc = df_add_df(acc, df_mul_ff(v, v));
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    DF other{__shfl_xor_sync(0xffffffffu, acc.hi, o), __shfl_xor_sync(0xffffffffu, acc.lo, o)};
    acc = df_add_df(acc, other);
  }
  if (lane == 0) {
    xn[row] = acc.hi;  // fp32 |x|^2 used with the BF16 scores (its error is part of eps)
    xn_hi[row] = acc.hi;
    xn_lo[row] = acc.lo;
  }
}

// Per query: normalise (cosine, as NormalizeVect: unfused sum, 1/sqrtf), bf16 copy, |q|^2 in
// double-float, and eps = a rigorous bound on |BF16 key - exact key| for every base row:
//   |q.x - bf(q).bf(x)| <= sum_i |bfq_i| dx_i + |dq_i| xt_i + |dq_i| dx_i   (representation)
//                        + (kp + 2) 2^-22 sum_i |bfq_i| xt_i               (FP32 accumulation, 4x slack)
// and for l2 keys (2 dot - |x|^2): 2 * that + 2^-20 (2 sum_i |bfq_i| xt_i + max |x|^2).
__global__ void prep_query_kernel(const float* __restrict__ qin, int nq, int dim, int kp, int mpad, int cosine,
                                  int l2, const unsigned* __restrict__ xt_max, const unsigned* __restrict__ dx_max,
                                  float max_xn, float* __restrict__ q32, __nv_bfloat16* __restrict__ q16,
                                  float* __restrict__ qn_hi, float* __restrict__ qn_lo, float* __restrict__ eps) {
  const int lane = threadIdx.x & 31;
  const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (q >= mpad) return;
  if (q >= nq) {  // zero padding rows of the last query block
    for (int e = lane; e < kp; e += 32) q16[(size_t)q * kp + e] = __float2bfloat16_rn(0.0f);
    return;
  }
  const float* src = qin + (size_t)q * dim;
  float scale = 1.0f;
  if (cosine) {
    float sum = 0.0f;
    if (lane == 0) {
      for (int e = 0; e < dim; ++e) sum = __fadd_rn(sum, __fmul_rn(src[e], src[e]));
    }
    sum = __shfl_sync(0xffffffffu, sum, 0);
    if (sum != 0.0f) scale = __fdiv_rn(1.0f, __fsqrt_rn(sum));
  }
  float rep = 0.0f, mag = 0.0f;
  DF acc{0.0f, 0.0f};
  for (int e = lane; e < kp; e += 32) {
    float v = 0.0f;
    if (e < dim) {
      v = src[e];
      if (cosine && scale != 1.0f) v = __fmul_rn(v, scale);
      q32[(size_t)q * dim + e] = v;
    }
    const __nv_bfloat16 b = __float2bfloat16_rn(v);
    q16[(size_t)q * kp + e] = b;
    if (e < dim) {
      const float bv = fabsf(__bfloat162float(b));
      const float dv = fabsf(__fsub_rn(v, __bfloat162float(b)));
      const float xt = __uint_as_float(xt_max[e]), dx = __uint_as_float(dx_max[e]);
      rep += bv * dx + dv * xt + dv * dx;
      mag += bv * xt;
      acc = df_add_df(acc, df_mul_ff(v, v));
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    rep += __shfl_xor_sync(0xffffffffu, rep, o);
    mag += __shfl_xor_sync(0xffffffffu, mag, o);
    DF other{__shfl_xor_sync(0xffffffffu, acc.hi, o), __shfl_xor_sync(0xffffffffu, acc.lo, o)};
    acc = df_add_df(acc, other);
  }
  if (lane == 0) {
    // the float sums above round; 1% slack covers them
    float e_dot = 1.01f * (rep + (float)(kp + 2) * 2.384185791e-7f * mag);
    float e = l2 ? 2.0f * e_dot + 9.5367431640625e-7f * (2.0f * mag + max_xn) : e_dot;
    eps[q] = e;
    qn_hi[q] = acc.hi;
    qn_lo[q] = acc.lo;
  }
}

// Final rows: external ids and distances in the index's space convention.
__global__ void finish_kernel(const int32_t* __restrict__ id_a, const DF* __restrict__ key_a,
                              const int32_t* __restrict__ cnt_a, const int32_t* __restrict__ id_b,
                              const DF* __restrict__ key_b, const int32_t* __restrict__ cnt_b,
                              const uint8_t* __restrict__ use_b, int nq, int k, int kmax, int space,
                              const float* __restrict__ qn_hi, const float* __restrict__ qn_lo,
                              const int32_t* __restrict__ ext_id, int32_t* __restrict__ ids, float* __restrict__ dists,
                              int32_t* __restrict__ counts) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nq) return;
  const bool b = use_b && use_b[q];
  const int32_t* id = (b ? id_b : id_a) + (size_t)q * k;
  const DF* key = (b ? key_b : key_a) + (size_t)q * k;
  const int cnt = b ? cnt_b[q] : cnt_a[q];
  for (int j = 0; j < kmax; ++j) {
    if (j < cnt && j < k) {
      ids[(size_t)q * kmax + j] = ext_id[id[j]];
      const DF kv = key[j];
      float d;
      if (space == NMSG_SPACE_L2) {
        DF t = df_add_df(DF{qn_hi[q], qn_lo[q]}, DF{-kv.hi, -kv.lo});
        d = __fadd_rn(t.hi, t.lo);
        if (d < 0.0f) d = 0.0f;
      } else if (space == NMSG_SPACE_COSINE) {
        const float c = __fadd_rn(kv.hi, kv.lo);
        const float mn = (c < 1.0f) ? c : 1.0f;
        const float mx = (-1.0f < mn) ? mn : -1.0f;
        const float v = __fsub_rn(1.0f, mx);
        d = (0.0f < v) ? v : 0.0f;
      } else {
        d = -__fadd_rn(kv.hi, kv.lo);
      }
      dists[(size_t)q * kmax + j] = d;
    } else {
      ids[(size_t)q * kmax + j] = -1;
      dists[(size_t)q * kmax + j] = __int_as_float(0x7f800000);
    }
  }
  counts[q] = min(cnt, k);
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult qr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &qr) == cudaSuccess &&
        qr == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// 2-D bf16 tensor map over a [rows][kp] matrix, 64 x box_rows tiles with the 128-byte swizzle.
bool make_tmap(CUtensorMap* m, void* base, int64_t rows, int kp, int box_rows) {
  auto enc = tensor_map_encoder();
  if (!enc) return false;
  cuuint64_t dims[2] = {(cuuint64_t)kp, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)kp * 2};
  cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int bf_fail(int code, const std::string& msg) {
  set_last_error(msg);
  return code;
}

#define BF_CUDA(call, what)                                                       \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess) return bf_fail(e_ == cudaErrorMemoryAllocation ? NMSG_ERR_OOM : NMSG_ERR_DEVICE, \
                                          std::string(what) + ": " + cudaGetErrorString(e_)); \
  } while (0)

int prepare_base(nmsg_index* h, BruteForceState* s) {
  const HostIndex& hi = h->host;
  const int64_t n = hi.n;
  const int dim = hi.dim;
  s->kp = ((dim + BK - 1) / BK) * BK;
  std::vector<float> x((size_t)n * dim);
  double max_xn = 0;
  for (int64_t i = 0; i < n; ++i) {
    const float* v = hi.vec(i);
    std::memcpy(x.data() + i * dim, v, 4 * dim);
    double a = 0;
    for (int e = 0; e < dim; ++e) a += (double)v[e] * v[e];
    max_xn = std::max(max_xn, a);
  }
  s->max_xn = (float)max_xn;
  BF_CUDA(s->x32.ensure(x.size() * 4, false), "cudaMalloc(brute-force fp32 base)");
  BF_CUDA(cudaMemcpy(s->x32.p, x.data(), x.size() * 4, cudaMemcpyHostToDevice), "upload base");
  BF_CUDA(s->x16.ensure((size_t)n * s->kp * 2, false), "cudaMalloc(bf16 base)");
  const int64_t npad = ((n + BN - 1) / BN) * BN;  // the scan reads norms 32 at a time per tile
  BF_CUDA(s->xn.ensure(npad * 4, true), "cudaMalloc(norms)");
  BF_CUDA(s->xn_hi.ensure(n * 4, false), "cudaMalloc(norms)");
  BF_CUDA(s->xn_lo.ensure(n * 4, false), "cudaMalloc(norms)");
  BF_CUDA(s->xt_max.ensure(dim * 4, true), "cudaMalloc(bounds)");
  BF_CUDA(s->dx_max.ensure(dim * 4, true), "cudaMalloc(bounds)");
  const int wpb = 8;
  prep_base_kernel<<<(unsigned)((n + wpb - 1) / wpb), 32 * wpb>>>(
      s->x32.as<float>(), n, dim, s->kp, s->x16.as<__nv_bfloat16>(), s->xn.as<float>(), s->xn_hi.as<float>(),
      s->xn_lo.as<float>(), s->xt_max.as<unsigned>(), s->dx_max.as<unsigned>());
  BF_CUDA(cudaGetLastError(), "prepare base");
  BF_CUDA(cudaDeviceSynchronize(), "prepare base");
  if (!make_tmap(&s->tmx, s->x16.p, n, s->kp, BN)) return bf_fail(NMSG_ERR_DEVICE, "cuTensorMapEncodeTiled (base)");
  return NMSG_OK;
}

}  // namespace
}  // namespace nmsg

using namespace nmsg;

extern "C" NMSG_API int nmsg_bruteforce_knn(nmsg_index* h, const float* queries, int64_t nq, int32_t dim, int32_t k,
                                            int32_t kmax, int32_t* ids, float* dists, int32_t* counts,
                                            int64_t* stats, uint32_t flags, void* stream) {
  if (!h) return bf_fail(NMSG_ERR_BAD_ARG, "Must call createIndex or loadIndex before this method");
  if (nq < 0 || k < 1 || kmax < k) return bf_fail(NMSG_ERR_BAD_ARG, "nq must be >= 0, k >= 1 and kmax >= k");
  if (k > CAND) return bf_fail(NMSG_ERR_UNSUPPORTED, "brute force supports k <= 32");
  if (nq > 0 && (!queries || !ids || !dists || !counts)) return bf_fail(NMSG_ERR_BAD_ARG, "null buffer");
  std::lock_guard<std::mutex> lk(h->mu);
  const bool dev_ptrs = flags & NMSG_DEVICE_PTRS;
  if (nq == 0) return NMSG_OK;
  const HostIndex& hi = h->host;
  const int64_t n = hi.n;
  if (n == 0) {
    if (dev_ptrs) return bf_fail(NMSG_ERR_BAD_ARG, "empty index");
    std::fill(counts, counts + nq, 0);
    std::fill(ids, ids + nq * kmax, -1);
    std::fill(dists, dists + nq * kmax, __builtin_inff());
    return NMSG_OK;
  }
  if (dim != hi.dim) return bf_fail(NMSG_ERR_BAD_ARG, "query dimension does not match the index dimension");
  if (((dim + BK - 1) / BK) > KB_MAX) return bf_fail(NMSG_ERR_UNSUPPORTED, "brute force supports dim <= 256");
  DeviceGuard g(h->device);
  cudaStream_t st = (cudaStream_t)stream;
  if (!h->bf) {
    h->bf = new BruteForceState();
    const int rc = prepare_base(h, h->bf);
    if (rc != NMSG_OK) {
      destroy_bruteforce(h->bf);
      h->bf = nullptr;
      return rc;
    }
  }
  BruteForceState* s = h->bf;
  const int kp = s->kp, kb = kp / BK;
  const int space = h->space;
  const int l2 = space == NMSG_SPACE_L2, cosine = space == NMSG_SPACE_COSINE;
  const int q_blocks = (int)((nq + BM - 1) / BM);
  const int mpad = q_blocks * BM;
  const int n_tiles = (int)((n + BN - 1) / BN);
  int n_chunks = std::max(1, std::min(n_tiles, (4 * h->num_sms + q_blocks - 1) / q_blocks));
  const int chunk_tiles = (n_tiles + n_chunks - 1) / n_chunks;
  n_chunks = (n_tiles + chunk_tiles - 1) / chunk_tiles;
  const int n_items = q_blocks * n_chunks;
  const int coll_cap = 16384;

  // inputs
  const float* qin = queries;
  if (!dev_ptrs) {
    BF_CUDA(s->h_q.ensure((size_t)nq * dim * 4, false), "cudaMalloc(query staging)");
    BF_CUDA(cudaMemcpyAsync(s->h_q.p, queries, (size_t)nq * dim * 4, cudaMemcpyHostToDevice, st), "copy queries");
    qin = s->h_q.as<float>();
  }
  BF_CUDA(s->q32.ensure((size_t)nq * dim * 4, false), "cudaMalloc");
  BF_CUDA(s->q16.ensure((size_t)mpad * kp * 2, false), "cudaMalloc");
  BF_CUDA(s->qn_hi.ensure(nq * 4, false), "cudaMalloc");
  BF_CUDA(s->qn_lo.ensure(nq * 4, false), "cudaMalloc");
  BF_CUDA(s->eps.ensure(nq * 4, false), "cudaMalloc");
  BF_CUDA(s->cand_key.ensure((size_t)nq * n_chunks * HALVES * CAND * 4, false), "cudaMalloc");
  BF_CUDA(s->cand_id.ensure((size_t)nq * n_chunks * HALVES * CAND * 4, false), "cudaMalloc");
  BF_CUDA(s->tau.ensure(nq * 4, false), "cudaMalloc");
  BF_CUDA(s->needs.ensure(mpad, false), "cudaMalloc");
  BF_CUDA(s->out_id.ensure((size_t)nq * k * 4, false), "cudaMalloc");
  BF_CUDA(s->out_key.ensure((size_t)nq * k * 8, false), "cudaMalloc");
  BF_CUDA(s->out_cnt.ensure(nq * 4, false), "cudaMalloc");
  BF_CUDA(s->status.ensure(4, true), "cudaMalloc");
  const float max_xn = s->max_xn;
  prep_query_kernel<<<(mpad + 7) / 8, 256, 0, st>>>(qin, (int)nq, dim, kp, mpad, cosine, l2, s->xt_max.as<unsigned>(),
                                                     s->dx_max.as<unsigned>(), max_xn * 1.0001f, s->q32.as<float>(),
                                                     s->q16.as<__nv_bfloat16>(), s->qn_hi.as<float>(),
                                                     s->qn_lo.as<float>(), s->eps.as<float>());
  BF_CUDA(cudaGetLastError(), "prepare queries");
  CUtensorMap tmq;
  if (!make_tmap(&tmq, s->q16.p, mpad, kp, BM)) return bf_fail(NMSG_ERR_DEVICE, "cuTensorMapEncodeTiled (queries)");
  BF_CUDA(cudaMemsetAsync(s->status.p, 0, 4, st), "reset status");

  GemmArgs ga;
  ga.kb = kb;
  ga.n = (int)n;
  ga.nq = (int)nq;
  ga.n_tiles = n_tiles;
  ga.chunk_tiles = chunk_tiles;
  ga.n_chunks = n_chunks;
  ga.q_blocks = q_blocks;
  ga.stages = kb <= 2 ? 3 : 2;
  ga.mode = 0;
  ga.key_l2 = l2;
  ga.xnorm2 = s->xn.as<float>();
  ga.cand_key = s->cand_key.as<float>();
  ga.cand_id = s->cand_id.as<int32_t>();
  ga.tau = s->tau.as<float>();
  ga.q_active = s->needs.as<uint8_t>();
  ga.status = s->status.as<int32_t>();
  const int smem = SmemLayout(kb, ga.stages).total + 1024;
  BF_CUDA(cudaFuncSetAttribute(bf16_scan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem), "smem attribute");
  const int grid = std::min(n_items, h->num_sms);
  bf16_scan_kernel<<<grid, kThreads, smem, st>>>(tmq, s->tmx, ga);
  BF_CUDA(cudaGetLastError(), "brute-force scan (pass A)");

  RerankArgs ra;
  ra.q = s->q32.as<float>();
  ra.x = s->x32.as<float>();
  ra.xn_hi = s->xn_hi.as<float>();
  ra.xn_lo = s->xn_lo.as<float>();
  ra.dim = dim;
  ra.n = (int)n;
  ra.nq = (int)nq;
  ra.k = k;
  ra.l2 = l2;
  ra.n_lists = n_chunks * HALVES;
  ra.list_len = CAND;
  ra.ids = s->cand_id.as<int32_t>();
  ra.bf_keys = s->cand_key.as<float>();
  ra.list_count = nullptr;
  ra.eps = s->eps.as<float>();
  ra.out_ids = s->out_id.as<int32_t>();
  ra.out_keys = s->out_key.as<DF>();
  ra.out_count = s->out_cnt.as<int32_t>();
  ra.tau = s->tau.as<float>();
  ra.needs = s->needs.as<uint8_t>();
  ra.coll_cap = coll_cap;
  BF_CUDA(cudaMemsetAsync(s->needs.p, 0, mpad, st), "reset flags");
  rerank_kernel<<<(unsigned)((nq + 7) / 8), 256, 0, st>>>(ra);
  BF_CUDA(cudaGetLastError(), "rerank (pass A)");

  // which queries are not certified?
  std::vector<uint8_t> needs(nq);
  BF_CUDA(cudaMemcpyAsync(needs.data(), s->needs.p, nq, cudaMemcpyDeviceToHost, st), "copy flags");
  int32_t dstatus = 0;
  BF_CUDA(cudaMemcpyAsync(&dstatus, s->status.p, 4, cudaMemcpyDeviceToHost, st), "copy status");
  BF_CUDA(cudaStreamSynchronize(st), "brute force pass A");
  if (dstatus) return bf_fail(dstatus, "brute-force scan reported a device-side error");
  int64_t n_uncert = 0;
  for (uint8_t v : needs) n_uncert += v;
  const bool pass_b = n_uncert > 0;
  if (pass_b) {
    BF_CUDA(s->coll_id.ensure((size_t)nq * coll_cap * 4, false), "cudaMalloc(collection)");
    BF_CUDA(s->coll_key.ensure((size_t)nq * coll_cap * 4, false), "cudaMalloc(collection)");
    BF_CUDA(s->coll_cnt.ensure(nq * 4, false), "cudaMalloc(collection)");
    BF_CUDA(s->fin_id.ensure((size_t)nq * k * 4, false), "cudaMalloc");
    BF_CUDA(s->fin_key.ensure((size_t)nq * k * 8, false), "cudaMalloc");
    BF_CUDA(s->fin_cnt.ensure(nq * 4, false), "cudaMalloc");
    BF_CUDA(s->qact.ensure(mpad, false), "cudaMalloc");
    BF_CUDA(cudaMemcpyAsync(s->qact.p, s->needs.p, mpad, cudaMemcpyDeviceToDevice, st), "copy flags");
    BF_CUDA(cudaMemsetAsync(s->coll_cnt.p, 0, nq * 4, st), "reset counts");
    ga.mode = 1;
    ga.q_active = s->qact.as<uint8_t>();
    ga.coll_id = s->coll_id.as<int32_t>();
    ga.coll_key = s->coll_key.as<float>();
    ga.coll_cnt = s->coll_cnt.as<int32_t>();
    ga.coll_cap = coll_cap;
    bf16_scan_kernel<<<grid, kThreads, smem, st>>>(tmq, s->tmx, ga);
    BF_CUDA(cudaGetLastError(), "brute-force scan (pass B)");
    RerankArgs rb = ra;
    rb.ids = s->coll_id.as<int32_t>();
    rb.bf_keys = s->coll_key.as<float>();
    rb.list_count = s->coll_cnt.as<int32_t>();
    rb.out_ids = s->fin_id.as<int32_t>();
    rb.out_keys = s->fin_key.as<DF>();
    rb.out_count = s->fin_cnt.as<int32_t>();
    rb.needs = s->needs.as<uint8_t>();  // now: 1 = collection overflowed
    rerank_kernel<<<(unsigned)((nq + 7) / 8), 256, 0, st>>>(rb);
    BF_CUDA(cudaGetLastError(), "rerank (pass B)");
  }
  // outputs
  int32_t* o_ids = ids;
  float* o_d = dists;
  int32_t* o_c = counts;
  if (!dev_ptrs) {
    BF_CUDA(s->h_ids.ensure((size_t)nq * kmax * 4, false), "cudaMalloc(staging)");
    BF_CUDA(s->h_dists.ensure((size_t)nq * kmax * 4, false), "cudaMalloc(staging)");
    BF_CUDA(s->h_counts.ensure(nq * 4, false), "cudaMalloc(staging)");
    o_ids = s->h_ids.as<int32_t>();
    o_d = s->h_dists.as<float>();
    o_c = s->h_counts.as<int32_t>();
  }
  finish_kernel<<<(unsigned)((nq + 127) / 128), 128, 0, st>>>(
      s->out_id.as<int32_t>(), s->out_key.as<DF>(), s->out_cnt.as<int32_t>(), s->fin_id.as<int32_t>(),
      s->fin_key.as<DF>(), s->fin_cnt.as<int32_t>(), pass_b ? s->qact.as<uint8_t>() : nullptr, (int)nq, k, kmax,
      space, s->qn_hi.as<float>(), s->qn_lo.as<float>(), h->dev.ext_id, o_ids, o_d, o_c);
  BF_CUDA(cudaGetLastError(), "finish");
  int64_t n_overflow = 0;
  if (pass_b) {
    std::vector<uint8_t> ov(nq);
    BF_CUDA(cudaMemcpyAsync(ov.data(), s->needs.p, nq, cudaMemcpyDeviceToHost, st), "copy flags");
    BF_CUDA(cudaMemcpyAsync(&dstatus, s->status.p, 4, cudaMemcpyDeviceToHost, st), "copy status");
    BF_CUDA(cudaStreamSynchronize(st), "brute force pass B");
    for (int64_t i = 0; i < nq; ++i) n_overflow += ov[i] && needs[i];
    if (dstatus) return bf_fail(dstatus, "brute-force scan reported a device-side error");
  }
  if (!dev_ptrs) {
    BF_CUDA(cudaMemcpyAsync(ids, o_ids, (size_t)nq * kmax * 4, cudaMemcpyDeviceToHost, st), "copy ids");
    BF_CUDA(cudaMemcpyAsync(dists, o_d, (size_t)nq * kmax * 4, cudaMemcpyDeviceToHost, st), "copy distances");
    BF_CUDA(cudaMemcpyAsync(counts, o_c, nq * 4, cudaMemcpyDeviceToHost, st), "copy counts");
    BF_CUDA(cudaStreamSynchronize(st), "copy results");
  }
  if (stats) {
    stats[0] = nq - n_uncert;  // certified after pass A
    stats[1] = n_uncert;       // resolved by pass B
    stats[2] = n_overflow;
    stats[3] = n_chunks;
  }
  if (n_overflow)
    return bf_fail(NMSG_ERR_CAPACITY, std::to_string(n_overflow) + " queries had more than 16384 vectors within the "
                                      "BF16 error bound of their k-th neighbour");
  return NMSG_OK;
}
