// Exact brute-force k-NN over the loaded index's vectors — the semantics of NMSLIB's sequential
// search (similarity_search/src/method/seqsearch.cc:143-177: every stored object is compared
// with the query and the k best are kept, knnquery.cc:67-75) — computed as:
//
//   sample  a tcgen05 BF16 x BF16 -> FP32 GEMM of 128-query tiles against a strided sample of
//           the 256-row base tiles (TMA-fed, accumulators double-buffered in TMEM) whose epilogue
//           keeps, per query, the C best of the sample's 32-column group maxima (one base
//           vector per group);
//   rerank  exact scores of those candidates in double-float arithmetic (error-free products and
//           sums on FP32 units, about 2^-44 relative); the exact k-th score of the sample is a
//           lower bound of the exact k-th score of the whole base, so with a rigorous per-query
//           bound eps on |BF16 score - exact score|, tau = (sample k-th - eps) is a BF16 score
//           that every true top-k vector reaches;
//   scan    the same GEMM over every base tile, collecting each vector whose BF16 score is
//           >= tau (a few hundred per query), then the exact rerank of that set. A query whose
//           set overflows the collection buffer is scanned once more with tau raised to the
//           exact k-th score of what it did collect less eps (again a lower bound).
//
// So the returned ids are the exact top-k (ties by id), independent of BF16 rounding.
// Scores ("keys", larger is better): negdot and cosine use q.x (queries of the cosine space
// are normalised as NormalizeVect does, base vectors are stored normalised); l2 uses
// 2 q.x - |x|^2, so distance = |q|^2 - key is the squared L2 the HNSW path reports.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
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
constexpr int KB_MAX = 4;               // padded dim <= 256 with the query block resident
constexpr int KB_STREAM_MAX = 64;       // padded dim <= 4096 with query K-blocks streamed per stage
constexpr int Q_BLOCK_BYTES = BM * BK * 2;   // 16 KB
constexpr int X_STAGE_BYTES = BN * BK * 2;   // 32 KB
constexpr int EPI_WARPS = 8;            // sample pass: two warps per TMEM lane quarter, one per column half
constexpr int HALVES = 2;
constexpr int SCAN_EPI_WARPS = 16;      // full scan: four warps per lane quarter, one per column quarter
constexpr int SCAN_PARTS = 4;
// Warps of each pass: its epilogue warps, then the TMA warp and the MMA warp.
template <int MODE>
struct Roles {
  static constexpr int kEpi = MODE == 1 ? SCAN_EPI_WARPS : EPI_WARPS;
  static constexpr int kThreads = (kEpi + 2) * 32;
};
constexpr int LIST_STRIDE = CAND + 1;   // +1: rows of a list on different banks
constexpr int kCollectLen = 64;         // entries of a full-scan list (query, chunk, column half)

struct GemmArgs {
  int kb;             // padded dim / 64
  int stages;         // base-tile pipeline depth (3 when kb <= 2, else 2; 3 when streaming)
  int stream_q;       // 1: rows wider than 256: each stage carries the query block's K-block with the
                      // base K-block (the whole query block does not fit in shared memory)
  int n;              // base rows
  int nq;             // queries
  int n_tiles;        // tiles visited: tile j of the scan is base tile j * tile_step
  int tile_step;      // 1 for the full scan, > 1 for the sample
  int chunk_tiles;    // visited tiles per work item
  int n_chunks;
  int q_blocks;
  int per_column;     // sample pass: offer every column, not only each 32-column group's best
  int key_l2;         // 1: key = 2 dot - |x|^2, 0: key = dot
  const float* xnorm2;  // |x|^2 (l2) or 0, +inf for the padding rows up to n_tiles * BN
  // one list of list_len entries per (query, chunk, column part), written only by the thread
  // that owns that query row in that work item: mode 0 the best group maxima of a column half
  // (list_len = CAND), mode 1 the rows of a column quarter whose key reaches tau (the count may
  // exceed list_len: the list overflowed)
  int list_len;
  float* list_key;    // [nq][n_chunks * parts][list_len], parts = HALVES (mode 0) or SCAN_PARTS (1)
  int32_t* list_id;
  int32_t* list_cnt;  // [nq][n_chunks * parts]
  const float* tau;   // [nq]
  const uint8_t* q_active;  // [q_blocks * BM]
  int32_t* status;
};

// Shared memory: Q blocks | base stages | candidate lists | barriers (1024-aligned base). When the
// query is streamed there is no resident Q region and each stage is a base K-block followed by
// the query block's K-block.
struct SmemLayout {
  int q_off, x_off, stage_bytes, key_off, id_off, nrm_off, bar_off, total;
  __host__ __device__ SmemLayout(int kb, int stages, int stream_q) {
    q_off = 0;
    x_off = q_off + (stream_q ? 0 : kb * Q_BLOCK_BYTES);
    stage_bytes = X_STAGE_BYTES + (stream_q ? Q_BLOCK_BYTES : 0);
    key_off = x_off + stages * stage_bytes;
    id_off = key_off + HALVES * BM * LIST_STRIDE * 4;
    nrm_off = id_off + HALVES * BM * LIST_STRIDE * 4;  // per epilogue warp: its 128 columns' |x|^2
    bar_off = (nrm_off + EPI_WARPS * (BN / HALVES) * 4 + 7) & ~7;
    total = bar_off + 8 * (2 * 4 + 2 + 4 + 1) + 16;
  }
};

template <int MODE>
__device__ __forceinline__ bool item_active(const GemmArgs& a, int qb) {
  if (MODE == 0) return true;
  const uint8_t* p = a.q_active + (size_t)qb * BM;
  for (int i = 0; i < BM; ++i)
    if (p[i]) return true;
  return false;
}

// First active work item at or after `item` in this CTA's round-robin sequence (n_items if none).
template <int MODE>
__device__ __forceinline__ int next_active_item(const GemmArgs& a, int item, int n_items) {
  while (item < n_items && !item_active<MODE>(a, item % a.q_blocks)) item += gridDim.x;
  return item;
}

// The largest of three floats in one instruction (max.f32 with three sources).
__device__ __forceinline__ float max3f(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

// v[i] of 16 values for a lane-dependent i, by four levels of selects.
__device__ __forceinline__ float pick16(const float (&v)[16], int i) {
  float a[8];
#pragma unroll
  for (int t = 0; t < 8; ++t) a[t] = (i & 8) ? v[t + 8] : v[t];
#pragma unroll
  for (int t = 0; t < 4; ++t) a[t] = (i & 4) ? a[t + 4] : a[t];
#pragma unroll
  for (int t = 0; t < 2; ++t) a[t] = (i & 2) ? a[t + 2] : a[t];
  return (i & 1) ? a[1] : a[0];
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

// MODE 0: the sample pass (per-row candidate heaps); MODE 1: the full scan (threshold lists).
// Compiled separately so that each carries only its own epilogue code.
template <int MODE>
__global__ void __launch_bounds__(Roles<MODE>::kThreads, 1)
    bf16_scan_kernel(const __grid_constant__ CUtensorMap tmq, const __grid_constant__ CUtensorMap tmx, GemmArgs a) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const SmemLayout L(a.kb, a.stages, a.stream_q);
  const int sbytes = L.stage_bytes;
  uint8_t* sq = base + L.q_off;
  uint8_t* sx = base + L.x_off;
  float* skey = reinterpret_cast<float*>(base + L.key_off);
  int32_t* sid = reinterpret_cast<int32_t*>(base + L.id_off);
  float* snrm = reinterpret_cast<float*>(base + L.nrm_off);
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + L.bar_off);
  uint64_t* x_full = bars;          // [4]
  uint64_t* x_empty = bars + 4;     // [4]
  uint64_t* q_full = bars + 8;
  uint64_t* q_empty = bars + 9;
  uint64_t* acc_full = bars + 10;   // [2]
  uint64_t* acc_empty = bars + 12;  // [2]
  uint64_t* mma_drain = bars + 14;  // the MMA thread's last commit, waited on before teardown
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 15);
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
      mbar_init(&acc_empty[i], Roles<MODE>::kEpi);  // one arrival per epilogue warp
    }
    mbar_init(mma_drain, 1);
    fence_barrier_init();
  }
  if (warp == 0) tmem_alloc(tmem_slot, 512);
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  bool ok = true;

  if (warp == Roles<MODE>::kEpi) {
    // ------------------------------------------------ TMA producer
    // A load is issued only after its slot's empty barrier completed. After a failed wait nothing
    // more is issued, and before the role ends it waits (bounded) for the last load armed on each
    // slot, so no TMA write into shared memory is in flight when the CTA tears down.
    if (lane == 0) {
      prefetch_tmap(&tmq);
      prefetch_tmap(&tmx);
      int stage = 0;
      uint32_t xphase = 0, qphase = 0;
      int prev_qb = -1;
      int x_armed = 0, q_armed = 0;  // loads armed on x_full (all stages) and on q_full
      // items are chunk-major: the CTAs running at the same time read the same base chunk, which
      // stays in L2 while every query block passes over it. The query block is loaded only when
      // it differs from the previous item's (for batches of <= 128 queries, once per CTA).
      for (int item = next_active_item<MODE>(a, blockIdx.x, n_items); item < n_items && ok;
           item = next_active_item<MODE>(a, item + gridDim.x, n_items)) {
        const int qb = item % a.q_blocks, chunk = item / a.q_blocks;
        if (qb != prev_qb && !a.stream_q) {
          if (prev_qb >= 0) {
            ok = mbar_wait(q_empty, qphase);
            qphase ^= 1;
            if (!ok) break;
          }
          mbar_arrive_expect_tx(q_full, a.kb * Q_BLOCK_BYTES);
          for (int kb = 0; kb < a.kb; ++kb) tma_load_2d(sq + kb * Q_BLOCK_BYTES, &tmq, q_full, kb * BK, qb * BM);
          ++q_armed;
          prev_qb = qb;
        }
        const int t0 = chunk * a.chunk_tiles, t1 = min(a.n_tiles, t0 + a.chunk_tiles);
        for (int vt = t0; vt < t1 && ok; ++vt) {
          const int t = vt * a.tile_step;
          for (int kb = 0; kb < a.kb && ok; ++kb) {
            ok = mbar_wait(&x_empty[stage], xphase ^ 1);
            if (!ok) break;
            mbar_arrive_expect_tx(&x_full[stage], (uint32_t)sbytes);
            tma_load_2d(sx + stage * sbytes, &tmx, &x_full[stage], kb * BK, t * BN);
            if (a.stream_q) tma_load_2d(sx + stage * sbytes + X_STAGE_BYTES, &tmq, &x_full[stage], kb * BK, qb * BM);
            ++x_armed;
            if (++stage == stages) {
              stage = 0;
              xphase ^= 1;
            }
          }
        }
      }
      // drain: the c-th arming of a barrier (from 0) completes its phase c, so the last load on
      // slot s has parity (arms(s) - 1) & 1; earlier loads on s completed before its reuse
      for (int s = 0; s < stages; ++s) {
        const int arms = x_armed / stages + (s < x_armed % stages ? 1 : 0);
        if (arms > 0 && !mbar_wait(&x_full[s], (uint32_t)((arms - 1) & 1))) ok = false;
      }
      if (q_armed > 0 && !mbar_wait(q_full, (uint32_t)((q_armed - 1) & 1))) ok = false;
    }
  } else if (warp == Roles<MODE>::kEpi + 1) {
    // ------------------------------------------------ MMA issuer
    // No MMA and no commit is issued after a failed wait. Every MMA reads operands whose full
    // barrier completed, and before the role ends one last commit (only if an MMA was ever issued)
    // is waited on (bounded), so no tensor-core work is in flight at the final barrier and TMEM
    // deallocation.
    if (lane == 0) {
      const uint32_t idesc = idesc_bf16_f32(BM, BN);
      int stage = 0;
      uint32_t xphase = 0, qphase = 0;
      uint32_t accphase[2] = {0, 0};
      int tcount = 0, prev_qb = -1;
      bool issued = false;  // some MMA was issued by this thread
      for (int item = next_active_item<MODE>(a, blockIdx.x, n_items); item < n_items && ok;) {
        const int next = next_active_item<MODE>(a, item + gridDim.x, n_items);
        const int qb = item % a.q_blocks, chunk = item / a.q_blocks;
        if (qb != prev_qb && !a.stream_q) {
          ok = mbar_wait(q_full, qphase);
          qphase ^= 1;
          if (!ok) break;
          tc_fence_after();
          prev_qb = qb;
        }
        const int t0 = chunk * a.chunk_tiles, t1 = min(a.n_tiles, t0 + a.chunk_tiles);
        for (int vt = t0; vt < t1 && ok; ++vt, ++tcount) {
          const int buf = tcount & 1;
          ok = mbar_wait(&acc_empty[buf], accphase[buf] ^ 1);
          accphase[buf] ^= 1;
          if (!ok) break;
          tc_fence_after();
          const uint32_t dcol = tmem + buf * BN;
          for (int kb = 0; kb < a.kb; ++kb) {
            ok = mbar_wait(&x_full[stage], xphase);
            if (!ok) break;
            tc_fence_after();
            const uint32_t xa = smem_u32(sx + stage * sbytes);
            const uint32_t qa = a.stream_q ? xa + X_STAGE_BYTES : smem_u32(sq + kb * Q_BLOCK_BYTES);
#pragma unroll
            for (int k = 0; k < BK / 16; ++k)
              umma_bf16(dcol, smem_desc_sw128(qa + 32 * k), smem_desc_sw128(xa + 32 * k), idesc, kb > 0 || k > 0);
            issued = true;
            umma_commit(&x_empty[stage]);
            if (++stage == stages) {
              stage = 0;
              xphase ^= 1;
            }
          }
          if (!ok) break;
          umma_commit(&acc_full[buf]);
        }
        if (!ok) break;
        // the query block's buffer is free for the next one once these MMAs complete
        if (issued && !a.stream_q && next < n_items && next % a.q_blocks != qb) umma_commit(q_empty);
        item = next;
      }
      if (issued) {
        umma_commit(mma_drain);
        if (!mbar_wait(mma_drain, 0)) ok = false;
      }
    }
  } else if constexpr (MODE == 1) {
    // ------------------------------------------------ epilogue of the full scan: warps 0-15. Warp w
    // reads TMEM lane quarter w & 3 (thread = one query row) and the 64 columns of part w >> 2 of
    // each tile, 16 at a time: four warps per scheduler hide the latency of the threshold test and
    // of the rare hit path, which two warps per scheduler left exposed.
    constexpr int CW = BN / SCAN_PARTS;  // columns per warp
    const int quarter = warp & 3, part = warp >> 2;
    const int row = quarter * 32 + lane;
    float* snw = snrm + warp * CW;  // |x|^2 of this warp's columns of the tile
    uint32_t accphase[2] = {0, 0};
    int tcount = 0;
    for (int item = blockIdx.x; item < n_items && ok; item += gridDim.x) {
      const int qb = item % a.q_blocks, chunk = item / a.q_blocks;
      if (!item_active<MODE>(a, qb)) continue;
      const int q = qb * BM + row;
      const bool qvalid = q < a.nq;
      // tau, with a finite floor so the -inf keys of columns past the last row never qualify
      const float thr = (qvalid && a.q_active[q]) ? fmaxf(a.tau[q], -FLT_MAX) : INFINITY;
      const int t0 = chunk * a.chunk_tiles, t1 = min(a.n_tiles, t0 + a.chunk_tiles);
      // |x|^2 of this part's columns, 4 per lane in lanes 0-15, loaded one tile ahead
      const float4* xn4 = reinterpret_cast<const float4*>(a.xnorm2) + part * (CW / 4) + (lane & 15);
      float4 nrm_next = make_float4(0.f, 0.f, 0.f, 0.f);
      if (t0 < t1) nrm_next = __ldg(xn4 + (size_t)t0 * a.tile_step * (BN / 4));
      const float ks = a.key_l2 ? 2.0f : 1.0f;
      const size_t list = ((size_t)q * a.n_chunks + chunk) * SCAN_PARTS + part;
      int32_t* cid = a.list_id + list * a.list_len;
      float* ckey = a.list_key + list * a.list_len;
      int ncoll = 0;
      for (int vt = t0; vt < t1 && ok; ++vt, ++tcount) {
        const int t = vt * a.tile_step;
        const int buf = tcount & 1;
        __syncwarp();  // every lane is done with the previous tile's norms
        if (lane < CW / 4) reinterpret_cast<float4*>(snw)[lane] = nrm_next;
        // the smallest |x|^2 of each 16-column group: lane 4g holds group g's
        float gmin = fminf(fminf(nrm_next.x, nrm_next.y), fminf(nrm_next.z, nrm_next.w));
        gmin = fminf(gmin, __shfl_xor_sync(0xffffffffu, gmin, 1));
        gmin = fminf(gmin, __shfl_xor_sync(0xffffffffu, gmin, 2));
        if (vt + 1 < t1) nrm_next = __ldg(xn4 + (size_t)(t + a.tile_step) * (BN / 4));
        __syncwarp();
        ok = mbar_wait(&acc_full[buf], accphase[buf]);
        accphase[buf] ^= 1;
        tc_fence_after();
        // the work on one 16-column group (cur: its accumulators)
        auto group = [&](const uint32_t (&cur)[16], int c) {
          const int col0 = t * BN + part * CW + c * 16;
          // An upper bound of the group's keys (ks * acc - xnorm2): ks * (largest acc) - (smallest
          // xnorm2), rounded as one FMA. The exact sum is at least every column's, and rounding to
          // nearest is monotone, so no key of the group exceeds the bound: below tau, the group
          // has no hit and its keys are never formed. The maximum: three-input max instructions.
          const float m0 = max3f(__uint_as_float(cur[0]), __uint_as_float(cur[1]), __uint_as_float(cur[2]));
          const float m1 = max3f(__uint_as_float(cur[3]), __uint_as_float(cur[4]), __uint_as_float(cur[5]));
          const float m2 = max3f(__uint_as_float(cur[6]), __uint_as_float(cur[7]), __uint_as_float(cur[8]));
          const float m3 = max3f(__uint_as_float(cur[9]), __uint_as_float(cur[10]), __uint_as_float(cur[11]));
          const float m4 = max3f(__uint_as_float(cur[12]), __uint_as_float(cur[13]), __uint_as_float(cur[14]));
          const float mx = fmaxf(max3f(m0, m1, m2), max3f(m3, m4, __uint_as_float(cur[15])));
          const float bound = __fmaf_rn(ks, mx, -__shfl_sync(0xffffffffu, gmin, 4 * c));
          // one warp vote first: the common case (no row of the warp passes) skips the rest
          if (__any_sync(0xffffffffu, bound >= thr)) {
            // the keys, as in the sample pass (rows past the base have key -inf)
            float v[16];
            const float4* nv = reinterpret_cast<const float4*>(snw + c * 16);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const float4 x4 = nv[j];  // same address in every lane: a broadcast
              v[4 * j + 0] = __fmaf_rn(ks, __uint_as_float(cur[4 * j + 0]), -x4.x);
              v[4 * j + 1] = __fmaf_rn(ks, __uint_as_float(cur[4 * j + 1]), -x4.y);
              v[4 * j + 2] = __fmaf_rn(ks, __uint_as_float(cur[4 * j + 2]), -x4.z);
              v[4 * j + 3] = __fmaf_rn(ks, __uint_as_float(cur[4 * j + 3]), -x4.w);
            }
            // this row's hits as a bit mask built with selects, then one store pair per hit in a
            // loop whose trip count is the warp's largest hit count, plain stores into the row's list
            unsigned hm = 0;
#pragma unroll
            for (int i = 0; i < 16; ++i) hm |= (v[i] >= thr ? 1u : 0u) << i;
            while (__any_sync(0xffffffffu, hm != 0)) {
              if (hm) {
                const int i = __ffs(hm) - 1;
                hm &= hm - 1;
                if (ncoll < a.list_len) {
                  cid[ncoll] = col0 + i;
                  ckey[ncoll] = pick16(v, i);
                }
                ++ncoll;
              }
            }
          }
          __syncwarp();
        };
        // TMEM loads of the next 16 columns overlap the work on the current ones, the groups
        // alternating between two register buffers (no copies between them)
        const uint32_t tb = tmem + ((uint32_t)(quarter * 32) << 16) + buf * BN + part * CW;
        uint32_t ra[16], rb[16];
        tmem_ld16_issue(tb, ra);
        tmem_ld_wait16(ra);
#pragma unroll 1
        for (int c = 0; c < CW / 16; c += 2) {
          tmem_ld16_issue(tb + 16 * (c + 1), rb);
          group(ra, c);
          tmem_ld_wait16(rb);
          if (c + 2 < CW / 16) {
            tmem_ld16_issue(tb + 16 * (c + 2), ra);
          } else {  // every load of this tile has completed
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[buf]);  // this warp's part of the accumulator is read
          }
          group(rb, c + 1);
          if (c + 2 < CW / 16) tmem_ld_wait16(ra);
        }
      }
      if (qvalid) a.list_cnt[list] = ncoll;
    }
  } else {
    // ------------------------------------------------ epilogue of the sample pass: warps 0-7; thread
    // = one query row (TMEM lane) for one half of the tile's columns, 32 columns at a time
    const int quarter = warp & 3, half = warp >> 2;
    const int row = quarter * 32 + lane;
    float* lk = skey + (half * BM + row) * LIST_STRIDE;
    int32_t* li = sid + (half * BM + row) * LIST_STRIDE;
    float* snw = snrm + warp * (BN / HALVES);  // |x|^2 of this warp's 128 columns of the tile
    uint32_t accphase[2] = {0, 0};
    int tcount = 0;
    for (int item = blockIdx.x; item < n_items && ok; item += gridDim.x) {
      const int qb = item % a.q_blocks, chunk = item / a.q_blocks;
      if (!item_active<MODE>(a, qb)) continue;
      const int q = qb * BM + row;
      const bool qvalid = q < a.nq;
      float thr = -INFINITY;  // the list's smallest key once full
      int nfill = 0;
      const int t0 = chunk * a.chunk_tiles, t1 = min(a.n_tiles, t0 + a.chunk_tiles);
      // |x|^2 of this half's 128 columns, 4 per lane, loaded one tile ahead
      const float4* xn4 = reinterpret_cast<const float4*>(a.xnorm2) + half * (BN / HALVES / 4) + lane;
      float4 nrm_next = make_float4(0.f, 0.f, 0.f, 0.f);
      if (t0 < t1) nrm_next = __ldg(xn4 + (size_t)t0 * a.tile_step * (BN / 4));
      const float ks = a.key_l2 ? 2.0f : 1.0f;
      const size_t list = ((size_t)q * a.n_chunks + chunk) * HALVES + half;
      int32_t* cid = a.list_id + list * a.list_len;
      float* ckey = a.list_key + list * a.list_len;
      for (int vt = t0; vt < t1 && ok; ++vt, ++tcount) {
        const int t = vt * a.tile_step;
        const int buf = tcount & 1;
        __syncwarp();  // every lane is done with the previous tile's norms
        reinterpret_cast<float4*>(snw)[lane] = nrm_next;
        if (vt + 1 < t1) nrm_next = __ldg(xn4 + (size_t)(t + a.tile_step) * (BN / 4));
        __syncwarp();
        ok = mbar_wait(&acc_full[buf], accphase[buf]);
        accphase[buf] ^= 1;
        tc_fence_after();
        // the work on one 32-column group (cur: its accumulators)
        auto group = [&](const uint32_t (&cur)[32], int c) {
          const int col0 = t * BN + half * (BN / HALVES) + c * 32;
          // keys: ks * acc - xnorm2 (l2: 2 q.x - |x|^2, where 2 acc is exact so one FMA rounds
          // as the two-step form would; dot spaces: acc - 0). Rows past the base have
          // xnorm2 = +inf, so their key is -inf.
          float v[32];
          const float4* nv = reinterpret_cast<const float4*>(snw + c * 32);
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const float4 x4 = nv[j];  // same address in every lane: a broadcast
            v[4 * j + 0] = __fmaf_rn(ks, __uint_as_float(cur[4 * j + 0]), -x4.x);
            v[4 * j + 1] = __fmaf_rn(ks, __uint_as_float(cur[4 * j + 1]), -x4.y);
            v[4 * j + 2] = __fmaf_rn(ks, __uint_as_float(cur[4 * j + 2]), -x4.z);
            v[4 * j + 3] = __fmaf_rn(ks, __uint_as_float(cur[4 * j + 3]), -x4.w);
          }
          // the group's largest key, with three-input max instructions
          float m[10];
#pragma unroll
          for (int i = 0; i < 10; ++i) m[i] = max3f(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
          const float mx = fmaxf(max3f(max3f(m[0], m[1], m[2]), max3f(m[3], m[4], m[5]), max3f(m[6], m[7], m[8])),
                                 max3f(m[9], v[30], v[31]));
          if (a.per_column) {
            // small bases (the sample is all of it): every column is offered
            if ((mx > thr || nfill < CAND) && mx > -INFINITY) {
              float vl[32];
#pragma unroll
              for (int i = 0; i < 32; ++i) vl[i] = v[i];
#pragma unroll 1
              for (int i = 0; i < 32; ++i)
                if ((vl[i] > thr || nfill < CAND) && vl[i] > -INFINITY)
                  list_offer(lk, li, nfill, thr, vl[i], col0 + i);
            }
          } else if ((mx > thr || nfill < CAND) && mx > -INFINITY) {
            // the group's best column is the candidate: the lists hold distinct base vectors,
            // so the exact k-th key among them still bounds the true k-th key from below
            int arg = 31;
#pragma unroll
            for (int i = 30; i >= 0; --i) arg = v[i] == mx ? i : arg;
            list_offer(lk, li, nfill, thr, mx, col0 + arg);
          }
          __syncwarp();
        };
        // TMEM loads of the next group of 32 columns overlap the work on the current one, the
        // groups alternating between two register buffers (no copies between them)
        const uint32_t tb = tmem + ((uint32_t)(quarter * 32) << 16) + buf * BN + half * (BN / HALVES);
        uint32_t ra[32], rb[32];
        tmem_ld32_issue(tb, ra);
        tmem_ld_wait(ra);
#pragma unroll 1
        for (int c = 0; c < BN / HALVES / 32; c += 2) {
          tmem_ld32_issue(tb + 32 * (c + 1), rb);
          group(ra, c);
          tmem_ld_wait(rb);
          if (c + 2 < BN / HALVES / 32) {
            tmem_ld32_issue(tb + 32 * (c + 2), ra);
          } else {  // every load of this tile has completed
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[buf]);  // the accumulator is read out
          }
          group(rb, c + 1);
          if (c + 2 < BN / HALVES / 32) tmem_ld_wait(ra);
        }
      }
      if (qvalid) {
        for (int j = 0; j < nfill; ++j) {
          ckey[j] = lk[j];
          cid[j] = li[j];
        }
        a.list_cnt[list] = nfill;
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

struct RerankArgs {
  const float* q;        // [nq][dim] (normalised for cosine)
  const float* x;        // [n][dim] natural order, fp32
  const float* xn_hi;    // l2: |x|^2 as double-float
  const float* xn_lo;
  int dim, n, nq, k, l2;
  int n_lists, list_len;       // lists of list_len entries per query
  int32_t* ids;                // [nq][n_lists][list_len] internal ids, compacted in place here
  float* bf_keys;              // BF16 keys, same layout
  const int32_t* list_count;   // [nq][n_lists] entries found per list (more than list_len: overflow)
  const float* eps;            // [nq] bound on |BF16 key - exact key|
  const uint8_t* only;         // optional: rerank only the queries flagged here
  // outputs
  int32_t* out_ids;            // [nq][k] internal ids, best first
  DF* out_keys;                // [nq][k]
  int32_t* out_count;          // [nq]
  float* tau;                  // [nq] BF16 threshold that every true top-k vector reaches
  uint8_t* needs;              // optional [nq]: 1 = some list overflowed
  int32_t* found;              // optional [nq]: entries found over all lists
};

// (key, id) order of the result: larger key first, then smaller id.
__device__ __forceinline__ bool better(DF ka, int ia, DF kb, int ib) {
  return df_greater(ka, kb) || (ka.hi == kb.hi && ka.lo == kb.lo && ia < ib);
}

// Exact key of one (query, row) pair computed by a single lane (sequential over the dimension), in
// FP64: a product of two floats is exact in a double and each FMA rounds the running sum once (a
// relative error of about dim * 2^-53, far below the BF16 bound eps), returned as a double-float
// pair (hi = the double rounded to float, lo = the rest rounded to float) like the other keys.
__device__ DF exact_key_lane(const float* __restrict__ q, const float* __restrict__ x, int dim, bool l2, DF xnorm) {
  double acc = 0.0;
  if ((dim & 3) == 0) {  // rows and queries start on 16-byte boundaries
    const float4* q4 = reinterpret_cast<const float4*>(q);
    const float4* x4 = reinterpret_cast<const float4*>(x);
    for (int e = 0; e < dim / 4; ++e) {
      const float4 a = q4[e];
      const float4 b = __ldg(x4 + e);
      acc = fma((double)a.x, (double)b.x, acc);
      acc = fma((double)a.y, (double)b.y, acc);
      acc = fma((double)a.z, (double)b.z, acc);
      acc = fma((double)a.w, (double)b.w, acc);
    }
  } else {
    for (int e = 0; e < dim; ++e) acc = fma((double)q[e], (double)__ldg(x + e), acc);
  }
  if (l2) acc = fma(2.0, acc, -((double)xnorm.hi + (double)xnorm.lo));
  const float hi = __double2float_rn(acc);
  return DF{hi, __double2float_rn(acc - (double)hi)};
}

// One warp per query:
//  1. B_k = the k-th largest BF16 key among the candidates (pairs (key, slot), k rounds of
//     warp max);
//  2. only candidates with BF16 key >= B_k - 2 eps can be in the exact top k (the k candidates
//     at or above B_k all have exact keys >= B_k - eps, anything below B_k - 2 eps has an exact
//     key < B_k - eps), so only they get exact keys, one candidate per lane;
//  3. the exact top k by (key desc, id asc), merged 32 candidates at a time;
//  4. tau = exact k-th key - eps (rounded down, less one ulp of the double-float's high part):
//     the candidates are real base vectors, so their exact k-th key is at most the true k-th
//     key, and every true top-k vector has a BF16 key >= tau.
__global__ void rerank_kernel(RerankArgs a) {
  const int lane = threadIdx.x & 31;
  const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (q >= a.nq) return;
  if (a.only && !a.only[q]) return;
  const size_t base = (size_t)q * a.n_lists * a.list_len;
  int32_t* ids = a.ids + base;
  float* bk = a.bf_keys + base;
  const float eps = a.eps[q];

  // 0. compact the lists in place: list l's first min(count, list_len) entries move to the running
  //    total (never past their own position, and each lane reads before any lane writes)
  int total = 0, found_all = 0;
  bool overflow = false;
  const int32_t* lc = a.list_count + (size_t)q * a.n_lists;
  for (int l0 = 0; l0 < a.n_lists; l0 += 32) {
    const int my_cnt = l0 + lane < a.n_lists ? lc[l0 + lane] : 0;
    found_all += my_cnt;
    overflow |= my_cnt > a.list_len;
    unsigned nonempty = __ballot_sync(0xffffffffu, my_cnt > 0);
    while (nonempty) {
      const int j = __ffs(nonempty) - 1;
      nonempty &= nonempty - 1;
      const int cnt = min(__shfl_sync(0xffffffffu, my_cnt, j), a.list_len);
      for (int c0 = 0; c0 < cnt; c0 += 32) {
        const int take = min(32, cnt - c0);
        const int src = (l0 + j) * a.list_len + c0 + lane;
        int32_t id = 0;
        float key = 0.0f;
        if (lane < take) {
          id = ids[src];
          key = bk[src];
        }
        __syncwarp();
        if (lane < take) {
          ids[total + lane] = id;
          bk[total + lane] = key;
        }
        __syncwarp();
        total += take;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) found_all += __shfl_xor_sync(0xffffffffu, found_all, o);
  overflow = __any_sync(0xffffffffu, overflow);

  // 1. k-th largest BF16 key (pairs ordered by key desc, slot asc)
  float prev_k = INFINITY;
  int prev_s = -1;
  int found = 0;
  for (int r = 0; r < a.k; ++r) {
    float bkey = -INFINITY;
    int bslot = 0x7fffffff;
    for (int t = lane; t < total; t += 32) {
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
      if (!(bk[t] >= cut)) id = -1;
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
    a.tau[q] = have == kk ? __fsub_rd(__fsub_rd(kth, eps), fabsf(kth) * 1.1920929e-7f) : -INFINITY;
    if (a.needs) a.needs[q] = overflow ? 1 : 0;
    if (a.found) a.found[q] = found_all;
  }
}

}  // namespace
}  // namespace nmsg

// ====================================================================== host side
#include <cudaTypedefs.h>

namespace nmsg {

struct BruteForceState {
  bool base_ready = false;  // the BF16 base and its bounds exist (the exact scan needs none of it)
  int kp = 0;       // padded dim (multiple of 64, <= 4096)
  float max_xn = 0; // largest |x|^2 over the base (l2 bound)
  DevBuf x16, x32, xn, xn_hi, xn_lo, xt_max, dx_max;
  DevBuf q32, q16, qn_hi, qn_lo, eps, cand_key, cand_id, cand_cnt, tau, needs, qact, coll_id, coll_key, coll_cnt, found;
  DevBuf out_id, out_key, out_cnt, scr_id, scr_key, fin_id, fin_key, fin_cnt, status;
  DevBuf h_q, h_ids, h_dists, h_counts;
  CUtensorMap tmx;
};

void destroy_bruteforce(BruteForceState* s) {
  if (!s) return;
  for (DevBuf* b : {&s->x16, &s->x32, &s->xn, &s->xn_hi, &s->xn_lo, &s->xt_max, &s->dx_max, &s->q32, &s->q16, &s->qn_hi,
                    &s->qn_lo, &s->eps, &s->cand_key, &s->cand_id, &s->cand_cnt, &s->tau, &s->needs, &s->qact,
                    &s->coll_id, &s->coll_key, &s->coll_cnt, &s->found, &s->out_id, &s->out_key, &s->out_cnt, &s->scr_id, &s->scr_key,
                    &s->fin_id, &s->fin_key, &s->fin_cnt, &s->status, &s->h_q, &s->h_ids, &s->h_dists, &s->h_counts})
    b->release();
  delete s;
}

namespace {

// bf16 copy of the base (row pitch kp, zero padded), |x|^2 in fp32 and double-float, and the
// per-dimension maxima of |bf16(x)| and |x - bf16(x)| (as float bits, non-negative, so integer
// max is float max). One warp per row.
__global__ void prep_base_kernel(const float* __restrict__ x, int64_t n, int dim, int kp, int l2, __nv_bfloat16* __restrict__ x16,
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
    xn[row] = l2 ? acc.hi : 0.0f;  // fp32 |x|^2 used with the BF16 scores (its error is part of eps)
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
__global__ void finish_kernel(const int32_t* __restrict__ id_in, const DF* __restrict__ key_in,
                              const int32_t* __restrict__ cnt_in, int nq, int k, int kmax, int space,
                              const float* __restrict__ qn_hi, const float* __restrict__ qn_lo,
                              const int32_t* __restrict__ ext_id, int32_t* __restrict__ ids, float* __restrict__ dists,
                              int32_t* __restrict__ counts) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nq) return;
  const int32_t* id = id_in + (size_t)q * k;
  const DF* key = key_in + (size_t)q * k;
  const int cnt = cnt_in[q];
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
// The driver's result code of the last failed encoding (for the error message).
thread_local int g_tmap_result = 0;

bool make_tmap(CUtensorMap* m, void* base, int64_t rows, int kp, int box_rows) {
  auto enc = tensor_map_encoder();
  if (!enc) return false;
  cuuint64_t dims[2] = {(cuuint64_t)kp, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)kp * 2};
  cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  g_tmap_result = (int)r;
  return r == CUDA_SUCCESS;
}

std::string tmap_error(const char* what, int64_t rows, int kp, const void* base) {
  return std::string("cuTensorMapEncodeTiled (") + what + "): CUresult " + std::to_string(g_tmap_result) +
         ", rows " + std::to_string(rows) + ", padded dim " + std::to_string(kp) + ", address " +
         std::to_string((uintptr_t)base % 1024) + " mod 1024";
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
      s->x32.as<float>(), n, dim, s->kp, h->space == NMSG_SPACE_L2, s->x16.as<__nv_bfloat16>(), s->xn.as<float>(), s->xn_hi.as<float>(),
      s->xn_lo.as<float>(), s->xt_max.as<unsigned>(), s->dx_max.as<unsigned>());
  BF_CUDA(cudaGetLastError(), "prepare base");
  if (npad > n) {
    const std::vector<float> inf((size_t)(npad - n), INFINITY);
    BF_CUDA(cudaMemcpy(s->xn.as<float>() + n, inf.data(), inf.size() * 4, cudaMemcpyHostToDevice), "pad norms");
  }
  BF_CUDA(cudaDeviceSynchronize(), "prepare base");
  if (!make_tmap(&s->tmx, s->x16.p, n, s->kp, BN)) return bf_fail(NMSG_ERR_DEVICE, tmap_error("base", n, s->kp, s->x16.p));
  return NMSG_OK;
}

// L1 / LInf and rows wider than 256: every distance exactly as the search computes it, on CUDA
// cores (exact_scan_knn); stats = {0, rows scanned per query, 0, base chunks per query block}.
int scan_fallback(nmsg_index* h, const float* queries, int64_t nq, int dim, int k, int kmax, int32_t* ids, float* dists,
                  int32_t* counts, int64_t* stats, bool dev_ptrs, cudaStream_t st) {
  BruteForceState* s = h->bf ? h->bf : (h->bf = new BruteForceState());
  const DevIndex& d = h->dev;
  const int64_t q_blocks = (nq + 7) / 8;
  // many small blocks (about 16 per SM) keep the last wave short
  const int n_chunks = (int)std::max<int64_t>(
      1, std::min<int64_t>((16 * h->num_sms + q_blocks - 1) / q_blocks, std::max<int64_t>(1, d.n / 2048)));
  const size_t n_part = (size_t)nq * n_chunks * exact_scan_lists(d) * k;
  const float* qin = queries;
  if (!dev_ptrs) {
    BF_CUDA(s->h_q.ensure((size_t)nq * dim * 4, false), "cudaMalloc(query staging)");
    const HostPiece up{s->h_q.p, queries, (size_t)nq * dim * 4};
    BF_CUDA(copy_to_device(h->pin_in, h->cfg.host_copy == 0, &up, 1, st), "copy queries");
    qin = s->h_q.as<float>();
  }
  BF_CUDA(s->scr_key.ensure(n_part * 4, false), "cudaMalloc(scan lists)");
  BF_CUDA(s->scr_id.ensure(n_part * 4, false), "cudaMalloc(scan lists)");
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
  const int rc = exact_scan_knn(d, qin, nq, k, kmax, s->scr_key.as<float>(), s->scr_id.as<int32_t>(), n_chunks, o_ids,
                                o_d, o_c, st);
  if (rc != 0)
    return bf_fail(NMSG_ERR_DEVICE, std::string("exact scan: ") + cudaGetErrorString((cudaError_t)rc) +
                                        (rc == (int)cudaErrorInvalidValue ? " (rows too wide for the scan)" : ""));
  if (!dev_ptrs) {
    const HostPiece down[3] = {{ids, o_ids, (size_t)nq * kmax * 4}, {dists, o_d, (size_t)nq * kmax * 4},
                               {counts, o_c, (size_t)nq * 4}};
    BF_CUDA(copy_to_host(h->pin_out, h->cfg.host_copy == 0, down, 3, st), "copy results");
  } else {
    BF_CUDA(cudaStreamSynchronize(st), "exact scan");
  }
  if (stats) {
    stats[0] = 0;
    stats[1] = d.n;
    stats[2] = 0;
    stats[3] = n_chunks;
  }
  return NMSG_OK;
}

}  // namespace
}  // namespace nmsg

using namespace nmsg;

extern "C" NMSG_API int nmsg_bruteforce_knn(nmsg_index* h, const float* queries, int64_t nq, int32_t dim, int32_t k,
                                            int32_t kmax, int32_t* ids, float* dists, int32_t* counts,
                                            int64_t* stats, uint32_t flags, void* stream) {
  if (!h) return bf_fail(NMSG_ERR_BAD_ARG, "Must call createIndex or loadIndex before this method");
  if (h->host.sift) return bf_fail(NMSG_ERR_UNSUPPORTED, "brute force over l2sqr_sift indices is not supported");
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
  DeviceGuard g(h->device);
  cudaStream_t st = (cudaStream_t)stream;
  const bool dot_space = h->space == NMSG_SPACE_L2 || h->space == NMSG_SPACE_COSINE || h->space == NMSG_SPACE_NEGDOT;
  if (!dot_space || ((dim + BK - 1) / BK) > KB_STREAM_MAX || (flags & NMSG_EXACT_SCAN))
    return scan_fallback(h, queries, nq, dim, k, kmax, ids, dists, counts, stats, dev_ptrs, st);
  if (!h->bf) h->bf = new BruteForceState();
  if (!h->bf->base_ready) {
    const int rc = prepare_base(h, h->bf);
    if (rc != NMSG_OK) {
      destroy_bruteforce(h->bf);
      h->bf = nullptr;
      return rc;
    }
    h->bf->base_ready = true;
  }
  BruteForceState* s = h->bf;
  const int kp = s->kp, kb = kp / BK;
  const int space = h->space;
  const int l2 = space == NMSG_SPACE_L2, cosine = space == NMSG_SPACE_COSINE;
  const int q_blocks = (int)((nq + BM - 1) / BM);
  const int mpad = q_blocks * BM;
  const int n_tiles = (int)((n + BN - 1) / BN);

  // the sample: every tile_step-th base tile, at least 16 tiles (or all of them), about 1/16
  // of the base; split into chunks so the sample pass also fills the GPU for small batches
  const int s_tiles = std::min(n_tiles, std::max(16, n_tiles / 16));
  const int s_step = n_tiles / s_tiles;
  // (chunks of at least 4 tiles; the split with the least of: tiles the busiest CTA visits plus the
  // rerank's cost of the candidate lists each chunk adds per query, which measured on B200 as about
  // 14 tile visits per chunk for 10K queries, in proportion to the query count)
  int s_chunks = 1, s_chunk_tiles = s_tiles;
  {
    const double per_chunk = 14.0 * (double)nq / 10000.0;
    double best = 1e300;
    for (int c = 1; c <= std::max(1, s_tiles / 4); ++c) {
      const int ct = (s_tiles + c - 1) / c, cc = (s_tiles + ct - 1) / ct;
      const int64_t rounds = ((int64_t)q_blocks * cc + h->num_sms - 1) / h->num_sms;
      const double cost = (double)rounds * ct + per_chunk * cc;
      if (cost < best - 1e-9) {
        best = cost;
        s_chunks = cc;
        s_chunk_tiles = ct;
      }
    }
  }
  // the full scan: about 8 or more work items per CTA, the split whose busiest CTA carries the
  // least excess over the average (items are dealt round-robin)
  int chunk_tiles = n_tiles, n_chunks = 1;
  {
    const int lo = std::max(1, std::min(n_tiles, (8 * h->num_sms + q_blocks - 1) / q_blocks));
    const int hi = std::min(n_tiles, 2 * lo);
    double best = 1e30;
    for (int c = lo; c <= hi; ++c) {
      const int ct = (n_tiles + c - 1) / c, cc = (n_tiles + ct - 1) / ct;
      const int64_t items = (int64_t)q_blocks * cc;
      const int64_t rounds = (items + h->num_sms - 1) / h->num_sms;
      const double cost = (double)rounds * ct / ((double)q_blocks * n_tiles / h->num_sms);
      if (cost < best - 1e-9) {
        best = cost;
        chunk_tiles = ct;
        n_chunks = cc;
      }
    }
  }

  // inputs
  const float* qin = queries;
  if (!dev_ptrs) {
    BF_CUDA(s->h_q.ensure((size_t)nq * dim * 4, false), "cudaMalloc(query staging)");
    const HostPiece up{s->h_q.p, queries, (size_t)nq * dim * 4};
    BF_CUDA(copy_to_device(h->pin_in, h->cfg.host_copy == 0, &up, 1, st), "copy queries");
    qin = s->h_q.as<float>();
  }
  BF_CUDA(s->q32.ensure((size_t)nq * dim * 4, false), "cudaMalloc");
  BF_CUDA(s->q16.ensure((size_t)mpad * kp * 2, false), "cudaMalloc");
  BF_CUDA(s->qn_hi.ensure(nq * 4, false), "cudaMalloc");
  BF_CUDA(s->qn_lo.ensure(nq * 4, false), "cudaMalloc");
  BF_CUDA(s->eps.ensure(nq * 4, false), "cudaMalloc");
  const size_t s_lists = (size_t)nq * s_chunks * HALVES, c_lists = (size_t)nq * n_chunks * SCAN_PARTS;
  BF_CUDA(s->cand_key.ensure(s_lists * CAND * 4, false), "cudaMalloc");
  BF_CUDA(s->cand_id.ensure(s_lists * CAND * 4, false), "cudaMalloc");
  BF_CUDA(s->cand_cnt.ensure(s_lists * 4, false), "cudaMalloc");
  BF_CUDA(s->tau.ensure(nq * 4, false), "cudaMalloc");
  BF_CUDA(s->needs.ensure(mpad, false), "cudaMalloc");
  BF_CUDA(s->qact.ensure(mpad, false), "cudaMalloc");
  BF_CUDA(s->out_id.ensure((size_t)nq * k * 4, false), "cudaMalloc");
  BF_CUDA(s->out_key.ensure((size_t)nq * k * 8, false), "cudaMalloc");
  BF_CUDA(s->out_cnt.ensure(nq * 4, false), "cudaMalloc");
  BF_CUDA(s->fin_id.ensure((size_t)nq * k * 4, false), "cudaMalloc");
  BF_CUDA(s->fin_key.ensure((size_t)nq * k * 8, false), "cudaMalloc");
  BF_CUDA(s->fin_cnt.ensure(nq * 4, false), "cudaMalloc");
  BF_CUDA(s->coll_id.ensure(c_lists * kCollectLen * 4, false), "cudaMalloc(collection)");
  BF_CUDA(s->coll_key.ensure(c_lists * kCollectLen * 4, false), "cudaMalloc(collection)");
  BF_CUDA(s->coll_cnt.ensure(c_lists * 4, false), "cudaMalloc(collection)");
  BF_CUDA(s->found.ensure(nq * 4, false), "cudaMalloc");
  BF_CUDA(s->status.ensure(4, true), "cudaMalloc");
  const float max_xn = s->max_xn;
  prep_query_kernel<<<(mpad + 7) / 8, 256, 0, st>>>(qin, (int)nq, dim, kp, mpad, cosine, l2, s->xt_max.as<unsigned>(),
                                                     s->dx_max.as<unsigned>(), max_xn * 1.0001f, s->q32.as<float>(),
                                                     s->q16.as<__nv_bfloat16>(), s->qn_hi.as<float>(),
                                                     s->qn_lo.as<float>(), s->eps.as<float>());
  BF_CUDA(cudaGetLastError(), "prepare queries");
  CUtensorMap tmq;
  if (!make_tmap(&tmq, s->q16.p, mpad, kp, BM)) return bf_fail(NMSG_ERR_DEVICE, tmap_error("queries", mpad, kp, s->q16.p));
  BF_CUDA(cudaMemsetAsync(s->status.p, 0, 4, st), "reset status");

  // 1. top-CAND BF16 candidates of the sample, exact rerank -> tau
  GemmArgs ga;
  std::memset(&ga, 0, sizeof(ga));
  ga.kb = kb;
  ga.n = (int)n;
  ga.nq = (int)nq;
  ga.n_tiles = s_tiles;
  ga.tile_step = s_step;
  ga.chunk_tiles = s_chunk_tiles;
  ga.n_chunks = s_chunks;
  ga.q_blocks = q_blocks;
  ga.stream_q = kb > KB_MAX ? 1 : 0;
  ga.stages = ga.stream_q ? 3 : (kb <= 2 ? 3 : 2);
  ga.per_column = s_tiles == n_tiles;
  ga.key_l2 = l2;
  ga.xnorm2 = s->xn.as<float>();
  ga.list_len = CAND;
  ga.list_key = s->cand_key.as<float>();
  ga.list_id = s->cand_id.as<int32_t>();
  ga.list_cnt = s->cand_cnt.as<int32_t>();
  ga.tau = s->tau.as<float>();
  ga.q_active = s->qact.as<uint8_t>();
  ga.status = s->status.as<int32_t>();
  const int smem = SmemLayout(kb, ga.stages, ga.stream_q).total + 1024;
  BF_CUDA((cudaError_t)allow_max_smem((const void*)bf16_scan_kernel<0>), "smem attribute");
  BF_CUDA((cudaError_t)allow_max_smem((const void*)bf16_scan_kernel<1>), "smem attribute");
  bf16_scan_kernel<0><<<std::min(q_blocks * s_chunks, h->num_sms), Roles<0>::kThreads, smem, st>>>(tmq, s->tmx, ga);
  BF_CUDA(cudaGetLastError(), "brute-force scan (sample)");

  RerankArgs ra;
  std::memset(&ra, 0, sizeof(ra));
  ra.q = s->q32.as<float>();
  ra.x = s->x32.as<float>();
  ra.xn_hi = s->xn_hi.as<float>();
  ra.xn_lo = s->xn_lo.as<float>();
  ra.dim = dim;
  ra.n = (int)n;
  ra.nq = (int)nq;
  ra.k = k;
  ra.l2 = l2;
  ra.n_lists = s_chunks * HALVES;
  ra.list_len = CAND;
  ra.ids = s->cand_id.as<int32_t>();
  ra.bf_keys = s->cand_key.as<float>();
  ra.list_count = s->cand_cnt.as<int32_t>();
  ra.eps = s->eps.as<float>();
  ra.out_ids = s->out_id.as<int32_t>();
  ra.out_keys = s->out_key.as<DF>();
  ra.out_count = s->out_cnt.as<int32_t>();
  ra.tau = s->tau.as<float>();
  const unsigned rr_blocks = (unsigned)((nq + 7) / 8);
  rerank_kernel<<<rr_blocks, 256, 0, st>>>(ra);
  BF_CUDA(cudaGetLastError(), "rerank (sample)");

  // 2. every base tile, collecting BF16 keys >= tau; exact rerank of the collection. A query
  //    whose collection overflowed is scanned again with the raised tau of what it collected
  //    (up to three times: tau rises each time unless the collected keys are all tied).
  GemmArgs gb = ga;
  gb.per_column = 0;
  gb.n_tiles = n_tiles;
  gb.tile_step = 1;
  gb.chunk_tiles = chunk_tiles;
  gb.n_chunks = n_chunks;
  gb.list_len = kCollectLen;
  gb.list_key = s->coll_key.as<float>();
  gb.list_id = s->coll_id.as<int32_t>();
  gb.list_cnt = s->coll_cnt.as<int32_t>();
  RerankArgs rb = ra;
  rb.n_lists = n_chunks * SCAN_PARTS;
  rb.list_len = kCollectLen;
  rb.ids = s->coll_id.as<int32_t>();
  rb.bf_keys = s->coll_key.as<float>();
  rb.list_count = s->coll_cnt.as<int32_t>();
  rb.out_ids = s->fin_id.as<int32_t>();
  rb.out_keys = s->fin_key.as<DF>();
  rb.out_count = s->fin_cnt.as<int32_t>();
  rb.needs = s->needs.as<uint8_t>();
  rb.found = s->found.as<int32_t>();
  BF_CUDA(cudaMemsetAsync(s->qact.p, 1, mpad, st), "reset flags");
  int64_t max_collected = 0, rescanned = 0, overflow = 0;
  std::vector<uint8_t> flags_h(nq);
  std::vector<int32_t> cnt_h(nq);
  int32_t dstatus = 0;
  constexpr int kScans = 4;
  for (int attempt = 0; attempt < kScans; ++attempt) {
    BF_CUDA(cudaMemsetAsync(s->found.p, 0, nq * 4, st), "reset counts");
    BF_CUDA(cudaMemsetAsync(s->needs.p, 0, mpad, st), "reset flags");
    bf16_scan_kernel<1><<<std::min(q_blocks * n_chunks, h->num_sms), Roles<1>::kThreads, smem, st>>>(tmq, s->tmx,
                                                                                                   gb);
    BF_CUDA(cudaGetLastError(), "brute-force scan");
    rb.only = attempt == 0 ? nullptr : s->qact.as<uint8_t>();  // the other queries keep their results
    rerank_kernel<<<rr_blocks, 256, 0, st>>>(rb);
    BF_CUDA(cudaGetLastError(), "rerank");
    BF_CUDA(cudaMemcpyAsync(flags_h.data(), s->needs.p, nq, cudaMemcpyDeviceToHost, st), "copy flags");
    BF_CUDA(cudaMemcpyAsync(cnt_h.data(), s->found.p, nq * 4, cudaMemcpyDeviceToHost, st), "copy counts");
    BF_CUDA(cudaMemcpyAsync(&dstatus, s->status.p, 4, cudaMemcpyDeviceToHost, st), "copy status");
    BF_CUDA(cudaStreamSynchronize(st), "brute-force scan");
    if (dstatus) return bf_fail(dstatus, "brute-force scan reported a device-side error");
    overflow = 0;
    for (int64_t i = 0; i < nq; ++i) {
      max_collected = std::max<int64_t>(max_collected, cnt_h[i]);
      overflow += flags_h[i];
    }
    if (!overflow || attempt + 1 == kScans) break;
    if (attempt == 0) rescanned = overflow;
    BF_CUDA(cudaMemcpyAsync(s->qact.p, s->needs.p, mpad, cudaMemcpyDeviceToDevice, st), "copy flags");
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
      s->fin_id.as<int32_t>(), s->fin_key.as<DF>(), s->fin_cnt.as<int32_t>(), (int)nq, k, kmax, space,
      s->qn_hi.as<float>(), s->qn_lo.as<float>(), h->dev.ext_id, o_ids, o_d, o_c);
  BF_CUDA(cudaGetLastError(), "finish");
  if (!dev_ptrs) {
    const HostPiece down[3] = {{ids, o_ids, (size_t)nq * kmax * 4}, {dists, o_d, (size_t)nq * kmax * 4},
                               {counts, o_c, (size_t)nq * 4}};
    BF_CUDA(copy_to_host(h->pin_out, h->cfg.host_copy == 0, down, 3, st), "copy results");
  } else {
    BF_CUDA(cudaStreamSynchronize(st), "brute-force results");
  }
  if (stats) {
    stats[0] = (int64_t)s_tiles * BN;  // sample rows (the last tile may be partial)
    stats[1] = max_collected;
    stats[2] = rescanned;
    stats[3] = n_chunks;
  }
  if (overflow)
    return bf_fail(NMSG_ERR_CAPACITY, std::to_string(overflow) + " queries had more vectors within the BF16 error "
                                      "bound of their k-th neighbour than the scan keeps (" + std::to_string(kCollectLen) +
                                      " per " + std::to_string(chunk_tiles * BN / SCAN_PARTS) + " base rows)");
  return NMSG_OK;
}
