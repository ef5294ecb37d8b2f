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
constexpr int STAGES = 3;               // base-tile pipeline depth
constexpr int CAND = 32;                // candidates kept per query per chunk (pass A)
constexpr int KB_MAX = 4;               // padded dim <= 256
constexpr int Q_BLOCK_BYTES = BM * BK * 2;   // 16 KB
constexpr int X_STAGE_BYTES = BN * BK * 2;   // 32 KB
constexpr int kThreads = 192;           // warps 0-3 epilogue, 4 TMA, 5 MMA

struct GemmArgs {
  int kb;             // padded dim / 64
  int n;              // base rows
  int nq;             // queries
  int n_tiles;        // ceil(n / BN)
  int chunk_tiles;    // base tiles per work item
  int n_chunks;
  int q_blocks;
  int mode;           // 0: top-CAND per chunk; 1: collect keys >= tau
  int key_l2;         // 1: key = 2 dot - |x|^2
  const float* xnorm2;
  float* cand_key;    // [nq][n_chunks][CAND]
  int32_t* cand_id;
  const float* tau;   // [nq]
  const uint8_t* q_active;  // [q_blocks * BM]
  int32_t* coll_id;   // [nq][coll_cap]
  float* coll_key;
  int32_t* coll_cnt;  // [nq]
  int coll_cap;
  int32_t* status;
};

struct __align__(1024) GemmSmem {
  uint8_t q[KB_MAX][Q_BLOCK_BYTES];
  uint8_t x[STAGES][X_STAGE_BYTES];
  float ckey[BM][CAND + 1];  // +1: rows on different banks
  int32_t cid[BM][CAND + 1];
  uint64_t x_full[STAGES], x_empty[STAGES];
  uint64_t q_full, q_empty;
  uint64_t acc_full[2], acc_empty[2];
  uint32_t tmem_base;
};

__device__ __forceinline__ bool item_active(const GemmArgs& a, int qb) {
  if (a.mode == 0) return true;
  const uint8_t* p = a.q_active + (size_t)qb * BM;
  for (int i = 0; i < BM; ++i)
    if (p[i]) return true;
  return false;
}

__global__ void __launch_bounds__(kThreads, 1)
    bf16_scan_kernel(const __grid_constant__ CUtensorMap tmq, const __grid_constant__ CUtensorMap tmx, GemmArgs a) {
  extern __shared__ uint8_t smem_raw[];
  GemmSmem& s = *reinterpret_cast<GemmSmem*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n_items = a.q_blocks * a.n_chunks;

  if (threadIdx.x == 0) {
    for (int i = 0; i < STAGES; ++i) {
      mbar_init(&s.x_full[i], 1);
      mbar_init(&s.x_empty[i], 1);
    }
    mbar_init(&s.q_full, 1);
    mbar_init(&s.q_empty, 1);
    for (int i = 0; i < 2; ++i) {
      mbar_init(&s.acc_full[i], 1);
      mbar_init(&s.acc_empty[i], 4);  // one arrival per epilogue warp
    }
    fence_barrier_init();
  }
  if (warp == 0) tmem_alloc(&s.tmem_base, 512);
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s.tmem_base;
  bool ok = true;

  if (warp == 4) {
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
          ok = mbar_wait(&s.q_empty, qphase);
          qphase ^= 1;
        }
        mbar_arrive_expect_tx(&s.q_full, a.kb * Q_BLOCK_BYTES);
        for (int kb = 0; kb < a.kb; ++kb) tma_load_2d(s.q[kb], &tmq, &s.q_full, kb * BK, qb * BM);
        const int t0 = chunk * a.chunk_tiles, t1 = min(a.n_tiles, t0 + a.chunk_tiles);
        for (int t = t0; t < t1 && ok; ++t) {
          for (int kb = 0; kb < a.kb && ok; ++kb) {
            ok = mbar_wait(&s.x_empty[stage], xphase ^ 1);
            mbar_arrive_expect_tx(&s.x_full[stage], X_STAGE_BYTES);
            tma_load_2d(s.x[stage], &tmx, &s.x_full[stage], kb * BK, t * BN);
            if (++stage == STAGES) {
              stage = 0;
              xphase ^= 1;
            }
          }
        }
        ++done_items;
      }
    }
  } else if (warp == 5) {
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
        ok = mbar_wait(&s.q_full, qphase);
        qphase ^= 1;
        tc_fence_after();
        const int t0 = chunk * a.chunk_tiles, t1 = min(a.n_tiles, t0 + a.chunk_tiles);
        for (int t = t0; t < t1 && ok; ++t, ++tcount) {
          const int buf = tcount & 1;
          ok = mbar_wait(&s.acc_empty[buf], accphase[buf] ^ 1);
          accphase[buf] ^= 1;
          tc_fence_after();
          const uint32_t dcol = tmem + buf * BN;
          for (int kb = 0; kb < a.kb && ok; ++kb) {
            ok = mbar_wait(&s.x_full[stage], xphase);
            tc_fence_after();
            const uint32_t qa = smem_u32(s.q[kb]), xa = smem_u32(s.x[stage]);
#pragma unroll
            for (int k = 0; k < BK / 16; ++k)
              umma_bf16(dcol, smem_desc_sw128(qa + 32 * k), smem_desc_sw128(xa + 32 * k), idesc, kb > 0 || k > 0);
            umma_commit(&s.x_empty[stage]);
            if (++stage == STAGES) {
              stage = 0;
              xphase ^= 1;
            }
          }
          umma_commit(&s.acc_full[buf]);
        }
        umma_commit(&s.q_empty);
      }
    }
  } else {
    // ------------------------------------------------ epilogue: warps 0-3, thread = query row
    const int row = warp * 32 + lane;
    uint32_t accphase[2] = {0, 0};
    int tcount = 0;
    for (int item = blockIdx.x; item < n_items && ok; item += gridDim.x) {
      const int qb = item / a.n_chunks, chunk = item % a.n_chunks;
      if (!item_active(a, qb)) continue;
      const int q = qb * BM + row;
      const bool qvalid = q < a.nq;
      float thr = -INFINITY;  // mode 0: current C-th best; mode 1: tau
      int nfill = 0, minpos = 0;
      if (a.mode == 1) thr = (qvalid && a.q_active[q]) ? a.tau[q] : INFINITY;
      const int t0 = chunk * a.chunk_tiles, t1 = min(a.n_tiles, t0 + a.chunk_tiles);
      for (int t = t0; t < t1 && ok; ++t, ++tcount) {
        const int buf = tcount & 1;
        ok = mbar_wait(&s.acc_full[buf], accphase[buf]);
        accphase[buf] ^= 1;
        tc_fence_after();
        for (int c = 0; c < BN / 32; ++c) {
          float v[32];
          tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + buf * BN + c * 32, v);
          const int col0 = t * BN + c * 32;
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            const int col = col0 + i;
            if (col >= a.n) continue;
            float key = v[i];
            if (a.key_l2) key = __fsub_rn(__fmul_rn(2.0f, key), __ldg(a.xnorm2 + col));
            if (a.mode == 0) {
              if (nfill < CAND) {
                s.ckey[row][nfill] = key;
                s.cid[row][nfill] = col;
                if (++nfill == CAND) {
                  thr = s.ckey[row][0];
                  minpos = 0;
                  for (int j = 1; j < CAND; ++j)
                    if (s.ckey[row][j] < thr) {
                      thr = s.ckey[row][j];
                      minpos = j;
                    }
                }
              } else if (key > thr) {
                s.ckey[row][minpos] = key;
                s.cid[row][minpos] = col;
                thr = s.ckey[row][0];
                minpos = 0;
                for (int j = 1; j < CAND; ++j)
                  if (s.ckey[row][j] < thr) {
                    thr = s.ckey[row][j];
                    minpos = j;
                  }
              }
            } else if (key >= thr) {
              const int slot = atomicAdd(a.coll_cnt + q, 1);
              if (slot < a.coll_cap) {
                a.coll_id[(size_t)q * a.coll_cap + slot] = col;
                a.coll_key[(size_t)q * a.coll_cap + slot] = key;
              }
            }
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&s.acc_empty[buf]);
      }
      if (a.mode == 0 && qvalid) {
        float* ok_out = a.cand_key + ((size_t)q * a.n_chunks + chunk) * CAND;
        int32_t* oi_out = a.cand_id + ((size_t)q * a.n_chunks + chunk) * CAND;
        for (int j = 0; j < CAND; ++j) {
          ok_out[j] = j < nfill ? s.ckey[row][j] : -INFINITY;
          oi_out[j] = j < nfill ? s.cid[row][j] : -1;
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
  int n_lists, list_len;       // candidate lists per query and their length
  const int32_t* ids;          // [nq][n_lists * list_len] (-1 = empty)
  const float* bf_keys;        // same shape, BF16 keys (pass A only, for the certificate)
  const int32_t* list_count;   // pass B: per-query count (null in pass A)
  const float* eps;            // [nq] bound on |BF16 key - exact key|
  // outputs
  int32_t* out_ids;            // [nq][k]
  DF* out_keys;                // [nq][k]
  int32_t* out_count;          // [nq]
  float* tau;                  // [nq] collection threshold (pass A), else unused
  uint8_t* needs;              // [nq] 1 = not certified (pass A) / overflowed (pass B)
  int coll_cap;
  int32_t* scratch_id;         // [nq][k] working top-k ids per warp slot
  DF* scratch_key;
};

// One warp per query: exact keys for every listed candidate, top-k by (key desc, id asc).
__global__ void rerank_kernel(RerankArgs a) {
  const int lane = threadIdx.x & 31;
  const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (q >= a.nq) return;
  const float* qv = a.q + (size_t)q * a.dim;
  int32_t* tid = a.scratch_id + (size_t)q * a.k;
  DF* tkey = a.scratch_key + (size_t)q * a.k;
  int have = 0;
  int total = a.n_lists * a.list_len;
  if (a.list_count) total = min(a.list_count[q], a.coll_cap);
  float worst_bf_chunk = -INFINITY;  // max over chunks of each chunk's C-th best BF16 key
  if (!a.list_count) {
    for (int c = 0; c < a.n_lists; ++c) {
      // a full chunk list bounds every vector of the chunk it dropped by its smallest key
      float mn = INFINITY;
      bool full = true;
      for (int j = lane; j < a.list_len; j += 32) {
        const int id = a.ids[(size_t)q * total + c * a.list_len + j];
        full &= id >= 0;
        mn = fminf(mn, a.bf_keys[(size_t)q * total + c * a.list_len + j]);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      full = __all_sync(0xffffffffu, full);
      if (full) worst_bf_chunk = fmaxf(worst_bf_chunk, mn);
    }
  }
  for (int t = 0; t < total; ++t) {
    const int id = a.list_count ? a.ids[(size_t)q * a.coll_cap + t] : a.ids[(size_t)q * total + t];
    if (id < 0) continue;
    DF xn{0.0f, 0.0f};
    if (a.l2) xn = DF{a.xn_hi[id], a.xn_lo[id]};
    const DF key = exact_key(qv, a.x + (size_t)id * a.dim, a.dim, a.l2, xn);
    // insert into the running top-k (sorted: best first); lane 0 does it
    if (lane == 0) {
      int pos = have;
      while (pos > 0) {
        const DF pk = tkey[pos - 1];
        const int pid = tid[pos - 1];
        if (df_greater(pk, key) || (pk.hi == key.hi && pk.lo == key.lo && pid < id)) break;
        if (pos < a.k) {
          tkey[pos] = pk;
          tid[pos] = pid;
        }
        --pos;
      }
      if (pos < a.k) {
        tkey[pos] = key;
        tid[pos] = id;
      }
    }
    have = min(have + 1, a.k);
    __syncwarp();
  }
  if (lane == 0) {
    for (int j = 0; j < a.k; ++j) {
      a.out_ids[(size_t)q * a.k + j] = j < have ? tid[j] : -1;
      a.out_keys[(size_t)q * a.k + j] = j < have ? tkey[j] : DF{-INFINITY, 0.0f};
    }
    a.out_count[q] = have;
    if (!a.list_count) {
      // certificate: every vector outside the candidates has BF16 key <= worst_bf_chunk, so
      // exact key <= worst_bf_chunk + eps; certified when that is below the k-th exact key
      // tau <= exact k-th key - eps: the hi part alone can exceed the exact value by half an ulp
      const float kth = have == a.k ? tkey[a.k - 1].hi : -INFINITY;
      const float tau = __fsub_rd(__fsub_rd(kth, a.eps[q]), fabsf(kth) * 1.1920929e-7f);
      const bool cert = have == a.n || (have == a.k && worst_bf_chunk < tau);
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
  BF_CUDA(s->xn.ensure(n * 4, false), "cudaMalloc(norms)");
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
  BF_CUDA(s->cand_key.ensure((size_t)nq * n_chunks * CAND * 4, false), "cudaMalloc");
  BF_CUDA(s->cand_id.ensure((size_t)nq * n_chunks * CAND * 4, false), "cudaMalloc");
  BF_CUDA(s->tau.ensure(nq * 4, false), "cudaMalloc");
  BF_CUDA(s->needs.ensure(mpad, false), "cudaMalloc");
  BF_CUDA(s->out_id.ensure((size_t)nq * k * 4, false), "cudaMalloc");
  BF_CUDA(s->out_key.ensure((size_t)nq * k * 8, false), "cudaMalloc");
  BF_CUDA(s->out_cnt.ensure(nq * 4, false), "cudaMalloc");
  BF_CUDA(s->scr_id.ensure((size_t)nq * k * 4, false), "cudaMalloc");
  BF_CUDA(s->scr_key.ensure((size_t)nq * k * 8, false), "cudaMalloc");
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
  ga.mode = 0;
  ga.key_l2 = l2;
  ga.xnorm2 = s->xn.as<float>();
  ga.cand_key = s->cand_key.as<float>();
  ga.cand_id = s->cand_id.as<int32_t>();
  ga.tau = s->tau.as<float>();
  ga.q_active = s->needs.as<uint8_t>();
  ga.status = s->status.as<int32_t>();
  const int smem = (int)sizeof(GemmSmem) + 1024;
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
  ra.n_lists = n_chunks;
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
  ra.scratch_id = s->scr_id.as<int32_t>();
  ra.scratch_key = s->scr_key.as<DF>();
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
