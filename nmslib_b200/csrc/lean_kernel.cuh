// The lean one-query-per-warp V1Merge kernel, instantiated per distance by lean_l2.cu,
// lean_cos.cu and lean_negdot.cu (so the three compile in parallel). See the comment at
// search_lean_kernel below.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "engine.h"
#include "search_device.cuh"
#include "sm100.cuh"
#include "../../include/nmslib_b200.h"

namespace nmsg {
namespace {

// ------------------------------------------------------------------ lean single-query kernel
// search_lean_kernel<NF, HALF, SP, NCH>: the persistent one-query-per-warp V1Merge search for the
// common index shapes, written for few instructions per expansion: rows of 32 * NF (+ 16 when
// HALF) floats, the distance code fixed at compile time (SP 0: L2Sqr16Ext, 1: NormCosine, 2:
// NegativeDotProduct, all through the reference's 16-wide kernels since the length is a multiple
// of 16), lists of up to 32 * NCH ids. The query sits in registers (lane j of an 8-lane group holds
// the float4 pieces it multiplies), every new neighbour's row is fetched by the lane that holds it
// with one bulk copy (TMA unit) into the warp's staging rows, and warp-uniform state stays in
// registers. The steps, arithmetic and tie rules are those of run_query above (greedy descent
// hnsw_distfunc_opt.cc:168-198, SearchV1Merge :200-283, push_or_replace_non_empty_exp
// sort_arr_bi.h:159-199), so results and per-query counts are identical to it bit for bit.

template <int SP>
__device__ __forceinline__ float lean_term(float q, float x, float acc) {
  if constexpr (SP == 0) {
    const float d = __fsub_rn(q, x);
    return __fmaf_rn(d, d, acc);
  } else {
    return __fmaf_rn(q, x, acc);
  }
}

// The reference's reduction of a group's 8 lane accumulators for rows whose length is a multiple
// of 16 (no remainder or scalar tail): hnsw_distfunc_opt_impl_inline.h:68-69 for L2Sqr16Ext;
// :100,152 and hnsw.cc:70-81 for the scalar product. Every lane of the group returns the value.
template <int SP>
__device__ __forceinline__ float lean_combine(float acc) {
  const int gb = lane_id() & ~7;
  if constexpr (SP == 0) {
    float s = __shfl_sync(kFull, acc, gb);
#pragma unroll
    for (int t = 1; t < 8; ++t) s = __fadd_rn(s, __shfl_sync(kFull, acc, gb + t));
    return s;
  } else {
    const float t4 = __fadd_rn(acc, __shfl_down_sync(kFull, acc, 4, 8));
    float s = __fadd_rn(__shfl_sync(kFull, t4, gb), __shfl_sync(kFull, t4, gb + 1));
    s = __fadd_rn(s, __shfl_sync(kFull, t4, gb + 2));
    s = __fadd_rn(s, __shfl_sync(kFull, t4, gb + 3));
    if constexpr (SP == 1) {
      const float mn = (s < 1.0f) ? s : 1.0f;
      const float mx = (-1.0f < mn) ? mn : -1.0f;
      const float v = __fsub_rn(1.0f, mx);
      return (0.0f < v) ? v : 0.0f;
    } else {
      return -s;
    }
  }
}

// Two single-precision subtractions in one packed instruction (sub.rn.f32x2): each half is the
// IEEE-754 binary32 difference rounded to nearest even, the same value as __fsub_rn on that half.
__device__ __forceinline__ float2 sub2_rn(float2 a, float2 b) {
  unsigned long long ra, rb, rd;
  asm("mov.b64 %0, {%1, %2};" : "=l"(ra) : "f"(a.x), "f"(a.y));
  asm("mov.b64 %0, {%1, %2};" : "=l"(rb) : "f"(b.x), "f"(b.y));
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(rd) : "l"(ra), "l"(rb));
  float2 d;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(d.x), "=f"(d.y) : "l"(rd));
  return d;
}

template <int NF, bool HALF>
struct LeanQuery {
  float4 c[NF > 0 ? NF : 1];
  float2 h;
};

template <int NF, bool HALF, int SP>
__device__ __forceinline__ float lean_row_dist(const LeanQuery<NF, HALF>& q, const float* __restrict__ row) {
  const int j = lane_id() & 7;
  float acc = 0.0f;
#pragma unroll
  for (int c = 0; c < NF; ++c) {
    const float4 x = reinterpret_cast<const float4*>(row + c * 32)[j];
    if constexpr (SP == 0) {  // the differences two at a time, the sum of squares in order
      const float2 d01 = sub2_rn(make_float2(q.c[c].x, q.c[c].y), make_float2(x.x, x.y));
      const float2 d23 = sub2_rn(make_float2(q.c[c].z, q.c[c].w), make_float2(x.z, x.w));
      acc = __fmaf_rn(d01.x, d01.x, acc);
      acc = __fmaf_rn(d01.y, d01.y, acc);
      acc = __fmaf_rn(d23.x, d23.x, acc);
      acc = __fmaf_rn(d23.y, d23.y, acc);
    } else {
      acc = lean_term<SP>(q.c[c].x, x.x, acc);
      acc = lean_term<SP>(q.c[c].y, x.y, acc);
      acc = lean_term<SP>(q.c[c].z, x.z, acc);
      acc = lean_term<SP>(q.c[c].w, x.w, acc);
    }
  }
  if constexpr (HALF) {
    const float2 x = reinterpret_cast<const float2*>(row + NF * 32)[j];
    if constexpr (SP == 0) {
      const float2 d = sub2_rn(q.h, x);
      acc = __fmaf_rn(d.x, d.x, acc);
      acc = __fmaf_rn(d.y, d.y, acc);
    } else {
      acc = lean_term<SP>(q.h.x, x.x, acc);
      acc = lean_term<SP>(q.h.y, x.y, acc);
    }
  }
  return lean_combine<SP>(acc);
}

struct LeanWarp {  // a warp's shared-memory pieces and counters
  uint2* items;
  int* nb_id;
  float* nb_d;
  float* sk;
  int* sv;
  float* stage;
  uint64_t* bar;
  uint8_t* vis;
  uint32_t phase;
  int stage_rows;
  bool bulk;  // rows by one bulk copy each (else 16-byte asynchronous copies spread over the lanes)
  int st_dist, st_expand, st_greedy, st_list_ints;
};

// Distances to the rows the lanes hold (lane l: up to NCH rows, has[h] / position pos[h] in the
// step's row list / vector id[h]) into w.nb_d[pos]. Rows go through the staging area in rounds of
// stage_rows: with w.bulk each row is one bulk copy issued by the lane that holds it, completing on
// the warp's mbarrier; otherwise the round's ids are posted in w.sv and every lane copies 16-byte
// pieces of the round's rows. Returns false if bulk copies did not complete within the wait bound.
template <int NF, bool HALF, int SP, int NCH>
__device__ bool lean_rows(const DevIndex& ix, LeanWarp& w, const LeanQuery<NF, HALF>& q, const bool (&has)[NCH],
                          const int (&pos)[NCH], const int (&id)[NCH], int nrows) {
  constexpr int kDim = NF * 32 + (HALF ? 16 : 0);
  constexpr uint32_t kRowBytes = kDim * 4;
  const int lane = lane_id(), g = lane >> 3;
  for (int base = 0; base < nrows; base += w.stage_rows) {
    const int rows = min(w.stage_rows, nrows - base);
    if (w.bulk) {
      if (lane == 0) sm100::mbar_arrive_expect_tx(w.bar, (uint32_t)rows * kRowBytes);
      __syncwarp();
#pragma unroll
      for (int h = 0; h < NCH; ++h) {
        if (has[h] && pos[h] >= base && pos[h] < base + rows) {
          sm100::fence_proxy_async_smem();
          sm100::bulk_copy_g2s(w.stage + (pos[h] - base) * kDim, ix.vecs + (int64_t)id[h] * ix.pitch, kRowBytes,
                               w.bar);
        }
      }
      const bool ok = sm100::mbar_wait(w.bar, w.phase);
      w.phase ^= 1;
      if (!ok) {
        sm100::mbar_wait(w.bar, w.phase ^ 1);  // bounded: no copy may be left writing the staging rows
        return false;
      }
    } else {
      constexpr int kPieces = kRowBytes / 16;  // 16-byte pieces per row
#pragma unroll
      for (int h = 0; h < NCH; ++h)
        if (has[h] && pos[h] >= base && pos[h] < base + rows) w.sv[pos[h] - base] = id[h];
      __syncwarp();
      for (int c = lane; c < rows * kPieces; c += 32) {
        const int r = c / kPieces, p = c - r * kPieces;
        cp_async16(w.stage + r * kDim + 4 * p, ix.vecs + (int64_t)w.sv[r] * ix.pitch + 4 * p);
      }
      cp_async_wait_all();
      __syncwarp();
    }
    for (int r0 = 0; r0 < rows; r0 += 4) {
      const int r = r0 + g;
      const bool act = r < rows;
      const float d = lean_row_dist<NF, HALF, SP>(q, w.stage + (act ? r : 0) * kDim);
      if (act && (lane & 7) == 0) w.nb_d[base + r] = d;
    }
    __syncwarp();
  }
  return true;
}

// One expansion's kept neighbours merged into items[0..num) (num <= cap <= 64) through registers:
// lane t holds list-order neighbour t (key d, id idt, kept or not), lane l array items l and l+32.
// Each array item moves right by the number of kept keys below it; each kept item lands at (array
// keys below it) + (kept keys below it). When no kept key equals another kept key or an array key,
// that is the array that sorting the batch and inserting its items one by one with
// push_or_replace_non_empty_exp (sort_arr_bi.h:159-199) leaves, truncated to cap, and the smallest
// insertion index is the kept minimum's. With such a tie it returns false and changes nothing.
__device__ __forceinline__ bool lean_merge64(uint2* items, int& num, int cap, float d, int idt, bool keep,
                                             int* first_pos) {
  const int lane = lane_id();
  const unsigned km = __ballot_sync(kFull, keep);
  const bool h0 = lane < num, h1 = lane + 32 < num;
  const uint2 it0 = h0 ? items[lane] : make_uint2(0u, 0u);
  const uint2 it1 = h1 ? items[lane + 32] : make_uint2(0u, 0u);
  const float k0 = key_of(it0), k1 = key_of(it1);
  int rank = 0, lb = 0, c0 = 0, c1 = 0;
  bool tie = false;
  for (unsigned mm = km; mm; mm &= mm - 1) {
    const int u = __ffs(mm) - 1;
    const float ku = __shfl_sync(kFull, d, u);
    rank += ku < d;
    tie |= (keep && u != lane && ku == d) || (h0 && k0 == ku) || (h1 && k1 == ku);
    const unsigned b0 = __ballot_sync(kFull, h0 && k0 < ku);
    const unsigned b1 = __ballot_sync(kFull, h1 && k1 < ku);
    if (lane == u) lb = __popc(b0) + __popc(b1);
    c0 += ku < k0;
    c1 += ku < k1;
  }
  if (__any_sync(kFull, tie)) return false;
  const int p = lb + rank;
  const int first = __shfl_sync(kFull, p, __ffs(__ballot_sync(kFull, keep && rank == 0)) - 1);
  __syncwarp();
  if (h0 && lane + c0 < cap) items[lane + c0] = it0;
  if (h1 && lane + 32 + c1 < cap) items[lane + 32 + c1] = it1;
  if (keep && p < cap) items[p] = make_item(d, idt, false);
  num = min(num + __popc(km), cap);
  *first_pos = first;
  __syncwarp();
  return true;
}

// Query qi in registers: lane j of each 8-lane group takes elements {32c + j + 8s} (s = 0..3) of
// every 32-element block c — the permuted order of the stored rows — and, with HALF, elements
// {32 NF + j + 8s} (s = 0, 1); a cosine query is normalised first as hnsw.h:486-497 does.
template <int NF, bool HALF, int SP>
__device__ LeanQuery<NF, HALF> lean_load_query(const SearchArgs& a, int64_t qi) {
  const int lane = lane_id(), j = lane & 7;
  constexpr int kDim = NF * 32 + (HALF ? 16 : 0);
  const float* src = a.queries + qi * kDim;
  float s = 1.0f;
  bool scale = false;
  if constexpr (SP == 1) {
    if (lane == 0) {
      float sum = 0.0f;
      for (int e = 0; e < kDim; ++e) {
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
  auto ld = [&](int e) {
    const float v = __ldg(src + e);
    return scale ? __fmul_rn(v, s) : v;
  };
  LeanQuery<NF, HALF> q;
#pragma unroll
  for (int c = 0; c < NF; ++c)
    q.c[c] = make_float4(ld(32 * c + j), ld(32 * c + j + 8), ld(32 * c + j + 16), ld(32 * c + j + 24));
  if constexpr (HALF) q.h = make_float2(ld(32 * NF + j), ld(32 * NF + j + 8));
  return q;
}

template <int NF, bool HALF, int SP, int NCH>
__device__ bool lean_query(const SearchArgs& a, LeanWarp& w, int64_t qi, uint8_t epoch) {
  const DevIndex& ix = a.ix;
  const int lane = lane_id();
  const LeanQuery<NF, HALF> q = lean_load_query<NF, HALF, SP>(a, qi);
  const int k = a.k_per_q ? a.k_per_q[qi] : a.k_default;
  const int ef = a.ef_per_q ? a.ef_per_q[qi] : a.ef_default;
  w.st_dist = w.st_expand = w.st_greedy = w.st_list_ints = 0;
  bool has[NCH];
  int pos[NCH], id[NCH];
  // ---- the entry point, then the greedy descent (hnsw_distfunc_opt.cc:168-198): at each level
  // move to the earliest list entry whose distance is strictly below every earlier one, while
  // one is below the current distance. In the level-0 pass of a split search the descent's end
  // (and its counts) come from the descent pass instead.
  int cur = ix.enterpoint;
  float curdist = 0.0f;
  if (a.split == 2) {
    cur = __ldg(a.entry_node + qi);
    curdist = __ldg(a.entry_dist + qi);
    w.st_dist = __ldg(a.entry_stats + 3 * qi + 0);
    w.st_greedy = __ldg(a.entry_stats + 3 * qi + 1);
    w.st_list_ints = __ldg(a.entry_stats + 3 * qi + 2);
    if (cur < 0 || cur >= ix.n) return false;  // the descent pass gave up on this query
  } else {
#pragma unroll
    for (int h = 0; h < NCH; ++h) {
      has[h] = h == 0 && lane == 0;
      pos[h] = 0;
      id[h] = cur;
    }
    if (!lean_rows<NF, HALF, SP, NCH>(ix, w, q, has, pos, id, 1)) return false;
    curdist = w.nb_d[0];
    w.st_dist += 1;
    for (int lev = ix.maxlevel; lev > 0; --lev) {
      while (true) {
        const int32_t* lst = ix.up_links + __ldg(ix.up_off + cur) + (int64_t)(ix.maxM + 1) * (lev - 1);
        const int cnt = __ldg(lst);
#pragma unroll
        for (int h = 0; h < NCH; ++h) {
          const int t = 32 * h + lane;
          has[h] = t < cnt;
          pos[h] = t;
          id[h] = has[h] ? __ldg(lst + 1 + t) : 0;
        }
        if (!lean_rows<NF, HALF, SP, NCH>(ix, w, q, has, pos, id, cnt)) return false;
        w.st_greedy += 1;
        w.st_dist += cnt;
        w.st_list_ints += 1 + cnt;
        float best = curdist;
        int bpos = 0x7fffffff, bid = 0;
#pragma unroll
        for (int h = 0; h < NCH; ++h) {
          if (has[h]) {
            const float d = w.nb_d[pos[h]];
            if (d < best) {
              best = d;
              bpos = pos[h];
              bid = id[h];
            }
          }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const float ob = __shfl_xor_sync(kFull, best, o);
          const int op = __shfl_xor_sync(kFull, bpos, o);
          const int oi = __shfl_xor_sync(kFull, bid, o);
          if (ob < best || (ob == best && op < bpos)) {
            best = ob;
            bpos = op;
            bid = oi;
          }
        }
        __syncwarp();
        if (!(bpos != 0x7fffffff && best < curdist)) break;
        cur = bid;
        curdist = best;
      }
    }
    if (a.split == 1) {  // the descent pass: record where level 0 starts, and the key it is ordered by
      if (lane == 0) {
        a.entry_node[qi] = cur;
        a.entry_dist[qi] = curdist;
        a.entry_stats[3 * qi + 0] = w.st_dist;
        a.entry_stats[3 * qi + 1] = w.st_greedy;
        a.entry_stats[3 * qi + 2] = w.st_list_ints;
        const uint32_t key = ordered_key(curdist);
        atomicMin(a.entry_range + 0, key);
        atomicMax(a.entry_range + 1, key);
      }
      __syncwarp();
      return true;
    }
  }
  // ---- level 0 (hnsw_distfunc_opt.cc:200-283)
  const int cap = max(ef, k);
  int num = 1, curr = 0;
  if (lane == 0) {
    w.items[0] = make_item(curdist, cur, false);
    w.vis[cur] = epoch;
  }
  __syncwarp();
  while (curr < min(num, ef)) {
    const uint2 e = w.items[curr];
    const int node = (int)(e.y & kIdMask);
    const float top_key = key_of(w.items[num - 1]);
    const int size_now = num;
    const int nxt = curr + 1 < num ? (int)(w.items[curr + 1].y & kIdMask) : -1;
    __syncwarp();
    if (lane == 0) w.items[curr].y = e.y | kUsedBit;
    ++curr;
    // the next candidate in line is usually expanded next: start pulling its list into L2
    if (lane < 2 && nxt >= 0 && 32 * lane < ix.l0_pitch) prefetch_l2(ix.l0 + (int64_t)nxt * ix.l0_pitch + 32 * lane);
    const int32_t* lst = ix.l0 + (int64_t)node * ix.l0_pitch;
    int idv[NCH];
#pragma unroll
    for (int h = 0; h < NCH; ++h) idv[h] = 32 * h + lane < ix.maxM0 ? __ldg(lst + 1 + 32 * h + lane) : 0;
    const int cnt = __ldg(lst);
    // visited check in list order, 32 entries at a time; an id listed twice counts once
    int nnew = 0;
#pragma unroll
    for (int h = 0; h < NCH; ++h) {
      const bool valid = 32 * h + lane < cnt;
      bool cand = valid;
      if (!ix.l0_unique) {  // the first of equal ids in the chunk is checked, as a serial walk would
        const unsigned same = __match_any_sync(kFull, valid ? idv[h] : -1 - lane);
        cand = valid && (__ffs(same) - 1) == lane;
      }
      bool isnew = false;
      if (cand) {
        isnew = w.vis[idv[h]] != epoch;
        if (isnew) w.vis[idv[h]] = epoch;
      }
      const unsigned m = __ballot_sync(kFull, isnew);
      has[h] = isnew;
      pos[h] = nnew + __popc(m & lanemask_lt());
      id[h] = idv[h];
      if (isnew) w.nb_id[pos[h]] = idv[h];
      nnew += __popc(m);
      if (NCH > 1) __syncwarp();
    }
    w.st_expand += 1;
    w.st_list_ints += 1 + cnt;
    w.st_dist += nnew;
    if (!lean_rows<NF, HALF, SP, NCH>(ix, w, q, has, pos, id, nnew)) return false;
    // keep d < topKey || size < ef (lists of up to 32 and arrays of up to 64: merged in registers
    // unless keys tie)
    bool merged = false;
    if constexpr (NCH == 1) {
      if (cap <= 64) {
        const bool valid = lane < nnew;
        const float d = valid ? w.nb_d[lane] : 0.0f;
        const int idt = valid ? w.nb_id[lane] : 0;
        const bool keep = valid && ((d < top_key) || (size_now < ef));
        int p0 = 0x7fffffff;
        merged = !__any_sync(kFull, keep) || lean_merge64(w.items, num, cap, d, idt, keep, &p0);
        if (p0 < curr) curr = p0;
      }
    }
    // otherwise: the kept ones in list order, then the batch merge or sort + insertion
    int qty = 0;
#pragma unroll
    for (int h = 0; h < NCH && !merged; ++h) {
      const int t = 32 * h + lane;
      bool keep = false;
      float d = 0.0f;
      int idt = 0;
      if (t < nnew) {
        d = w.nb_d[t];
        idt = w.nb_id[t];
        keep = (d < top_key) || (size_now < ef);
      }
      const unsigned mk = __ballot_sync(kFull, keep);
      if (keep) {
        const int p = qty + __popc(mk & lanemask_lt());
        w.sk[p] = d;
        w.sv[p] = idt;
      }
      qty += __popc(mk);
    }
    __syncwarp();
    if (qty && !merged) {
      int p0;
      if (merge_unsorted_batch(w.items, num, cap, w.sk, w.sv, qty, w.nb_d, w.nb_id, &p0)) {
        if (p0 < curr) curr = p0;
      } else {
        sort_like_std(w.sk, w.sv, qty, w.nb_d, w.nb_id);
        for (int i = 0; i < qty; ++i) {
          const int ins = sorted_insert(w.items, num, cap, w.sk[i], w.sv[i]);
          if (ins < curr) curr = ins;
        }
      }
    }
    // advance to the first unused item
    while (curr < num) {
      const int t = curr + lane;
      const bool unused = t < num && !(w.items[t].y & kUsedBit);
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
  write_result_row(a, qi, w.items, min(k, num), false);
  if (a.stats && lane == 0) {
    a.stats[qi * 4 + 0] = w.st_dist;
    a.stats[qi * 4 + 1] = w.st_expand;
    a.stats[qi * 4 + 2] = w.st_greedy;
    a.stats[qi * 4 + 3] = (int64_t)ix.row_bytes * w.st_dist + 4LL * w.st_list_ints;
  }
  __syncwarp();
  return true;
}

template <int NF, bool HALF, int SP, int NCH>
__global__ void __launch_bounds__(128, 8) search_lean_kernel(SearchArgs a) {
  extern __shared__ __align__(16) char smem[];
  constexpr int kDim = NF * 32 + (HALF ? 16 : 0);
  const int warp = threadIdx.x >> 5, lane = lane_id();
  char* ws = smem + warp * a.warp_smem;
  const int slot = blockIdx.x * (blockDim.x >> 5) + warp;
  if (slot >= a.num_slots) return;
  LeanWarp w;
  w.items = reinterpret_cast<uint2*>(ws);
  w.nb_id = reinterpret_cast<int*>(w.items + a.region_items);
  w.nb_d = reinterpret_cast<float*>(w.nb_id + a.nbpad);
  w.sk = w.nb_d + a.nbpad;
  w.sv = reinterpret_cast<int*>(w.sk + a.nbpad);
  w.stage = reinterpret_cast<float*>(w.sv + a.nbpad);
  w.bar = reinterpret_cast<uint64_t*>(w.stage + (size_t)a.stage_rows * kDim);
  w.vis = a.visited + (int64_t)slot * a.visited_pitch;
  w.phase = 0;
  w.stage_rows = a.stage_rows;
  w.bulk = a.bulk_rows != 0;
  if (lane == 0) {
    sm100::mbar_init(w.bar, 1);
    sm100::fence_barrier_init();
  }
  __syncwarp();
  while (true) {
    int item = 0;
    if (lane == 0) item = atomicAdd(a.work_counter, 1);
    item = __shfl_sync(kFull, item, 0);
    if (item >= a.nq) break;
    const int64_t qi = a.order ? a.order[item] : a.q_base + item;
    // next epoch of this slot's visited bytes; cleared when the byte wraps (hnsw.h:582-589). The
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
    if (!lean_query<NF, HALF, SP, NCH>(a, w, qi, (uint8_t)ep)) {
      if (lane == 0) set_status(a.status, NMSG_ERR_TIMEOUT);
      return;
    }
  }
}

// The instantiation for this index's row length and list length (SP fixed by the file), or null.
template <int SP>
void* lean_kernel_select(const DevIndex& ix) {
  const bool two = std::max(ix.maxM, ix.maxM0) > 32;
  switch (ix.dim) {
    case 16: return two ? (void*)search_lean_kernel<0, true, SP, 2> : (void*)search_lean_kernel<0, true, SP, 1>;
    case 48: return two ? (void*)search_lean_kernel<1, true, SP, 2> : (void*)search_lean_kernel<1, true, SP, 1>;
    case 64: return two ? (void*)search_lean_kernel<2, false, SP, 2> : (void*)search_lean_kernel<2, false, SP, 1>;
    case 96: return two ? (void*)search_lean_kernel<3, false, SP, 2> : (void*)search_lean_kernel<3, false, SP, 1>;
    case 128: return two ? (void*)search_lean_kernel<4, false, SP, 2> : (void*)search_lean_kernel<4, false, SP, 1>;
    case 256: return two ? (void*)search_lean_kernel<8, false, SP, 2> : (void*)search_lean_kernel<8, false, SP, 1>;
  }
  return nullptr;
}

}  // namespace
}  // namespace nmsg
