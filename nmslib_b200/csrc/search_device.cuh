// Device helpers shared by the HNSW search kernels (hnsw_search.cu and the lean kernels): warp
// basics, the libstdc++ std::sort order restated for neighbour batches, the SortArrBI insertion
// and batch merge, and the result-row writer. Included inside namespace nmsg (anonymous
// namespace per translation unit).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "engine.h"
#include "../../include/nmslib_b200.h"

namespace nmsg {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kUsedBit = 0x80000000u;
constexpr uint32_t kIdMask = 0x7fffffffu;

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ unsigned lanemask_lt() { return (1u << lane_id()) - 1u; }
__device__ __forceinline__ float key_of(uint2 it) { return __uint_as_float(it.x); }
__device__ __forceinline__ uint2 make_item(float key, int id, bool used) {
  return make_uint2(__float_as_uint(key), (uint32_t)id | (used ? kUsedBit : 0u));
}

__device__ __forceinline__ void set_status(int32_t* status, int code) { atomicCAS(status, 0, code); }

// A float as an unsigned key with the same order (negative values flipped entirely, positive ones
// with the sign bit set), so that atomicMin / atomicMax and integer buckets order floats.
__device__ __forceinline__ uint32_t ordered_key(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// asynchronous 16-byte global -> shared copies (cp.async, L2 only)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

// waits until at most N of this thread's committed copy groups are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait_keep() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// ------------------------------------------------------------------ libstdc++ sort order
// Restatement of the algorithm libstdc++ uses for std::sort on random-access ranges
// (introsort with median-of-three pivot into the first slot, unguarded partition, a 16-element
// threshold, heapsort fallback, final insertion sort). Comparison is on the key only, exactly as
// SortArrBI::Item::operator< (sort_arr_bi.h:43-45). Single-lane code on shared memory; used for
// neighbour batches that contain equal keys and more than 16 items.
struct KV {
  float* k;
  int* v;
  __device__ void swap(int a, int b) {
    float tk = k[a];
    k[a] = k[b];
    k[b] = tk;
    int tv = v[a];
    v[a] = v[b];
    v[b] = tv;
  }
};

__device__ void lib_adjust_heap(KV a, int first, int hole, int len, float vk, int vv) {
  const int top = hole;
  int child = hole;
  while (child < (len - 1) / 2) {
    child = 2 * (child + 1);
    if (a.k[first + child] < a.k[first + child - 1]) child--;
    a.k[first + hole] = a.k[first + child];
    a.v[first + hole] = a.v[first + child];
    hole = child;
  }
  if ((len & 1) == 0 && child == (len - 2) / 2) {
    child = 2 * (child + 1);
    a.k[first + hole] = a.k[first + child - 1];
    a.v[first + hole] = a.v[first + child - 1];
    hole = child - 1;
  }
  int parent = (hole - 1) / 2;
  while (hole > top && a.k[first + parent] < vk) {
    a.k[first + hole] = a.k[first + parent];
    a.v[first + hole] = a.v[first + parent];
    hole = parent;
    parent = (hole - 1) / 2;
  }
  a.k[first + hole] = vk;
  a.v[first + hole] = vv;
}

__device__ void lib_heap_sort_range(KV a, int first, int last) {
  const int len = last - first;
  if (len >= 2) {  // make_heap
    for (int parent = (len - 2) / 2;; --parent) {
      lib_adjust_heap(a, first, parent, len, a.k[first + parent], a.v[first + parent]);
      if (parent == 0) break;
    }
  }
  for (int end = last; end - first > 1;) {  // sort_heap via pop_heap
    --end;
    const float vk = a.k[end];
    const int vv = a.v[end];
    a.k[end] = a.k[first];
    a.v[end] = a.v[first];
    lib_adjust_heap(a, first, 0, end - first, vk, vv);
  }
}

__device__ void lib_move_median_to_first(KV a, int result, int x, int y, int z) {
  if (a.k[x] < a.k[y]) {
    if (a.k[y] < a.k[z])
      a.swap(result, y);
    else if (a.k[x] < a.k[z])
      a.swap(result, z);
    else
      a.swap(result, x);
  } else if (a.k[x] < a.k[z]) {
    a.swap(result, x);
  } else if (a.k[y] < a.k[z]) {
    a.swap(result, z);
  } else {
    a.swap(result, y);
  }
}

__device__ int lib_unguarded_partition(KV a, int first, int last, int pivot) {
  while (true) {
    while (a.k[first] < a.k[pivot]) ++first;
    --last;
    while (a.k[pivot] < a.k[last]) --last;
    if (!(first < last)) return first;
    a.swap(first, last);
    ++first;
  }
}

__device__ void lib_linear_insert(KV a, int last) {
  const float vk = a.k[last];
  const int vv = a.v[last];
  int next = last - 1;
  while (vk < a.k[next]) {
    a.k[last] = a.k[next];
    a.v[last] = a.v[next];
    last = next;
    --next;
  }
  a.k[last] = vk;
  a.v[last] = vv;
}

__device__ void lib_insertion_sort(KV a, int first, int last) {
  if (first == last) return;
  for (int i = first + 1; i != last; ++i) {
    if (a.k[i] < a.k[first]) {
      const float vk = a.k[i];
      const int vv = a.v[i];
      for (int t = i; t > first; --t) {
        a.k[t] = a.k[t - 1];
        a.v[t] = a.v[t - 1];
      }
      a.k[first] = vk;
      a.v[first] = vv;
    } else {
      lib_linear_insert(a, i);
    }
  }
}

__device__ void lib_std_sort(KV a, int n) {
  if (n < 2) return;
  int lg = 31 - __clz(n);
  // introsort loop with an explicit stack instead of recursion on the right part
  int stk_first[64], stk_last[64], stk_depth[64];
  int sp = 0;
  stk_first[sp] = 0;
  stk_last[sp] = n;
  stk_depth[sp] = 2 * lg;
  ++sp;
  while (sp > 0) {
    --sp;
    int first = stk_first[sp], last = stk_last[sp], depth = stk_depth[sp];
    while (last - first > 16) {
      if (depth == 0) {
        lib_heap_sort_range(a, first, last);
        break;
      }
      --depth;
      const int mid = first + (last - first) / 2;
      lib_move_median_to_first(a, first, first + 1, mid, last - 1);
      const int cut = lib_unguarded_partition(a, first + 1, last, first);
      // libstdc++ recurses on [cut, last) first, then loops on [first, cut); the two parts are
      // disjoint, so processing order does not change the result.
      // (segments of 16 or fewer are left to the final insertion sort, so only longer ones are
      // stacked; stacked segments are disjoint and longer than 16, which bounds the stack)
      if (last - cut > 16) {
        stk_first[sp] = cut;
        stk_last[sp] = last;
        stk_depth[sp] = depth;
        ++sp;
      }
      last = cut;
    }
  }
  // final insertion sort
  if (n > 16) {
    lib_insertion_sort(a, 0, 16);
    for (int i = 16; i < n; ++i) lib_linear_insert(a, i);
  } else {
    lib_insertion_sort(a, 0, n);
  }
}

// Order sk/sv[0..n) as std::sort would. Warp-cooperative; tmpk/tmpv are scratch of length n.
// Without equal keys every correct sort gives the same order, and for n <= 16 libstdc++ runs a
// stable insertion sort, so a stable rank sort is exact in both cases; otherwise one lane runs
// the restated introsort.
__device__ void sort_like_std(float* sk, int* sv, int n, float* tmpk, int* tmpv) {
  const int lane = lane_id();
  bool tie = false;
  for (int t = lane; t < n; t += 32) {
    const float kt = sk[t];
    int rank = 0;
    for (int u = 0; u < n; ++u) {
      const float ku = sk[u];
      rank += (ku < kt) || (ku == kt && u < t);
      tie |= (ku == kt && u != t);
    }
    tmpk[rank] = kt;
    tmpv[rank] = sv[t];
  }
  const bool anytie = __any_sync(kFull, tie);
  __syncwarp();
  if (!anytie || n <= 16) {
    for (int t = lane; t < n; t += 32) {
      sk[t] = tmpk[t];
      sv[t] = tmpv[t];
    }
  } else if (lane == 0) {
    lib_std_sort(KV{sk, sv}, n);
  }
  __syncwarp();
}

// ------------------------------------------------------------------ sorted candidate array
// push_or_replace_non_empty_exp (sort_arr_bi.h:159-199) over items[0..num) with capacity cap.
// Returns the insertion index (num before the call when the item is appended, num when it is
// dropped). Warp-cooperative; all lanes return the same values.
__device__ int sorted_insert(uint2* items, int& num, int cap, float key, int id) {
  const int lane = lane_id();
  const float last_key = key_of(items[num - 1]);
  if (last_key <= key) {
    int ins = num;
    if (num < cap) {
      if (lane == 0) items[num] = make_item(key, id, false);
      ++num;
    }
    __syncwarp();
    return ins;
  }
  // The exponential probe from the tail visits num-1, num-2, num-4, ..., num-2^i (while > 0)
  // and then stops at 0. It stops early at the first probe whose key is <= the new key.
  const int c = (lane < 31) ? num - (1 << lane) : 0;
  const bool valid = lane < 31 && c > 0;
  const bool cond = valid && key_of(items[c]) <= key;
  const unsigned cm = __ballot_sync(kFull, cond);
  const unsigned vm = __ballot_sync(kFull, valid);
  int p, prev;
  if (cm) {
    const int f = __ffs(cm) - 1;  // f >= 1: the probe at num-1 has a larger key
    p = num - (1 << f);
    prev = num - (1 << (f - 1));
  } else {
    p = 0;
    prev = vm ? num - (1 << (31 - __clz(vm))) : 0;  // the last probe taken (none when num == 1)
  }
  int pos;
  if (cm && key_of(items[p]) == key) {
    pos = p;  // lower_bound over [p, prev) returns p itself
  } else {
    // lower_bound over [p, prev): count keys below `key` in that range (the array is sorted)
    int cnt = 0;
    for (int t = p + lane; t < prev; t += 32) cnt += key_of(items[t]) < key;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(kFull, cnt, o);
    pos = p + cnt;
  }
  // shift [pos, last) right by one; the tail item falls off when the array is full
  const int last = (num < cap) ? num : num - 1;
  for (int hi = last; hi > pos; hi -= 32) {
    const int src = hi - 1 - lane;
    const bool act = src >= pos;
    uint2 v;
    if (act) v = items[src];
    __syncwarp();
    if (act) items[src + 1] = v;
    __syncwarp();
  }
  if (lane == 0) items[pos] = make_item(key, id, false);
  if (num < cap) ++num;
  __syncwarp();
  return pos;
}

// Inserts the batch sk/sv[0..m) (in list order, not yet sorted) into items[0..num) in one
// parallel pass, in place. Exact only when no key of the batch equals another batch key or a key
// already in the array: then push_or_replace_non_empty_exp always lands on the lower bound, so
// sorting the batch and inserting it item by item equals a stable merge truncated to `cap`, and
// the smallest insertion index is the merged position of the smallest batch item. Every item's
// merged position is its lower bound in the array plus its rank in the batch; array items from
// the first insertion point on move right by the number of batch keys below them (processed
// from the tail, so nothing is overwritten before it is read). Returns false, with nothing
// changed, when a tie exists.
__device__ bool merge_unsorted_batch(uint2* items, int& num, int cap, const float* sk, const int* sv, int m,
                                     float* tk, int* tv, int* first_pos) {
  const int lane = lane_id();
  bool tie = false;
  int pmin = 0x7fffffff;
  int rk[4];  // m <= nbpad <= 128: ranks of this lane's items
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int i = lane + 32 * r;
    if (i >= m) break;
    const float key = sk[i];
    int rank = 0;
    for (int u = 0; u < m; ++u) {
      const float ku = sk[u];
      rank += ku < key;
      tie |= (ku == key) && (u != i);
    }
    rk[r] = rank;
    int lo = 0, hi = num;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (key_of(items[mid]) < key)
        lo = mid + 1;
      else
        hi = mid;
    }
    tie |= lo < num && key_of(items[lo]) == key;
    tk[rank] = key;  // the batch in sorted order (ranks are distinct when there is no tie)
    tv[rank] = lo;   // and each item's lower bound in the array
    pmin = min(pmin, lo + rank);
  }
  if (__any_sync(kFull, tie)) {
    __syncwarp();
    return false;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) pmin = min(pmin, __shfl_xor_sync(kFull, pmin, o));
  __syncwarp();
  // shift the array tail [p0, num): each item moves right by the count of batch keys below it
  // (binary search over the sorted batch), from the tail so nothing is overwritten before it is read
  const int p0 = min(pmin, num);
  for (int hi = num; hi > p0; hi -= 32) {
    const int t = hi - 1 - lane;
    const bool act = t >= p0;
    uint2 it;
    int dst = cap;
    if (act) {
      it = items[t];
      const float key = key_of(it);
      int lo = 0, h2 = m;
      while (lo < h2) {
        const int mid = (lo + h2) >> 1;
        if (tk[mid] < key)
          lo = mid + 1;
        else
          h2 = mid;
      }
      dst = t + lo;
    }
    __syncwarp();
    if (act && dst < cap) items[dst] = it;
    __syncwarp();
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int i = lane + 32 * r;
    if (i >= m) break;
    const int p = tv[rk[r]] + rk[r];
    if (p < cap) items[p] = make_item(sk[i], sv[i], false);
  }
  num = min(num + m, cap);
  *first_pos = pmin;
  __syncwarp();
  return true;
}

__device__ void write_result_row(const SearchArgs& a, int64_t qi, const uint2* res, int cnt, bool node_sorted) {
  // res[0..cnt) sorted by key; order equal keys by node index (the reference orders them by
  // Object address, allocated in node order at load time, hnsw.cc:1071)
  const int lane = lane_id();
  const DevIndex& ix = a.ix;
  for (int i = lane; i < a.kmax; i += 32) {
    if (i < cnt) {
      const float ki = key_of(res[i]);
      const int ni = (int)(res[i].y & kIdMask);
      int rank = i;
      if (!node_sorted) {
        int s = i;
        while (s > 0 && key_of(res[s - 1]) == ki) --s;
        int e = i + 1;
        while (e < cnt && key_of(res[e]) == ki) ++e;
        rank = s;
        for (int t = s; t < e; ++t) rank += (int)(res[t].y & kIdMask) < ni;
      }
      a.ids[qi * a.kmax + rank] = __ldg(ix.ext_id + ni);
      if (a.dists_int)  // l2sqr_sift: the key is an exact integer
        reinterpret_cast<int32_t*>(a.dists)[qi * a.kmax + rank] = __float2int_rn(ki);
      else
        a.dists[qi * a.kmax + rank] = ki;
    } else {
      a.ids[qi * a.kmax + i] = -1;
      if (a.dists_int)
        reinterpret_cast<int32_t*>(a.dists)[qi * a.kmax + i] = 0x7fffffff;
      else
        a.dists[qi * a.kmax + i] = __int_as_float(0x7f800000);
    }
  }
  if (lane == 0) a.counts[qi] = cnt;
}

}  // namespace
}  // namespace nmsg
