// Level-0 neighbour selection and linking of the device-assisted HNSW build, on the GPU.
//
// After a batch of new nodes has searched the graph (the engine's search kernel, ef = k =
// efConstruction, candidates sorted by distance), two kernels do what Hnsw::add does at level 0
// (similarity_search/src/method/hnsw.cc:576-600) for the whole batch:
//   select  one warp per new node: getNeighborsByHeuristic2 (similarity_search/include/method/
//           hnsw.h:129-169) keeps a candidate unless an already kept one is strictly closer to it
//           than the new node is, up to M; the node's level-0 list becomes the kept ids, farthest
//           first (the order the reference's max-heap pops them), and every (new node -> kept
//           neighbour) link is queued on the neighbour (up to kPend per neighbour and batch);
//   merge   one warp per neighbour with queued links: they are appended while the list has room
//           (addFriendlevel, hnsw.h:258-314); past maxM0 the list and the queued nodes are ranked
//           by distance to the neighbour and cut back to maxM0 with the same heuristic.
// The reference links each new node to its neighbours one at a time; here a batch's links reach a
// neighbour together, so the graph differs as two multi-threaded builds of the reference differ.
// Construction distances are squared L2, 1 - dot (unit vectors) and -dot in FP32, in any order:
// the query path never uses them.
#include <cuda_runtime.h>

#include <cstdint>

#include "engine.h"
#include "../../include/nmslib_b200.h"

namespace nmsg {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kPend = 32;       // queued links per neighbour and batch (more are dropped)
constexpr int kMaxCand = 96;    // merge: maxM0 (<= 64 here) + kPend
constexpr int kWarps = 4;

// Distance between two stored rows (both in the permuted, zero-padded layout, so elements
// correspond), by one 8-lane group; every lane of the group gets it. Every lane of the warp must
// call it (the shuffles span the warp).
__device__ __forceinline__ float group_dist(const DevIndex& ix, int space, const float* __restrict__ a,
                                           const float* __restrict__ b) {
  const int j = threadIdx.x & 7;
  float s = 0.0f;
  for (int e = j; e < ix.pitch; e += 8) {
    const float x = __ldg(a + e), y = __ldg(b + e);
    if (space == NMSG_SPACE_L2) {
      const float d = x - y;
      s = fmaf(d, d, s);
    } else {
      s = fmaf(x, y, s);
    }
  }
  s += __shfl_xor_sync(kFull, s, 4, 8);
  s += __shfl_xor_sync(kFull, s, 2, 8);
  s += __shfl_xor_sync(kFull, s, 1, 8);
  if (space == NMSG_SPACE_L2) return s;
  return space == NMSG_SPACE_COSINE ? 1.0f - s : -s;
}

__device__ __forceinline__ const float* row_of(const DevIndex& ix, int id) { return ix.vecs + (int64_t)id * ix.pitch; }

// Heuristic 2 over cand[0..nc) (ascending distance dc to the base point): returns how many were
// kept (<= keep_max) in kept[]; the warp cooperates, 4 candidate-vs-kept distances per pass.
__device__ int heuristic2(const DevIndex& ix, int space, const int* cand, const float* dc, int nc, int keep_max,
                          int* kept) {
  const int lane = threadIdx.x & 31, g = lane >> 3;
  int nk = 0;
  for (int t = 0; t < nc && nk < keep_max; ++t) {
    const int c = cand[t];
    const float d = dc[t];
    bool good = true;
    for (int i0 = 0; i0 < nk && good; i0 += 4) {
      // groups past nk compute with a valid row and ignore the result
      const int i = i0 + g;
      const float dk = group_dist(ix, space, row_of(ix, kept[min(i, nk - 1)]), row_of(ix, c));
      good = !__any_sync(kFull, i < nk && dk < d);
    }
    if (good) {
      if (lane == 0) kept[nk] = c;
      ++nk;
      __syncwarp();
    }
  }
  return nk;
}

struct SelectArgs {
  DevIndex ix;
  int space, M, efc;
  int64_t nb;                  // nodes in the batch
  const int32_t* nodes;        // [nb]
  const int32_t* cand_ids;     // [nb][efc], ascending distance
  const float* cand_d;         // [nb][efc]
  const int32_t* cand_cnt;     // [nb]
  int32_t* l0;                 // [n][l0_pitch] (writable view of ix.l0)
  int32_t* pend;               // [n][kPend]
  int32_t* pend_cnt;           // [n]
  int32_t* touched;            // [nb * M] neighbours with queued links
  int32_t* n_touched;
};

__global__ void __launch_bounds__(32 * kWarps) select_kernel(SelectArgs a) {
  __shared__ int kept_s[kWarps][64];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t j = (int64_t)blockIdx.x * kWarps + warp;
  if (j >= a.nb) return;
  int* kept = kept_s[warp];
  const int node = a.nodes[j];
  const int nc = a.cand_cnt[j];
  const int nk = heuristic2(a.ix, a.space, a.cand_ids + j * a.efc, a.cand_d + j * a.efc, nc, a.M, kept);
  // the node's list, farthest first; each kept neighbour gets a queued link back
  int32_t* lst = a.l0 + (int64_t)node * a.ix.l0_pitch;
  for (int i = lane; i < nk; i += 32) {
    const int r = kept[nk - 1 - i];
    lst[1 + i] = r;
    const int slot = atomicAdd(a.pend_cnt + r, 1);
    if (slot == 0) a.touched[atomicAdd(a.n_touched, 1)] = r;
    if (slot < kPend) a.pend[(int64_t)r * kPend + slot] = node;
  }
  if (lane == 0) lst[0] = nk;
}

struct MergeArgs {
  DevIndex ix;
  int space;
  int32_t* l0;
  int32_t* pend;
  int32_t* pend_cnt;
  const int32_t* touched;
  const int32_t* n_touched;
};

__global__ void __launch_bounds__(32 * kWarps) merge_kernel(MergeArgs a) {
  __shared__ int cid_s[kWarps][kMaxCand];
  __shared__ float cd_s[kWarps][kMaxCand];
  __shared__ int sid_s[kWarps][kMaxCand];
  __shared__ float sd_s[kWarps][kMaxCand];
  __shared__ int kept_s[kWarps][64];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 3;
  const int t = blockIdx.x * kWarps + warp;
  if (t >= *a.n_touched) return;
  const int r = a.touched[t];
  int32_t* lst = a.l0 + (int64_t)r * a.ix.l0_pitch;
  const int cnt = lst[0];
  const int p = min(a.pend_cnt[r], kPend);
  const int32_t* pend = a.pend + (int64_t)r * kPend;
  const int cap = a.ix.maxM0;
  if (cnt + p <= cap) {
    for (int i = lane; i < p; i += 32) lst[1 + cnt + i] = pend[i];
    __syncwarp();
    if (lane == 0) {
      lst[0] = cnt + p;
      a.pend_cnt[r] = 0;
    }
    return;
  }
  // the list and the queued nodes, ranked by distance to r, cut back to maxM0 by heuristic 2
  int* cid = cid_s[warp];
  float* cd = cd_s[warp];
  const int nc = cnt + p;
  for (int i = lane; i < nc; i += 32) cid[i] = i < cnt ? lst[1 + i] : pend[i - cnt];
  __syncwarp();
  for (int i0 = 0; i0 < nc; i0 += 4) {
    const int i = i0 + g;
    const float d = group_dist(a.ix, a.space, row_of(a.ix, r), row_of(a.ix, cid[min(i, nc - 1)]));
    if (i < nc && (lane & 7) == 0) cd[i] = d;
  }
  __syncwarp();
  // stable rank sort by (distance, position)
  int* sid = sid_s[warp];
  float* sd = sd_s[warp];
  for (int i = lane; i < nc; i += 32) {
    const float di = cd[i];
    int rank = 0;
    for (int u = 0; u < nc; ++u) rank += (cd[u] < di) || (cd[u] == di && u < i);
    sid[rank] = cid[i];
    sd[rank] = di;
  }
  __syncwarp();
  int* kept = kept_s[warp];
  const int nk = heuristic2(a.ix, a.space, sid, sd, nc, cap, kept);
  for (int i = lane; i < nk; i += 32) lst[1 + i] = kept[nk - 1 - i];  // farthest first
  __syncwarp();
  if (lane == 0) {
    lst[0] = nk;
    a.pend_cnt[r] = 0;
  }
}

}  // namespace

int level0_select_and_link(const DevIndex& ix, int space, int M, int efc, int64_t nb, const int32_t* nodes,
                           const int32_t* cand_ids, const float* cand_d, const int32_t* cand_cnt, int32_t* l0,
                           int32_t* pend, int32_t* pend_cnt, int32_t* touched, int32_t* n_touched, void* stream) {
  if (nb == 0) return 0;
  if (ix.maxM0 > 64 || M > 64) return (int)cudaErrorInvalidValue;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(n_touched, 0, 4, st);
  if (e != cudaSuccess) return (int)e;
  SelectArgs sa;
  sa.ix = ix;
  sa.space = space;
  sa.M = M;
  sa.efc = efc;
  sa.nb = nb;
  sa.nodes = nodes;
  sa.cand_ids = cand_ids;
  sa.cand_d = cand_d;
  sa.cand_cnt = cand_cnt;
  sa.l0 = l0;
  sa.pend = pend;
  sa.pend_cnt = pend_cnt;
  sa.touched = touched;
  sa.n_touched = n_touched;
  select_kernel<<<(unsigned)((nb + kWarps - 1) / kWarps), 32 * kWarps, 0, st>>>(sa);
  e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  MergeArgs ma;
  ma.ix = ix;
  ma.space = space;
  ma.l0 = l0;
  ma.pend = pend;
  ma.pend_cnt = pend_cnt;
  ma.touched = touched;
  ma.n_touched = n_touched;
  // at most nb * M neighbours are touched; warps past *n_touched return at once
  const int64_t max_touched = nb * M;
  merge_kernel<<<(unsigned)((max_touched + kWarps - 1) / kWarps), 32 * kWarps, 0, st>>>(ma);
  return (int)cudaGetLastError();
}

}  // namespace nmsg
