// Shared host/device declarations of the B200 HNSW query engine.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <driver_types.h>
#include <vector_types.h>

#ifdef __CUDACC__
#define NMSG_HD __host__ __device__
#else
#define NMSG_HD
#endif

namespace nmsg {

// Optimized-index distance codes (similarity_search/include/method/hnsw.h:50-58).
// kSiftL2 is the engine's own code for space l2sqr_sift (128 uint8 values per object, int
// distance; similarity_search/src/distcomp_l2sqr_sift.cc:40-50), whose indices exist only in the
// regular format: it is not a reference DistFuncType and never appears in an optimized file.
enum DistCode { kL2Sqr16Ext = 1, kL2SqrExt = 2, kNormCosine = 3, kNegDot = 4, kL1 = 5, kLInf = 6, kSiftL2 = 7 };
// Gather code of the kernels compiled for L1 / LInf (one row per 8-lane group in registers);
// 0 = rows staged in shared memory, 1 / 2 / 4 = register rows per group for the other codes.
constexpr int kLpGather = 3;
// Gather code of the kernels compiled for l2sqr_sift rows (one 128-byte row per 4-lane group).
constexpr int kSiftGather = 5;
constexpr int kSiftDim = 128;
constexpr int kSiftRowBytes = kSiftDim + 4;  // the reference's object payload: values + int norm

// The index as read from an optimized HNSW file, in host memory.
// File layout (similarity_search/src/method/hnsw.cc:774-806):
//   u32 optimIndexFlag(=1) | u32 N | u64 memoryPerObject | u64 offsetLevel0 | u64 offsetData
//   | i32 maxlevel | u32 enterpointId | u64 maxM | u64 maxM0 | i32 dist_func_type
//   | u64 searchMethod | N * memoryPerObject level-0 block | per node: u32 sizemass + bytes.
// Level-0 row i: [i32 ext id][i32 label][u64 datalength][dim x f32][i32 cnt][maxM0 x i32].
struct HostIndex {
  uint32_t n = 0;
  uint64_t mem_per_obj = 0, off_level0 = 0, off_data = 0;
  int32_t maxlevel = 0;
  uint32_t enterpoint = 0;
  uint64_t maxM = 0, maxM0 = 0;
  int32_t dist_type = 0;
  uint64_t search_method = 3;
  int dim = 0;
  bool empty_regular = false;        // the reference saves an empty index in the regular format
  std::vector<char> level0;          // N * mem_per_obj bytes, verbatim
  std::vector<uint32_t> link_bytes;  // per node sizemass
  std::vector<int64_t> up_off;       // per node offset (ints) into up_links, -1 if level 0 only
  std::vector<int32_t> up_links;     // concatenated upper-level lists, verbatim
  std::vector<int32_t> level;        // per node top level
  // l2sqr_sift indices (regular graph file + objects file): no level0 block; the lists, vectors,
  // norms and object ids are kept here, and M / the saved maxlevel for writing the file back
  bool sift = false;
  uint64_t M = 0;
  int32_t saved_maxlevel = 0;
  uint32_t cap0 = 0, capu = 0;       // longest level-0 / upper-level list
  std::vector<int32_t> sift_l0;      // n x (cap0 + 1): count, then ids
  std::vector<uint8_t> sift_vecs;    // n x 128
  std::vector<int32_t> sift_norms;   // n, as stored with each object
  std::vector<int32_t> sift_ids, sift_labels;

  const float* vec(int64_t i) const {
    return reinterpret_cast<const float*>(level0.data() + i * mem_per_obj + off_data + 16);
  }
  const int32_t* l0(int64_t i) const {
    return reinterpret_cast<const int32_t*>(level0.data() + i * mem_per_obj + off_level0);
  }
  int32_t ext_id(int64_t i) const {
    return *reinterpret_cast<const int32_t*>(level0.data() + i * mem_per_obj + off_data);
  }
};

// Returns an nmsg_status code; `err` gets the message.
int read_index_file(const char* path, HostIndex& ix, std::string& err);
int validate_index(const HostIndex& ix, std::string& err);
int write_index_file(const char* path, const HostIndex& ix, std::string& err);
// l2sqr_sift: the regular graph file (hnsw.cc:810-842 / 943-991) and the objects file
// (python_bindings/nmslib.cc:98-125, space.cc WriteObjectVectorBinData). Validated on read.
int read_sift_index(const char* graph_path, const char* data_path, HostIndex& ix, std::string& err);
int write_sift_index(const char* graph_path, const char* data_path, const HostIndex& ix, std::string& err);

// Device-resident index. Vectors are stored with a row pitch of round_up(dim, 32) floats and,
// inside each 32-float chunk of the first (dim & ~15) elements, permuted so that lane j of an
// 8-lane group reads elements {j, j+8, j+16, j+24} of the chunk as one float4 — the exact
// accumulation order of the reference's 8-wide AVX loop. Elements from (dim & ~15) on keep their
// natural position. A final 16-float half chunk is permuted the same way into float2 pairs.
struct DevIndex {
  const float* vecs = nullptr;      // [n][pitch]
  const uint8_t* vecs_u8 = nullptr; // l2sqr_sift: [n][128]
  const int32_t* norms = nullptr;   // l2sqr_sift: stored norms, or null when every stored norm is
                                    // the sum of squares of its values (recomputed from the row)
  const int32_t* l0 = nullptr;      // [n][l0_pitch]: cnt, neighbour ids (internal)
  const int64_t* up_off = nullptr;  // [n]
  const int32_t* up_links = nullptr;
  const int32_t* ext_id = nullptr;  // [n]
  int64_t n = 0;
  int dim = 0, pitch = 0, l0_pitch = 0;
  int n16 = 0, n4 = 0;
  int maxM = 0, maxM0 = 0, maxlevel = 0, enterpoint = 0, dist_type = 0;
  int row_bytes = 0;                // algorithmic bytes of one row: 4 dim, or 132 for l2sqr_sift
  int l0_unique = 0;                // 1: no level-0 list repeats an id (checked at upload), so a
                                    // list's visited checks need no duplicate vote
};

// Position of element e of a vector in the permuted device row.
NMSG_HD inline int permuted_pos(int e, int dim) {
  const int n16 = dim & ~15;
  if (e >= n16) return e;
  const int c = e >> 5, r = e & 31, s = r >> 3, j = r & 7;
  if (c * 32 + 32 <= n16) return c * 32 + j * 4 + s;
  return c * 32 + j * 2 + s;  // final half chunk of 16
}

struct SearchArgs {
  DevIndex ix;
  const float* queries = nullptr;   // [nq][dim]
  const uint8_t* queries_u8 = nullptr;  // l2sqr_sift: [nq][128]
  int dists_int = 0;                // write distances as int32 (l2sqr_sift)
  int64_t nq = 0;
  int k_default = 10, ef_default = 20, algo = 0;
  const int32_t* k_per_q = nullptr;
  const int32_t* ef_per_q = nullptr;
  const int32_t* order = nullptr;   // optional work order (query index per work item)
  int kmax = 10;
  int32_t* ids = nullptr;
  float* dists = nullptr;
  int32_t* counts = nullptr;
  int64_t* stats = nullptr;         // optional [nq][4]
  uint8_t* visited = nullptr;       // [num_slots][visited_pitch] epoch bytes
  int64_t visited_pitch = 0;
  uint8_t* epochs = nullptr;        // [num_slots]
  // Split lean search (split 1: upper-level descent only; 2: level 0 from the stored entries):
  // where each query enters level 0, its distance there (the work order key), the descent's
  // counts (distances, upper-level list scans, list ints) and the range of the keys.
  int split = 0;
  int32_t* entry_node = nullptr;    // [nq]
  float* entry_dist = nullptr;      // [nq]
  int32_t* entry_stats = nullptr;   // [nq][3]
  uint32_t* entry_range = nullptr;  // [2]: smallest and largest ordered key
  int32_t* entry_order = nullptr;   // [nq]: the level-0 pass's work order (largest entry distance first)
  int64_t q_base = 0;               // a lean descent pass over part of the batch: queries q_base + [0, nq)
  int32_t* slot_locks = nullptr;    // [num_slots] (one-query-per-block kernel only)
  int num_slots = 0;
  uint2* old_heap = nullptr;        // [num_slots][old_heap_cap] SearchOld candidate heaps
  int64_t old_heap_cap = 0;
  int32_t* work_counter = nullptr;
  int32_t* status = nullptr;
  int region_items = 0;             // uint2 items per warp in the shared region
  int nbpad = 32;                   // neighbour buffer length per warp
  int hash_log2 = 0;                // shared-memory visited table of 2^hash_log2 ids (0: none)
  int stage_rows = 0;               // rows per staged-gather round (gather mode 0)
  int warp_smem = 0;                // bytes of shared memory per warp
  int ctx_per_warp = 1;             // queries a persistent warp carries at once (search_multi_kernel)
  int bulk_rows = 0;                // search_multi_kernel: stage each row with one bulk copy (TMA
                                    // unit, mbarrier completion) instead of 16-byte copies per lane
  int lean = 0;                     // run search_lean_kernel (V1Merge, common index shapes)
};

// Per-warp shared memory needed for the given caps.
int warp_smem_bytes(const DevIndex& ix, int region_items, int nbpad, int hash_log2, int stage_rows);
// The several-queries-per-warp kernel: list chunks of 32 it reads (1 or 2; it takes lists of up to
// 64 ids) and its shared memory per warp (ctx contexts plus the staging rows).
int multi_list_chunks(const DevIndex& ix);
int multi_warp_smem_bytes(const DevIndex& ix, int region_items, int nbpad, int stage_rows, int ctx);
// The lean one-query-per-warp kernel (V1Merge; l2 / cosine / negdot rows of 16, 48, 64, 96, 128 or
// 256 floats; lists of up to 64 ids): whether it covers an index, its occupancy and its shared
// memory per warp.
bool lean_supported(const DevIndex& ix);
// The lean kernel for an index of the matching distance (lean_l2.cu / lean_cos.cu /
// lean_negdot.cu), or null when its row or list length has no instantiation.
void* lean_kernel_l2(const DevIndex& ix);
void* lean_kernel_cos(const DevIndex& ix);
void* lean_kernel_negdot(const DevIndex& ix);
NMSG_HD inline int lean_warp_smem_bytes(int dim, int region_items, int nbpad, int stage_rows) {
  return region_items * 8 + nbpad * 16 + stage_rows * dim * 4 + 16;  // + the row mbarrier
}
int lean_occupancy(const DevIndex& ix, int warps_per_block, int smem_per_block, int* blocks_per_sm);
int lean_smem_bytes(const DevIndex& ix, int region_items, int nbpad, int stage_rows);
// Bytes one bulk row copy moves: the row rounded up to 16 bytes (the padding is zeros).
NMSG_HD inline int bulk_row_bytes(const DevIndex& ix) { return ((ix.dim * 4 + 15) / 16) * 16; }

// Launch / occupancy of the search kernels (defined in hnsw_search.cu). `gather` selects how
// vector rows are fetched: 0 = asynchronous copies into shared memory (stage_rows per round),
// 1/2/4 = registers, that many rows per 8-lane group. `with_old` includes the SearchOld path.
// Return a cudaError_t value.
// Queries of a split lean search that reach the device in two parts (host uploads on another
// stream): the descent pass of queries [0, first) waits for ready[0], that of the rest for ready[1].
struct QueryParts {
  int64_t first = 0;
  cudaEvent_t ready[2] = {nullptr, nullptr};
};
int launch_search(const SearchArgs& a, bool plain, int gather, bool with_old, int blocks, int warps_per_block,
                  void* stream, const QueryParts* parts = nullptr);

// Opt-in dynamic shared memory of the current device (227 KB on B200).
constexpr int kMaxDynamicSmem = 227 * 1024;

// Lets `kern` launch with up to kMaxDynamicSmem of dynamic shared memory, once per device and
// kernel. The limit is a process-wide property of the function, so it is raised once and never
// set per launch: a per-launch value would race with launches of the same kernel from other
// threads (serving lanes, concurrent callers) that need more. Returns a cudaError_t value.
int allow_max_smem(const void* kern);
// Exact k-NN (k <= 32) by scanning every row with the query path's distance arithmetic, on CUDA
// cores (hnsw_search.cu): rows split into n_chunks per query block, each chunk kept as
// exact_scan_lists(ix) partial lists; part_d / part_id are [nq][n_chunks * exact_scan_lists(ix)][k]
// scratch. Outputs as the search writes them (external ids, -1 / +inf padding). Returns a
// cudaError_t value.
int exact_scan_lists(const DevIndex& ix);
int exact_scan_knn(const DevIndex& ix, const float* queries, int64_t nq, int k, int kmax, float* part_d,
                   int32_t* part_id, int n_chunks, int32_t* ids, float* dists, int32_t* counts, void* stream);

// Device-assisted build (build_gpu.cu): heuristic-2 selection for a searched batch of new nodes,
// their lists, and the reverse links merged into their neighbours' lists (maxM0 <= 64). pend /
// pend_cnt ([n][32] / [n], zero at the first call) and touched ([nb * M]) are scratch. Returns a
// cudaError_t value.
int level0_select_and_link(const DevIndex& ix, int space, int M, int efc, int64_t nb, const int32_t* nodes,
                           const int32_t* cand_ids, const float* cand_d, const int32_t* cand_cnt, int32_t* l0,
                           int32_t* pend, int32_t* pend_cnt, int32_t* touched, int32_t* n_touched, void* stream);

int search_occupancy(bool plain, int gather, bool with_old, int warps_per_block, int smem_per_block,
                     int* blocks_per_sm, int ctx = 1, int nch = 1);

}  // namespace nmsg
