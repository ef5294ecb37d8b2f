/*
 * nmslib_b200 — C ABI of the B200 (sm_100a) engine for NMSLIB's HNSW query path.
 *
 * Plain pointers and sizes only. Each entry point replaces one piece of the reference's
 * Python-facing interface (paths are relative to the reference project root):
 *
 *   nmsg_index_load        IndexWrapper::loadIndex        python_bindings/nmslib.cc:98-113
 *                          -> Hnsw::LoadIndex / LoadOptimizedIndex  similarity_search/src/method/hnsw.cc:993-1074
 *   nmsg_set_query_params  setQueryTimeParams lambda      python_bindings/nmslib.cc:599-607
 *                          -> Hnsw::SetQueryTimeParams    similarity_search/src/method/hnsw.cc:472-507
 *   nmsg_knn_batch         IndexWrapper::knnQueryBatch    python_bindings/nmslib.cc:142-168
 *                          -> Hnsw::Search(KNNQuery*)     similarity_search/src/method/hnsw.cc:717-746
 *                          -> SearchV1Merge / SearchOld   similarity_search/src/method/hnsw_distfunc_opt.cc:46-283
 *   nmsg_knn_batch (nq=1)  IndexWrapper::knnQuery         python_bindings/nmslib.cc:127-140
 *   nmsg_index_save        IndexWrapper::saveIndex        python_bindings/nmslib.cc:115-125
 *                          -> Hnsw::SaveOptimizedIndex    similarity_search/src/method/hnsw.cc:774-806
 *   nmsg_index_free        IndexWrapper destructor (index.reset)
 *   nmsg_last_error        the message of the C++ exception the reference would throw
 *                          (CHECK_MSG / runtime_error, similarity_search/include/logging.h:123-135)
 *
 * Every call returns NMSG_OK (0) or a negative status; nmsg_last_error() then holds a message
 * (thread-local). Kernels never trap: device-side failures are written to a status word and
 * reported as a status here.
 */
#ifndef NMSLIB_B200_H_
#define NMSLIB_B200_H_

#include <stdint.h>

#if defined(__GNUC__)
#define NMSG_API __attribute__((visibility("default")))
#else
#define NMSG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nmsg_index nmsg_index;

enum nmsg_status {
  NMSG_OK = 0,
  NMSG_ERR_BAD_FILE = -1,      /* missing, truncated or malformed index file */
  NMSG_ERR_UNSUPPORTED = -2,   /* e.g. a non-optimized (regular) index, or L1/LInf codes */
  NMSG_ERR_BAD_ARG = -3,       /* argument out of range, dimension mismatch, ... */
  NMSG_ERR_OOM = -4,           /* device or pinned-host allocation failed */
  NMSG_ERR_DEVICE = -5,        /* CUDA runtime error */
  NMSG_ERR_TIMEOUT = -6,       /* a bounded device wait gave up */
  NMSG_ERR_CORRUPT_GRAPH = -7, /* neighbour id out of range, count above maxM/maxM0, ... */
  NMSG_ERR_CAPACITY = -8       /* a per-query device buffer would overflow */
};

/* Space names of nmslib.init(space=...): 'l2', 'cosinesimil', 'negdotprod', 'l1', 'linf'. The
 * last two are the optimized index's distance codes 5 and 6 (L1NormSIMD / LInfNormSIMD,
 * similarity_search/src/method/hnsw.cc:83-89, src/distcomp_lp.cc:77-251). */
enum nmsg_space { NMSG_SPACE_L2 = 0, NMSG_SPACE_COSINE = 1, NMSG_SPACE_NEGDOT = 2, NMSG_SPACE_L1 = 3, NMSG_SPACE_LINF = 4,
                  /* 'l2sqr_sift' with data_type DENSE_UINT8_VECTOR and dtype INT: 128 uint8 values per
                   * object, int squared L2 (similarity_search/src/space/space_l2sqr_sift.cc,
                   * src/distcomp_l2sqr_sift.cc:40-50); indices in the regular format + objects file */
                  NMSG_SPACE_L2SQR_SIFT = 5 };

/* algoType of setQueryTimeParams (hnsw.cc:486-497): hybrid uses SearchOld when ef >= 1000. */
enum nmsg_algo { NMSG_ALGO_HYBRID = 0, NMSG_ALGO_OLD = 1, NMSG_ALGO_V1MERGE = 2 };

/* nmsg_knn_batch flags */
enum nmsg_flags {
  NMSG_DEVICE_PTRS = 1, /* queries and outputs are device pointers; no host copies, no sync */
  NMSG_PLAIN_KERNEL = 2, /* one query per CUDA block (the unbatched kernel) instead of the
                           persistent work-queue kernel */
  NMSG_CUDA_GRAPH = 4,   /* with NMSG_DEVICE_PTRS: launch through a CUDA graph captured on the
                           first call and replayed while every argument stays the same */
  NMSG_EXACT_SCAN = 8    /* nmsg_bruteforce_knn: scan on CUDA cores with the search's own distance
                           arithmetic (every distance bit-identical to the HNSW search's) instead
                           of the tensor-core path */
};

typedef struct nmsg_index_info {
  int64_t n;            /* stored elements (totalElementsStored_) */
  int32_t dim;          /* vector length */
  int32_t dist_type;    /* DistFuncType code from the file: 1 L2Sqr16Ext, 2 L2SqrExt,
                           3 NormCosine, 4 NegativeDotProduct (hnsw.h:50-58) */
  int32_t maxlevel;
  int32_t enterpoint;
  int32_t maxM;
  int32_t maxM0;
  int32_t ef;           /* current query-time ef (20 after load, hnsw.cc:483) */
  int32_t algo;         /* current nmsg_algo */
  int32_t device;
  int64_t device_bytes; /* resident index bytes on the device */
} nmsg_index_info;

/* Load an optimized HNSW index file (the output of the reference's saveIndex) onto `device`.
 * `space` must agree with the file's distance code. ef is reset to 20 and algo to hybrid,
 * as IndexWrapper::loadIndex does through ResetQueryTimeParams (nmslib.cc:112). */
NMSG_API int nmsg_index_load(const char* path, int space, int device, nmsg_index** out);

/* Load an index whose vectors live in a separate objects file, like IndexWrapper::loadIndex(path,
 * load_data=True) (python_bindings/nmslib.cc:98-113): the objects from `data_path` (the
 * reference's `path + ".dat"`, Space::ReadObjectVectorFromBinData, space.cc) and the regular graph
 * file from `path` (Hnsw::LoadRegularIndexBin, similarity_search/src/method/hnsw.cc:943-991).
 * Space NMSG_SPACE_L2SQR_SIFT only (the reference has no optimized layout for it). Every count,
 * id and level is validated before the upload. ef is 20 and algo hybrid after the load. */
NMSG_API int nmsg_index_load_with_data(const char* path, const char* data_path, int space, int device,
                                       nmsg_index** out);

/* saveIndex(path, save_data=True) for an index loaded with nmsg_index_load_with_data
 * (nmslib.cc:115-125): the regular graph file (Hnsw::SaveRegularIndexBin, hnsw.cc:810-842) and the
 * objects file (Space::WriteObjectVectorBinData, space.cc); byte-identical to the reference's. */
NMSG_API int nmsg_index_save_with_data(const nmsg_index* index, const char* path, const char* data_path);

/* Write the loaded index back in the reference's optimized format (hnsw.cc:774-806). */
NMSG_API int nmsg_index_save(const nmsg_index* index, const char* path);

NMSG_API void nmsg_index_free(nmsg_index* index);

NMSG_API int nmsg_index_info_get(const nmsg_index* index, nmsg_index_info* out);

/* efSearch (>= 1) and algoType; applied to later nmsg_knn_batch calls. */
NMSG_API int nmsg_set_query_params(nmsg_index* index, int ef, int algo);

/* k-NN for nq queries of length dim (row-major float32).
 *   k_per_q / ef_per_q: optional per-query k and ef (NULL -> `k` / the index's ef).
 *   kmax: row stride of ids/dists (>= every k used).
 *   ids   [nq * kmax]: external ids (the ids stored in each node's object header), -1 padding.
 *   dists [nq * kmax]: distances in ascending order, +inf padding. l2 reports SQUARED
 *                      distance, as the reference's optimized path does.
 *   counts[nq]: results per query, min(k, found).
 *   stats [nq * 4] (optional): distance evaluations, level-0 expansions, upper-level list
 *                      scans, algorithmic bytes read.
 *   stream: a cudaStream_t (NULL = the legacy default stream).
 * Host pointers (default): copies in and out, synchronous. NMSG_DEVICE_PTRS: device pointers,
 * asynchronous on `stream`. Calls on one handle are serialised. */
NMSG_API int nmsg_knn_batch(nmsg_index* index, const float* queries, int64_t nq, int32_t dim, int32_t k,
                   const int32_t* k_per_q, const int32_t* ef_per_q, int32_t kmax, int32_t* ids,
                   float* dists, int32_t* counts, int64_t* stats, uint32_t flags, void* stream);

/* nmsg_knn_batch for l2sqr_sift indices: IndexWrapper<int>::knnQueryBatch over
 * DENSE_UINT8_VECTOR queries (nmslib.cc:142-168, :258-272: each query row becomes an object
 * with its int sum of squares) -> the generic Hnsw searches (hnsw.cc:1078-1290, the same steps as
 * the optimized ones). queries: nq x 128 uint8; dists: int32 squared L2 (INT32_MAX padding);
 * every other argument as nmsg_knn_batch. */
NMSG_API int nmsg_knn_batch_u8(nmsg_index* index, const uint8_t* queries, int64_t nq, int32_t dim, int32_t k,
                               const int32_t* k_per_q, const int32_t* ef_per_q, int32_t kmax, int32_t* ids,
                               int32_t* dists, int32_t* counts, int64_t* stats, uint32_t flags, void* stream);

/* Build an HNSW index on the host and write it in the optimized format, like
 * IndexWrapper::createIndex + saveIndex (python_bindings/nmslib.cc:89-96, :115-125)
 * -> Hnsw::CreateIndex (similarity_search/src/method/hnsw.cc:183-470): M, efConstruction,
 * maxM = M, maxM0 = 2M, mult = 1/ln M, neighbour heuristic 2. `ids` (optional) are the
 * external ids (addDataPointBatch ids=...), else row numbers. nthreads <= 0: all cores.
 * Node levels are a deterministic function of `seed`; the links depend on thread timing, as in
 * the reference's multi-threaded build. Spaces l2, cosinesimil and negdotprod (l1 / linf
 * indices come from the reference's createIndex: NMSG_ERR_UNSUPPORTED). */
NMSG_API int nmsg_build_index(const float* data, int64_t n, int32_t dim, const int32_t* ids, int space, int M,
                              int ef_construction, int nthreads, uint64_t seed, const char* out_path);

/* The same build with the efConstruction-wide level-0 searches on `device`: nodes with an upper
 * level and the first 4096 nodes are inserted on the host as above; every other node (level 0
 * only) joins in a batch whose searches run in the engine's search kernel (greedy descent, then
 * the level-0 beam with ef = k = efConstruction) over the graph as it stands before the batch,
 * after which the host selects its neighbours with heuristic 2 and adds the reverse links as
 * Hnsw::add does (hnsw.cc:534-609). A batch is an eighth of the graph so far; its nodes do not see
 * one another while searching. Same file format and parameters; the graph differs from a host
 * build as two multi-threaded builds of the reference differ. No reference counterpart for the
 * device part (the reference builds on the host only). */
NMSG_API int nmsg_build_index_device(const float* data, int64_t n, int32_t dim, const int32_t* ids, int space, int M,
                                     int ef_construction, int nthreads, uint64_t seed, int device,
                                     const char* out_path);

NMSG_API const char* nmsg_build_last_error(void);

/* Launch shape of the search kernels; 0 in a field = chosen automatically. */
typedef struct nmsg_launch_config {
  int32_t warps_per_block;   /* persistent kernel: 1, 2 or 4 queries (warps) per block */
  int32_t rows_per_group;    /* register gather: vector rows each 8-lane group loads per round
                                (1, 2 or 4) */
  int32_t stage_rows;        /* staged gather: rows copied into shared memory per round with
                                asynchronous copies (1..64); -1 = use the register gather */
  int32_t visited_hash_log2; /* per-query shared-memory visited table of 2^x ids (8..14);
                                -1 = visited set in HBM only */
  int32_t plain_slots;       /* one-query-per-block kernel: query slots (visited sets) its blocks
                                share; 0 = one per resident block. With fewer slots than resident
                                blocks, a block that finds no free slot in one bounded pass gives up:
                                its query returns nothing and the call fails with NMSG_ERR_TIMEOUT
                                (a way to exercise that bounded wait) */
  int32_t queries_per_warp;  /* persistent kernel: queries one warp carries at once (1..4); their
                                list reads, visited checks and row copies overlap. Used for
                                V1Merge batches over float rows staged in shared memory with lists
                                of up to 64 ids; other batches run one query per warp */
  int32_t row_copy;          /* that kernel's row staging: 0 = automatic, 1 = 16-byte asynchronous
                                copies spread over the lanes, 2 = one bulk copy (TMA unit) per row */
  int32_t query_order;       /* V1Merge batches of one efSearch on the lean kernel with more queries
                                than resident warps: 0 = automatic (every query's upper-level descent
                                first, then level 0 with the queries that enter it farthest from
                                their query first), -1 = one pass in batch order */
  int32_t host_copy;         /* calls on host buffers (no NMSG_DEVICE_PTRS): 0 = automatic (pageable
                                buffers of 512 KB and more go through page-locked staging that
                                several host threads fill and empty, with full-rate DMAs in between;
                                page-locked buffers are copied directly), 1 = copy the caller's
                                buffers directly */
} nmsg_launch_config;

/* Set (cfg != NULL) or reset to automatic (cfg == NULL) the launch shape used by later
 * nmsg_knn_batch calls on this handle. Results do not depend on it; speed does. */
NMSG_API int nmsg_set_launch_config(nmsg_index* index, const nmsg_launch_config* cfg);

/* nmsg_knn_batch for callers that cannot allocate device memory — no counterpart in the
 * reference (NMSLIB is CPU-only). Some callers must not call cudaMalloc at query time: real-time
 * serving threads that may not enter the allocator (its latency is unbounded), processes whose
 * device memory is reserved up front by another framework's pool, and plug-ins inside such an
 * engine. This entry point allocates nothing: queries, ids, dists and counts are caller-owned
 * DEVICE buffers (row stride kmax), k is uniform and ef/algoType are the handle's, and all per-call
 * scratch comes from one fixed 32 MiB device array that every GPU loading this library holds until
 * the process exits. One query slot needs round_up(n, 16) + 1 bytes (plus 8 * min(n + 1, 131072)
 * bytes when SearchOld runs), so the array bounds the queries in flight (33 at n = 1M) and the call
 * fails with NMSG_ERR_CAPACITY when not even one slot fits. The first call on a device looks up the
 * array's device address; make it before any stream capture. Calls share the array, which keeps
 * the last call's contents (a call with the previous call's slot layout reuses its visited-set
 * epochs; any other call clears what it uses): calls that overlap on the GPU race with each other.
 * Returns after the search has finished. */
NMSG_API int nmsg_knn_batch_noalloc(nmsg_index* index, const float* queries, int64_t nq, int32_t dim, int32_t k,
                                    int32_t kmax, int32_t* ids, float* dists, int32_t* counts, void* stream);

/* Exact k-NN by scanning every stored vector, the semantics of the reference's sequential
 * search (similarity_search/src/method/seqsearch.cc:143-177), on the tensor cores: a BF16 GEMM
 * (FP32 accumulation) over a sample of the base and an exact rerank in double-float arithmetic
 * give each query a threshold that, by a rigorous bound on the BF16 error, every true neighbour
 * reaches; a second BF16 GEMM over the whole base collects the vectors at or above it and the
 * exact rerank orders them. The ids are the exact top-k (ties by id); distances follow the
 * index's space as the HNSW path reports them (squared L2, 1 - cos on normalised vectors, -dot).
 * k <= 32. That is the path for l2 / cosinesimil / negdotprod rows of up to 4096 floats (up to 256
 * the query block stays in shared memory, wider rows stream its K-blocks beside the base's); L1,
 * LInf, wider rows and calls with NMSG_EXACT_SCAN are scanned exactly on CUDA cores with the query
 * path's own distance arithmetic (every distance bit-identical to the HNSW search's; stats then
 * {0, n, 0, chunks}). The full scan keeps
 * up to 64 vectors per query and per half of a base
 * chunk; a query that finds more in some chunk is scanned again with a raised threshold (up to
 * three times), and if it still overflows the call returns NMSG_ERR_CAPACITY (many vectors tied
 * with the k-th neighbour within the BF16 error bound). stats (optional, 4 values): sample rows
 * of the first pass, most vectors at or above the threshold for one query, queries rescanned,
 * base chunks per query block. Buffer conventions as nmsg_knn_batch. */
NMSG_API int nmsg_bruteforce_knn(nmsg_index* index, const float* queries, int64_t nq, int32_t dim, int32_t k,
                                 int32_t kmax, int32_t* ids, float* dists, int32_t* counts, int64_t* stats,
                                 uint32_t flags, void* stream);

/* ---- Serving: continuous batching over a loaded index (no reference counterpart; per-request
 * semantics are knnQueryBatch's, python_bindings/nmslib.cc:142-168). Requests of 1..max_batch
 * queries, each with its own k (<= max_k) and efSearch (< 1000, V1Merge), are admitted oldest
 * first as device memory frees up: a request takes one search slot per query (up to max_batch,
 * in whole blocks of 4) from a pool that memory_budget_bytes sizes (one slot = one visited byte
 * per stored element), and one of max_lanes lanes (a stream with staging buffers). Requests in
 * different lanes run concurrently on the device; each request's results do not depend on the
 * others. */
typedef struct nmsg_server nmsg_server;

NMSG_API int nmsg_server_create(nmsg_index* index, int64_t memory_budget_bytes, int32_t max_batch, int32_t max_k,
                                int32_t max_lanes, nmsg_server** out);
NMSG_API int nmsg_server_lanes(const nmsg_server* server);
/* Copies the queries; returns at once with a request id. */
NMSG_API int nmsg_server_submit(nmsg_server* server, const float* queries, int32_t nq, int32_t k, int32_t ef,
                                int64_t* request_id);
/* Blocks until the request finished; ids/dists are nq x k, counts nq; latency from submission. */
NMSG_API int nmsg_server_wait(nmsg_server* server, int64_t request_id, int32_t* ids, float* dists, int32_t* counts,
                              double* latency_s);
/* Open-loop replay of a request trace (arrival times in seconds from the start); per-request
 * latency from the scheduled arrival to completion, and the wall time of the whole trace. */
NMSG_API int nmsg_server_run_trace(nmsg_server* server, const float* queries, const int64_t* q_offset,
                                   const int32_t* nq, const int32_t* k, const int32_t* ef, const double* arrival_s,
                                   int64_t nreq, double* latency_s, double* wall_s);
NMSG_API void nmsg_server_free(nmsg_server* server);

/* ---- Query server: NMSLIB's Thrift QueryService (query_server/protocol.thrift;
 * query_server/cpp_client_server/QueryService_server.cpp:150-640) on a TCP port, binary protocol
 * over a buffered (unframed) stream, in front of a loaded index, so the reference's clients work
 * unchanged. knnQuery / knnQueryBatch return ReplyEntry lists in ascending distance
 * (QueryService_server.cpp:392-440); setQueryTimeParams("efSearch=64,algoType=v1merge") waits for
 * the queries in flight; rangeQuery answers QueryException "Range search is not supported!"
 * (hnsw.cc:712-715); getDistance computes the space's distance of two text objects on the GPU.
 * Float indices are searched through the continuous-batching serving loop where it applies.
 * port 0 picks a free port (nmsg_query_server_port tells which); at most max_connections clients
 * are served at once. The server uses the index's query-time parameters; do not change them
 * through other calls while it runs. */
typedef struct nmsg_query_server nmsg_query_server;
NMSG_API int nmsg_query_server_start(nmsg_index* index, int port, int max_connections, int debug,
                                     nmsg_query_server** out);
NMSG_API int nmsg_query_server_port(const nmsg_query_server* server);
NMSG_API void nmsg_query_server_stop(nmsg_query_server* server);

/* Device status of the last batch on this handle (NMSG_OK or a device-side error code). */
NMSG_API int nmsg_last_device_status(const nmsg_index* index);

/* Search kernels the last nmsg_knn_batch / nmsg_knn_batch_u8 call on this handle launched (under
 * NMSG_CUDA_GRAPH: launched by the graph it replayed): 1 for one pass, 3 for a batch that runs the
 * upper-level descent, the entry ordering and level 0 as separate passes, 4 when that descent runs
 * in two halves (pageable host queries copied in two parts, the first half's descents overlapping
 * the second half's copy); 0 when it launched none (an empty batch or index, or a call that failed
 * before launching). */
NMSG_API int nmsg_last_kernel_launches(const nmsg_index* index);

NMSG_API const char* nmsg_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* NMSLIB_B200_H_ */
