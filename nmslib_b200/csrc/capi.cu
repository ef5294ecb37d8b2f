// C ABI of the engine (declared in include/nmslib_b200.h): index upload, query-time parameters,
// batch search with host or device buffers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "engine.h"
#include "handle.h"
#include "../../include/nmslib_b200.h"

using namespace nmsg;

namespace nmsg {
void set_last_error(const std::string& msg);
}

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? NMSG_ERR_OOM : NMSG_ERR_DEVICE;
}

#define NMSG_CUDA(call, what)                      \
  do {                                             \
    cudaError_t e_ = (call);                       \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)


}  // namespace

namespace {

int upload_index(nmsg_index* h) {
  const HostIndex& hi = h->host;
  DevIndex& d = h->dev;
  d = DevIndex();
  d.n = hi.n;
  if (hi.n == 0) return NMSG_OK;
  d.dim = hi.dim;
  d.pitch = (hi.dim + 31) & ~31;
  d.n16 = hi.dim & ~15;
  d.n4 = hi.dim & ~3;
  d.row_bytes = 4 * hi.dim;
  d.maxM = (int)hi.maxM;
  d.maxM0 = (int)hi.maxM0;
  d.l0_pitch = ((int)hi.maxM0 + 1 + 7) & ~7;
  d.maxlevel = hi.maxlevel;
  d.enterpoint = (int)hi.enterpoint;
  d.dist_type = hi.dist_type;

  const int64_t n = hi.n;
  std::vector<float> vec((size_t)n * d.pitch, 0.0f);
  std::vector<int32_t> l0((size_t)n * d.l0_pitch, 0);
  std::vector<int32_t> ext(n);
  std::vector<uint32_t> seen_in(n, 0);  // 1 + the last node whose list held each id
  bool unique = true;
  for (int64_t i = 0; i < n; ++i) {
    const float* src = hi.vec(i);
    float* dst = vec.data() + i * d.pitch;
    for (int e = 0; e < hi.dim; ++e) dst[permuted_pos(e, hi.dim)] = src[e];
    const int32_t* lst = hi.l0(i);
    std::memcpy(l0.data() + i * d.l0_pitch, lst, 4 * (1 + lst[0]));
    for (int t = 1; t <= lst[0]; ++t) {  // ids were validated (< n) when the file was read
      if (seen_in[lst[t]] == (uint32_t)(i + 1)) unique = false;
      seen_in[lst[t]] = (uint32_t)(i + 1);
    }
    ext[i] = hi.ext_id(i);
  }
  d.l0_unique = unique ? 1 : 0;
  std::vector<int32_t> links = hi.up_links;
  if (links.empty()) links.push_back(0);
  NMSG_CUDA(h->vecs.ensure(vec.size() * 4, false), "cudaMalloc(vectors)");
  NMSG_CUDA(h->l0.ensure(l0.size() * 4, false), "cudaMalloc(level-0 lists)");
  NMSG_CUDA(h->up_off.ensure(n * 8, false), "cudaMalloc(upper offsets)");
  NMSG_CUDA(h->up_links.ensure(links.size() * 4, false), "cudaMalloc(upper lists)");
  NMSG_CUDA(h->ext_id.ensure(n * 4, false), "cudaMalloc(ids)");
  NMSG_CUDA(cudaMemcpy(h->vecs.p, vec.data(), vec.size() * 4, cudaMemcpyHostToDevice), "upload vectors");
  NMSG_CUDA(cudaMemcpy(h->l0.p, l0.data(), l0.size() * 4, cudaMemcpyHostToDevice), "upload lists");
  NMSG_CUDA(cudaMemcpy(h->up_off.p, hi.up_off.data(), n * 8, cudaMemcpyHostToDevice), "upload offsets");
  NMSG_CUDA(cudaMemcpy(h->up_links.p, links.data(), links.size() * 4, cudaMemcpyHostToDevice), "upload links");
  NMSG_CUDA(cudaMemcpy(h->ext_id.p, ext.data(), n * 4, cudaMemcpyHostToDevice), "upload ids");
  d.vecs = h->vecs.as<float>();
  d.l0 = h->l0.as<int32_t>();
  d.up_off = h->up_off.as<int64_t>();
  d.up_links = h->up_links.as<int32_t>();
  d.ext_id = h->ext_id.as<int32_t>();
  h->resident_bytes = (int64_t)(vec.size() * 4 + l0.size() * 4 + n * 12 + links.size() * 4);
  return NMSG_OK;
}

// l2sqr_sift index: 128-byte rows (the values only; the stored norms go to the device only if
// some stored norm differs from the sum of squares of its values, else the kernel recomputes
// them from the row it has read), the level-0 lists padded to l0_pitch, upper lists as CSR with
// a stride of capu + 1.
int upload_sift(nmsg_index* h) {
  const HostIndex& hi = h->host;
  DevIndex& d = h->dev;
  d = DevIndex();
  d.n = hi.n;
  d.dim = kSiftDim;
  d.pitch = kSiftDim / 4 + 4;  // shared-memory query: 128 values, the norm, padding to 16 bytes
  d.row_bytes = kSiftRowBytes;
  d.dist_type = kSiftL2;
  if (hi.n == 0) return NMSG_OK;
  d.maxM = (int)hi.capu;
  d.maxM0 = (int)hi.cap0;
  d.l0_pitch = ((int)hi.cap0 + 1 + 7) & ~7;
  d.maxlevel = hi.maxlevel;
  d.enterpoint = (int)hi.enterpoint;
  const int64_t n = hi.n;
  std::vector<int32_t> l0((size_t)n * d.l0_pitch, 0);
  bool norms_match = true;
  for (int64_t i = 0; i < n; ++i) {
    const int32_t* lst = hi.sift_l0.data() + i * (hi.cap0 + 1);
    std::memcpy(l0.data() + i * d.l0_pitch, lst, 4 * (1 + lst[0]));
    const uint8_t* v = hi.sift_vecs.data() + i * kSiftDim;
    int32_t s2 = 0;
    for (int e = 0; e < kSiftDim; ++e) s2 += int32_t(v[e]) * int32_t(v[e]);
    norms_match &= s2 == hi.sift_norms[i];
  }
  std::vector<int32_t> links = hi.up_links;
  if (links.empty()) links.push_back(0);
  NMSG_CUDA(h->vecs.ensure((size_t)n * kSiftDim, false), "cudaMalloc(vectors)");
  NMSG_CUDA(h->l0.ensure(l0.size() * 4, false), "cudaMalloc(level-0 lists)");
  NMSG_CUDA(h->up_off.ensure(n * 8, false), "cudaMalloc(upper offsets)");
  NMSG_CUDA(h->up_links.ensure(links.size() * 4, false), "cudaMalloc(upper lists)");
  NMSG_CUDA(h->ext_id.ensure(n * 4, false), "cudaMalloc(ids)");
  NMSG_CUDA(cudaMemcpy(h->vecs.p, hi.sift_vecs.data(), (size_t)n * kSiftDim, cudaMemcpyHostToDevice), "upload vectors");
  NMSG_CUDA(cudaMemcpy(h->l0.p, l0.data(), l0.size() * 4, cudaMemcpyHostToDevice), "upload lists");
  NMSG_CUDA(cudaMemcpy(h->up_off.p, hi.up_off.data(), n * 8, cudaMemcpyHostToDevice), "upload offsets");
  NMSG_CUDA(cudaMemcpy(h->up_links.p, links.data(), links.size() * 4, cudaMemcpyHostToDevice), "upload links");
  NMSG_CUDA(cudaMemcpy(h->ext_id.p, hi.sift_ids.data(), n * 4, cudaMemcpyHostToDevice), "upload ids");
  if (!norms_match) {
    NMSG_CUDA(h->norms.ensure(n * 4, false), "cudaMalloc(norms)");
    NMSG_CUDA(cudaMemcpy(h->norms.p, hi.sift_norms.data(), n * 4, cudaMemcpyHostToDevice), "upload norms");
    d.norms = h->norms.as<int32_t>();
  }
  d.vecs_u8 = h->vecs.as<uint8_t>();
  d.l0 = h->l0.as<int32_t>();
  d.up_off = h->up_off.as<int64_t>();
  d.up_links = h->up_links.as<int32_t>();
  d.ext_id = h->ext_id.as<int32_t>();
  h->resident_bytes = (int64_t)((size_t)n * kSiftDim + l0.size() * 4 + n * 12 + links.size() * 4 +
                                (norms_match ? 0 : n * 4));
  return NMSG_OK;
}

int space_matches(int space, int dist_type) {
  switch (space) {
    case NMSG_SPACE_L2: return dist_type == kL2Sqr16Ext || dist_type == kL2SqrExt;
    case NMSG_SPACE_COSINE: return dist_type == kNormCosine;
    case NMSG_SPACE_NEGDOT: return dist_type == kNegDot;
    case NMSG_SPACE_L1: return dist_type == kL1;
    case NMSG_SPACE_LINF: return dist_type == kLInf;
  }
  return 0;
}

}  // namespace

namespace nmsg {

// Rows per staging round when every row is one bulk copy completing on the warp's mbarrier: at most
// kBulkRoundBytes per round (one mbarrier phase). On B200, rounds of 122,880 and 153,600 bytes ran
// out of the wait bound (NMSG_ERR_TIMEOUT, the device still answering) while the general kernels
// re-initialised the mbarrier at every query of a warp; they now initialise it once per warp, and
// with that, 8-row rounds of 3,840-byte rows complete at full scale. Larger rounds have not been
// run since, so they are still not issued. Returns whether *rows changed.
static bool cap_bulk_round(const DevIndex& d, int* rows) {
  const int cap = std::max(1, kBulkRoundBytes / bulk_row_bytes(d));
  if (*rows <= cap) return false;
  *rows = cap;
  return true;
}

int plan_launch(const DevIndex& d, const nmsg_launch_config& cfg, int region, bool with_old, bool plain,
                LaunchPlan* out, std::string* err) {
  LaunchPlan p;
  p.with_old = with_old;
  p.nbpad = ((std::max(d.maxM, d.maxM0) + 1 + 31) / 32) * 32;
  p.region = (region + 1) & ~1;  // keeps the following shared-memory pieces 16-byte aligned
  // Launch shape: explicit configuration, else defaults by vector width and beam size.
  // Measured on B200 (1M x 128 SIFT-like, 10K queries, k 10): staging rows through shared memory
  // beats register gathers at every beam size; 8 rows per round is best up to efSearch 128
  // (4.10M q/s at 64 vs 3.47M for two register rows per 8-lane group), 4 rows at efSearch 256
  // (1.90M vs 1.64M), where the larger beam array leaves less shared memory per warp.
  p.stage_rows = 0;
  if (d.dist_type == kSiftL2) {
    p.gather = kSiftGather;  // the only kernels compiled with the uint8 distance
  } else if (d.dist_type == kL1 || d.dist_type == kLInf) {
    p.gather = kLpGather;  // the only kernels compiled with the L1 / LInf distances
  } else if (cfg.stage_rows > 0) {
    p.gather = 0;
    p.stage_rows = cfg.stage_rows;
  } else if (cfg.stage_rows == 0 && cfg.rows_per_group == 0 && d.pitch <= 256) {
    p.gather = 0;
    p.stage_rows = p.region <= 160 ? 8 : 4;
  } else if (cfg.stage_rows == 0 && cfg.rows_per_group == 0) {
    // wider rows: staged too, by one bulk copy per row unless 16-byte copies are asked for (rounds
    // capped below). Measured on B200 for the 1M x 960 negdot mixed batch (8000 queries, per-query
    // k and efSearch up to 1024): 41.95 ms staged by bulk copies, 47.91 ms staged by 16-byte copies,
    // 56.04 ms with the rows gathered into registers.
    p.gather = 0;
    p.stage_rows = 8;
  } else {
    p.gather = cfg.rows_per_group ? cfg.rows_per_group : (d.pitch <= 256 ? 2 : 1);
  }
  const int hl = cfg.visited_hash_log2 == 0 ? -1 : cfg.visited_hash_log2;  // default: visited set in HBM
  p.hash_log2 = hl > 0 ? hl : 0;
  p.warp_smem = warp_smem_bytes(d, p.region, p.nbpad, p.hash_log2, p.stage_rows);
  while (p.gather == 0 && p.stage_rows > 1 && p.warp_smem > kMaxSmemPerBlock) {  // wide rows: fewer per round
    p.stage_rows = (p.stage_rows + 1) / 2;
    p.warp_smem = warp_smem_bytes(d, p.region, p.nbpad, p.hash_log2, p.stage_rows);
  }
  // several queries per warp (search_multi_kernel): V1Merge over staged float rows, lists of up
  // to 64 ids, no shared-memory visited table
  p.ctx = 1;
  const int want_ctx = cfg.queries_per_warp ? cfg.queries_per_warp : kDefaultQueriesPerWarp;
  if (!plain && !with_old && p.gather == 0 && p.hash_log2 == 0 && want_ctx > 1 && p.stage_rows <= 32 &&
      std::max(d.maxM, d.maxM0) <= 64) {
    const int nbpad = std::max(32, ((std::max(d.maxM, d.maxM0) + 31) / 32) * 32);
    for (int c = want_ctx; c > 1; --c) {
      const int ws = multi_warp_smem_bytes(d, p.region, nbpad, p.stage_rows, c);
      if (ws <= kMaxSmemPerBlock) {
        p.ctx = c;
        p.nbpad = nbpad;
        p.warp_smem = ws;
        break;
      }
    }
    if (p.ctx > 1) {
      p.bulk_rows = cfg.row_copy == 2 || (cfg.row_copy == 0 && d.dim * 4 >= kBulkRowMinBytes);
      if (p.bulk_rows && cap_bulk_round(d, &p.stage_rows))
        p.warp_smem = multi_warp_smem_bytes(d, p.region, p.nbpad, p.stage_rows, p.ctx);
    }
  }
  // the general kernels stage wide rows with one bulk copy each (row_copy 2 asks for it always)
  if (p.gather == 0 && p.ctx == 1) {
    p.bulk_rows = cfg.row_copy == 2 || (cfg.row_copy == 0 && d.dim * 4 >= kBulkRowMinBytes);
    if (p.bulk_rows && cap_bulk_round(d, &p.stage_rows))
      p.warp_smem = warp_smem_bytes(d, p.region, p.nbpad, p.hash_log2, p.stage_rows);
  }
  // the lean kernel: V1Merge with one query per warp over the index shapes it is compiled for,
  // rows staged by one bulk copy each, or by 16-byte copies spread over the lanes (row_copy 1)
  p.lean = false;
  if (!plain && !with_old && p.gather == 0 && p.hash_log2 == 0 && p.ctx == 1 && lean_supported(d)) {
    const int nbpad = std::max(32, ((std::max(d.maxM, d.maxM0) + 31) / 32) * 32);
    const bool bulk = cfg.row_copy != 1;
    int rows = p.stage_rows;
    if (bulk) cap_bulk_round(d, &rows);
    const int ws = lean_smem_bytes(d, p.region, nbpad, rows);
    if (ws <= kMaxSmemPerBlock) {
      p.lean = true;
      p.bulk_rows = bulk;
      p.nbpad = nbpad;
      p.stage_rows = rows;
      p.warp_smem = ws;
    }
  }
  p.wpb = plain ? 1 : (cfg.warps_per_block ? cfg.warps_per_block : kWarpsPerBlock);
  while (p.wpb > 1 && p.wpb * p.warp_smem > kMaxSmemPerBlock) p.wpb >>= 1;
  if (p.wpb * p.warp_smem > kMaxSmemPerBlock) {
    *err = "max(ef, k) = " + std::to_string(p.region) + " needs more shared memory per query than a block has";
    return NMSG_ERR_CAPACITY;
  }
  p.blocks_per_sm = 0;
  const int rc = p.lean ? lean_occupancy(d, p.wpb, p.wpb * p.warp_smem, &p.blocks_per_sm)
                        : search_occupancy(plain, p.gather, with_old, p.wpb, p.wpb * p.warp_smem, &p.blocks_per_sm,
                                           p.ctx, multi_list_chunks(d));
  if (rc != 0 || p.blocks_per_sm < 1) {
    *err = "no resident block fits this configuration";
    return NMSG_ERR_DEVICE;
  }
  *out = p;
  return NMSG_OK;
}

}  // namespace nmsg

extern "C" {

const char* nmsg_last_error(void) { return g_err.c_str(); }

}  // extern "C"

void nmsg::set_last_error(const std::string& msg) { g_err = msg; }

extern "C" {

int nmsg_index_load(const char* path, int space, int device, nmsg_index** out) {
  if (!out || !path) return fail(NMSG_ERR_BAD_ARG, "null argument");
  *out = nullptr;
  if (space < NMSG_SPACE_L2 || space > NMSG_SPACE_LINF) return fail(NMSG_ERR_BAD_ARG, "unknown space code");
  auto* h = new nmsg_index();
  h->device = device;
  h->space = space;
  std::string err;
  int rc = read_index_file(path, h->host, err);
  if (rc == NMSG_OK) rc = validate_index(h->host, err);
  if (rc == NMSG_OK && !h->host.empty_regular && h->host.n > 0 && !space_matches(space, h->host.dist_type)) {
    rc = NMSG_ERR_BAD_ARG;
    err = "the index file was built for a different space (distance code " + std::to_string(h->host.dist_type) + ")";
  }
  if (rc != NMSG_OK) {
    delete h;
    return fail(rc, err);
  }
  // the file is read and validated before any device is touched
  int ndev = 0;
  cudaError_t ce = cudaGetDeviceCount(&ndev);
  if (ce != cudaSuccess || ndev == 0) {
    delete h;
    return fail(NMSG_ERR_DEVICE, "no CUDA device is available");
  }
  if (device < 0 || device >= ndev) {
    delete h;
    return fail(NMSG_ERR_BAD_ARG, "device ordinal out of range");
  }
  {
    DeviceGuard g(device);
    cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device);
    rc = upload_index(h);
  }
  if (rc != NMSG_OK) {
    nmsg_index_free(h);
    return rc;
  }
  *out = h;
  return NMSG_OK;
}

int nmsg_index_save(const nmsg_index* h, const char* path) {
  if (!h || !path) return fail(NMSG_ERR_BAD_ARG, "null argument");
  if (h->host.sift)
    return fail(NMSG_ERR_BAD_ARG, "an l2sqr_sift index is saved with its objects file: nmsg_index_save_with_data");
  std::string err;
  int rc = write_index_file(path, h->host, err);
  return rc == NMSG_OK ? rc : fail(rc, err);
}

int nmsg_index_load_with_data(const char* path, const char* data_path, int space, int device, nmsg_index** out) {
  if (!out || !path || !data_path) return fail(NMSG_ERR_BAD_ARG, "null argument");
  *out = nullptr;
  if (space != NMSG_SPACE_L2SQR_SIFT)
    return fail(NMSG_ERR_UNSUPPORTED, "loading with a data file is supported for the l2sqr_sift space only");
  auto* h = new nmsg_index();
  h->device = device;
  h->space = space;
  std::string err;
  const int rc0 = read_sift_index(path, data_path, h->host, err);
  if (rc0 != NMSG_OK) {
    delete h;
    return fail(rc0, err);
  }
  int ndev = 0;
  cudaError_t ce = cudaGetDeviceCount(&ndev);
  if (ce != cudaSuccess || ndev == 0) {
    delete h;
    return fail(NMSG_ERR_DEVICE, "no CUDA device is available");
  }
  if (device < 0 || device >= ndev) {
    delete h;
    return fail(NMSG_ERR_BAD_ARG, "device ordinal out of range");
  }
  int rc;
  {
    DeviceGuard g(device);
    cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device);
    rc = upload_sift(h);
  }
  if (rc != NMSG_OK) {
    nmsg_index_free(h);
    return rc;
  }
  *out = h;
  return NMSG_OK;
}

int nmsg_index_save_with_data(const nmsg_index* h, const char* path, const char* data_path) {
  if (!h || !path || !data_path) return fail(NMSG_ERR_BAD_ARG, "null argument");
  if (!h->host.sift) return fail(NMSG_ERR_UNSUPPORTED, "saving with a data file is supported for l2sqr_sift indices only");
  std::string err;
  const int rc = write_sift_index(path, data_path, h->host, err);
  return rc == NMSG_OK ? rc : fail(rc, err);
}

void nmsg_index_free(nmsg_index* h) {
  if (!h) return;
  {
    DeviceGuard g(h->device);
    if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
    if (h->capture_stream) cudaStreamDestroy(h->capture_stream);
    if (h->copy_stream) {
      cudaStreamSynchronize(h->copy_stream);
      cudaStreamDestroy(h->copy_stream);
    }
    for (cudaEvent_t ev : h->part_ev)
      if (ev) cudaEventDestroy(ev);
    destroy_bruteforce(h->bf);
    h->bf = nullptr;
    for (DevBuf* b : {&h->vecs, &h->norms, &h->l0, &h->up_off, &h->up_links, &h->ext_id, &h->visited, &h->epochs, &h->locks,
                      &h->old_heap, &h->counter, &h->status, &h->order, &h->kq, &h->efq, &h->q_stage,
                      &h->ids_stage, &h->dists_stage, &h->counts_stage, &h->stats_stage, &h->entry})
      b->release();
    h->pin_in.release();
    h->pin_out.release();
  }
  delete h;
}

int nmsg_index_info_get(const nmsg_index* h, nmsg_index_info* out) {
  if (!h || !out) return fail(NMSG_ERR_BAD_ARG, "null argument");
  out->n = h->host.n;
  out->dim = h->host.dim;
  out->dist_type = h->host.dist_type;
  out->maxlevel = h->host.maxlevel;
  out->enterpoint = (int32_t)h->host.enterpoint;
  out->maxM = (int32_t)h->host.maxM;
  out->maxM0 = (int32_t)h->host.maxM0;
  out->ef = h->ef;
  out->algo = h->algo;
  out->device = h->device;
  out->device_bytes = h->resident_bytes;
  return NMSG_OK;
}

int nmsg_set_query_params(nmsg_index* h, int ef, int algo) {
  if (!h) return fail(NMSG_ERR_BAD_ARG, "null index");
  if (ef < 0) return fail(NMSG_ERR_BAD_ARG, "ef must be non-negative");
  if (algo < 0 || algo > 2) return fail(NMSG_ERR_BAD_ARG, "algoType should be one of the following: old, v1merge");
  std::lock_guard<std::mutex> lk(h->mu);
  h->ef = ef;
  h->algo = algo;
  return NMSG_OK;
}

int nmsg_last_device_status(const nmsg_index* h) { return h ? h->last_status : NMSG_ERR_BAD_ARG; }

int nmsg_last_kernel_launches(const nmsg_index* h) { return h ? h->last_launches : NMSG_ERR_BAD_ARG; }

int nmsg_set_launch_config(nmsg_index* h, const nmsg_launch_config* cfg) {
  if (!h) return fail(NMSG_ERR_BAD_ARG, "null index");
  nmsg_launch_config c{0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (cfg) {
    c = *cfg;
    if (c.plain_slots < 0) return fail(NMSG_ERR_BAD_ARG, "plain_slots must be >= 0");
    if (c.queries_per_warp < 0 || c.queries_per_warp > 4) return fail(NMSG_ERR_BAD_ARG, "queries_per_warp must be 0..4");
    if (c.row_copy < 0 || c.row_copy > 2) return fail(NMSG_ERR_BAD_ARG, "row_copy must be 0, 1 or 2");
    if (c.query_order != 0 && c.query_order != -1) return fail(NMSG_ERR_BAD_ARG, "query_order must be 0 or -1");
    if (c.host_copy != 0 && c.host_copy != 1) return fail(NMSG_ERR_BAD_ARG, "host_copy must be 0 or 1");
    const int w = c.warps_per_block, r = c.rows_per_group, hl = c.visited_hash_log2, sr = c.stage_rows;
    if (!(w == 0 || w == 1 || w == 2 || w == 4)) return fail(NMSG_ERR_BAD_ARG, "warps_per_block must be 0, 1, 2 or 4");
    if (!(r == 0 || r == 1 || r == 2 || r == 4)) return fail(NMSG_ERR_BAD_ARG, "rows_per_group must be 0, 1, 2 or 4");
    if (!(sr == -1 || (sr >= 0 && sr <= 64))) return fail(NMSG_ERR_BAD_ARG, "stage_rows must be -1 or 0..64");
    if (!(hl == 0 || hl == -1 || (hl >= 8 && hl <= 14)))
      return fail(NMSG_ERR_BAD_ARG, "visited_hash_log2 must be 0, -1 or 8..14");
  }
  std::lock_guard<std::mutex> lk(h->mu);
  h->cfg = c;
  return NMSG_OK;
}

}  // extern "C"

namespace {

// The batch search behind nmsg_knn_batch (float queries and distances) and nmsg_knn_batch_u8
// (l2sqr_sift: uint8 queries, int distances).
int knn_batch_impl(nmsg_index* h, const void* queries_v, bool u8, int64_t nq, int32_t dim, int32_t k,
                   const int32_t* k_per_q, const int32_t* ef_per_q, int32_t kmax, int32_t* ids, void* dists_v,
                   int32_t* counts, int64_t* stats, uint32_t flags, void* stream) {
  const float* queries = static_cast<const float*>(queries_v);
  float* dists = static_cast<float*>(dists_v);
  if (nq < 0) return fail(NMSG_ERR_BAD_ARG, "negative query count");
  if (nq > 0 && (!queries || !ids || !dists || !counts)) return fail(NMSG_ERR_BAD_ARG, "null buffer");
  const bool dev_ptrs = flags & NMSG_DEVICE_PTRS;
  if (dev_ptrs && (k_per_q || ef_per_q))
    return fail(NMSG_ERR_BAD_ARG, "per-query k/ef arrays are host arrays; pass host buffers for mixed batches");
  std::lock_guard<std::mutex> lk(h->mu);
  h->last_launches = 0;
  const int ef = h->ef, algo = h->algo;
  // per-query parameters and capacity of the shared-memory region
  int region = 1;
  bool any_old = false;
  for (int64_t i = 0; i < nq; ++i) {
    const int kq = k_per_q ? k_per_q[i] : k;
    const int eq = ef_per_q ? ef_per_q[i] : ef;
    if (kq < 1) return fail(NMSG_ERR_BAD_ARG, "k must be at least 1");
    if (kq > kmax) return fail(NMSG_ERR_BAD_ARG, "k exceeds the output row stride kmax");
    if (eq < 0) return fail(NMSG_ERR_BAD_ARG, "ef must be non-negative");
    const bool old = algo == NMSG_ALGO_OLD || (algo == NMSG_ALGO_HYBRID && eq >= 1000);
    any_old |= old;
    // V1Merge keeps its sorted array of max(ef, k) items; SearchOld its closest-set heap (ef + 1)
    // and the k results
    region = std::max(region, old ? eq + 1 + kq : std::max(eq, kq));
    if (!k_per_q && !ef_per_q) break;  // uniform batch: one check covers every query
  }
  if (nq == 0) return NMSG_OK;
  const DevIndex& d = h->dev;
  if (d.n == 0) {  // empty index: every query returns nothing (hnsw.cc:721-723)
    if (dev_ptrs) {
      DeviceGuard g(h->device);
      NMSG_CUDA(cudaMemsetAsync(counts, 0, nq * 4, (cudaStream_t)stream), "memset counts");
      NMSG_CUDA(cudaMemsetAsync(ids, 0xff, nq * kmax * 4, (cudaStream_t)stream), "memset ids");
    } else {
      std::fill(counts, counts + nq, 0);
      std::fill(ids, ids + nq * kmax, -1);
      if (u8)
        std::fill(static_cast<int32_t*>(dists_v), static_cast<int32_t*>(dists_v) + nq * kmax, 0x7fffffff);
      else
        std::fill(dists, dists + nq * kmax, __builtin_inff());
      if (stats) std::fill(stats, stats + nq * 4, 0);
    }
    return NMSG_OK;
  }
  if (dim != d.dim)
    return fail(NMSG_ERR_BAD_ARG, "query dimension " + std::to_string(dim) + " does not match the index dimension " +
                                      std::to_string(d.dim));
  DeviceGuard g(h->device);
  cudaStream_t st = (cudaStream_t)stream;
  const bool plain = flags & NMSG_PLAIN_KERNEL;

  SearchArgs a;
  std::memset(&a, 0, sizeof(a));  // padding too: the CUDA-graph cache compares argument bytes
  a.ix = d;
  a.nq = nq;
  a.dists_int = u8 ? 1 : 0;
  a.k_default = k;
  a.ef_default = ef;
  a.algo = algo;
  a.kmax = kmax;
  LaunchPlan plan;
  std::string perr;
  int rc = plan_launch(d, h->cfg, region, any_old, plain, &plan, &perr);
  if (rc != NMSG_OK) return fail(rc, perr);
  region = plan.region;
  a.region_items = plan.region;
  a.hash_log2 = plan.hash_log2;
  a.stage_rows = plan.stage_rows;
  a.warp_smem = plan.warp_smem;
  const int gather = plan.gather, wpb = plan.wpb, bps = plan.blocks_per_sm;
  const int blocks = plain ? 0 : bps * h->num_sms;
  const int slots = plain ? (h->cfg.plain_slots > 0 ? std::min(h->cfg.plain_slots, bps * h->num_sms)
                                                   : bps * h->num_sms)
                          : blocks * wpb * plan.ctx;
  a.ctx_per_warp = plan.ctx;
  a.bulk_rows = plan.bulk_rows ? 1 : 0;
  a.lean = plan.lean ? 1 : 0;
  // scratch
  const int64_t vpitch = ((d.n + 15) / 16) * 16;
  if (slots > h->slots || (int64_t)h->visited.bytes < (int64_t)slots * vpitch) {
    h->visited.release();
    h->epochs.release();
    h->locks.release();
    NMSG_CUDA(h->visited.ensure((size_t)slots * vpitch, true), "cudaMalloc(visited sets)");
    NMSG_CUDA(h->epochs.ensure(slots, true), "cudaMalloc(epochs)");
    NMSG_CUDA(h->locks.ensure((size_t)slots * 4, true), "cudaMalloc(slot locks)");
    h->slots = slots;
  }
  if (any_old) {
    const int64_t cap = std::min<int64_t>(d.n + 1, 1 << 17);
    if (cap > h->old_cap || (int64_t)h->old_heap.bytes < (int64_t)h->slots * cap * 8) {
      h->old_heap.release();
      NMSG_CUDA(h->old_heap.ensure((size_t)h->slots * cap * 8, false), "cudaMalloc(SearchOld heaps)");
      h->old_cap = cap;
    }
  }
  NMSG_CUDA(h->counter.ensure(4, true), "cudaMalloc(counter)");
  NMSG_CUDA(h->status.ensure(4, true), "cudaMalloc(status)");
  a.visited = h->visited.as<uint8_t>();
  a.visited_pitch = vpitch;
  a.epochs = h->epochs.as<uint8_t>();
  a.slot_locks = h->locks.as<int32_t>();
  a.num_slots = slots;
  a.old_heap = h->old_heap.as<uint2>();
  a.old_heap_cap = h->old_cap;
  a.work_counter = h->counter.as<int32_t>();
  a.status = h->status.as<int32_t>();

  // Split search: worth it once the batch outnumbers the resident warps (some warps then run
  // several queries, and which queries start last decides when the batch ends). V1Merge batches of
  // one efSearch on the one-query-per-warp kernels.
  const bool split =
      (plan.lean || (plan.ctx == 1 && !any_old)) && !plain && !ef_per_q && nq > slots && h->cfg.query_order != -1;
  QueryParts parts;
  bool use_parts = false;

  // inputs / outputs
  const size_t qbytes = (size_t)nq * dim * (u8 ? 1 : 4), obytes = (size_t)nq * kmax * 4;
  if (dev_ptrs) {
    if (u8)
      a.queries_u8 = static_cast<const uint8_t*>(queries_v);
    else
      a.queries = queries;
    a.ids = ids;
    a.dists = dists;
    a.counts = counts;
    a.stats = stats;
  } else {
    NMSG_CUDA(h->q_stage.ensure(qbytes, false), "cudaMalloc(query staging)");
    NMSG_CUDA(h->ids_stage.ensure(obytes, false), "cudaMalloc(id staging)");
    NMSG_CUDA(h->dists_stage.ensure(obytes, false), "cudaMalloc(distance staging)");
    NMSG_CUDA(h->counts_stage.ensure((size_t)nq * 4, false), "cudaMalloc(count staging)");
    if (stats) NMSG_CUDA(h->stats_stage.ensure((size_t)nq * 32, false), "cudaMalloc(stats staging)");
    HostPiece up[3];
    int nup = 0;
    up[nup++] = HostPiece{h->q_stage.p, queries_v, qbytes};
    if (u8)
      a.queries_u8 = h->q_stage.as<uint8_t>();
    else
      a.queries = h->q_stage.as<float>();
    a.ids = h->ids_stage.as<int32_t>();
    a.dists = h->dists_stage.as<float>();
    a.counts = h->counts_stage.as<int32_t>();
    a.stats = stats ? h->stats_stage.as<int64_t>() : nullptr;
    if (k_per_q) {
      NMSG_CUDA(h->kq.ensure((size_t)nq * 4, false), "cudaMalloc(k per query)");
      up[nup++] = HostPiece{h->kq.p, k_per_q, (size_t)nq * 4};
      a.k_per_q = h->kq.as<int32_t>();
    }
    if (ef_per_q) {
      NMSG_CUDA(h->efq.ensure((size_t)nq * 4, false), "cudaMalloc(ef per query)");
      up[nup++] = HostPiece{h->efq.p, ef_per_q, (size_t)nq * 4};
      a.ef_per_q = h->efq.as<int32_t>();
      // most expensive queries first, so the persistent warps finish together
      std::vector<int32_t> order(nq);
      std::iota(order.begin(), order.end(), 0);
      std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return ef_per_q[x] > ef_per_q[y]; });
      NMSG_CUDA(h->order.ensure((size_t)nq * 4, false), "cudaMalloc(order)");
      NMSG_CUDA(cudaMemcpy(h->order.p, order.data(), nq * 4, cudaMemcpyHostToDevice), "copy order");
      a.order = h->order.as<int32_t>();
    }
    const bool staged = use_staging(h->pin_in, h->cfg.host_copy == 0, up, nup, true);
    const bool locked = !staged && h->cfg.host_copy == 0 && host_range_page_locked(up[0].src, up[0].bytes);
    if (split && plan.lean && (staged || locked)) {
      // Two halves on the handle's copy stream: the first half's descents start while the second
      // half is still being copied (pageable queries through staging, page-locked ones directly).
      if (!h->copy_stream) {
        NMSG_CUDA(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking), "copy stream");
        for (cudaEvent_t& ev : h->part_ev) NMSG_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "event");
      }
      NMSG_CUDA(cudaEventRecord(h->part_ev[2], st), "record");  // after the caller's earlier work on st
      NMSG_CUDA(cudaStreamWaitEvent(h->copy_stream, h->part_ev[2], 0), "wait");
      parts.first = nq / 2;
      parts.ready[0] = h->part_ev[0];
      parts.ready[1] = h->part_ev[1];
      if (staged)
        NMSG_CUDA(upload_staged_parts(h->pin_in, up, nup, (size_t)parts.first * dim * 4, h->copy_stream, h->part_ev),
                  "copy queries");
      else
        NMSG_CUDA(upload_parts_direct(up, nup, (size_t)parts.first * dim * 4, h->copy_stream, h->part_ev),
                  "copy queries");
      use_parts = true;
    } else {
      NMSG_CUDA(copy_to_device(h->pin_in, h->cfg.host_copy == 0, up, nup, st), "copy queries");
    }
  }
  a.nbpad = plan.nbpad;
  if (split) {
    const size_t words = (size_t)nq * 6 + 4;  // node, distance, 3 counts, order; range
    NMSG_CUDA(h->entry.ensure(words * 4, false), "cudaMalloc(level-0 entries)");
    int32_t* e = h->entry.as<int32_t>();
    a.entry_node = e;
    a.entry_dist = reinterpret_cast<float*>(e + nq);
    a.entry_stats = e + 2 * nq;
    a.entry_order = e + 5 * nq;
    a.entry_range = reinterpret_cast<uint32_t*>(e + 6 * nq);
  }
  // launch_search runs the descent, the order kernel and level 0 when the entry arrays are set
  const int split_launches = (!plain && a.entry_node) ? 3 : 1;
  if (dev_ptrs && (flags & NMSG_CUDA_GRAPH)) {
    // Replay the captured launch when every argument is the same as last time; otherwise
    // capture (counter and status resets + kernel) into a new graph.
    const bool same = h->graph_exec && std::memcmp(&h->graph_args, &a, sizeof(SearchArgs)) == 0 &&
                      h->graph_shape[0] == (int)plain && h->graph_shape[1] == gather &&
                      h->graph_shape[2] == (int)any_old && h->graph_shape[3] == blocks && h->graph_shape[4] == wpb;
    if (!same) {
      if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
      h->graph_exec = nullptr;
      // capture on the handle's own stream (the legacy default stream cannot be captured); the
      // graph is then launched on the caller's stream
      if (!h->capture_stream) NMSG_CUDA(cudaStreamCreateWithFlags(&h->capture_stream, cudaStreamNonBlocking), "stream");
      cudaStream_t cs = h->capture_stream;
      NMSG_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "begin capture");
      cudaMemsetAsync(a.work_counter, 0, 4, cs);
      cudaMemsetAsync(a.status, 0, 4, cs);
      const int lrc = launch_search(a, plain, gather, any_old, blocks, wpb, cs);
      cudaGraph_t graph = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(cs, &graph);
      if (lrc != 0 || ce != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return cuda_fail(ce != cudaSuccess ? ce : (cudaError_t)lrc, "capture search launch");
      }
      const cudaError_t ie = cudaGraphInstantiate(&h->graph_exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ie != cudaSuccess) return cuda_fail(ie, "instantiate search graph");
      std::memcpy(&h->graph_args, &a, sizeof(SearchArgs));
      h->graph_shape[0] = (int)plain;
      h->graph_shape[1] = gather;
      h->graph_shape[2] = (int)any_old;
      h->graph_shape[3] = blocks;
      h->graph_shape[4] = wpb;
    }
    NMSG_CUDA(cudaGraphLaunch(h->graph_exec, st), "graph launch");
    h->last_launches = split_launches;
    return NMSG_OK;
  }
  NMSG_CUDA(cudaMemsetAsync(a.work_counter, 0, 4, st), "reset counter");
  NMSG_CUDA(cudaMemsetAsync(a.status, 0, 4, st), "reset status");
  rc = launch_search(a, plain, gather, any_old, blocks, wpb, stream, use_parts ? &parts : nullptr);
  if (rc != 0) return cuda_fail((cudaError_t)rc, "search kernel launch");
  h->last_launches = split_launches + (use_parts ? 1 : 0);
  if (dev_ptrs) return NMSG_OK;
  int32_t dstatus = 0;
  const HostPiece down[5] = {{ids, a.ids, obytes},
                             {dists_v, a.dists, obytes},
                             {counts, a.counts, (size_t)nq * 4},
                             {&dstatus, a.status, 4},
                             {stats, a.stats, stats ? (size_t)nq * 32 : 0}};
  NMSG_CUDA(copy_to_host(h->pin_out, h->cfg.host_copy == 0, down, stats ? 5 : 4, st), "copy results");
  h->last_status = dstatus;
  if (dstatus != 0) return fail(dstatus, "the search kernel reported a device-side error (status " + std::to_string(dstatus) + ")");
  return NMSG_OK;
}

}  // namespace

extern "C" {

int nmsg_knn_batch(nmsg_index* h, const float* queries, int64_t nq, int32_t dim, int32_t k,
                   const int32_t* k_per_q, const int32_t* ef_per_q, int32_t kmax, int32_t* ids, float* dists,
                   int32_t* counts, int64_t* stats, uint32_t flags, void* stream) {
  if (!h) return fail(NMSG_ERR_BAD_ARG, "Must call createIndex or loadIndex before this method");
  if (h->host.sift)
    return fail(NMSG_ERR_BAD_ARG, "this index holds uint8 (l2sqr_sift) vectors: search it with nmsg_knn_batch_u8");
  return knn_batch_impl(h, queries, false, nq, dim, k, k_per_q, ef_per_q, kmax, ids, dists, counts, stats, flags,
                        stream);
}

int nmsg_knn_batch_u8(nmsg_index* h, const uint8_t* queries, int64_t nq, int32_t dim, int32_t k,
                      const int32_t* k_per_q, const int32_t* ef_per_q, int32_t kmax, int32_t* ids, int32_t* dists,
                      int32_t* counts, int64_t* stats, uint32_t flags, void* stream) {
  if (!h) return fail(NMSG_ERR_BAD_ARG, "Must call createIndex or loadIndex before this method");
  if (!h->host.sift) return fail(NMSG_ERR_BAD_ARG, "nmsg_knn_batch_u8 searches l2sqr_sift indices only");
  if (h->host.n > 0 && nq > 0 && dim != kSiftDim)
    return fail(NMSG_ERR_BAD_ARG, "query dimension " + std::to_string(dim) + " does not match the index dimension 128");
  return knn_batch_impl(h, queries, true, nq, dim, k, k_per_q, ef_per_q, kmax, ids, dists, counts, stats, flags,
                        stream);
}

}  // extern "C"
