// Reader and writer of an l2sqr_sift HNSW index: the regular graph file and the objects file.
//
// The reference has no optimized layout for this space (the optimized packing covers float
// vectors only, similarity_search/src/method/hnsw.cc:370-400), so saveIndex(path, save_data=True)
// writes two files:
//   <path>      SaveRegularIndexBin (hnsw.cc:810-842) after the u32 flag 0: u32 N | i32 maxlevel |
//               u32 entry point | u64 M | u64 maxM | u64 maxM0, then per node u32 level and, for
//               every level 0..level, u32 count and that many i32 neighbour ids
//               (read back by LoadRegularIndexBin, hnsw.cc:943-991);
//   <path>.dat  WriteObjectVectorBinData (space.cc): u64 count, then per object u64 length and the
//               object: i32 id | i32 label | u64 data length (132) | 128 uint8 values | i32 sum of
//               their squares (space_l2sqr_sift.cc:137-150); loadIndex(path, load_data=True) reads
//               it first (python_bindings/nmslib.cc:98-113).
// Everything is validated before it can reach the device: counts, ids, list lengths, and that
// every upper-level neighbour exists at that level (the greedy descent reads its list there).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "engine.h"
#include "../../include/nmslib_b200.h"

namespace nmsg {

namespace {
struct FileCloser {
  void operator()(FILE* f) const {
    if (f) std::fclose(f);
  }
};
template <typename T>
bool rd(FILE* f, T& v) {
  return std::fread(&v, sizeof(T), 1, f) == 1;
}
template <typename T>
bool wr(FILE* f, const T& v) {
  return std::fwrite(&v, sizeof(T), 1, f) == 1;
}
int64_t file_size(FILE* f) {
  if (std::fseek(f, 0, SEEK_END) != 0) return -1;
  const long sz = std::ftell(f);
  if (std::fseek(f, 0, SEEK_SET) != 0) return -1;
  return sz;
}
constexpr uint64_t kObjectBytes = 16 + kSiftRowBytes;  // id, label, data length, payload
constexpr uint32_t kMaxLevel = 64;
constexpr uint32_t kMaxList0 = 100;  // the kernels read level-0 lists of up to 100 ids
}  // namespace

int read_sift_index(const char* graph_path, const char* data_path, HostIndex& ix, std::string& err) {
  ix = HostIndex();
  ix.sift = true;
  ix.dist_type = kSiftL2;
  ix.dim = kSiftDim;
  // ---- objects
  std::unique_ptr<FILE, FileCloser> d(std::fopen(data_path, "rb"));
  if (!d) {
    err = std::string("Cannot open file '") + data_path + "' for reading";
    return NMSG_ERR_BAD_FILE;
  }
  const int64_t dsize = file_size(d.get());
  uint64_t qty = 0;
  if (dsize < 8 || !rd(d.get(), qty)) {
    err = "objects file is empty";
    return NMSG_ERR_BAD_FILE;
  }
  if (qty > (uint64_t)(dsize - 8) / (8 + kObjectBytes) || qty > 0x7fffffffull) {
    err = "objects file: object count " + std::to_string(qty) + " does not fit the file";
    return NMSG_ERR_BAD_FILE;
  }
  try {
    ix.sift_vecs.resize(qty * kSiftDim);
    ix.sift_norms.resize(qty);
    ix.sift_ids.resize(qty);
    ix.sift_labels.resize(qty);
  } catch (const std::bad_alloc&) {
    err = "out of host memory reading the objects";
    return NMSG_ERR_OOM;
  }
  for (uint64_t i = 0; i < qty; ++i) {
    uint64_t len = 0, dlen = 0;
    int32_t id = 0, label = 0;
    if (!rd(d.get(), len) || !rd(d.get(), id) || !rd(d.get(), label) || !rd(d.get(), dlen) ||
        len != kObjectBytes || dlen != (uint64_t)kSiftRowBytes ||
        std::fread(ix.sift_vecs.data() + i * kSiftDim, 1, kSiftDim, d.get()) != (size_t)kSiftDim ||
        !rd(d.get(), ix.sift_norms[i])) {
      err = "objects file: object " + std::to_string(i) + " is not a 128-value l2sqr_sift object";
      return NMSG_ERR_BAD_FILE;
    }
    ix.sift_ids[i] = id;
    ix.sift_labels[i] = label;
  }
  // ---- graph
  std::unique_ptr<FILE, FileCloser> g(std::fopen(graph_path, "rb"));
  if (!g) {
    err = std::string("Cannot open file '") + graph_path + "' for reading";
    return NMSG_ERR_BAD_FILE;
  }
  uint32_t flag = 1, n = 0;
  if (!rd(g.get(), flag) || !rd(g.get(), n) || !rd(g.get(), ix.saved_maxlevel) || !rd(g.get(), ix.enterpoint) ||
      !rd(g.get(), ix.M) || !rd(g.get(), ix.maxM) || !rd(g.get(), ix.maxM0)) {
    err = "truncated regular index header";
    return NMSG_ERR_BAD_FILE;
  }
  if (flag != 0) {
    err = "the graph file is an optimized index; l2sqr_sift indices are saved in the regular format";
    return NMSG_ERR_BAD_FILE;
  }
  if (n != qty) {
    // the reference's message for this case (hnsw.cc:955-958)
    err = "The number of stored elements " + std::to_string(n) + " doesn't match the number of data points " +
          std::to_string(qty) + "! Did you forget to re-load data?";
    return NMSG_ERR_BAD_FILE;
  }
  ix.n = n;
  if (n == 0) return NMSG_OK;
  if (ix.enterpoint >= n) {
    err = "entry point out of range";
    return NMSG_ERR_CORRUPT_GRAPH;
  }
  const int64_t gsize = file_size(g.get());
  std::fseek(g.get(), 4 + 4 + 4 + 4 + 8 * 3, SEEK_SET);
  // per node: its level and every list, read once; lists are kept flat per node
  std::vector<uint32_t> lev(n);
  std::vector<int64_t> start(n + 1, 0);  // offset of node i's lists in `flat`
  std::vector<int32_t> flat;
  uint32_t cap0 = 0, capu = 0;
  for (uint32_t i = 0; i < n; ++i) {
    start[i] = (int64_t)flat.size();
    uint32_t level = 0;
    if (!rd(g.get(), level) || level > kMaxLevel) {
      err = "graph file: bad level at node " + std::to_string(i);
      return NMSG_ERR_BAD_FILE;
    }
    lev[i] = level;
    for (uint32_t l = 0; l <= level; ++l) {
      uint32_t cnt = 0;
      if (!rd(g.get(), cnt) || cnt > n || (int64_t)cnt * 4 > gsize) {
        err = "graph file: bad list at node " + std::to_string(i);
        return NMSG_ERR_BAD_FILE;
      }
      const size_t at = flat.size();
      flat.push_back((int32_t)cnt);
      flat.resize(at + 1 + cnt);
      if (cnt && std::fread(flat.data() + at + 1, 4, cnt, g.get()) != cnt) {
        err = "graph file is truncated";
        return NMSG_ERR_BAD_FILE;
      }
      for (uint32_t t = 0; t < cnt; ++t) {
        const int32_t f = flat[at + 1 + t];
        if (f < 0 || (uint32_t)f >= n) {  // the reference's check (hnsw.cc:982-984)
          err = "Invalid friendId = " + std::to_string(f) + " for node id: " + std::to_string(i);
          return NMSG_ERR_CORRUPT_GRAPH;
        }
      }
      if (l == 0)
        cap0 = std::max(cap0, cnt);
      else
        capu = std::max(capu, cnt);
    }
  }
  start[n] = (int64_t)flat.size();
  if (cap0 > kMaxList0) {
    err = "level-0 lists longer than 100 are not supported by the B200 engine";
    return NMSG_ERR_UNSUPPORTED;
  }
  ix.cap0 = cap0;
  ix.capu = capu;
  ix.level.assign(n, 0);
  ix.up_off.assign(n, -1);
  ix.sift_l0.assign((size_t)n * (cap0 + 1), 0);
  for (uint32_t i = 0; i < n; ++i) {
    ix.level[i] = (int32_t)lev[i];
    const int32_t* p = flat.data() + start[i];
    std::memcpy(ix.sift_l0.data() + (size_t)i * (cap0 + 1), p, 4 * (1 + p[0]));
    p += 1 + p[0];
    if (lev[i] == 0) continue;
    ix.up_off[i] = (int64_t)ix.up_links.size();
    for (uint32_t l = 1; l <= lev[i]; ++l) {
      const size_t at = ix.up_links.size();
      ix.up_links.resize(at + capu + 1, 0);
      std::memcpy(ix.up_links.data() + at, p, 4 * (1 + p[0]));
      for (int t = 1; t <= p[0]; ++t) {
        // the greedy descent reads the level-l list of every node it moves to
        if (lev[p[t]] < l) {
          err = "upper-level neighbour " + std::to_string(p[t]) + " of node " + std::to_string(i) +
                " does not exist at level " + std::to_string(l);
          return NMSG_ERR_CORRUPT_GRAPH;
        }
      }
      p += 1 + p[0];
    }
  }
  // the generic search starts at the entry point's own level (hnsw.cc:1183)
  ix.maxlevel = (int32_t)lev[ix.enterpoint];
  return NMSG_OK;
}

int write_sift_index(const char* graph_path, const char* data_path, const HostIndex& ix, std::string& err) {
  std::unique_ptr<FILE, FileCloser> g(std::fopen(graph_path, "wb"));
  if (!g) {
    err = std::string("Cannot open file '") + graph_path + "' for writing";
    return NMSG_ERR_BAD_FILE;
  }
  const uint32_t flag = 0;
  bool ok = wr(g.get(), flag) && wr(g.get(), ix.n) && wr(g.get(), ix.saved_maxlevel) && wr(g.get(), ix.enterpoint) &&
            wr(g.get(), ix.M) && wr(g.get(), ix.maxM) && wr(g.get(), ix.maxM0);
  for (uint32_t i = 0; ok && i < ix.n; ++i) {
    const uint32_t level = (uint32_t)ix.level[i];
    ok = wr(g.get(), level);
    const int32_t* l0 = ix.sift_l0.data() + (size_t)i * (ix.cap0 + 1);
    ok = ok && std::fwrite(l0, 4, 1 + l0[0], g.get()) == (size_t)(1 + l0[0]);
    for (uint32_t l = 1; ok && l <= level; ++l) {
      const int32_t* u = ix.up_links.data() + ix.up_off[i] + (int64_t)(ix.capu + 1) * (l - 1);
      ok = std::fwrite(u, 4, 1 + u[0], g.get()) == (size_t)(1 + u[0]);
    }
  }
  if (!ok) {
    err = std::string("write to '") + graph_path + "' failed";
    return NMSG_ERR_BAD_FILE;
  }
  std::unique_ptr<FILE, FileCloser> d(std::fopen(data_path, "wb"));
  if (!d) {
    err = std::string("Cannot open file '") + data_path + "' for writing";
    return NMSG_ERR_BAD_FILE;
  }
  const uint64_t qty = ix.n, len = kObjectBytes, dlen = kSiftRowBytes;
  ok = wr(d.get(), qty);
  for (uint64_t i = 0; ok && i < qty; ++i) {
    ok = wr(d.get(), len) && wr(d.get(), ix.sift_ids[i]) && wr(d.get(), ix.sift_labels[i]) && wr(d.get(), dlen) &&
         std::fwrite(ix.sift_vecs.data() + i * kSiftDim, 1, kSiftDim, d.get()) == (size_t)kSiftDim &&
         wr(d.get(), ix.sift_norms[i]);
  }
  if (!ok) {
    err = std::string("write to '") + data_path + "' failed";
    return NMSG_ERR_BAD_FILE;
  }
  return NMSG_OK;
}

}  // namespace nmsg
