// Reader, validator and writer of NMSLIB's optimized HNSW index file.
//
// Format: similarity_search/src/method/hnsw.cc:774-806 (SaveOptimizedIndex) and :1025-1074
// (LoadOptimizedIndex); the per-node row is packed at hnsw.cc:353-465. An empty index is saved
// by the reference in the regular format (flag 0, hnsw.cc:808-840) with zero elements; that case
// is accepted as an empty index. Regular (non-optimized) files with elements are outside the
// B200 engine (they need the separately stored data objects) and are reported as unsupported.
//
// The reference trusts the optimized file; this reader validates every count and neighbour id
// before anything reaches the device, so a corrupt file becomes an error, never a device fault.
#include <cstdio>
#include <cstring>
#include <memory>

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
}  // namespace

int read_index_file(const char* path, HostIndex& ix, std::string& err) {
  std::unique_ptr<FILE, FileCloser> f(std::fopen(path, "rb"));
  if (!f) {
    err = std::string("Cannot open file '") + path + "' for reading";
    return NMSG_ERR_BAD_FILE;
  }
  uint32_t flag = 0;
  if (!rd(f.get(), flag)) {
    err = "index file is empty";
    return NMSG_ERR_BAD_FILE;
  }
  if (flag == 0) {
    uint32_t n = 0;
    if (!rd(f.get(), n)) {
      err = "truncated regular index header";
      return NMSG_ERR_BAD_FILE;
    }
    if (n != 0) {
      err = "regular (non-optimized) HNSW index files are not supported by the B200 engine; "
            "save the index with the optimized layout (skip_optimized_index=0)";
      return NMSG_ERR_UNSUPPORTED;
    }
    ix = HostIndex();
    ix.empty_regular = true;
    return NMSG_OK;
  }
  if (flag != 1) {
    err = "unknown index flag " + std::to_string(flag);
    return NMSG_ERR_BAD_FILE;
  }
  bool ok = rd(f.get(), ix.n) && rd(f.get(), ix.mem_per_obj) && rd(f.get(), ix.off_level0) &&
            rd(f.get(), ix.off_data) && rd(f.get(), ix.maxlevel) && rd(f.get(), ix.enterpoint) &&
            rd(f.get(), ix.maxM) && rd(f.get(), ix.maxM0) && rd(f.get(), ix.dist_type) &&
            rd(f.get(), ix.search_method);
  if (!ok) {
    err = "truncated optimized index header";
    return NMSG_ERR_BAD_FILE;
  }
  if (ix.mem_per_obj == 0 || ix.mem_per_obj > (1ull << 24) || ix.maxM > 4096 || ix.maxM0 > 4096) {
    err = "implausible index header";
    return NMSG_ERR_BAD_FILE;
  }
  const uint64_t total = (uint64_t)ix.n * ix.mem_per_obj;
  try {
    ix.level0.resize(total);
    ix.link_bytes.assign(ix.n, 0);
    ix.up_off.assign(ix.n, -1);
    ix.level.assign(ix.n, 0);
  } catch (const std::bad_alloc&) {
    err = "out of host memory reading the index";
    return NMSG_ERR_OOM;
  }
  if (total && std::fread(ix.level0.data(), 1, total, f.get()) != total) {
    err = "truncated level-0 block";
    return NMSG_ERR_BAD_FILE;
  }
  const uint64_t list_bytes = (ix.maxM + 1) * 4;
  for (uint32_t i = 0; i < ix.n; ++i) {
    uint32_t sz = 0;
    if (!rd(f.get(), sz)) {
      err = "truncated upper-level link lists";
      return NMSG_ERR_BAD_FILE;
    }
    ix.link_bytes[i] = sz;
    if (sz == 0) continue;
    if (sz % list_bytes != 0) {
      err = "upper-level list size of node " + std::to_string(i) + " is not a multiple of (maxM+1)*4";
      return NMSG_ERR_BAD_FILE;
    }
    ix.up_off[i] = (int64_t)ix.up_links.size();
    ix.level[i] = (int32_t)(sz / list_bytes);
    ix.up_links.resize(ix.up_links.size() + sz / 4);
    if (std::fread(ix.up_links.data() + ix.up_off[i], 1, sz, f.get()) != sz) {
      err = "truncated upper-level link list";
      return NMSG_ERR_BAD_FILE;
    }
  }
  ix.dim = (ix.off_level0 >= ix.off_data + 16) ? (int)((ix.off_level0 - ix.off_data - 16) / 4) : -1;
  return NMSG_OK;
}

int validate_index(const HostIndex& ix, std::string& err) {
  if (ix.empty_regular) return NMSG_OK;
  if (ix.dist_type < 1 || ix.dist_type > 6) {
    err = "Unknown distance function code: " + std::to_string(ix.dist_type);
    return NMSG_ERR_BAD_FILE;
  }
  if (ix.n == 0) return NMSG_OK;
  if (ix.dim <= 0 || ix.off_data != 0 || ix.mem_per_obj != ix.off_level0 + (ix.maxM0 + 1) * 4) {
    err = "inconsistent row layout in the index header";
    return NMSG_ERR_BAD_FILE;
  }
  if (ix.maxM0 > 100) {
    // SearchV1Merge switches to an in-place merge for more than 100 buffered neighbours
    // (hnsw_distfunc_opt.cc:36,254-260); the engine implements the insertion path only.
    err = "maxM0 > 100 is not supported by the B200 engine";
    return NMSG_ERR_UNSUPPORTED;
  }
  if (ix.enterpoint >= ix.n || ix.maxlevel < 0 || ix.level[ix.enterpoint] < ix.maxlevel) {
    err = "entry point or maximum level out of range";
    return NMSG_ERR_CORRUPT_GRAPH;
  }
  for (int64_t i = 0; i < ix.n; ++i) {
    uint64_t dl = 0;
    std::memcpy(&dl, ix.level0.data() + i * ix.mem_per_obj + ix.off_data + 8, 8);
    if (dl != (uint64_t)ix.dim * 4) {
      err = "object " + std::to_string(i) + " has a data length different from the index vectors";
      return NMSG_ERR_BAD_FILE;
    }
    const int32_t* l0 = ix.l0(i);
    if (l0[0] < 0 || (uint64_t)l0[0] > ix.maxM0) {
      err = "level-0 neighbour count of node " + std::to_string(i) + " exceeds maxM0";
      return NMSG_ERR_CORRUPT_GRAPH;
    }
    for (int j = 1; j <= l0[0]; ++j) {
      if (l0[j] < 0 || (uint32_t)l0[j] >= ix.n) {
        err = "level-0 neighbour id out of range at node " + std::to_string(i);
        return NMSG_ERR_CORRUPT_GRAPH;
      }
    }
    for (int lev = 1; lev <= ix.level[i]; ++lev) {
      const int32_t* lst = ix.up_links.data() + ix.up_off[i] + (ix.maxM + 1) * (lev - 1);
      if (lst[0] < 0 || (uint64_t)lst[0] > ix.maxM) {
        err = "upper-level neighbour count of node " + std::to_string(i) + " exceeds maxM";
        return NMSG_ERR_CORRUPT_GRAPH;
      }
      for (int j = 1; j <= lst[0]; ++j) {
        // the greedy descent reads the level-`lev` list of every node it moves to
        if (lst[j] < 0 || (uint32_t)lst[j] >= ix.n || ix.level[lst[j]] < lev) {
          err = "upper-level neighbour id out of range at node " + std::to_string(i);
          return NMSG_ERR_CORRUPT_GRAPH;
        }
      }
    }
  }
  return NMSG_OK;
}

int write_index_file(const char* path, const HostIndex& ix, std::string& err) {
  std::unique_ptr<FILE, FileCloser> f(std::fopen(path, "wb"));
  if (!f) {
    err = std::string("Cannot open file '") + path + "' for writing";
    return NMSG_ERR_BAD_FILE;
  }
  bool ok = true;
  if (ix.empty_regular) {
    // regular-format header of an empty index: flag 0, then N maxlevel ep M maxM maxM0
    uint32_t zero = 0;
    int32_t maxlevel = 0, ep = 0;
    uint64_t m = 0;
    ok = wr(f.get(), zero) && wr(f.get(), zero) && wr(f.get(), maxlevel) && wr(f.get(), ep) &&
         wr(f.get(), m) && wr(f.get(), m) && wr(f.get(), m);
  } else {
    uint32_t flag = 1;
    ok = wr(f.get(), flag) && wr(f.get(), ix.n) && wr(f.get(), ix.mem_per_obj) && wr(f.get(), ix.off_level0) &&
         wr(f.get(), ix.off_data) && wr(f.get(), ix.maxlevel) && wr(f.get(), ix.enterpoint) &&
         wr(f.get(), ix.maxM) && wr(f.get(), ix.maxM0) && wr(f.get(), ix.dist_type) &&
         wr(f.get(), ix.search_method);
    ok = ok && std::fwrite(ix.level0.data(), 1, ix.level0.size(), f.get()) == ix.level0.size();
    for (uint32_t i = 0; ok && i < ix.n; ++i) {
      uint32_t sz = ix.link_bytes[i];
      ok = wr(f.get(), sz);
      if (ok && sz) ok = std::fwrite(ix.up_links.data() + ix.up_off[i], 1, sz, f.get()) == sz;
    }
  }
  if (!ok) {
    err = std::string("write to '") + path + "' failed";
    return NMSG_ERR_BAD_FILE;
  }
  return NMSG_OK;
}

}  // namespace nmsg
