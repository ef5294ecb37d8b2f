// The query server: NMSLIB's Thrift QueryService (query_server/protocol.thrift) over TCP in front of
// a loaded index, so clients of the reference's server (query_server/cpp_client_server/
// QueryService_server.cpp, the Java and Python clients) can talk to the B200 engine unchanged.
//
// Wire format: Thrift's binary protocol over a plain (buffered, unframed) TCP stream, as the
// reference's server uses (TBinaryProtocolFactory + TBufferedTransportFactory over TServerSocket).
// This file implements that protocol itself (the Thrift library is not a dependency):
//   message  = i32 (0x80010000 | type) | string name | i32 seqid      (strict form; the old
//              non-strict form, string name | i8 type | i32 seqid, is accepted on input)
//   struct   = { i8 field type | i16 field id | value }* | i8 0
//   string   = i32 length | bytes; list = i8 element type | i32 count | elements; big-endian ints.
// Methods (QueryService_server.cpp:150-460):
//   setQueryTimeParams(string)  waits for running queries, then sets efSearch / algoType
//   knnQuery(k, queryObj, retExternId, retObj) -> list<ReplyEntry>, ascending distance
//   knnQueryBatch(k, list<queryObj>, retExternId, retObj, numThreads) -> list<list<ReplyEntry>>
//   rangeQuery(...)             QueryException "Range search is not supported!" (hnsw.cc:712-715)
//   getDistance(obj1, obj2)     the space's distance of two objects, computed on the GPU
// Query objects are the space's text form (space_vector.cc:53-75, read_data.h): an optional
// "label:N" prefix, then numbers separated by white space, ',' or ':'; l2sqr_sift values must be
// integers in 0..255. Errors reach the client as QueryException{message}, unknown methods as a
// TApplicationException, as the generated processor would send them.
//
// Searches go through the engine's serving loop (nmsg_server_*: continuous batching of
// concurrent requests onto lanes) when it can take them (float index, V1Merge, k within its
// limit), else through nmsg_knn_batch / nmsg_knn_batch_u8 directly; both run the search on the GPU.
#include <arpa/inet.h>
#include <netinet/in.h>
#include <netinet/tcp.h>
#include <sys/socket.h>
#include <unistd.h>

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cctype>
#include <cerrno>
#include <chrono>
#include <cstdio>
#include <list>
#include <memory>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <iomanip>
#include <limits>
#include <mutex>
#include <shared_mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "engine.h"
#include "handle.h"
#include "../../include/nmslib_b200.h"

namespace nmsg {
namespace {

// ---------------------------------------------------------------- binary protocol
enum TType : int8_t { T_STOP = 0, T_BOOL = 2, T_BYTE = 3, T_DOUBLE = 4, T_I16 = 6, T_I32 = 8, T_I64 = 10,
                      T_STRING = 11, T_STRUCT = 12, T_MAP = 13, T_SET = 14, T_LIST = 15 };
enum MsgType : int32_t { M_CALL = 1, M_REPLY = 2, M_EXCEPTION = 3, M_ONEWAY = 4 };
constexpr uint32_t kVersion1 = 0x80010000u;
constexpr int32_t kMaxString = 256 << 20;  // refuse absurd lengths instead of allocating them
constexpr int32_t kMaxList = 1 << 24;

struct ProtocolError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// A buffered socket stream (the TBufferedTransport of the reference's server).
class Stream {
 public:
  explicit Stream(int fd) : fd_(fd) {}
  void read(void* dst, size_t n) {
    char* p = static_cast<char*>(dst);
    while (n) {
      if (rpos_ == rlen_) fill();
      const size_t m = std::min(n, rlen_ - rpos_);
      std::memcpy(p, rbuf_ + rpos_, m);
      rpos_ += m;
      p += m;
      n -= m;
    }
  }
  void write(const void* src, size_t n) {
    const char* p = static_cast<const char*>(src);
    wbuf_.insert(wbuf_.end(), p, p + n);
  }
  void flush() {
    size_t off = 0;
    while (off < wbuf_.size()) {
      const ssize_t w = ::send(fd_, wbuf_.data() + off, wbuf_.size() - off, MSG_NOSIGNAL);
      if (w <= 0) {
        if (w < 0 && errno == EINTR) continue;
        throw ProtocolError("connection closed while writing");
      }
      off += (size_t)w;
    }
    wbuf_.clear();
  }

 private:
  void fill() {
    while (true) {
      const ssize_t r = ::recv(fd_, rbuf_, sizeof(rbuf_), 0);
      if (r > 0) {
        rpos_ = 0;
        rlen_ = (size_t)r;
        return;
      }
      if (r < 0 && errno == EINTR) continue;
      throw ProtocolError("connection closed");
    }
  }
  int fd_;
  char rbuf_[1 << 16];
  size_t rpos_ = 0, rlen_ = 0;
  std::vector<char> wbuf_;
};

class Proto {
 public:
  explicit Proto(Stream& s) : s_(s) {}
  // readers
  int8_t i8() {
    int8_t v;
    s_.read(&v, 1);
    return v;
  }
  int16_t i16() {
    uint16_t v;
    s_.read(&v, 2);
    return (int16_t)ntohs(v);
  }
  int32_t i32() {
    uint32_t v;
    s_.read(&v, 4);
    return (int32_t)ntohl(v);
  }
  int64_t i64() {
    const uint64_t hi = (uint32_t)i32(), lo = (uint32_t)i32();
    return (int64_t)((hi << 32) | lo);
  }
  double dbl() {
    const int64_t b = i64();
    double d;
    std::memcpy(&d, &b, 8);
    return d;
  }
  bool boolean() { return i8() != 0; }
  std::string str() {
    const int32_t n = i32();
    if (n < 0 || n > kMaxString) throw ProtocolError("bad string length");
    std::string v((size_t)n, '\0');
    if (n) s_.read(&v[0], (size_t)n);
    return v;
  }
  void skip(int8_t t, int depth = 0) {
    if (depth > 64) throw ProtocolError("nesting too deep");
    switch (t) {
      case T_BOOL:
      case T_BYTE: i8(); break;
      case T_I16: i16(); break;
      case T_I32: i32(); break;
      case T_DOUBLE:
      case T_I64: i64(); break;
      case T_STRING: str(); break;
      case T_STRUCT:
        while (true) {
          const int8_t ft = i8();
          if (ft == T_STOP) break;
          i16();
          skip(ft, depth + 1);
        }
        break;
      case T_MAP: {
        const int8_t kt = i8(), vt = i8();
        const int32_t n = i32();
        if (n < 0 || n > kMaxList) throw ProtocolError("bad map size");
        for (int32_t i = 0; i < n; ++i) {
          skip(kt, depth + 1);
          skip(vt, depth + 1);
        }
        break;
      }
      case T_SET:
      case T_LIST: {
        const int8_t et = i8();
        const int32_t n = i32();
        if (n < 0 || n > kMaxList) throw ProtocolError("bad list size");
        for (int32_t i = 0; i < n; ++i) skip(et, depth + 1);
        break;
      }
      default: throw ProtocolError("unknown field type");
    }
  }
  // writers
  void w8(int8_t v) { s_.write(&v, 1); }
  void w16(int16_t v) {
    const uint16_t b = htons((uint16_t)v);
    s_.write(&b, 2);
  }
  void w32(int32_t v) {
    const uint32_t b = htonl((uint32_t)v);
    s_.write(&b, 4);
  }
  void w64(int64_t v) {
    w32((int32_t)((uint64_t)v >> 32));
    w32((int32_t)(uint64_t)v);
  }
  void wdbl(double d) {
    int64_t b;
    std::memcpy(&b, &d, 8);
    w64(b);
  }
  void wstr(const std::string& v) {
    w32((int32_t)v.size());
    s_.write(v.data(), v.size());
  }
  void field(int8_t t, int16_t id) {
    w8(t);
    w16(id);
  }
  void stop() { w8(T_STOP); }
  void msg_begin(const std::string& name, int32_t type, int32_t seqid) {
    w32((int32_t)(kVersion1 | (uint32_t)type));
    wstr(name);
    w32(seqid);
  }
  void flush() { s_.flush(); }

 private:
  Stream& s_;
};

// ---------------------------------------------------------------- query objects
struct ReplyEntry {
  int32_t id;
  double dist;
  bool has_extern = false, has_obj = false;
  std::string extern_id, obj;
};

struct QueryError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// The text form of a dense object (VectorSpace::ReadVec, space_vector.cc:122-138, with
// Object::extractLabel and ReadVecDataEfficiently): an optional "label:N" prefix, then strtof
// over the rest with ',' and ':' read as white space.
std::vector<float> parse_vector(std::string s) {
  static const std::string kLabel = "label:";
  if (s.size() > kLabel.size() + 1 && s.compare(0, kLabel.size(), kLabel) == 0) {
    size_t p = kLabel.size();
    while (p < s.size() && !std::isspace((unsigned char)s[p])) ++p;
    if (p < s.size()) {
      const std::string num = s.substr(kLabel.size(), p - kLabel.size());
      char* end = nullptr;
      std::strtol(num.c_str(), &end, 10);
      if (num.empty() || *end != '\0') throw QueryError("Cannot extract label from the file line: '" + s + "'");
      s = s.substr(p);
    }
  }
  for (char& c : s)
    if (c == ',' || c == ':') c = ' ';
  std::vector<float> v;
  const char* ptr = s.c_str();
  char* end = nullptr;
  errno = 0;
  for (float val = std::strtof(ptr, &end); ptr != end; val = std::strtof(ptr, &end)) {
    ptr = end;
    if (errno == ERANGE) throw QueryError("Failed to parse the line: '" + s + "'");
    v.push_back(val);
  }
  if (errno == ERANGE) throw QueryError("Failed to parse the line: '" + s + "'");
  return v;
}

// Dense float object -> text (VectorSpace::CreateStrFromObj, space_vector.cc:96-108).
std::string vector_text(const float* p, int n) {
  std::ostringstream out;
  for (int i = 0; i < n; ++i) {
    if (i) out << " ";
    out.unsetf(std::ios_base::floatfield);
    out << std::setprecision(std::numeric_limits<float>::max_digits10) << std::noshowpoint << p[i];
  }
  return out.str();
}

// l2sqr_sift object -> text (SpaceL2SqrSift::CreateStrFromObj, space_l2sqr_sift.cc:75-85): the
// reference streams each uint8_t value as a character, so the bytes themselves, space-separated.
std::string sift_text(const uint8_t* p) {
  std::string out;
  for (int i = 0; i < kSiftDim; ++i) {
    if (i) out += ' ';
    out += (char)p[i];
  }
  return out;
}

// ---------------------------------------------------------------- the distance of two objects
// getDistance: the space's own distance (Space::IndexTimeDistance), in double precision on the
// GPU: l2 = the Euclidean norm (the l2 space's distance is not squared), cosinesimil =
// 1 - cos clamped to [0, 2], negdotprod = -dot, l1, linf, l2sqr_sift = the squared integer norm.
__global__ void pair_distance_kernel(int space, const float* a, const float* b, int n, double* out) {
  double s0 = 0, s1 = 0, s2 = 0;
  for (int i = threadIdx.x; i < n; i += 32) {
    const double x = a[i], y = b[i];
    switch (space) {
      case NMSG_SPACE_L2:
      case NMSG_SPACE_L2SQR_SIFT: s0 += (x - y) * (x - y); break;
      case NMSG_SPACE_L1: s0 += fabs(x - y); break;
      case NMSG_SPACE_LINF: s0 = fmax(s0, fabs(x - y)); break;
      default:
        s0 += x * y;
        s1 += x * x;
        s2 += y * y;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double t0 = __shfl_xor_sync(0xffffffffu, s0, o);
    s0 = space == NMSG_SPACE_LINF ? fmax(s0, t0) : s0 + t0;
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if (threadIdx.x == 0) {
    double r = s0;
    if (space == NMSG_SPACE_L2) r = sqrt(s0);
    if (space == NMSG_SPACE_NEGDOT) r = -s0;
    if (space == NMSG_SPACE_COSINE) {
      const double nn = sqrt(s1) * sqrt(s2);
      const double c = nn > 0 ? s0 / nn : 0.0;
      r = fmax(0.0, 1.0 - fmin(1.0, fmax(-1.0, c)));
    }
    *out = r;
  }
}

// ---------------------------------------------------------------- the service
struct Service {
  nmsg_index* h = nullptr;
  nmsg_server* srv = nullptr;  // continuous batching (float indices), or null
  int srv_max_batch = 0, srv_max_k = 0;
  bool debug = false;
  std::shared_mutex params_mu;  // queries share it; setQueryTimeParams takes it alone
  int ef = 20, algo = NMSG_ALGO_HYBRID;

  bool sift() const { return h->host.sift; }
  int dim() const { return h->host.dim; }

  // a request's queries, parsed and checked against the index
  std::vector<float> parse_float_query(const std::string& s) const {
    std::vector<float> v = parse_vector(s);
    if ((int)v.size() != dim())
      throw QueryError("query dimension " + std::to_string(v.size()) + " does not match the index dimension " +
                       std::to_string(dim()));
    return v;
  }
  std::vector<uint8_t> parse_sift_query(const std::string& s) const {
    const std::vector<float> f = parse_vector(s);
    if ((int)f.size() != kSiftDim)
      throw QueryError("Bug or internal error, SIFT vectors dim " + std::to_string(f.size()) + " isn't == 128");
    std::vector<uint8_t> v(kSiftDim);
    for (int i = 0; i < kSiftDim; ++i) {
      // space_l2sqr_sift.cc:117-132
      if (f[i] < 0 || f[i] > 255) throw QueryError("Out-of range integer values (for SIFT) in the line: '" + s + "'");
      v[i] = (uint8_t)f[i];
      if (std::fabs(v[i] - f[i]) > std::numeric_limits<float>::min())
        throw QueryError("Non-integer values (for SIFT) in the line: '" + s + "'");
    }
    return v;
  }

  void set_params(const std::string& desc) {
    int new_ef = 20, new_algo = NMSG_ALGO_HYBRID;
    bool has_ef = false, has_efs = false;
    std::stringstream ss(desc);
    std::string item;
    while (!desc.empty() && std::getline(ss, item, ',')) {
      const size_t eq = item.find('=');
      if (eq == std::string::npos) throw QueryError("Wrong format of the parameter: '" + item + "'");
      std::string key = item.substr(0, eq), val = item.substr(eq + 1);
      auto trim = [](std::string& x) {
        while (!x.empty() && std::isspace((unsigned char)x.back())) x.pop_back();
        size_t i = 0;
        while (i < x.size() && std::isspace((unsigned char)x[i])) ++i;
        x = x.substr(i);
      };
      trim(key);
      trim(val);
      auto as_int = [&](const std::string& k, const std::string& v) {
        char* end = nullptr;
        const long r = std::strtol(v.c_str(), &end, 10);
        if (v.empty() || *end != '\0')
          throw QueryError("Failed to convert value '" + v + "' of parameter '" + k + "' to an integer");
        return (int)r;
      };
      if (key == "ef" || key == "efSearch") {
        (key == "ef" ? has_ef : has_efs) = true;
        new_ef = as_int(key, val);
      } else if (key == "algoType") {
        std::string a = val;
        for (char& c : a) c = (char)std::tolower((unsigned char)c);
        if (a == "old")
          new_algo = NMSG_ALGO_OLD;
        else if (a == "v1merge")
          new_algo = NMSG_ALGO_V1MERGE;
        else if (a == "hybrid")
          new_algo = NMSG_ALGO_HYBRID;
        else
          throw QueryError("algoType should be one of the following: old, v1merge");
      } else if (key == "searchMethod") {
        as_int(key, val);
      } else {
        throw QueryError("Unknown parameters found!");
      }
    }
    if (has_ef && has_efs)
      throw QueryError("The user shouldn't specify parameters ef and efSearch at the same time (they are synonyms)");
    std::unique_lock<std::shared_mutex> lk(params_mu);  // waits for the queries in flight
    const int rc = nmsg_set_query_params(h, new_ef, new_algo);
    if (rc != NMSG_OK) throw QueryError(nmsg_last_error());
    ef = new_ef;
    algo = new_algo;
  }

  // k-NN of `nq` queries (float or uint8 rows); results ascending, `counts` per query
  void search(const void* q, int nq, int k, std::vector<int32_t>& ids, std::vector<float>& dists,
              std::vector<int32_t>& counts) {
    if (k < 1) throw QueryError("k must be at least 1");
    ids.assign((size_t)nq * k, -1);
    dists.assign((size_t)nq * k, 0.0f);
    counts.assign(nq, 0);
    if (nq == 0) return;
    std::shared_lock<std::shared_mutex> lk(params_mu);
    const bool via_server = srv && !sift() && algo != NMSG_ALGO_OLD && ef < 1000 && k <= srv_max_k;
    if (via_server) {
      // every chunk of the request is admitted at once; the lanes overlap them with other requests
      std::vector<int64_t> rid;
      for (int s = 0; s < nq; s += srv_max_batch) {
        const int n = std::min(srv_max_batch, nq - s);
        int64_t id = 0;
        const int rc = nmsg_server_submit(srv, static_cast<const float*>(q) + (size_t)s * dim(), n, k, ef, &id);
        if (rc != NMSG_OK) throw QueryError(nmsg_last_error());
        rid.push_back(id);
      }
      int idx = 0;
      for (int s = 0; s < nq; s += srv_max_batch, ++idx) {
        double lat = 0;
        const int rc = nmsg_server_wait(srv, rid[idx], ids.data() + (size_t)s * k, dists.data() + (size_t)s * k,
                                        counts.data() + s, &lat);
        if (rc != NMSG_OK) throw QueryError(nmsg_last_error());
      }
      return;
    }
    int rc;
    if (sift()) {
      std::vector<int32_t> di((size_t)nq * k);
      rc = nmsg_knn_batch_u8(h, static_cast<const uint8_t*>(q), nq, kSiftDim, k, nullptr, nullptr, k, ids.data(),
                             di.data(), counts.data(), nullptr, 0, nullptr);
      for (size_t i = 0; i < di.size(); ++i) dists[i] = (float)di[i];
    } else {
      rc = nmsg_knn_batch(h, static_cast<const float*>(q), nq, dim(), k, nullptr, nullptr, k, ids.data(), dists.data(),
                          counts.data(), nullptr, 0, nullptr);
    }
    if (rc != NMSG_OK) throw QueryError(nmsg_last_error());
  }

  // The stored object with external id `id` (ids of a loaded index are its node order when
  // created with default ids; otherwise found by search of the id column).
  int64_t node_of(int32_t id) const {
    const HostIndex& hi = h->host;
    if (hi.sift) {
      if (id >= 0 && id < (int32_t)hi.n && hi.sift_ids[id] == id) return id;
      for (int64_t i = 0; i < hi.n; ++i)
        if (hi.sift_ids[i] == id) return i;
      return -1;
    }
    if (id >= 0 && id < (int32_t)hi.n && hi.ext_id(id) == id) return id;
    for (int64_t i = 0; i < hi.n; ++i)
      if (hi.ext_id(i) == id) return i;
    return -1;
  }

  std::vector<ReplyEntry> entries(const int32_t* ids, const float* d, int cnt, bool ret_extern, bool ret_obj) const {
    std::vector<ReplyEntry> out(cnt);
    for (int i = 0; i < cnt; ++i) {
      ReplyEntry& e = out[i];
      e.id = ids[i];
      e.dist = (double)d[i];
      if (ret_extern || ret_obj) {
        // the engine's index files carry integer object ids; the external id is their decimal form
        e.has_extern = true;
        e.extern_id = std::to_string(ids[i]);
      }
      if (ret_obj) {
        const int64_t node = node_of(ids[i]);
        e.has_obj = true;
        if (node >= 0)
          e.obj = h->host.sift ? sift_text(h->host.sift_vecs.data() + node * kSiftDim)
                               : vector_text(h->host.vec(node), dim());
      }
    }
    return out;
  }

  double distance(const std::string& s1, const std::string& s2) {
    std::vector<float> a, b;
    if (sift()) {
      const std::vector<uint8_t> x = parse_sift_query(s1), y = parse_sift_query(s2);
      a.assign(x.begin(), x.end());
      b.assign(y.begin(), y.end());
    } else {
      a = parse_vector(s1);
      b = parse_vector(s2);
      if (a.size() != b.size()) throw QueryError("the two objects have different dimensions");
    }
    DeviceGuard g(h->device);
    float* d = nullptr;
    double* r = nullptr;
    double res = 0;
    cudaError_t e = cudaMalloc(&d, 8 * std::max<size_t>(1, a.size()));
    if (e == cudaSuccess) e = cudaMalloc(&r, 8);
    if (e == cudaSuccess) e = cudaMemcpy(d, a.data(), 4 * a.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + a.size(), b.data(), 4 * b.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
      pair_distance_kernel<<<1, 32>>>(h->space, d, d + a.size(), (int)a.size(), r);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(&res, r, 8, cudaMemcpyDeviceToHost);
    if (d) cudaFree(d);
    if (r) cudaFree(r);
    if (e != cudaSuccess) throw QueryError(std::string("getDistance: ") + cudaGetErrorString(e));
    return res;
  }
};

void write_entry(Proto& p, const ReplyEntry& e) {
  p.field(T_I32, 1);
  p.w32(e.id);
  p.field(T_DOUBLE, 2);
  p.wdbl(e.dist);
  if (e.has_extern) {
    p.field(T_STRING, 3);
    p.wstr(e.extern_id);
  }
  if (e.has_obj) {
    p.field(T_STRING, 4);
    p.wstr(e.obj);
  }
  p.stop();
}

void write_entry_list(Proto& p, const std::vector<ReplyEntry>& v) {
  p.w8(T_STRUCT);
  p.w32((int32_t)v.size());
  for (const ReplyEntry& e : v) write_entry(p, e);
}

// Reads one call, runs it and writes the reply. Returns false when the connection should close.
bool serve_one(Service& svc, Proto& p) {
  std::string name;
  int32_t type, seqid;
  const int32_t first = p.i32();
  if (first < 0) {
    if (((uint32_t)first & 0xffff0000u) != kVersion1) throw ProtocolError("bad protocol version");
    type = first & 0xff;
    name = p.str();
    seqid = p.i32();
  } else {
    if (first > kMaxString) throw ProtocolError("bad method name length");
    name.assign((size_t)first, '\0');
    for (int32_t i = 0; i < first; ++i) name[i] = (char)p.i8();
    type = p.i8();
    seqid = p.i32();
  }
  if (type != M_CALL && type != M_ONEWAY) throw ProtocolError("expected a call");
  // arguments, by field id
  int32_t k = 0;
  [[maybe_unused]] int32_t num_threads = 0;  // the GPU takes the whole batch at once
  [[maybe_unused]] double r = 0;             // range search is refused
  bool ret_extern = false, ret_obj = false;
  std::string s1, s2;
  std::vector<std::string> objs;
  const bool known = name == "setQueryTimeParams" || name == "knnQuery" || name == "knnQueryBatch" ||
                     name == "rangeQuery" || name == "getDistance";
  while (true) {
    const int8_t ft = p.i8();
    if (ft == T_STOP) break;
    const int16_t fid = p.i16();
    bool used = false;
    if (known) {
      if (name == "setQueryTimeParams" && fid == 1 && ft == T_STRING) {
        s1 = p.str();
        used = true;
      } else if ((name == "knnQuery" || name == "knnQueryBatch") && fid == 1 && ft == T_I32) {
        k = p.i32();
        used = true;
      } else if (name == "rangeQuery" && fid == 1 && ft == T_DOUBLE) {
        r = p.dbl();
        used = true;
      } else if ((name == "knnQuery" || name == "rangeQuery") && fid == 2 && ft == T_STRING) {
        s1 = p.str();
        used = true;
      } else if (name == "knnQueryBatch" && fid == 2 && ft == T_LIST) {
        const int8_t et = p.i8();
        const int32_t n = p.i32();
        if (et != T_STRING || n < 0 || n > kMaxList) throw ProtocolError("bad query list");
        objs.resize(n);
        for (int32_t i = 0; i < n; ++i) objs[i] = p.str();
        used = true;
      } else if (name != "getDistance" && name != "setQueryTimeParams" && fid == 3 && ft == T_BOOL) {
        ret_extern = p.boolean();
        used = true;
      } else if (name != "getDistance" && name != "setQueryTimeParams" && fid == 4 && ft == T_BOOL) {
        ret_obj = p.boolean();
        used = true;
      } else if (name == "knnQueryBatch" && fid == 5 && ft == T_I32) {
        num_threads = p.i32();
        used = true;
      } else if (name == "getDistance" && (fid == 1 || fid == 2) && ft == T_STRING) {
        (fid == 1 ? s1 : s2) = p.str();
        used = true;
      }
    }
    if (!used) p.skip(ft);
  }
  if (!known) {
    // TApplicationException{1: message, 2: type UNKNOWN_METHOD (1)}
    p.msg_begin(name, M_EXCEPTION, seqid);
    p.field(T_STRING, 1);
    p.wstr("Invalid method name: '" + name + "'");
    p.field(T_I32, 2);
    p.w32(1);
    p.stop();
    p.flush();
    return true;
  }
  // run it: the result struct's field 0 is the success value, field 1 the QueryException
  std::string error;
  std::vector<ReplyEntry> one;
  std::vector<std::vector<ReplyEntry>> many;
  double dist = 0;
  try {
    if (name == "setQueryTimeParams") {
      if (svc.debug) std::fprintf(stderr, "[query server] setQueryTimeParams(%s)\n", s1.c_str());
      svc.set_params(s1);
    } else if (name == "rangeQuery") {
      throw QueryError("Range search is not supported!");
    } else if (name == "getDistance") {
      dist = svc.distance(s1, s2);
    } else {
      const bool batch = name == "knnQueryBatch";
      if (!batch) objs.assign(1, s1);
      const int nq = (int)objs.size();
      std::vector<int32_t> ids, counts;
      std::vector<float> dists;
      if (svc.sift()) {
        std::vector<uint8_t> q((size_t)nq * kSiftDim);
        for (int i = 0; i < nq; ++i) {
          const std::vector<uint8_t> v = svc.parse_sift_query(objs[i]);
          std::memcpy(q.data() + (size_t)i * kSiftDim, v.data(), kSiftDim);
        }
        svc.search(q.data(), nq, k, ids, dists, counts);
      } else {
        std::vector<float> q((size_t)nq * svc.dim());
        for (int i = 0; i < nq; ++i) {
          const std::vector<float> v = svc.parse_float_query(objs[i]);
          std::memcpy(q.data() + (size_t)i * svc.dim(), v.data(), 4 * v.size());
        }
        svc.search(q.data(), nq, k, ids, dists, counts);
      }
      if (svc.debug) std::fprintf(stderr, "[query server] %s: %d queries, k=%d\n", name.c_str(), nq, k);
      if (batch) {
        many.resize(nq);
        for (int i = 0; i < nq; ++i)
          many[i] = svc.entries(ids.data() + (size_t)i * k, dists.data() + (size_t)i * k, counts[i], ret_extern,
                                ret_obj);
      } else {
        one = svc.entries(ids.data(), dists.data(), counts[0], ret_extern, ret_obj);
      }
    }
  } catch (const QueryError& e) {
    error = e.what();
  } catch (const std::exception& e) {
    error = e.what();
  }
  if (type == M_ONEWAY) return true;
  p.msg_begin(name, M_REPLY, seqid);
  if (!error.empty()) {
    p.field(T_STRUCT, 1);  // QueryException err
    p.field(T_STRING, 1);
    p.wstr(error);
    p.stop();
  } else if (name == "knnQuery") {
    p.field(T_LIST, 0);
    write_entry_list(p, one);
  } else if (name == "knnQueryBatch") {
    p.field(T_LIST, 0);
    p.w8(T_LIST);
    p.w32((int32_t)many.size());
    for (const auto& v : many) write_entry_list(p, v);
  } else if (name == "getDistance") {
    p.field(T_DOUBLE, 0);
    p.wdbl(dist);
  }
  p.stop();
  p.flush();
  return true;
}

}  // namespace
}  // namespace nmsg

using namespace nmsg;

struct QsConn {  // one client connection and the thread serving it
  int fd = -1;
  std::thread t;
  std::atomic<bool> done{false};
};

struct nmsg_query_server {
  Service svc;
  int listen_fd = -1;
  int port = 0;
  int max_conns = 8;
  std::atomic<bool> stopping{false};
  std::thread acceptor;
  std::mutex mu;
  std::list<std::unique_ptr<QsConn>> conns;
  std::atomic<int> active{0};
};

namespace {

void connection_loop(nmsg_query_server* s, QsConn* c) {
  try {
    Stream st(c->fd);
    Proto p(st);
    while (!s->stopping.load() && serve_one(s->svc, p)) {
    }
  } catch (const std::exception&) {
    // a closed or malformed connection ends quietly, as TThreadPoolServer does
  }
  s->active.fetch_sub(1);
  c->done.store(true);
}

// Joins and forgets the connections that have ended (mu held).
void reap(nmsg_query_server* s) {
  for (auto it = s->conns.begin(); it != s->conns.end();) {
    if ((*it)->done.load()) {
      if ((*it)->t.joinable()) (*it)->t.join();
      ::close((*it)->fd);
      it = s->conns.erase(it);
    } else {
      ++it;
    }
  }
}

void accept_loop(nmsg_query_server* s) {
  while (!s->stopping.load()) {
    sockaddr_in addr{};
    socklen_t len = sizeof(addr);
    const int fd = ::accept(s->listen_fd, reinterpret_cast<sockaddr*>(&addr), &len);
    if (fd < 0) {
      if (s->stopping.load()) break;
      if (errno == EINTR || errno == ECONNABORTED) continue;
      std::this_thread::sleep_for(std::chrono::milliseconds(10));
      continue;
    }
    // at most max_conns connections are served at once (the reference's thread pool size)
    while (s->active.load() >= s->max_conns && !s->stopping.load())
      std::this_thread::sleep_for(std::chrono::milliseconds(1));
    if (s->stopping.load()) {
      ::close(fd);
      break;
    }
    const int one = 1;
    setsockopt(fd, IPPROTO_TCP, TCP_NODELAY, &one, sizeof(one));
    s->active.fetch_add(1);
    std::lock_guard<std::mutex> lk(s->mu);
    reap(s);
    auto c = std::make_unique<QsConn>();
    c->fd = fd;
    QsConn* raw = c.get();
    s->conns.push_back(std::move(c));
    raw->t = std::thread(connection_loop, s, raw);
  }
}

int qs_fail(int code, const std::string& msg) {
  set_last_error(msg);
  return code;
}

}  // namespace

extern "C" {

NMSG_API int nmsg_query_server_start(nmsg_index* index, int port, int max_connections, int debug,
                                     nmsg_query_server** out) {
  if (!index || !out) return qs_fail(NMSG_ERR_BAD_ARG, "null argument");
  if (port < 0 || port > 65535 || max_connections < 1) return qs_fail(NMSG_ERR_BAD_ARG, "bad port or connection count");
  *out = nullptr;
  auto* s = new nmsg_query_server();
  s->svc.h = index;
  s->svc.debug = debug != 0;
  s->svc.ef = index->ef;
  s->svc.algo = index->algo;
  s->max_conns = max_connections;
  if (!index->host.sift && index->host.n > 0) {
    // continuous batching for the float indices; requests of up to 256 queries per lane slot
    s->svc.srv_max_batch = 256;
    s->svc.srv_max_k = 100;
    const int64_t budget = std::max<int64_t>(1ll << 30, (int64_t)16 * 256 * ((index->host.n + 15) / 16 * 16 + 1));
    if (nmsg_server_create(index, budget, s->svc.srv_max_batch, s->svc.srv_max_k, 16, &s->svc.srv) != NMSG_OK)
      s->svc.srv = nullptr;  // then every request goes through nmsg_knn_batch
  }
  s->listen_fd = ::socket(AF_INET, SOCK_STREAM, 0);
  if (s->listen_fd < 0) {
    nmsg_query_server_stop(s);
    return qs_fail(NMSG_ERR_DEVICE, std::string("socket: ") + std::strerror(errno));
  }
  const int one = 1;
  setsockopt(s->listen_fd, SOL_SOCKET, SO_REUSEADDR, &one, sizeof(one));
  sockaddr_in addr{};
  addr.sin_family = AF_INET;
  addr.sin_addr.s_addr = htonl(INADDR_ANY);
  addr.sin_port = htons((uint16_t)port);
  if (::bind(s->listen_fd, reinterpret_cast<sockaddr*>(&addr), sizeof(addr)) != 0 || ::listen(s->listen_fd, 64) != 0) {
    const std::string msg = std::string("bind/listen on port ") + std::to_string(port) + ": " + std::strerror(errno);
    nmsg_query_server_stop(s);
    return qs_fail(NMSG_ERR_BAD_ARG, msg);
  }
  socklen_t len = sizeof(addr);
  getsockname(s->listen_fd, reinterpret_cast<sockaddr*>(&addr), &len);
  s->port = ntohs(addr.sin_port);
  s->acceptor = std::thread(accept_loop, s);
  *out = s;
  return NMSG_OK;
}

NMSG_API int nmsg_query_server_port(const nmsg_query_server* s) { return s ? s->port : -1; }

NMSG_API void nmsg_query_server_stop(nmsg_query_server* s) {
  if (!s) return;
  s->stopping.store(true);
  if (s->listen_fd >= 0) {
    ::shutdown(s->listen_fd, SHUT_RDWR);
    ::close(s->listen_fd);
    s->listen_fd = -1;
  }
  if (s->acceptor.joinable()) s->acceptor.join();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (auto& c : s->conns) ::shutdown(c->fd, SHUT_RDWR);  // wakes the connection threads
    for (auto& c : s->conns)
      if (c->t.joinable()) c->t.join();
    for (auto& c : s->conns) ::close(c->fd);
    s->conns.clear();
  }
  if (s->svc.srv) nmsg_server_free(s->svc.srv);
  delete s;
}

}  // extern "C"
