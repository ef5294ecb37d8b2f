"""nmslib_b200 — a B200 (sm_100a) engine behind NMSLIB's Python surface for the HNSW query path.

Drop-in for the reference's ``nmslib`` module on this path::

    import nmslib_b200 as nmslib
    index = nmslib.init(method='hnsw', space='l2')        # 'l2' | 'cosinesimil' | 'negdotprod' | 'l1' | 'linf'
    index.loadIndex('index.hnsw')                          # a file written by the reference's saveIndex
    index.setQueryTimeParams({'efSearch': 100})
    results = index.knnQueryBatch(queries, k=10)           # [(ids int32[], dists float32[]), ...]

Names, argument meaning and error behaviour follow python_bindings/nmslib.cc (``init`` :470-510,
``IndexWrapper`` :67-376, ``loadParams`` :658-692). The search itself runs in the CUDA engine
(include/nmslib_b200.h); there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import enum
import os

import numpy as np

from . import _capi

__version__ = "0.1.0"

SPACES = {"l2": _capi.SPACE_L2, "cosinesimil": _capi.SPACE_COSINE, "negdotprod": _capi.SPACE_NEGDOT,
          "l1": _capi.SPACE_L1, "linf": _capi.SPACE_LINF}
METHODS = ("hnsw",)
_ALGOS = {"hybrid": _capi.ALGO_HYBRID, "old": _capi.ALGO_OLD, "v1merge": _capi.ALGO_V1MERGE}


class DistType(enum.IntEnum):
    FLOAT = 0
    INT = 1


class DataType(enum.IntEnum):
    DENSE_VECTOR = 0
    DENSE_UINT8_VECTOR = 1
    SPARSE_VECTOR = 2
    OBJECT_AS_STRING = 3


def _load_params(o):
    """dict or ['key=value', ...] -> {key: str}; python_bindings/nmslib.cc:658-692."""
    if o is None:
        return {}
    if isinstance(o, list):
        out = {}
        for item in o:
            if not isinstance(item, str) or "=" not in item:
                raise ValueError(f"Wrong format of the parameter string: {item!r}")
            key, val = item.split("=", 1)
            out[key.strip()] = val.strip()
        return out
    if isinstance(o, dict):
        out = {}
        for key, val in o.items():
            if isinstance(val, bool) or not isinstance(val, (int, float, str)):
                raise ValueError(f"Unknown type for parameter '{key}'")
            out[str(key)] = str(int(val)) if isinstance(val, float) and float(val).is_integer() else str(val)
        return out
    raise ValueError("Unknown type for parameters")


def _as_int(key, val):
    try:
        return int(val)
    except ValueError:
        raise RuntimeError(f"Failed to convert value '{val}' of parameter '{key}' to an integer") from None


class FloatIndex:
    """Mirror of ``IndexWrapper<float>`` for method='hnsw' over dense float vectors."""

    def __init__(self, method, space, space_params, data_type, dtype, device=0):
        if method not in METHODS:
            raise ValueError(f"The B200 engine implements method 'hnsw' only, got {method!r}")
        if space not in SPACES:
            raise ValueError(f"The B200 engine implements spaces {sorted(SPACES)}, got {space!r}")
        if _load_params(space_params):
            raise RuntimeError("Unknown parameters found!")
        if data_type != DataType.DENSE_VECTOR:
            raise ValueError(f"The space type {space} is not compatible with the type {DataType(data_type).name}, "
                             "only dense vector spaces are allowed!")
        if dtype != DistType.FLOAT:
            raise ValueError("The B200 engine implements DistType.FLOAT only")
        self.method, self.space, self.device = method, space, int(device)
        self.dataType, self.distType = DataType(data_type), DistType(dtype)
        self._h = ctypes.c_void_p()
        self._info = None
        self._data = []   # rows added with addDataPoint(Batch), consumed by createIndex
        self._ids = []

    # ------------------------------------------------------------------ lifecycle
    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(_capi, "_lib", None) if _capi is not None else None
        if h and lib is not None:
            lib.nmsg_index_free(h)
            self._h = None

    def _require(self):
        if not self._h:
            raise ValueError("Must call createIndex or loadIndex before this method")
        return self._h

    # ------------------------------------------------------------------ building
    def addDataPointBatch(self, data, ids=None):
        """IndexWrapper::addDataPointBatch (nmslib.cc:313-334): rows to index; ids default to the
        row numbers. Returns the number of rows added."""
        x = self._queries(data)
        if ids is None:
            start = sum(len(d) for d in self._data)
            idv = np.arange(start, start + len(x), dtype=np.int64)
        else:
            idv = np.asarray(ids, dtype=np.int64).reshape(-1)
            if len(idv) != len(x):
                raise ValueError("ids must have one entry per row")
        self._data.append(x)
        self._ids.append(idv)
        return len(x)

    def addDataPoint(self, id, data):
        self.addDataPointBatch(np.asarray(data, dtype=np.float32).reshape(1, -1), ids=[id])
        return sum(len(d) for d in self._data) - 1

    def createIndex(self, index_params=None, print_progress=False):
        """IndexWrapper::createIndex (nmslib.cc:89-96) -> Hnsw::CreateIndex (hnsw.cc:183-470),
        built by the engine's builder (M, efConstruction, indexThreadQty; maxM = M, maxM0 = 2M,
        heuristic 2) and loaded onto the device. ``gpuBuild=1`` runs the level-0 construction
        searches on this index's GPU (nmsg_build_index_device); the default builds on the host."""
        p = _load_params(index_params)
        known = {"M", "efConstruction", "indexThreadQty", "maxM", "maxM0", "delaunay_type", "post",
                 "skip_optimized_index", "searchMethod", "seed", "gpuBuild"}
        if set(p) - known:
            raise RuntimeError("Unknown parameters found!")
        m = _as_int("M", p.get("M", "16"))
        efc = _as_int("efConstruction", p.get("efConstruction", "200"))
        threads = _as_int("indexThreadQty", p.get("indexThreadQty", "0"))
        if _as_int("maxM", p.get("maxM", str(m))) != m or _as_int("maxM0", p.get("maxM0", str(2 * m))) != 2 * m \
                or p.get("delaunay_type", "2") != "2" or p.get("post", "0") != "0" \
                or p.get("skip_optimized_index", "0") != "0":
            raise ValueError("the B200 builder implements maxM=M, maxM0=2M, delaunay_type=2, post=0 and the "
                             "optimized layout only")
        data = np.concatenate(self._data) if self._data else np.zeros((0, 1), np.float32)
        ids = np.concatenate(self._ids) if self._ids else np.zeros(0, np.int64)
        import tempfile
        with tempfile.TemporaryDirectory() as tmp:
            path = os.path.join(tmp, "index.hnsw")
            gpu = _as_int("gpuBuild", p.get("gpuBuild", "0")) != 0
            _capi.build_index(data, SPACES[self.space], m, efc, ids=ids.astype(np.int32), nthreads=threads,
                              seed=_as_int("seed", p.get("seed", "0")), out_path=path,
                              device=self.device if gpu else None)
            self.loadIndex(path)

    def loadIndex(self, filename, load_data=False):
        """IndexWrapper::loadIndex (nmslib.cc:98-113): reads the optimized index file and resets
        the query-time parameters (ef = 20, algoType = hybrid)."""
        if load_data:
            raise ValueError("load_data=True is not supported: the optimized index file already holds the vectors")
        lib = _capi.load()
        h = ctypes.c_void_p()
        _capi.check(lib.nmsg_index_load(os.fsencode(filename), SPACES[self.space], self.device, ctypes.byref(h)))
        if self._h:
            lib.nmsg_index_free(self._h)
        self._h = h
        self._refresh_info()

    def saveIndex(self, filename, save_data=False):
        if save_data:
            raise ValueError("save_data=True is not supported by the B200 engine")
        _capi.check(_capi.load().nmsg_index_save(self._require(), os.fsencode(filename)))

    def _refresh_info(self):
        info = _capi.IndexInfo()
        _capi.check(_capi.load().nmsg_index_info_get(self._h, ctypes.byref(info)))
        self._info = info

    @property
    def info(self) -> dict:
        self._require()
        self._refresh_info()
        return {name: getattr(self._info, name) for name, _ in _capi.IndexInfo._fields_}

    def __len__(self):
        return int(self._info.n) if self._h else 0

    def __repr__(self):
        return f"<nmslib_b200.FloatIndex method={self.method} space={self.space} n={len(self)}>"

    # ------------------------------------------------------------------ parameters
    def setQueryTimeParams(self, params=None):
        """Hnsw::SetQueryTimeParams (hnsw.cc:472-507): keys ef | efSearch (default 20),
        algoType old | v1merge | hybrid (default hybrid), searchMethod (accepted, ignored).
        Keys left out return to their defaults."""
        h = self._require()
        p = _load_params(params)
        if "ef" in p and "efSearch" in p:
            raise RuntimeError("The user shouldn't specify parameters ef and efSearch at the same time "
                               "(they are synonyms)")
        unknown = set(p) - {"ef", "efSearch", "algoType", "searchMethod"}
        if unknown:
            raise RuntimeError("Unknown parameters found!")
        ef = _as_int("ef", p.get("ef", p.get("efSearch", "20")))
        algo = p.get("algoType", "hybrid").lower()
        if algo not in _ALGOS:
            raise RuntimeError("algoType should be one of the following: old, v1merge")
        if "searchMethod" in p:
            _as_int("searchMethod", p["searchMethod"])
        _capi.check(_capi.load().nmsg_set_query_params(h, ef, _ALGOS[algo]))

    def setLaunchConfig(self, warps_per_block=0, rows_per_group=0, visited_hash_log2=0, stage_rows=0,
                        plain_slots=0, queries_per_warp=0, row_copy=0, query_order=0, host_copy=0):
        """Launch shape of the search kernels (0 = automatic); results do not depend on it, except
        that plain_slots below the resident block count makes one-query-per-block launches give up
        with a timeout error (the bounded slot wait). host_copy=1 copies host arrays directly
        instead of through page-locked staging."""
        cfg = _capi.LaunchConfig(warps_per_block, rows_per_group, stage_rows, visited_hash_log2, plain_slots,
                                 queries_per_warp, row_copy, query_order, host_copy)
        _capi.check(_capi.load().nmsg_set_launch_config(self._require(), ctypes.byref(cfg)))

    # ------------------------------------------------------------------ search
    def _queries(self, input):
        if isinstance(input, list):
            rows = [np.ascontiguousarray(np.asarray(r, dtype=np.float32).reshape(-1)) for r in input]
            if not rows:
                return np.zeros((0, self._info.dim if self._info else 0), np.float32)
            return np.ascontiguousarray(np.stack(rows))
        q = np.ascontiguousarray(np.asarray(input, dtype=np.float32))
        if q.ndim != 2:
            raise RuntimeError("data must be a 2d array")
        return q

    def knnQueryBatchArrays(self, queries, k=10, ef=None, plain=False, stats=False):
        """Batch search returning dense arrays: (ids [nq, kmax] int32 with -1 padding,
        dists [nq, kmax] float32 with +inf padding, counts [nq] int32[, stats [nq, 4] int64]).
        ``k`` and ``ef`` may be per-query integer arrays (mixed batches in one launch)."""
        h = self._require()
        q = self._queries(queries)
        nq = q.shape[0]
        k_arr = None
        if np.ndim(k):
            k_arr = np.ascontiguousarray(np.asarray(k, dtype=np.int32).reshape(-1))
            if k_arr.shape[0] != nq:
                raise ValueError("per-query k must have one entry per query")
            kmax = int(k_arr.max()) if nq else 1
        else:
            kmax = int(k)
        ef_arr = None
        if ef is not None:
            ef_arr = np.ascontiguousarray(np.broadcast_to(np.asarray(ef, dtype=np.int32), (nq,)))
        kmax = max(kmax, 1)
        ids = np.empty((nq, kmax), np.int32)
        dists = np.empty((nq, kmax), np.float32)
        counts = np.empty(nq, np.int32)
        st = np.empty((nq, 4), np.int64) if stats else None
        ptr = lambda a: None if a is None else a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
        flags = _capi.FLAG_PLAIN_KERNEL if plain else 0
        dim = q.shape[1] if nq else (self._info.dim if self._info else 0)
        _capi.check(_capi.load().nmsg_knn_batch(h, ptr(q), nq, dim, 1 if k_arr is not None else kmax, ptr(k_arr),
                                                ptr(ef_arr), kmax, ptr(ids), ptr(dists), ptr(counts), ptr(st),
                                                flags, None))
        return (ids, dists, counts, st) if stats else (ids, dists, counts)

    def bruteForceBatchArrays(self, queries, k=10, stats=False, exact_scan=False):
        """Exact k-NN over every stored vector (seq_search semantics) on the tensor cores:
        (ids [nq, k] external, dists [nq, k], counts [nq][, stats [4]]). k <= 32. l2 / cosinesimil /
        negdotprod rows of up to 4096 floats use BF16 tensor cores with an exact rerank; L1, LInf,
        wider rows and ``exact_scan=True`` an exact CUDA-core scan whose distances are the search's
        own values bit for bit."""
        h = self._require()
        q = self._queries(queries)
        nq = q.shape[0]
        ids = np.empty((nq, k), np.int32)
        dists = np.empty((nq, k), np.float32)
        counts = np.empty(nq, np.int32)
        st = np.zeros(4, np.int64)
        ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
        dim = q.shape[1] if nq else (self._info.dim if self._info else 0)
        _capi.check(_capi.load().nmsg_bruteforce_knn(h, ptr(q), nq, dim, int(k), int(k), ptr(ids), ptr(dists),
                                                     ptr(counts), ptr(st),
                                                     _capi.FLAG_EXACT_SCAN if exact_scan else 0, None))
        return (ids, dists, counts, st) if stats else (ids, dists, counts)

    def knnQueryBatch(self, queries, k=10, num_threads=0):
        """IndexWrapper::knnQueryBatch (nmslib.cc:142-168): a list of (ids int32[], dists float32[])
        per query, ascending distance. num_threads is accepted for compatibility and unused."""
        ids, dists, counts = self.knnQueryBatchArrays(queries, k)
        # each query's arrays are views of its rows in the batch's result arrays: no per-query copy
        # (10K queries of k = 10: 3 ms against 11 ms with copies)
        if counts.size and int(counts.min()) == ids.shape[1]:
            return list(zip(ids, dists))  # every row full: iterating the arrays yields the row views
        return [(ids[i, :c], dists[i, :c]) for i, c in enumerate(counts.tolist())]

    def knnQuery(self, vector, k=10):
        """IndexWrapper::knnQuery (nmslib.cc:127-140)."""
        v = np.asarray(vector, dtype=np.float32).reshape(1, -1)
        return self.knnQueryBatch(v, k)[0]


class IntIndex(FloatIndex):
    """Mirror of ``IndexWrapper<int>`` for method='hnsw', space='l2sqr_sift' over
    DENSE_UINT8_VECTOR data (128 uint8 values per object, int squared L2 distances,
    similarity_search/src/space/space_l2sqr_sift.cc). The reference saves such an index only in the
    regular format with a separate objects file, so ``loadIndex`` needs ``load_data=True`` (or
    rows added first with ``addDataPointBatch``) and ``saveIndex`` writes both files with
    ``save_data=True``. Building is the reference's job (``createIndex`` is not offered)."""

    def __init__(self, method, space, space_params, data_type, dtype, device=0):
        if method not in METHODS:
            raise ValueError(f"The B200 engine implements method 'hnsw' only, got {method!r}")
        if space != "l2sqr_sift":
            raise ValueError(f"The B200 engine implements integer distances for space 'l2sqr_sift' only, got {space!r}")
        if _load_params(space_params):
            raise RuntimeError("Unknown parameters found!")
        if data_type != DataType.DENSE_UINT8_VECTOR:
            raise ValueError(f"The space type {space} is not compatible with the type {DataType(data_type).name}!")
        self.method, self.space, self.device = method, space, int(device)
        self.dataType, self.distType = DataType(data_type), DistType(dtype)
        self._h = ctypes.c_void_p()
        self._info = None
        self._data = []
        self._ids = []

    def __repr__(self):
        return f"<nmslib_b200.IntIndex method={self.method} space={self.space} n={len(self)}>"

    def _queries(self, input):
        """py::array_t<uint8_t, c_style | forcecast> (nmslib.cc:258-272): 2-D rows of uint8."""
        if isinstance(input, list):
            input = np.stack([np.asarray(r).reshape(-1) for r in input]) if input else np.zeros((0, 128))
        q = np.ascontiguousarray(np.asarray(input).astype(np.uint8, copy=False))
        if q.ndim != 2:
            raise RuntimeError("data must be a 2d array")
        return q

    def addDataPointBatch(self, data, ids=None):
        x = self._queries(data)
        if x.shape[1] != 128:
            raise RuntimeError(f"Bug or internal error, SIFT vectors dim {x.shape[1]} isn't == 128")
        start = sum(len(d) for d in self._data)
        idv = np.arange(start, start + len(x), dtype=np.int64) if ids is None else np.asarray(ids, np.int64).reshape(-1)
        if len(idv) != len(x):
            raise ValueError("ids must have one entry per row")
        self._data.append(x)
        self._ids.append(idv)
        return len(x)

    def addDataPoint(self, id, data):
        self.addDataPointBatch(np.asarray(data).reshape(1, -1), ids=[id])
        return sum(len(d) for d in self._data) - 1

    def createIndex(self, index_params=None, print_progress=False):
        raise RuntimeError("the B200 engine loads l2sqr_sift indices built by the reference's createIndex; "
                           "it does not build them")

    def _objects_file(self, path):
        """Objects added with addDataPointBatch written in the reference's objects-file format
        (u64 count; per object u64 length, i32 id, i32 label -1, u64 132, 128 values, i32 norm)."""
        data = np.concatenate(self._data)
        ids = np.concatenate(self._ids).astype(np.int32)
        norms = (data.astype(np.int64) ** 2).sum(1).astype(np.int32)
        rec = np.zeros(len(data), dtype=[("len", "<u8"), ("id", "<i4"), ("label", "<i4"), ("dlen", "<u8"),
                                         ("v", "u1", 128), ("norm", "<i4")])
        rec["len"], rec["id"], rec["label"], rec["dlen"], rec["v"], rec["norm"] = 148, ids, -1, 132, data, norms
        with open(path, "wb") as f:
            f.write(np.uint64(len(data)).tobytes())
            f.write(rec.tobytes())

    def loadIndex(self, filename, load_data=False):
        """IndexWrapper::loadIndex (nmslib.cc:98-113): with load_data the objects come from
        ``filename + '.dat'``, else from rows added before; then the regular graph file."""
        lib = _capi.load()
        h = ctypes.c_void_p()
        if load_data:
            rc = lib.nmsg_index_load_with_data(os.fsencode(filename), os.fsencode(filename + ".dat"),
                                               _capi.SPACE_L2SQR_SIFT, self.device, ctypes.byref(h))
        else:
            import tempfile
            with tempfile.TemporaryDirectory() as tmp:
                dat = os.path.join(tmp, "objects.dat")
                if self._data:
                    self._objects_file(dat)
                else:
                    with open(dat, "wb") as f:
                        f.write(np.uint64(0).tobytes())
                rc = lib.nmsg_index_load_with_data(os.fsencode(filename), os.fsencode(dat), _capi.SPACE_L2SQR_SIFT,
                                                   self.device, ctypes.byref(h))
        _capi.check(rc)
        if self._h:
            lib.nmsg_index_free(self._h)
        self._h = h
        self._refresh_info()

    def saveIndex(self, filename, save_data=False):
        """saveIndex (nmslib.cc:115-125): the regular graph file, and with save_data the objects
        file ``filename + '.dat'``."""
        h = self._require()
        import tempfile
        with tempfile.TemporaryDirectory() as tmp:
            dat = filename + ".dat" if save_data else os.path.join(tmp, "objects.dat")
            _capi.check(_capi.load().nmsg_index_save_with_data(h, os.fsencode(filename), os.fsencode(dat)))

    def knnQueryBatchArrays(self, queries, k=10, ef=None, plain=False, stats=False):
        """Batch search returning dense arrays: (ids [nq, kmax] int32, -1 padding; dists
        [nq, kmax] int32, INT32_MAX padding; counts [nq][, stats [nq, 4]])."""
        h = self._require()
        q = self._queries(queries)
        nq = q.shape[0]
        k_arr = None
        if np.ndim(k):
            k_arr = np.ascontiguousarray(np.asarray(k, dtype=np.int32).reshape(-1))
            if k_arr.shape[0] != nq:
                raise ValueError("per-query k must have one entry per query")
            kmax = int(k_arr.max()) if nq else 1
        else:
            kmax = int(k)
        ef_arr = None
        if ef is not None:
            ef_arr = np.ascontiguousarray(np.broadcast_to(np.asarray(ef, dtype=np.int32), (nq,)))
        kmax = max(kmax, 1)
        ids = np.empty((nq, kmax), np.int32)
        dists = np.empty((nq, kmax), np.int32)
        counts = np.empty(nq, np.int32)
        st = np.empty((nq, 4), np.int64) if stats else None
        ptr = lambda a: None if a is None else a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
        flags = _capi.FLAG_PLAIN_KERNEL if plain else 0
        dim = q.shape[1] if nq else 128
        _capi.check(_capi.load().nmsg_knn_batch_u8(h, ptr(q), nq, dim, 1 if k_arr is not None else kmax, ptr(k_arr),
                                                   ptr(ef_arr), kmax, ptr(ids), ptr(dists), ptr(counts), ptr(st),
                                                   flags, None))
        return (ids, dists, counts, st) if stats else (ids, dists, counts)

    def knnQuery(self, vector, k=10):
        return self.knnQueryBatch(np.asarray(vector).reshape(1, -1), k)[0]

    def bruteForceBatchArrays(self, queries, k=10, stats=False):
        raise RuntimeError("brute force over l2sqr_sift indices is not supported")


def init(space="cosinesimil", space_params=None, method="hnsw", data_type=DataType.DENSE_VECTOR,
         dtype=DistType.FLOAT, device=0):
    """nmslib.init (python_bindings/nmslib.cc:470-510): DistType.FLOAT gives the float index,
    DistType.INT the integer one (space 'l2sqr_sift'); ``device`` selects the CUDA device."""
    if dtype == DistType.INT:
        return IntIndex(method, space, space_params, data_type, dtype, device)
    return FloatIndex(method, space, space_params, data_type, dtype, device)
