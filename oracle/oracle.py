"""ORACLE — test infrastructure only (the checker, never the thing measured or shipped).

Python side of the CPU restatement in ``oracle/hnsw_oracle.cc`` plus an FP64 brute-force
ground truth. Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.

* ``OracleIndex`` — loads an NMSLIB optimized HNSW file (similarity_search/src/method/
  hnsw.cc:1025-1074) and searches it with the reference's SearchV1Merge / SearchOld semantics
  (src/method/hnsw_distfunc_opt.cc:46-283), FMA lane order of
  include/method/hnsw_distfunc_opt_impl_inline.h:42-173.
* ``OracleSiftIndex`` — loads an ``l2sqr_sift`` index (the regular graph file of
  hnsw.cc:810-842 and the ``<file>.dat`` objects of python_bindings/nmslib.cc:115-125) and
  searches it with the same steps (the generic search of hnsw.cc:1078-1290) and the reference's
  int distance (distcomp_l2sqr_sift.cc:40-50).
* ``bruteforce_fp64`` — exact kNN in float64 with ties broken by id; the recall ground truth.
* ``reference_module`` — the reference's own pybind module built by ``make -C oracle ref``
  into ``oracle/_ref`` (present only where the reference sources were available to build it).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_hnsw.so")
REF_DIR = os.path.join(HERE, "_ref")

SPACE_CODES = {"l2": 0, "cosinesimil": 1, "negdotprod": 2}


def build_oracle(force: bool = False) -> str:
    """Compile the CPU restatement (g++, a few seconds) if it is not built yet."""
    src = os.path.join(HERE, "hnsw_oracle.cc")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE, "liboracle_hnsw.so"], check=True)
    return LIB_PATH


_lib = None


def _load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(build_oracle())
        P, I64, I32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
        lib.oracle_load.restype = P
        lib.oracle_load.argtypes = [ctypes.c_char_p]
        lib.oracle_free.argtypes = [P]
        lib.oracle_info.argtypes = [P, P]
        lib.oracle_export.argtypes = [P, P, P, P, P]
        lib.oracle_dist.restype = ctypes.c_float
        lib.oracle_dist.argtypes = [I32, P, P, I32]
        lib.oracle_normalize.argtypes = [P, I32, I32]
        lib.oracle_search.restype = I32
        lib.oracle_search.argtypes = [P, P, I64, I32, I32, P, I32, P, I32, I32, P, P, P, P, I32]
        lib.oracle_std_sort_items.argtypes = [P, P, I32]
        lib.oracle_sift_load.restype = P
        lib.oracle_sift_load.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
        lib.oracle_sift_free.argtypes = [P]
        lib.oracle_sift_info.argtypes = [P, P]
        lib.oracle_sift_search.restype = I32
        lib.oracle_sift_search.argtypes = [P, P, I64, I32, I32, I32, I32, P, P, P, P, I32]
        lib.oracle_last_error.restype = ctypes.c_char_p
        _lib = lib
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class OracleIndex:
    """CPU restatement of the reference's optimized HNSW query path over one index file."""

    INFO_KEYS = ("n", "dim", "maxlevel", "enterpoint", "maxM", "maxM0", "dist_type",
                 "mem_per_obj", "off_level0")

    def __init__(self, path: str):
        lib = _load()
        self._h = lib.oracle_load(os.fsencode(path))
        if not self._h:
            raise RuntimeError(lib.oracle_last_error().decode())
        info = np.zeros(9, np.int64)
        lib.oracle_info(self._h, _ptr(info))
        self.info = dict(zip(self.INFO_KEYS, (int(v) for v in info)))
        self.n, self.dim = self.info["n"], self.info["dim"]

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.oracle_free(self._h)
            self._h = None

    def export(self):
        """(vectors [n, dim] f32, external ids [n], level-0 lists [n, maxM0+1], levels [n])."""
        n, d, m0 = self.n, self.dim, self.info["maxM0"]
        vecs = np.zeros((n, d), np.float32)
        ext = np.zeros(n, np.int32)
        l0 = np.zeros((n, m0 + 1), np.int32)
        lev = np.zeros(n, np.int32)
        _load().oracle_export(self._h, _ptr(vecs), _ptr(ext), _ptr(l0), _ptr(lev))
        return vecs, ext, l0, lev

    def search(self, queries, k=10, ef=20, algo=0, k_per_q=None, ef_per_q=None, nthreads=0):
        """Returns (ids [nq,kmax], dists [nq,kmax], counts [nq], stats [nq,4]).

        algo: 0 hybrid, 1 old, 2 v1merge (hnsw.cc:472-507, :724). stats columns are
        n_dist, n_expand, n_greedy, algorithmic bytes.
        """
        q = np.ascontiguousarray(queries, dtype=np.float32)
        nq = q.shape[0]
        kp = None if k_per_q is None else np.ascontiguousarray(k_per_q, np.int32)
        ep = None if ef_per_q is None else np.ascontiguousarray(ef_per_q, np.int32)
        kmax = int(kp.max()) if kp is not None and nq else int(k)
        kmax = max(kmax, 1)
        ids = np.empty((nq, kmax), np.int32)
        dists = np.empty((nq, kmax), np.float32)
        counts = np.empty(nq, np.int32)
        stats = np.empty((nq, 4), np.int64)
        rc = _load().oracle_search(self._h, _ptr(q), nq, q.shape[1] if q.ndim == 2 else 0, int(k),
                                   _ptr(kp), int(ef), _ptr(ep), int(algo), kmax, _ptr(ids),
                                   _ptr(dists), _ptr(counts), _ptr(stats), int(nthreads))
        if rc != 0:
            raise ValueError(_load().oracle_last_error().decode())
        return ids, dists, counts, stats


def dist(dist_type: int, a, b) -> float:
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return float(_load().oracle_dist(int(dist_type), _ptr(a), _ptr(b), a.shape[0]))


def normalize(v, use_double: bool = False):
    v = np.array(v, np.float32, copy=True)
    _load().oracle_normalize(_ptr(v), v.shape[0], int(use_double))
    return v


def std_sort_items(keys, payload):
    """libstdc++ std::sort of (key, payload) compared by key only."""
    k = np.array(keys, np.float32, copy=True)
    p = np.array(payload, np.int32, copy=True)
    _load().oracle_std_sort_items(_ptr(k), _ptr(p), k.shape[0])
    return k, p


class OracleSiftIndex:
    """CPU restatement of the reference's generic HNSW search over an ``l2sqr_sift`` index: 128
    uint8 values per object, int distances."""

    INFO_KEYS = ("n", "maxlevel", "enterpoint", "M", "maxM", "maxM0")

    def __init__(self, path: str, data_path: str | None = None):
        lib = _load()
        self._h = lib.oracle_sift_load(path.encode(), (data_path or path + ".dat").encode())
        if not self._h:
            raise ValueError(lib.oracle_last_error().decode())
        info = np.zeros(len(self.INFO_KEYS), np.int64)
        lib.oracle_sift_info(self._h, _ptr(info))
        self.info = dict(zip(self.INFO_KEYS, (int(v) for v in info)))

    def __del__(self):
        if getattr(self, "_h", None):
            _load().oracle_sift_free(self._h)
            self._h = None

    def search(self, queries, k, ef, algo=0, nthreads=0, stats=False):
        """(ids [nq,k], int32 dists [nq,k], counts [nq][, stats [nq,4]]); algo 0 hybrid, 1 old,
        2 v1merge. stats: distance evaluations, level-0 expansions, upper-level list scans,
        algorithmic bytes."""
        q = np.ascontiguousarray(queries, np.uint8)
        if q.ndim != 2 or q.shape[1] != 128:
            raise ValueError("l2sqr_sift queries are [nq, 128] uint8")
        nq = q.shape[0]
        ids = np.empty((nq, k), np.int32)
        dists = np.empty((nq, k), np.int32)
        counts = np.empty(nq, np.int32)
        st = np.zeros((nq, 4), np.int64)
        rc = _load().oracle_sift_search(self._h, _ptr(q), nq, int(k), int(ef), int(algo), int(k), _ptr(ids),
                                        _ptr(dists), _ptr(counts), _ptr(st), int(nthreads))
        if rc != 0:
            raise ValueError(_load().oracle_last_error().decode())
        return (ids, dists, counts, st) if stats else (ids, dists, counts)


def bruteforce_fp64(base, queries, k, space, ids=None, chunk=256):
    """Exact kNN in float64, ties broken by id. Returns (ids [nq,k], dists [nq,k]).

    l2 uses squared distance (the value the optimized HNSW path reports); cosinesimil uses
    1 - cos on float64-normalised vectors; negdotprod uses -dot.
    """
    b = np.asarray(base, np.float64)
    q = np.asarray(queries, np.float64)
    ext = np.arange(b.shape[0]) if ids is None else np.asarray(ids)
    if space == "cosinesimil":
        bn = np.linalg.norm(b, axis=1, keepdims=True)
        qn = np.linalg.norm(q, axis=1, keepdims=True)
        b = b / np.where(bn == 0, 1, bn)
        q = q / np.where(qn == 0, 1, qn)
    k = min(k, b.shape[0])
    out_i = np.empty((q.shape[0], k), np.int64)
    out_d = np.empty((q.shape[0], k), np.float64)
    bsq = (b * b).sum(1)
    for s in range(0, q.shape[0], chunk):
        qq = q[s:s + chunk]
        if space == "l2":
            d = (qq * qq).sum(1)[:, None] - 2 * qq @ b.T + bsq[None, :]
        elif space == "cosinesimil":
            d = 1 - qq @ b.T
        else:
            d = -(qq @ b.T)
        part = np.argpartition(d, k - 1, axis=1)[:, :k + 0] if k < b.shape[0] else np.tile(
            np.arange(b.shape[0]), (qq.shape[0], 1))
        # exact recheck + id tie-break: widen to every candidate within the kth distance
        for r in range(qq.shape[0]):
            kth = d[r, part[r]].max()
            cand = np.nonzero(d[r] <= kth)[0]
            if space == "l2":  # recompute exactly for the candidates
                dd = ((b[cand] - qq[r]) ** 2).sum(1)
            else:
                dd = d[r, cand]
            order = np.lexsort((ext[cand], dd))[:k]
            out_i[s + r] = ext[cand[order]]
            out_d[s + r] = dd[order]
    return out_i, out_d


def recall(found_ids, true_ids, counts=None) -> float:
    """Mean |found ∩ true| / k (benchmark/eval.py recall definition: set overlap)."""
    k = true_ids.shape[1]
    hits = 0
    for r in range(true_ids.shape[0]):
        f = found_ids[r] if counts is None else found_ids[r][: counts[r]]
        hits += len(np.intersect1d(f, true_ids[r]))
    return hits / (k * max(1, true_ids.shape[0]))


def reference_module():
    """Import the reference's own pybind module from oracle/_ref, or return None."""
    if not os.path.isdir(REF_DIR):
        return None
    if REF_DIR not in sys.path:
        sys.path.insert(0, REF_DIR)
    try:
        import nmslib as ref  # noqa: WPS433 — the reference module built from its sources
    except ImportError:
        return None
    return ref
