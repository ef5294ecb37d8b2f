"""Continuous-batching server over a loaded index (C ABI nmsg_server_*).

    srv = Server(index, memory_budget_bytes=8 << 30, max_batch=256, max_k=100)
    rid = srv.submit(queries, k=10, ef=100)      # returns at once
    ids, dists, counts, latency = srv.wait(rid)  # ids/dists are [nq, k]
    lat, wall = srv.run_trace(pool, offsets, sizes, ks, efs, arrivals)   # open-loop replay

Requests are admitted oldest first as device memory frees up: each takes one search slot per
query (the visited-set bytes; up to max_batch) from a pool the memory budget sizes, and one of
max_lanes lanes (a CUDA stream with staging). Requests in different lanes run concurrently on the
GPU and each request's results are independent of the others.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Server:
    def __init__(self, index, memory_budget_bytes=8 << 30, max_batch=256, max_k=100, max_lanes=32):
        self._lib = _capi.load()
        self._index = index  # keeps the index alive
        self.max_batch, self.max_k = int(max_batch), int(max_k)
        h = ctypes.c_void_p()
        _capi.check(self._lib.nmsg_server_create(index._require(), int(memory_budget_bytes), self.max_batch,
                                                 self.max_k, int(max_lanes), ctypes.byref(h)))
        self._h = h
        self.dim = index.info["dim"]

    @property
    def lanes(self) -> int:
        return self._lib.nmsg_server_lanes(self._h)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.nmsg_server_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 — interpreter shutdown
            pass

    def submit(self, queries, k=10, ef=100) -> int:
        q = np.ascontiguousarray(queries, dtype=np.float32).reshape(-1, self.dim)
        rid = ctypes.c_int64()
        _capi.check(self._lib.nmsg_server_submit(self._h, _p(q), q.shape[0], int(k), int(ef), ctypes.byref(rid)))
        self._pending = getattr(self, "_pending", {})
        self._pending[rid.value] = (q.shape[0], int(k))
        return rid.value

    def wait(self, rid):
        nq, k = self._pending.pop(rid)
        ids = np.empty((nq, k), np.int32)
        dists = np.empty((nq, k), np.float32)
        counts = np.empty(nq, np.int32)
        lat = ctypes.c_double()
        _capi.check(self._lib.nmsg_server_wait(self._h, ctypes.c_int64(rid), _p(ids), _p(dists), _p(counts),
                                               ctypes.byref(lat)))
        return ids, dists, counts, lat.value

    def run_trace(self, pool, offsets, sizes, ks, efs, arrivals):
        pool = np.ascontiguousarray(pool, dtype=np.float32)
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        sz = np.ascontiguousarray(sizes, dtype=np.int32)
        kk = np.ascontiguousarray(ks, dtype=np.int32)
        ee = np.ascontiguousarray(efs, dtype=np.int32)
        arr = np.ascontiguousarray(arrivals, dtype=np.float64)
        lat = np.empty(len(arr), np.float64)
        wall = ctypes.c_double()
        _capi.check(self._lib.nmsg_server_run_trace(self._h, _p(pool), _p(off), _p(sz), _p(kk), _p(ee), _p(arr),
                                                    len(arr), _p(lat), ctypes.byref(wall)))
        return lat, wall.value
