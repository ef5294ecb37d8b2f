"""Launch-shape autotuner for the HNSW search kernels.

What varies is how many queries one persistent warp carries at once (1..4: their list reads,
visited checks and row copies overlap), how many warps share a block, how a round of vector rows
is gathered (asynchronous copies of 4..16 rows into shared memory, or 1..2 rows per 8-lane group
in registers) and whether the visited set starts in a shared-memory hash table. None of it changes
results (the GPU parity tests run every shape); all of it changes speed with the vector width, the
beam size (efSearch, which sets the shared memory each query needs) and the batch size.
``autotune`` times the candidate shapes on the caller's own queries and leaves the fastest one set
on the index.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi

# (warps_per_block, rows_per_group, visited_hash_log2, stage_rows, queries_per_warp, row_copy)
DEFAULT_CANDIDATES = (
    (4, 0, -1, 8, 1, 0), (2, 0, -1, 8, 1, 0), (4, 2, -1, -1, 1, 0),
    (4, 0, -1, 8, 2, 0), (4, 0, -1, 16, 2, 0), (2, 0, -1, 8, 2, 0), (4, 0, -1, 8, 2, 2),
    (4, 0, -1, 8, 3, 0), (4, 0, -1, 8, 4, 0), (4, 0, -1, 16, 4, 0), (2, 0, -1, 16, 4, 0), (4, 0, -1, 16, 4, 2),
)


def _config(shape):
    return _capi.LaunchConfig(shape[0], shape[1], shape[3], shape[2], 0, shape[4] if len(shape) > 4 else 0,
                              shape[5] if len(shape) > 5 else 0)


def autotune(index, queries, k=10, ef=None, candidates=DEFAULT_CANDIDATES, reps=5):
    """Times every candidate shape on `queries` (host array) at the index's current efSearch
    (or `ef`), sets the fastest on the index and returns (best_shape, [(shape, ms), ...])."""
    import torch

    lib = _capi.load()
    h = index._require()
    if ef is not None:
        index.setQueryTimeParams({"efSearch": int(ef)})
    q = np.ascontiguousarray(queries, dtype=np.float32)
    nq, dim = q.shape
    dq = torch.from_numpy(q).cuda()
    ids = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    dists = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    counts = torch.empty((nq,), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()

    def run():
        _capi.check(lib.nmsg_knn_batch(h, dq.data_ptr(), nq, dim, k, None, None, k, ids.data_ptr(),
                                       dists.data_ptr(), counts.data_ptr(), None, _capi.FLAG_DEVICE_PTRS,
                                       stream.cuda_stream))

    table = []
    for shape in candidates:
        cfg = _config(shape)
        _capi.check(lib.nmsg_set_launch_config(h, ctypes.byref(cfg)))
        run()
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(reps):
            run()
        end.record(stream)
        torch.cuda.synchronize()
        table.append((shape, start.elapsed_time(end) / reps))
    best = min(table, key=lambda t: t[1])[0]
    cfg = _config(best)
    _capi.check(lib.nmsg_set_launch_config(h, ctypes.byref(cfg)))
    return best, table
