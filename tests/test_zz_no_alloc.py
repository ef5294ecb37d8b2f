"""nmsg_knn_batch_noalloc: the search entry point for callers that cannot allocate device memory
(real-time threads kept away from the allocator, processes whose device memory another pool has
reserved). It must return exactly what nmsg_knn_batch returns, call after call, while taking all
of its scratch from the library's fixed device array.

Collected last on purpose (file name), so a stop-at-first-failure run has already run every
other test when it gets here; it also passes when run alone in a fresh process."""
import struct

import numpy as np
import pytest

import nmslib_b200 as nmslib
from nmslib_b200 import _capi
from nmslib_b200.build import build

from conftest import golden_manifest, golden_path, load_golden

pytestmark = pytest.mark.gpu


def _loaded(name, ef, algo):
    idx = nmslib.init(method="hnsw", space=golden_manifest()[name]["space"])
    idx.loadIndex(golden_path(name))
    idx.setQueryTimeParams({"efSearch": ef, "algoType": algo})
    return idx


def _noalloc(lib, idx, q, k):
    """One call through the C ABI on device buffers pre-filled with junk; returns host copies."""
    import torch
    nq, dim = q.shape
    dq = torch.from_numpy(q).cuda()
    ids = torch.full((nq, k), -7, dtype=torch.int32, device="cuda")
    dists = torch.full((nq, k), -7.0, dtype=torch.float32, device="cuda")
    counts = torch.full((nq,), -7, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = lib.nmsg_knn_batch_noalloc(idx._h, dq.data_ptr(), nq, dim, k, k, ids.data_ptr(), dists.data_ptr(),
                                    counts.data_ptr(), None)
    assert rc == 0, _capi.last_error()
    return ids.cpu().numpy(), dists.cpu().numpy(), counts.cpu().numpy()


def _assert_same(got, want, what):
    ids, d, c = got
    want_ids, want_d, want_c = want
    np.testing.assert_array_equal(c, want_c, err_msg=what)
    np.testing.assert_array_equal(ids, want_ids, err_msg=what)
    np.testing.assert_array_equal(d.view(np.int32), want_d.view(np.int32), err_msg=what)


@pytest.mark.parametrize("name,ef,algo,k", [("c1_l2_d128", 100, "hybrid", 10),
                                           ("cos_d100", 1000, "hybrid", 10),
                                           ("negdot_d960", 64, "v1merge", 100)])
def test_no_alloc_matches_the_allocating_entry_point(name, ef, algo, k):
    build()
    lib = _capi.load()
    idx = _loaded(name, ef, algo)
    q = np.ascontiguousarray(load_golden(name)["queries"])
    want = idx.knnQueryBatchArrays(q, k)  # the existing entry point
    for call in range(2):  # the scratch keeps the previous call's contents; results must not change
        _assert_same(_noalloc(lib, idx, q, k), want, f"{name} call {call}")


def test_no_alloc_across_slot_layouts():
    """Calls alternating between indices and efSearch values (so the slot layout of the shared
    array changes from call to call, and sometimes repeats) give the allocating path's results."""
    build()
    lib = _capi.load()
    a = _loaded("c1_l2_d128", 100, "hybrid")
    b = _loaded("sift_l2_ties", 50, "hybrid")
    qa = np.ascontiguousarray(load_golden("c1_l2_d128")["queries"][:300])
    qb = np.ascontiguousarray(load_golden("sift_l2_ties")["queries"][:300])
    want_a, want_b = a.knnQueryBatchArrays(qa, 10), b.knnQueryBatchArrays(qb, 10)
    a.setQueryTimeParams({"efSearch": 300})
    want_a300 = a.knnQueryBatchArrays(qa, 10)
    seq = [(b, qb, want_b, 50), (a, qa, want_a300, 300), (a, qa, want_a300, 300), (b, qb, want_b, 50),
           (a, qa, want_a, 100), (b, qb, want_b, 50), (b, qb, want_b, 50), (a, qa, want_a, 100)]
    for i, (idx, q, want, ef) in enumerate(seq):
        idx.setQueryTimeParams({"efSearch": ef})
        _assert_same(_noalloc(lib, idx, q, 10), want, f"call {i}")


def test_no_alloc_empty_index_and_empty_batch(tmp_path):
    import torch
    build()
    lib = _capi.load()
    p = tmp_path / "empty.hnsw"
    p.write_bytes(struct.pack("<IIiiQQQ", 0, 0, 0, 0, 0, 0, 0))  # the reference's empty index
    idx = nmslib.init(method="hnsw", space="l2")
    idx.loadIndex(str(p))
    ids, d, c = _noalloc(lib, idx, np.zeros((3, 5), np.float32), 4)
    np.testing.assert_array_equal(c, np.zeros(3, np.int32))
    np.testing.assert_array_equal(ids, np.full((3, 4), -1, np.int32))
    # nq == 0: nothing to do, buffers untouched, no error
    full = _loaded("c1_l2_d128", 100, "hybrid")
    out = torch.full((4,), -7, dtype=torch.int32, device="cuda")
    rc = lib.nmsg_knn_batch_noalloc(full._h, out.data_ptr(), 0, 128, 10, 10, out.data_ptr(), out.data_ptr(),
                                    out.data_ptr(), None)
    assert rc == 0, _capi.last_error()
    assert (out.cpu().numpy() == -7).all()


def test_no_alloc_rejects_bad_arguments():
    build()
    lib = _capi.load()
    idx = _loaded("c1_l2_d128", 100, "hybrid")
    rc = lib.nmsg_knn_batch_noalloc(idx._h, None, 4, 128, 10, 5, None, None, None, None)  # kmax < k
    assert rc == _capi.ERR_BAD_ARG and "kmax" in _capi.last_error()
    rc = lib.nmsg_knn_batch_noalloc(None, None, 4, 128, 10, 10, None, None, None, None)
    assert rc == _capi.ERR_BAD_ARG
