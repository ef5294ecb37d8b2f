"""nmsg_knn_batch_noalloc: the search entry point for callers that cannot allocate device memory
(allocation-free stream captures, real-time threads kept away from the allocator, processes whose
device memory another pool has reserved). It must return exactly what nmsg_knn_batch returns,
call after call, while taking all of its scratch from the library's fixed device array.

Collected last on purpose (file name), so a stop-at-first-failure run has already run every
other test when it gets here; it also passes when run alone in a fresh process."""
import ctypes

import numpy as np
import pytest

import nmslib_b200 as nmslib
from nmslib_b200 import _capi
from nmslib_b200.build import build

from conftest import golden_manifest, golden_path, load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,ef,algo,k", [("c1_l2_d128", 100, "hybrid", 10),
                                           ("cos_d100", 1000, "hybrid", 10),
                                           ("negdot_d960", 64, "v1merge", 100)])
def test_no_alloc_matches_the_allocating_entry_point(name, ef, algo, k):
    import torch

    build()
    lib = _capi.load()
    idx = nmslib.init(method="hnsw", space=golden_manifest()[name]["space"])
    idx.loadIndex(golden_path(name))
    idx.setQueryTimeParams({"efSearch": ef, "algoType": algo})
    q = np.ascontiguousarray(load_golden(name)["queries"])
    nq, dim = q.shape
    want_ids, want_d, want_c = idx.knnQueryBatchArrays(q, k)  # the existing entry point

    dq = torch.from_numpy(q).cuda()
    ids = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    dists = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    counts = torch.empty((nq,), dtype=torch.int32, device="cuda")
    for call in range(2):  # the scratch keeps the previous call's contents; results must not change
        ids.fill_(-7)
        dists.fill_(-7.0)
        counts.fill_(-7)
        torch.cuda.synchronize()
        rc = lib.nmsg_knn_batch_noalloc(idx._h, dq.data_ptr(), nq, dim, k, k, ids.data_ptr(), dists.data_ptr(),
                                        counts.data_ptr(), None)
        assert rc == 0, _capi.last_error()
        np.testing.assert_array_equal(counts.cpu().numpy(), want_c, err_msg=f"call {call}")
        np.testing.assert_array_equal(ids.cpu().numpy(), want_ids, err_msg=f"call {call}")
        np.testing.assert_array_equal(dists.cpu().numpy().view(np.int32), want_d.view(np.int32),
                                      err_msg=f"call {call}")


def test_no_alloc_rejects_bad_arguments():
    build()
    lib = _capi.load()
    idx = nmslib.init(method="hnsw", space="l2")
    idx.loadIndex(golden_path("c1_l2_d128"))
    rc = lib.nmsg_knn_batch_noalloc(idx._h, None, 4, 128, 10, 5, None, None, None, None)  # kmax < k
    assert rc == _capi.ERR_BAD_ARG and "kmax" in _capi.last_error()
    rc = lib.nmsg_knn_batch_noalloc(None, None, 4, 128, 10, 10, None, None, None, None)
    assert rc == _capi.ERR_BAD_ARG
