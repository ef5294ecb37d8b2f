"""The continuous-batching server: each request's results are identical alone and in a mix of
concurrently running requests, and identical to a plain batch search with the same k and ef."""
import numpy as np
import pytest

import nmslib_b200 as nmslib
from nmslib_b200.build import build
from nmslib_b200.serving import Server

from conftest import golden_path, load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def served():
    build()
    idx = nmslib.init(method="hnsw", space="l2")
    idx.loadIndex(golden_path("c1_l2_d128"))
    srv = Server(idx, memory_budget_bytes=64 << 20, max_batch=64, max_k=100, max_lanes=8)
    yield idx, srv
    srv.close()


def _requests(n_queries):
    rng = np.random.default_rng(3)
    reqs, start = [], 0
    while start < n_queries:
        b = int(min(n_queries - start, max(1, np.exp(rng.uniform(0, np.log(64))))))
        reqs.append((start, b, int(rng.choice([10, 100])), int(rng.choice([50, 100, 400]))))
        start += b
    return reqs


def test_results_same_alone_and_in_mix(served):
    idx, srv = served
    assert srv.lanes >= 2
    q = load_golden("c1_l2_d128")["queries"]
    reqs = _requests(len(q))
    alone = []
    for s, b, k, ef in reqs:
        alone.append(srv.wait(srv.submit(q[s:s + b], k, ef))[:3])
    rids = [srv.submit(q[s:s + b], k, ef) for s, b, k, ef in reqs]  # all in flight together
    for (s, b, k, ef), rid, ref in zip(reqs, rids, alone):
        got = srv.wait(rid)[:3]
        for x, y in zip(got, ref):
            np.testing.assert_array_equal(x, y)
        idx.setQueryTimeParams({"efSearch": ef})
        bi, bd, bc = idx.knnQueryBatchArrays(q[s:s + b], k)
        np.testing.assert_array_equal(got[0], bi)
        np.testing.assert_array_equal(got[1].view(np.int32), bd.view(np.int32))
        np.testing.assert_array_equal(got[2], bc)


def test_trace_replay(served):
    _, srv = served
    q = load_golden("c1_l2_d128")["queries"]
    reqs = _requests(len(q))
    rng = np.random.default_rng(5)
    arrivals = np.cumsum(rng.exponential(200e-6, len(reqs)))
    lat, wall = srv.run_trace(q, [r[0] for r in reqs], [r[1] for r in reqs], [r[2] for r in reqs],
                              [r[3] for r in reqs], arrivals)
    assert (lat > 0).all() and wall >= arrivals[-1]
    assert np.percentile(lat, 99) < 1.0  # seconds; generous bound, the bench reports the real figures


def test_rejects_bad_requests(served):
    _, srv = served
    q = load_golden("c1_l2_d128")["queries"]
    with pytest.raises(ValueError):
        srv.submit(q[:65], 10, 50)     # above max_batch
    with pytest.raises(ValueError):
        srv.submit(q[:4], 101, 50)     # above max_k
    with pytest.raises(RuntimeError):
        srv.submit(q[:4], 10, 1000)    # SearchOld is not served


def test_admission_waits_for_memory():
    """A budget that holds the slots of one full request only (64 slots of 10K visited bytes,
    besides the lanes' staging): requests wait for memory rather than for a lane, all complete,
    and each result is the plain batch search's."""
    idx = nmslib.init(method="hnsw", space="l2")
    idx.loadIndex(golden_path("c1_l2_d128"))
    lane_staging = 64 * (128 * 4 + 100 * 8 + 8)
    budget = 8 * lane_staging + 64 * (10_000 + 1) + 100
    srv = Server(idx, memory_budget_bytes=budget, max_batch=64, max_k=100, max_lanes=8)
    try:
        q = load_golden("c1_l2_d128")["queries"]
        reqs = _requests(len(q))
        rids = [srv.submit(q[s:s + b], k, ef) for s, b, k, ef in reqs]
        for (s, b, k, ef), rid in zip(reqs, rids):
            got = srv.wait(rid)[:3]
            idx.setQueryTimeParams({"efSearch": ef})
            bi, bd, bc = idx.knnQueryBatchArrays(q[s:s + b], k)
            np.testing.assert_array_equal(got[0], bi)
            np.testing.assert_array_equal(got[2], bc)
    finally:
        srv.close()
    with pytest.raises(MemoryError):
        Server(idx, memory_budget_bytes=8 * lane_staging, max_batch=64, max_k=100, max_lanes=8)
