"""Parity of the CUDA engine (through the C ABI) with the oracle and with the reference's own
recorded outputs, on every committed fixture. Distances must be bit-identical; ids identical to
the oracle (both order equal distances by node index) and identical to the reference except
inside runs of equal distance (the reference orders those by object address)."""
import os
import struct

import numpy as np
import pytest

import nmslib_b200 as nmslib
from nmslib_b200.build import build
from oracle.oracle import OracleIndex

from conftest import ALGO_CODES, assert_same_results, golden_cases, golden_manifest, golden_path, load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    build()


_cache = {}


def _gpu_index(name):
    if name not in _cache:
        space = golden_manifest()[name]["space"]
        idx = nmslib.init(method="hnsw", space=space)
        idx.loadIndex(golden_path(name))
        _cache[name] = idx
    return _cache[name]


def _oracle(name):
    key = ("oracle", name)
    if key not in _cache:
        _cache[key] = OracleIndex(golden_path(name))
    return _cache[key]


@pytest.mark.parametrize("plain", [False, True], ids=["batched", "plain"])
@pytest.mark.parametrize("name,si,k,ef,algo", golden_cases())
def test_gpu_matches_oracle_and_reference(name, si, k, ef, algo, plain):
    g = load_golden(name)
    q = g["queries"]
    idx = _gpu_index(name)
    idx.setQueryTimeParams({"efSearch": ef, "algoType": algo})
    ids, d, cnt, st = idx.knnQueryBatchArrays(q, k, plain=plain, stats=True)
    oi, od, oc, ost = _oracle(name).search(q, k=k, ef=ef, algo=ALGO_CODES[algo])
    np.testing.assert_array_equal(cnt, oc)
    np.testing.assert_array_equal(d.view(np.int32), od.view(np.int32))
    np.testing.assert_array_equal(ids, oi)
    np.testing.assert_array_equal(st, ost)  # same distance evaluations, expansions, bytes
    assert_same_results(ids, d, cnt, g[f"ids_{si}"], g[f"dists_{si}"], g[f"counts_{si}"])


def test_mixed_batch_matches_oracle():
    """One launch with per-query k and ef (both V1Merge and SearchOld queries)."""
    rng = np.random.default_rng(7)
    for name in ("c1_l2_d128", "sift_l2_ties", "negdot_d960"):
        q = load_golden(name)["queries"]
        k = rng.choice([1, 10, 100], size=len(q)).astype(np.int32)
        ef = rng.integers(16, 1100, size=len(q)).astype(np.int32)
        idx = _gpu_index(name)
        idx.setQueryTimeParams({"efSearch": 20})
        ids, d, cnt, st = idx.knnQueryBatchArrays(q, k, ef=ef, stats=True)
        oi, od, oc, ost = _oracle(name).search(q, k_per_q=k, ef_per_q=ef)
        np.testing.assert_array_equal(cnt, oc)
        np.testing.assert_array_equal(d.view(np.int32), od.view(np.int32))
        np.testing.assert_array_equal(ids, oi)
        np.testing.assert_array_equal(st, ost)


def test_repeat_is_deterministic():
    idx = _gpu_index("sift_l2_ties")
    idx.setQueryTimeParams({"efSearch": 64})
    q = load_golden("sift_l2_ties")["queries"]
    a = idx.knnQueryBatchArrays(q, 10)
    for _ in range(3):
        b = idx.knnQueryBatchArrays(q, 10)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)


def test_python_surface_matches_reference_shapes(tmp_path):
    g = load_golden("c1_l2_d128")
    idx = nmslib.init(method="hnsw", space="l2")
    idx.loadIndex(golden_path("c1_l2_d128"))
    # after loadIndex ef is 20 (hnsw.cc:483): setting 1 of the fixture is ef=20
    res = idx.knnQueryBatch(g["queries"][:50], k=10)
    assert len(res) == 50
    for r, (ri, rd) in enumerate(res):
        assert ri.dtype == np.int32 and rd.dtype == np.float32
        np.testing.assert_array_equal(rd, g["dists_1"][r])
    # list input, Fortran-ordered input and knnQuery agree with the array path
    a = idx.knnQueryBatch(np.asfortranarray(g["queries"][:5]), k=10)
    b = idx.knnQueryBatch([list(v) for v in g["queries"][:5]], k=10)
    c = [idx.knnQuery(v, k=10) for v in g["queries"][:5]]
    for x, y, z in zip(a, b, c):
        np.testing.assert_array_equal(x[0], y[0])
        np.testing.assert_array_equal(x[0], z[0])
    with pytest.raises(ValueError, match="dimension"):
        idx.knnQueryBatch(np.zeros((2, 64), np.float32))
    # save -> load round trip gives identical results
    p = str(tmp_path / "re.hnsw")
    idx.saveIndex(p)
    with open(p, "rb") as f1, open(golden_path("c1_l2_d128"), "rb") as f2:
        assert f1.read() == f2.read()
    idx2 = nmslib.init(method="hnsw", space="l2")
    idx2.loadIndex(p)
    res2 = idx2.knnQueryBatch(g["queries"][:50], k=10)
    for x, y in zip(res, res2):
        np.testing.assert_array_equal(x[0], y[0])


def test_empty_index(tmp_path):
    import struct
    p = tmp_path / "empty.hnsw"
    p.write_bytes(struct.pack("<IIiiQQQ", 0, 0, 0, 0, 0, 0, 0))
    idx = nmslib.init(method="hnsw", space="l2")
    idx.loadIndex(str(p))
    res = idx.knnQueryBatch(np.zeros((3, 5), np.float32), k=4)
    assert [len(r[0]) for r in res] == [0, 0, 0]


def test_zero_query_cosine():
    """A zero query is left unnormalised and every cosine distance is 1 (bindings_test.py:72-91)."""
    idx = _gpu_index("cos_d100")
    idx.setQueryTimeParams({"efSearch": 50})
    ids, d = idx.knnQuery(np.zeros(100, np.float32), k=5)
    np.testing.assert_array_equal(d, np.ones(5, np.float32))


@pytest.mark.parametrize("cfg", [(4, 1, -1, -1), (2, 4, 8, -1), (1, 2, 10, -1), (4, 4, 14, -1), (4, 0, -1, 16), (2, 0, 9, 3), (1, 0, -1, 64)],
                         ids=["hbm-visited", "tiny-table-spills", "table-1k", "table-16k", "staged16", "staged3-spill", "staged64"])
@pytest.mark.parametrize("name,si", [("c1_l2_d128", 0), ("sift_l2_ties", 1), ("sift_l2_ties", 2),
                                     ("negdot_d960", 2), ("cos_d100", 0), ("dup_l2_d16", 2)])
def test_launch_shapes_do_not_change_results(name, si, cfg):
    """Every launch shape (visited set in HBM only, a table small enough to spill mid-query,
    different rows in flight and warps per block) gives the oracle's results."""
    k, ef, algo = golden_manifest()[name]["settings"][si]
    q = load_golden(name)["queries"]
    idx = _gpu_index(name)
    idx.setLaunchConfig(*cfg)
    try:
        idx.setQueryTimeParams({"efSearch": ef, "algoType": algo})
        for plain in (False, True):
            ids, d, cnt, st = idx.knnQueryBatchArrays(q, k, plain=plain, stats=True)
            oi, od, oc, ost = _oracle(name).search(q, k=k, ef=ef, algo=ALGO_CODES[algo])
            np.testing.assert_array_equal(ids, oi)
            np.testing.assert_array_equal(d.view(np.int32), od.view(np.int32))
            np.testing.assert_array_equal(st, ost)
    finally:
        idx.setLaunchConfig(0, 0, 0)


def test_cuda_graph_launch_matches():
    """NMSG_CUDA_GRAPH: the captured launch replays with identical results, and a change of
    arguments (efSearch) re-captures."""
    import torch

    from nmslib_b200 import _capi
    idx = _gpu_index("c1_l2_d128")
    lib = _capi.load()
    q = np.ascontiguousarray(load_golden("c1_l2_d128")["queries"])
    nq, dim = q.shape
    dq = torch.from_numpy(q).cuda()
    for ef in (100, 40, 100):
        idx.setQueryTimeParams({"efSearch": ef})
        want = idx.knnQueryBatchArrays(q, 10)
        for _ in range(3):
            ids = torch.full((nq, 10), -7, dtype=torch.int32, device="cuda")
            d = torch.zeros((nq, 10), dtype=torch.float32, device="cuda")
            c = torch.zeros((nq,), dtype=torch.int32, device="cuda")
            rc = lib.nmsg_knn_batch(idx._h, dq.data_ptr(), nq, dim, 10, None, None, 10, ids.data_ptr(),
                                    d.data_ptr(), c.data_ptr(), None,
                                    _capi.FLAG_DEVICE_PTRS | _capi.FLAG_CUDA_GRAPH, None)
            assert rc == 0, _capi.last_error()
            torch.cuda.synchronize()
            np.testing.assert_array_equal(ids.cpu().numpy(), want[0])
            np.testing.assert_array_equal(c.cpu().numpy(), want[2])


def test_concurrent_launches_with_different_shared_memory():
    """Two handles searched from two threads at once, with beams of very different sizes: the
    same kernels launch concurrently with different shared-memory sizes, and neither launch may
    be refused (the shared-memory limit is a process-wide property of each kernel)."""
    import threading
    q = np.ascontiguousarray(load_golden("c1_l2_d128")["queries"])
    handles = []
    for _ in range(2):
        idx = nmslib.init(method="hnsw", space="l2")
        idx.loadIndex(golden_path("c1_l2_d128"))
        handles.append(idx)
    want = []
    for idx, (ef, k) in zip(handles, [(16, 5), (800, 100)]):
        idx.setQueryTimeParams({"efSearch": ef})
        want.append(idx.knnQueryBatchArrays(q, k)[0])
    errors = []

    def run(idx, k, ref):
        try:
            for _ in range(40):
                ids = idx.knnQueryBatchArrays(q, k)[0]
                np.testing.assert_array_equal(ids, ref)
        except Exception as e:  # noqa: BLE001 - reported below
            errors.append(e)

    threads = [threading.Thread(target=run, args=(handles[0], 5, want[0])),
               threading.Thread(target=run, args=(handles[1], 100, want[1]))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors


def test_plain_kernel_slot_wait_gives_up_with_timeout():
    """The one-query-per-block kernel takes a visited-set slot with one bounded pass over the slot
    locks. With a single slot for a whole batch, the blocks that find it taken give up: the call
    reports NMSG_ERR_TIMEOUT (no spin, no fault), and the next call with the normal slot count is
    clean and exact."""
    from nmslib_b200 import _capi
    name = "c1_l2_d128"
    q = load_golden(name)["queries"]
    idx = _gpu_index(name)
    idx.setQueryTimeParams({"efSearch": 100})
    idx.setLaunchConfig(plain_slots=1)
    try:
        with pytest.raises(RuntimeError, match=f"status {_capi.ERR_TIMEOUT}"):
            idx.knnQueryBatchArrays(q, 10, plain=True)
        assert _capi.load().nmsg_last_device_status(idx._h) == _capi.ERR_TIMEOUT
    finally:
        idx.setLaunchConfig()
    oi, od, oc, _ = _oracle(name).search(q, k=10, ef=100)
    for plain in (True, False):
        ids, d, cnt = idx.knnQueryBatchArrays(q, 10, plain=plain)
        np.testing.assert_array_equal(cnt, oc)
        np.testing.assert_array_equal(ids, oi)
        np.testing.assert_array_equal(d.view(np.int32), od.view(np.int32))
    assert _capi.load().nmsg_last_device_status(idx._h) == 0


@pytest.mark.parametrize("row_copy", [1, 2], ids=["cp16", "bulk"])
@pytest.mark.parametrize("qpw", [1, 2, 3, 4])
@pytest.mark.parametrize("stage", [4, 8, 16])
@pytest.mark.parametrize("name,si", [("c1_l2_d128", 0), ("c1_l2_d128", 6), ("sift_l2_ties", 1), ("cos_d100", 0),
                                     ("negdot_d960", 1), ("dup_l2_d16", 2), ("tiny_l2_d20_sqids", 1),
                                     ("one_l2_d3", 0)])
def test_queries_per_warp_do_not_change_results(name, si, stage, qpw, row_copy):
    """Several queries per persistent warp (their list reads, visited checks and row copies
    overlapping) take the single-query steps in the same order: ids, distances and per-query
    counts are the oracle's, for every context count, staging depth and row-copy kind (16-byte
    copies per lane, or one bulk copy per row)."""
    k, ef, algo = golden_manifest()[name]["settings"][si]
    q = load_golden(name)["queries"]
    idx = _gpu_index(name)
    idx.setLaunchConfig(stage_rows=stage, queries_per_warp=qpw, row_copy=row_copy)
    try:
        idx.setQueryTimeParams({"efSearch": ef, "algoType": algo})
        ids, d, cnt, st = idx.knnQueryBatchArrays(q, k, stats=True)
        oi, od, oc, ost = _oracle(name).search(q, k=k, ef=ef, algo=ALGO_CODES[algo])
        np.testing.assert_array_equal(cnt, oc)
        np.testing.assert_array_equal(ids, oi)
        np.testing.assert_array_equal(d.view(np.int32), od.view(np.int32))
        np.testing.assert_array_equal(st, ost)
        # a batch smaller than the warps' contexts, and a single query
        for sub in (q[:37], q[5:6]):
            ids, d, cnt, st = idx.knnQueryBatchArrays(sub, k, stats=True)
            oi, od, oc, ost = _oracle(name).search(sub, k=k, ef=ef, algo=ALGO_CODES[algo])
            np.testing.assert_array_equal(ids, oi)
            np.testing.assert_array_equal(st, ost)
    finally:
        idx.setLaunchConfig()


def test_queries_per_warp_mixed_k_ef():
    """Per-query k and efSearch (all V1Merge) with four queries per warp."""
    name = "c1_l2_d128"
    q = load_golden(name)["queries"]
    rng = np.random.default_rng(7)
    ks = rng.choice([1, 10, 100], len(q)).astype(np.int32)
    efs = rng.integers(0, 600, len(q)).astype(np.int32)
    idx = _gpu_index(name)
    idx.setQueryTimeParams({"efSearch": 20, "algoType": "hybrid"})
    idx.setLaunchConfig(queries_per_warp=4)
    try:
        ids, d, cnt, st = idx.knnQueryBatchArrays(q, ks, ef=efs, stats=True)
    finally:
        idx.setLaunchConfig()
    oi, od, oc, ost = _oracle(name).search(q, k=int(ks.max()), ef=20, k_per_q=ks, ef_per_q=efs)
    np.testing.assert_array_equal(cnt, oc)
    np.testing.assert_array_equal(ids, oi)
    np.testing.assert_array_equal(d.view(np.int32), od.view(np.int32))
    np.testing.assert_array_equal(st, ost)


@pytest.mark.parametrize("stage", [3, 8, 40])
@pytest.mark.parametrize("name,si", [("negdot_d960", 0), ("negdot_d960", 2), ("cos_d100", 1), ("l1_d22", 1),
                                     ("c1_l2_d128", 5), ("sift_l2_ties", 2)])
def test_bulk_row_copies_in_the_general_kernel(name, si, stage):
    """The single-query kernels (SearchOld batches, L1 / LInf, shapes without a lean kernel, the
    plain kernel) with each staged row fetched by one bulk copy: the oracle's results and counts."""
    k, ef, algo = golden_manifest()[name]["settings"][si]
    q = load_golden(name)["queries"]
    idx = _gpu_index(name)
    idx.setLaunchConfig(stage_rows=stage, row_copy=2)
    try:
        idx.setQueryTimeParams({"efSearch": ef, "algoType": algo})
        oi, od, oc, ost = _oracle(name).search(q, k=k, ef=ef, algo=ALGO_CODES[algo])
        for plain in (False, True):
            ids, d, cnt, st = idx.knnQueryBatchArrays(q, k, plain=plain, stats=True)
            np.testing.assert_array_equal(cnt, oc)
            np.testing.assert_array_equal(ids, oi)
            np.testing.assert_array_equal(d.view(np.int32), od.view(np.int32))
            np.testing.assert_array_equal(st, ost)
    finally:
        idx.setLaunchConfig()


def test_lists_that_repeat_an_id(tmp_path):
    """Level-0 lists that name one neighbour twice (the reference visits it once: the second
    occurrence finds it visited). Such a file turns off the lean kernel's duplicate-free fast path;
    ids, distances and per-query counts stay the oracle's. The unmodified fixture, whose lists are
    duplicate-free, takes the fast path in every other test."""
    name = "c1_l2_d128"
    raw = bytearray(open(golden_path(name), "rb").read())
    n, mem, off0 = struct.unpack_from("<IQQ", raw, 4)
    header = 68  # flag, n, mem_per_obj, off_level0, off_data, maxlevel, enterpoint, maxM, maxM0, dist, method
    changed = 0
    for i in range(0, n, 3):
        p = header + i * mem + off0
        cnt = struct.unpack_from("<i", raw, p)[0]
        if cnt >= 3:
            struct.pack_into("<i", raw, p + 12, struct.unpack_from("<i", raw, p + 4)[0])  # ids[2] = ids[0]
            changed += 1
    assert changed > 100
    path = tmp_path / "repeated_ids.hnsw"
    path.write_bytes(bytes(raw))
    idx = nmslib.init(method="hnsw", space="l2")
    idx.loadIndex(str(path))
    orc = OracleIndex(str(path))
    q = load_golden(name)["queries"]
    for ef in (10, 64, 300):
        idx.setQueryTimeParams({"efSearch": ef, "algoType": "v1merge"})
        oi, od, oc, ost = orc.search(q, k=10, ef=ef, algo=ALGO_CODES["v1merge"])
        for plain in (False, True):
            ids, d, cnt, st = idx.knnQueryBatchArrays(q, 10, plain=plain, stats=True)
            np.testing.assert_array_equal(cnt, oc)
            np.testing.assert_array_equal(ids, oi)
            np.testing.assert_array_equal(d.view(np.int32), od.view(np.int32))
            np.testing.assert_array_equal(st, ost)


@pytest.mark.parametrize("row_copy", [2, 1], ids=["bulk", "cp16"])
def test_staged_wide_rows_many_queries_per_warp(row_copy):
    """3840-byte rows staged 8 per round through the general kernel for a batch large enough that
    every warp runs many queries in a row (the row-copy mbarrier is set up once per warp and its
    phase carried from query to query), SearchOld and V1Merge queries mixed: the oracle's results."""
    name = "negdot_d960"
    q = load_golden(name)["queries"]
    reps = max(1, 24000 // len(q))
    big = np.ascontiguousarray(np.tile(q, (reps, 1)))
    rng = np.random.default_rng(11)
    efs = np.tile(rng.integers(16, 1100, len(q)).astype(np.int32), reps)
    ks = np.tile(rng.choice([1, 10, 100], len(q)).astype(np.int32), reps)
    idx = _gpu_index(name)
    idx.setQueryTimeParams({"efSearch": 20, "algoType": "hybrid"})
    idx.setLaunchConfig(stage_rows=8, row_copy=row_copy)
    try:
        ids, d, cnt, st = idx.knnQueryBatchArrays(big, ks, ef=efs, stats=True)
    finally:
        idx.setLaunchConfig()
    oi, od, oc, ost = _oracle(name).search(q, k=int(ks.max()), ef=20, k_per_q=ks[:len(q)], ef_per_q=efs[:len(q)])
    np.testing.assert_array_equal(cnt, np.tile(oc, reps))
    np.testing.assert_array_equal(ids, np.tile(oi, (reps, 1)))
    np.testing.assert_array_equal(d.view(np.int32), np.tile(od, (reps, 1)).view(np.int32))
    np.testing.assert_array_equal(st, np.tile(ost, (reps, 1)))


@pytest.mark.parametrize("order", [0, -1], ids=["split", "one-pass"])
@pytest.mark.parametrize("name,si", [("c1_l2_d128", 0), ("c1_l2_d128", 3), ("c1_l2_d128", 6), ("sift_l2_ties", 0),
                                     ("dup_l2_d16", 2), ("tiny_cos_d48", 0), ("cos_d100", 0), ("negdot_d960", 0),
                                     ("l1_d22", 0), ("linf_d128", 0), ("tiny_l2_d20_sqids", 0)])
def test_batches_larger_than_the_resident_warps(name, si, order):
    """A V1Merge batch with more queries than resident warps: by default the lean kernel (and the
    general kernel for the other row shapes and distances) runs every query's upper-level descent
    first, orders the queries by their level-0 entry distance and then searches level 0 from the
    stored entries (query_order -1: one pass in batch order). Either way ids, distances and
    per-query counts (the descent's included) are the oracle's."""
    k, ef, algo = golden_manifest()[name]["settings"][si]
    q = load_golden(name)["queries"]
    reps = -(-12000 // len(q))
    big = np.ascontiguousarray(np.tile(q, (reps, 1)))
    idx = _gpu_index(name)
    idx.setLaunchConfig(query_order=order)
    try:
        idx.setQueryTimeParams({"efSearch": ef, "algoType": algo})
        ids, d, cnt, st = idx.knnQueryBatchArrays(big, k, stats=True)
    finally:
        idx.setLaunchConfig()
    oi, od, oc, ost = _oracle(name).search(q, k=k, ef=ef, algo=ALGO_CODES[algo])
    np.testing.assert_array_equal(cnt, np.tile(oc, reps))
    np.testing.assert_array_equal(ids, np.tile(oi, (reps, 1)))
    np.testing.assert_array_equal(d.view(np.int32), np.tile(od, (reps, 1)).view(np.int32))
    np.testing.assert_array_equal(st, np.tile(ost, (reps, 1)))


def test_cuda_graph_replays_the_split_search():
    """NMSG_CUDA_GRAPH with a batch larger than the resident warps: the captured sequence (descent,
    order, level 0) replays with the results of the uncaptured search."""
    import torch

    from nmslib_b200 import _capi
    idx = _gpu_index("c1_l2_d128")
    lib = _capi.load()
    q = np.ascontiguousarray(np.tile(load_golden("c1_l2_d128")["queries"], (12, 1)))
    nq, dim = q.shape
    dq = torch.from_numpy(q).cuda()
    idx.setQueryTimeParams({"efSearch": 64})
    want = idx.knnQueryBatchArrays(q, 10)
    for _ in range(3):
        ids = torch.full((nq, 10), -7, dtype=torch.int32, device="cuda")
        d = torch.zeros((nq, 10), dtype=torch.float32, device="cuda")
        c = torch.zeros((nq,), dtype=torch.int32, device="cuda")
        rc = lib.nmsg_knn_batch(idx._h, dq.data_ptr(), nq, dim, 10, None, None, 10, ids.data_ptr(),
                                d.data_ptr(), c.data_ptr(), None,
                                _capi.FLAG_DEVICE_PTRS | _capi.FLAG_CUDA_GRAPH, None)
        assert rc == 0, _capi.last_error()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(ids.cpu().numpy(), want[0])
        np.testing.assert_array_equal(d.cpu().numpy().view(np.int32), want[1].view(np.int32))
        np.testing.assert_array_equal(c.cpu().numpy(), want[2])


@pytest.mark.parametrize("rows", [1000, 2049, 12000])
def test_host_copies_staged_and_direct(rows):
    """Host-buffer batches of 512 KB and more travel through page-locked staging that host threads
    fill in 1 MB chunks (host_copy 0, the default); host_copy 1 copies the caller's arrays
    directly, and page-locked caller arrays are copied directly either way. Per-query k and
    efSearch arrays travel with the queries. Every route returns the oracle's results."""
    import torch

    name = "c1_l2_d128"
    q0 = load_golden(name)["queries"]
    reps = -(-rows // len(q0))
    base = np.arange(rows) % len(q0)
    q = np.ascontiguousarray(np.tile(q0, (reps, 1))[:rows])
    rng = np.random.default_rng(rows)
    ks = rng.choice([1, 10, 32], size=rows).astype(np.int32)
    efs = rng.choice([10, 64, 100], size=rows).astype(np.int32)
    pinned = torch.empty(q.shape, dtype=torch.float32, pin_memory=True).numpy()
    pinned[:] = q
    idx = _gpu_index(name)
    orc = _oracle(name)
    want = {}
    for kk in (1, 10, 32):
        for ee in (10, 64, 100):
            want[kk, ee] = orc.search(q0, k=kk, ef=ee, algo=ALGO_CODES["v1merge"])
    try:
        idx.setQueryTimeParams({"efSearch": 64, "algoType": "v1merge"})
        for host_copy in (0, 1):
            idx.setLaunchConfig(host_copy=host_copy)
            for arr in (q, pinned):
                ids, d, cnt, st = idx.knnQueryBatchArrays(arr, 10, stats=True)
                oi, od, oc, ost = want[10, 64]
                np.testing.assert_array_equal(cnt, oc[base])
                np.testing.assert_array_equal(ids, oi[base])
                np.testing.assert_array_equal(d.view(np.int32), od[base].view(np.int32))
                np.testing.assert_array_equal(st, ost[base])
                ids, d, cnt = idx.knnQueryBatchArrays(arr, ks, ef=efs)
                for (kk, ee), (oi, od, oc, _) in want.items():
                    m = (ks == kk) & (efs == ee)
                    b = base[m]
                    np.testing.assert_array_equal(cnt[m], oc[b])
                    live = np.arange(kk)[None, :] < oc[b][:, None]
                    np.testing.assert_array_equal(np.where(live, ids[m, :kk], -1), np.where(live, oi[b], -1))
                    np.testing.assert_array_equal(np.where(live, d[m, :kk].view(np.int32), 0),
                                                  np.where(live, od[b].view(np.int32), 0))
    finally:
        idx.setLaunchConfig()


def test_kernel_launch_count_of_the_last_batch():
    """nmsg_last_kernel_launches: one launch for a batch that fits the resident warps, for the
    one-query-per-block kernel and with query_order -1; three (descent, entry order, level 0) for a
    larger V1Merge batch copied directly, four when its queries travel in two halves (pageable ones
    through staging, page-locked ones directly; the descent split in two)."""
    from nmslib_b200 import _capi

    lib = _capi.load()
    idx = _gpu_index("c1_l2_d128")
    q = load_golden("c1_l2_d128")["queries"]
    big = np.ascontiguousarray(np.tile(q, (-(-12000 // len(q)), 1)))
    idx.setQueryTimeParams({"efSearch": 64, "algoType": "v1merge"})
    idx.knnQueryBatchArrays(q[:100], 10)
    assert lib.nmsg_last_kernel_launches(idx._h) == 1
    idx.knnQueryBatchArrays(q[:100], 10, plain=True)
    assert lib.nmsg_last_kernel_launches(idx._h) == 1
    idx.knnQueryBatchArrays(big, 10)
    assert lib.nmsg_last_kernel_launches(idx._h) == 4
    import torch

    pinned = torch.empty(big.shape, dtype=torch.float32, pin_memory=True).numpy()
    pinned[:] = big
    got = idx.knnQueryBatchArrays(pinned, 10)  # page-locked: two halves copied directly
    assert lib.nmsg_last_kernel_launches(idx._h) == 4
    want = idx.knnQueryBatchArrays(big, 10)
    for g, w in zip(got, want):
        np.testing.assert_array_equal(g, w)
    idx.setLaunchConfig(host_copy=1)
    try:
        idx.knnQueryBatchArrays(big, 10)
        assert lib.nmsg_last_kernel_launches(idx._h) == 3
    finally:
        idx.setLaunchConfig()
    idx.setLaunchConfig(query_order=-1)
    try:
        idx.knnQueryBatchArrays(big, 10)
        assert lib.nmsg_last_kernel_launches(idx._h) == 1
    finally:
        idx.setLaunchConfig()
    idx.knnQueryBatchArrays(q[:0], 10)
    assert lib.nmsg_last_kernel_launches(idx._h) == 0


def test_host_buffers_on_a_caller_stream():
    """nmsg_knn_batch with pageable host buffers on the caller's own stream, which still has work
    queued: a batch larger than the resident warps copies its queries in two halves on the
    handle's copy stream after that work, and returns the results of the default-stream call."""
    import ctypes

    import torch

    from nmslib_b200 import _capi

    lib = _capi.load()
    idx = _gpu_index("c1_l2_d128")
    q0 = load_golden("c1_l2_d128")["queries"]
    q = np.ascontiguousarray(np.tile(q0, (-(-12000 // len(q0)), 1)))
    nq, dim = q.shape
    idx.setQueryTimeParams({"efSearch": 64, "algoType": "v1merge"})
    want = idx.knnQueryBatchArrays(q, 10)
    s = torch.cuda.Stream()
    busy = torch.empty(1 << 28, dtype=torch.uint8, device="cuda")
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    for _ in range(2):
        with torch.cuda.stream(s):
            busy.fill_(7)  # earlier work on the caller's stream
        ids = np.full((nq, 10), -7, np.int32)
        d = np.zeros((nq, 10), np.float32)
        c = np.zeros(nq, np.int32)
        rc = lib.nmsg_knn_batch(idx._h, ptr(q), nq, dim, 10, None, None, 10, ptr(ids), ptr(d), ptr(c), None, 0,
                                s.cuda_stream)
        assert rc == 0, _capi.last_error()
        assert lib.nmsg_last_kernel_launches(idx._h) == 4
        np.testing.assert_array_equal(c, want[2])
        np.testing.assert_array_equal(ids, want[0])
        np.testing.assert_array_equal(d.view(np.int32), want[1].view(np.int32))
