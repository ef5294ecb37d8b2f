"""l2sqr_sift in the engine (uint8 rows, int distances, regular graph + objects file), on the GPU
through the C ABI: parity with the oracle's restatement of the reference's generic search (ids,
int distances and per-query traversal counts identical) and with the reference's recorded
knnQueryBatch output on the committed reference-built fixtures.

The reference orders equal distances by Object address (its objects are separate allocations made
while loading the objects file), the engine and the oracle by node index; against the reference
the comparison is therefore exact for every distance and for the ids below the k-th distance, and
by count at the k-th distance (as in the oracle's own pinning test)."""
import json
import os

import numpy as np
import pytest

import nmslib_b200 as nmslib
from nmslib_b200.build import build
from oracle.oracle import OracleSiftIndex

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ALGO = {"hybrid": 0, "old": 1, "v1merge": 2}


@pytest.fixture(scope="module", autouse=True)
def _built():
    build()


def _manifest():
    with open(os.path.join(HERE, "manifest_sift.json")) as f:
        return json.load(f)


def _cases():
    return [(name, si) for name, c in _manifest().items() for si in range(len(c["settings"]))]


_cache = {}


def _index(name):
    if name not in _cache:
        idx = nmslib.init(method="hnsw", space="l2sqr_sift", data_type=nmslib.DataType.DENSE_UINT8_VECTOR,
                          dtype=nmslib.DistType.INT)
        idx.loadIndex(os.path.join(HERE, name + ".hnsw"), load_data=True)
        _cache[name] = idx
    return _cache[name]


def _oracle(name):
    key = ("oracle", name)
    if key not in _cache:
        _cache[key] = OracleSiftIndex(os.path.join(HERE, name + ".hnsw"))
    return _cache[key]


def assert_same_up_to_address_ties(ids, dists, counts, want_ids, want_dists, want_counts):
    np.testing.assert_array_equal(counts, want_counts)
    for qi in range(len(counts)):
        c = counts[qi]
        d, i = dists[qi, :c], ids[qi, :c]
        wd, wi = want_dists[qi, :c], want_ids[qi, :c]
        np.testing.assert_array_equal(d, wd)
        if c == 0:
            continue
        np.testing.assert_array_equal(np.sort(i[d < d[-1]]), np.sort(wi[wd < wd[-1]]))
        assert len(set(i.tolist())) == c


@pytest.mark.parametrize("plain", [False, True], ids=["batched", "plain"])
@pytest.mark.parametrize("name,si", _cases())
def test_sift_gpu_matches_oracle_and_reference(name, si, plain):
    k, ef, algo = _manifest()[name]["settings"][si]
    g = np.load(os.path.join(HERE, name + ".npz"))
    q = g["queries"]
    idx = _index(name)
    idx.setQueryTimeParams({"efSearch": ef, "algoType": algo})
    ids, d, cnt, st = idx.knnQueryBatchArrays(q, k, plain=plain, stats=True)
    oi, od, oc, ost = _oracle(name).search(q, k, ef, ALGO[algo], stats=True)
    np.testing.assert_array_equal(cnt, oc)
    np.testing.assert_array_equal(ids, oi)
    np.testing.assert_array_equal(d, od)
    np.testing.assert_array_equal(st, ost)  # the same traversal, not only the same answer
    assert_same_up_to_address_ties(ids, d, cnt, g[f"ids_{si}"], g[f"dists_{si}"], g[f"counts_{si}"])


def test_sift_exact_where_no_ties():
    """Without tied distances the engine reproduces the reference's output exactly, order included."""
    g = np.load(os.path.join(HERE, "sift_u8_d128.npz"))
    idx = _index("sift_u8_d128")
    for si, (k, ef, algo) in enumerate(_manifest()["sift_u8_d128"]["settings"]):
        idx.setQueryTimeParams({"efSearch": ef, "algoType": algo})
        ids, d, cnt = idx.knnQueryBatchArrays(g["queries"], k)
        np.testing.assert_array_equal(ids, g[f"ids_{si}"])
        np.testing.assert_array_equal(d, g[f"dists_{si}"])


def test_sift_python_surface_and_round_trip(tmp_path):
    name = "sift_u8_d128"
    g = np.load(os.path.join(HERE, name + ".npz"))
    idx = _index(name)
    idx.setQueryTimeParams({"efSearch": 40})
    res = idx.knnQueryBatch(g["queries"], k=10)
    assert len(res) == len(g["queries"])
    assert res[0][0].dtype == np.int32 and res[0][1].dtype == np.int32
    one = idx.knnQuery(g["queries"][3], k=10)
    np.testing.assert_array_equal(one[0], res[3][0])
    # saveIndex(save_data=True) writes the reference's two files byte for byte
    p = str(tmp_path / "re.hnsw")
    idx.saveIndex(p, save_data=True)
    for suffix in ("", ".dat"):
        with open(p + suffix, "rb") as f1, open(os.path.join(HERE, name + ".hnsw" + suffix), "rb") as f2:
            assert f1.read() == f2.read(), suffix
    # the graph file without load_data needs the objects: the reference's message
    bare = nmslib.init(method="hnsw", space="l2sqr_sift", data_type=nmslib.DataType.DENSE_UINT8_VECTOR,
                       dtype=nmslib.DistType.INT)
    with pytest.raises(Exception, match="Did you forget to re-load data"):
        bare.loadIndex(p)
    # objects added first, then the graph alone: the same index
    raw = open(p + ".dat", "rb").read()
    n = int(np.frombuffer(raw[:8], np.uint64)[0])
    rows = np.stack([np.frombuffer(raw, np.uint8, 128, 8 + i * 156 + 24) for i in range(n)])
    bare.addDataPointBatch(rows)
    bare.loadIndex(p)
    bare.setQueryTimeParams({"efSearch": 40})
    res2 = bare.knnQueryBatch(g["queries"], k=10)
    for a, b in zip(res, res2):
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1], b[1])


def test_sift_mixed_batch_matches_oracle():
    """Per-query k and efSearch in one launch (SearchOld for ef >= 1000 under hybrid)."""
    name = "sift_u8_ties"
    q = np.load(os.path.join(HERE, name + ".npz"))["queries"]
    rng = np.random.default_rng(5)
    ks = rng.choice([1, 10, 30], len(q)).astype(np.int32)
    efs = rng.choice([10, 64, 300, 1000], len(q)).astype(np.int32)
    idx = _index(name)
    idx.setQueryTimeParams({"efSearch": 20})
    ids, d, cnt = idx.knnQueryBatchArrays(q, ks, ef=efs)
    o = _oracle(name)
    for i in range(len(q)):
        oi, od, oc = o.search(q[i:i + 1], int(ks[i]), int(efs[i]), 0)
        assert cnt[i] == oc[0]
        np.testing.assert_array_equal(ids[i, :cnt[i]], oi[0, :cnt[i]])
        np.testing.assert_array_equal(d[i, :cnt[i]], od[0, :cnt[i]])


def test_sift_rejects_float_paths():
    idx = _index("sift_u8_tiny")
    from nmslib_b200 import _capi
    lib = _capi.load()
    q = np.zeros((2, 128), np.float32)
    out = np.zeros(20, np.int32)
    rc = lib.nmsg_knn_batch(idx._h, q.ctypes.data, 2, 128, 10, None, None, 10, out.ctypes.data, out.ctypes.data,
                            out.ctypes.data, None, 0, None)
    assert rc == _capi.ERR_BAD_ARG and "nmsg_knn_batch_u8" in _capi.last_error()
    rc = lib.nmsg_bruteforce_knn(idx._h, q.ctypes.data, 2, 128, 10, 10, out.ctypes.data, out.ctypes.data,
                                 out.ctypes.data, None, 0, None)
    assert rc == _capi.ERR_UNSUPPORTED
    with pytest.raises(ValueError):
        idx.knnQueryBatchArrays(np.zeros((2, 64), np.uint8), 5)


@pytest.mark.parametrize("name,si", [c for c in _cases() if _manifest()[c[0]]["settings"][c[1]][2] != "old"
                                     and _manifest()[c[0]]["settings"][c[1]][1] < 1000])
def test_sift_batch_larger_than_the_resident_warps(name, si):
    """A V1Merge batch of uint8 queries with more queries than resident warps (descent pass, order by
    entry distance, level-0 pass): ids, int distances and per-query counts are the oracle's."""
    k, ef, algo = _manifest()[name]["settings"][si]
    q = np.load(os.path.join(HERE, name + ".npz"))["queries"]
    reps = -(-12000 // len(q))
    big = np.ascontiguousarray(np.tile(q, (reps, 1)))
    idx = _index(name)
    idx.setQueryTimeParams({"efSearch": ef, "algoType": algo})
    ids, d, cnt, st = idx.knnQueryBatchArrays(big, k, stats=True)
    oi, od, oc, ost = _oracle(name).search(q, k, ef, ALGO[algo], stats=True)
    np.testing.assert_array_equal(cnt, np.tile(oc, reps))
    np.testing.assert_array_equal(ids, np.tile(oi, (reps, 1)))
    np.testing.assert_array_equal(d, np.tile(od, (reps, 1)))
    np.testing.assert_array_equal(st, np.tile(ost, (reps, 1)))
