"""The Thrift query server (NMSLIB's QueryService, query_server/protocol.thrift) in front of the
engine, driven over TCP by a binary-protocol client: every reply equals the engine's own batch
search through the C ABI, in the reference server's shape (ascending ReplyEntry lists,
QueryService_server.cpp:392-440), and errors come back as QueryException / application
exceptions the way the reference's server sends them."""
import os
import threading

import numpy as np
import pytest

import nmslib_b200 as nmslib
from nmslib_b200.build import build
from nmslib_b200.query_server import QueryServer
from oracle.oracle import OracleIndex

from conftest import golden_path, load_golden
from thrift_client import ApplicationException, QueryClient, QueryException

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _text(v):
    return " ".join(repr(float(x)) for x in v)


@pytest.fixture(scope="module")
def served():
    build()
    idx = nmslib.init(method="hnsw", space="l2")
    idx.loadIndex(golden_path("c1_l2_d128"))
    idx.setQueryTimeParams({"efSearch": 100})
    srv = QueryServer(idx, port=0, max_connections=8)
    yield idx, srv
    srv.stop()


def _same(entries, ids, dists, cnt):
    assert len(entries) == cnt
    assert [e["id"] for e in entries] == ids[:cnt].tolist()
    np.testing.assert_array_equal(np.array([e["dist"] for e in entries], np.float32), dists[:cnt])


def test_knn_query_and_batch_match_the_engine(served):
    idx, srv = served
    q = load_golden("c1_l2_d128")["queries"][:40]
    ids, d, cnt = idx.knnQueryBatchArrays(q, 10)
    c = QueryClient("127.0.0.1", srv.port)
    try:
        for i in range(5):
            _same(c.knnQuery(10, _text(q[i])), ids[i], d[i], cnt[i])
        batch = c.knnQueryBatch(10, [_text(v) for v in q])
        for i in range(len(q)):
            _same(batch[i], ids[i], d[i], cnt[i])
        # the text form accepts ',' and ':' as separators and a label prefix
        _same(c.knnQuery(10, "label:7 " + ",".join(repr(float(x)) for x in q[3])), ids[3], d[3], cnt[3])
    finally:
        c.close()


def test_extern_ids_and_objects(served):
    idx, srv = served
    vecs, ext, _, _ = OracleIndex(golden_path("c1_l2_d128")).export()
    q = load_golden("c1_l2_d128")["queries"][0]
    c = QueryClient("127.0.0.1", srv.port)
    try:
        res = c.knnQuery(5, _text(q), retExternId=True, retObj=True)
    finally:
        c.close()
    for e in res:
        assert e["externId"] == str(e["id"])
        row = np.array([float(x) for x in e["obj"].decode().split()], np.float32)
        np.testing.assert_array_equal(row, vecs[list(ext).index(e["id"])])  # max_digits10: exact


def test_query_time_params_and_errors(served):
    idx, srv = served
    q = load_golden("c1_l2_d128")["queries"][:20]
    c = QueryClient("127.0.0.1", srv.port, strict=False)  # the old message header is accepted too
    try:
        for params, ef, algo in (("efSearch=300", 300, "hybrid"), ("ef=40,algoType=old", 40, "old"),
                                 ("efSearch=1200", 1200, "hybrid")):
            c.setQueryTimeParams(params)
            idx.setQueryTimeParams({"efSearch": ef, "algoType": algo})
            ids, d, cnt = idx.knnQueryBatchArrays(q, 10)
            batch = c.knnQueryBatch(10, [_text(v) for v in q])
            for i in range(len(q)):
                _same(batch[i], ids[i], d[i], cnt[i])
        # k above the serving loop's limit goes straight to the batch search
        ids, d, cnt = idx.knnQueryBatchArrays(q[:3], 150)
        for i, e in enumerate(c.knnQueryBatch(150, [_text(v) for v in q[:3]])):
            _same(e, ids[i], d[i], cnt[i])
        with pytest.raises(QueryException, match="Unknown parameters found"):
            c.setQueryTimeParams("efSearch=10,bogus=1")
        with pytest.raises(QueryException, match="synonyms"):
            c.setQueryTimeParams("ef=10,efSearch=20")
        with pytest.raises(QueryException, match="Range search is not supported"):
            c.rangeQuery(1.0, _text(q[0]))
        with pytest.raises(QueryException, match="dimension"):
            c.knnQuery(10, "1 2 3")
        with pytest.raises(ApplicationException) as ei:
            c.call_unknown("noSuchMethod")
        assert ei.value.kind == 1  # UNKNOWN_METHOD
        # the connection keeps working after errors
        c.setQueryTimeParams("efSearch=100")
        idx.setQueryTimeParams({"efSearch": 100})
        ids, d, cnt = idx.knnQueryBatchArrays(q[:1], 10)
        _same(c.knnQuery(10, _text(q[0])), ids[0], d[0], cnt[0])
    finally:
        c.close()


def test_get_distance(served):
    _, srv = served
    rng = np.random.default_rng(3)
    a, b = rng.standard_normal(128).astype(np.float32), rng.standard_normal(128).astype(np.float32)
    c = QueryClient("127.0.0.1", srv.port)
    try:
        got = c.getDistance(_text(a), _text(b))
    finally:
        c.close()
    want = float(np.sqrt(((a.astype(np.float64) - b) ** 2).sum()))  # the l2 space's (unsquared) norm
    assert abs(got - want) <= 1e-9 * want


def test_concurrent_clients(served):
    idx, srv = served
    q = load_golden("c1_l2_d128")["queries"][:64]
    idx.setQueryTimeParams({"efSearch": 100})
    ids, d, cnt = idx.knnQueryBatchArrays(q, 10)
    errors = []

    def client(part):
        try:
            c = QueryClient("127.0.0.1", srv.port)
            for rep in range(5):
                rows = list(range(part, len(q), 4))
                res = c.knnQueryBatch(10, [_text(q[i]) for i in rows])
                for r, i in zip(res, rows):
                    _same(r, ids[i], d[i], cnt[i])
            c.close()
        except Exception as e:  # noqa: BLE001 - reported below
            errors.append(e)

    ts = [threading.Thread(target=client, args=(p,)) for p in range(4)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errors, errors


def test_sift_index_served():
    build()
    name = "sift_u8_d128"
    g = np.load(os.path.join(HERE, name + ".npz"))
    idx = nmslib.init(method="hnsw", space="l2sqr_sift", data_type=nmslib.DataType.DENSE_UINT8_VECTOR,
                      dtype=nmslib.DistType.INT)
    idx.loadIndex(os.path.join(HERE, name + ".hnsw"), load_data=True)
    idx.setQueryTimeParams({"efSearch": 40})
    ids, d, cnt = idx.knnQueryBatchArrays(g["queries"][:10], 10)
    with QueryServer(idx) as srv:
        c = QueryClient("127.0.0.1", srv.port)
        try:
            res = c.knnQueryBatch(10, [" ".join(str(int(x)) for x in v) for v in g["queries"][:10]])
            for i, r in enumerate(res):
                assert [e["id"] for e in r] == ids[i, :cnt[i]].tolist()
                assert [e["dist"] for e in r] == d[i, :cnt[i]].astype(float).tolist()
            with pytest.raises(QueryException, match="Non-integer"):
                c.knnQuery(5, " ".join(["1.5"] * 128))
            assert c.getDistance(" ".join(["1"] * 128), " ".join(["3"] * 128)) == 4 * 128
        finally:
            c.close()
