"""The device-assisted builder (nmsg_build_index_device): the file it writes is a valid optimized
index whose search quality matches a host build of the same data and parameters, the oracle finds
exactly what the engine finds in it, and the reference reads it."""
import numpy as np
import pytest

import nmslib_b200 as nmslib
from nmslib_b200 import _capi
from nmslib_b200.build import build
from nmslib_b200.datasets import mixture
from oracle.oracle import OracleIndex, bruteforce_fp64, recall, reference_module

pytestmark = pytest.mark.gpu

KIND = {"l2": "gauss", "cosinesimil": "glove", "negdotprod": "absgauss"}


@pytest.mark.parametrize("space", ["l2", "cosinesimil", "negdotprod"])
def test_device_build_matches_host_build(tmp_path, space):
    build()
    x = mixture(KIND[space], 30_200, 48, 60, 7, 0.4)
    base, q = x[:30_000], x[30_000:]
    found = {}
    for dev in (None, 0):
        p = str(tmp_path / f"{space}_{'dev' if dev is not None else 'host'}.hnsw")
        _capi.build_index(base, nmslib.SPACES[space], 12, 100, nthreads=0, seed=3, out_path=p, device=dev)
        idx = nmslib.init(method="hnsw", space=space)
        idx.loadIndex(p)
        assert idx.info["n"] == len(base)
        idx.setQueryTimeParams({"efSearch": 64})
        ids, d, cnt = idx.knnQueryBatchArrays(q, 10)
        found[dev] = (p, ids, d)
    true_i, _ = bruteforce_fp64(base, q, 10, space)
    r_host, r_dev = recall(found[None][1], true_i), recall(found[0][1], true_i)
    assert r_dev >= r_host - 0.02, (r_host, r_dev)
    # the device-built file: the oracle's restatement of the query path finds the same lists
    p, ids, d = found[0]
    oi, od, oc, _ = OracleIndex(p).search(q, k=10, ef=64)
    np.testing.assert_array_equal(oi, ids)
    np.testing.assert_array_equal(od, d)
    ref = reference_module()
    if ref is not None:  # and the reference's own loader and search accept it
        r = ref.init(method="hnsw", space=space)
        r.loadIndex(p)
        r.setQueryTimeParams({"efSearch": 64})
        for i, (ri, rd) in enumerate(r.knnQueryBatch(q[:20], k=10, num_threads=1)):
            np.testing.assert_array_equal(rd, d[i, : len(rd)])


def test_device_build_through_create_index():
    build()
    x = mixture("gauss", 8_100, 32, 20, 9, 0.4)
    idx = nmslib.init(method="hnsw", space="l2")
    idx.addDataPointBatch(x[:8_000], ids=np.arange(8_000) * 3)
    idx.createIndex({"M": 8, "efConstruction": 60, "gpuBuild": 1})
    idx.setQueryTimeParams({"efSearch": 50})
    ids, d, cnt = idx.knnQueryBatchArrays(x[8_000:], 5)
    true_i, _ = bruteforce_fp64(x[:8_000], x[8_000:], 5, "l2", ids=np.arange(8_000) * 3)
    assert recall(ids, true_i) > 0.9
