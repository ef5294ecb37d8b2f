"""Parity of the lean kernel's instantiations that the reference-built fixtures do not reach: rows
of 64, 96 and 256 floats, and level-0 lists of more than 32 ids (M 24 and 32: lists of up to 48
and 64), for each of its three distances. The indices are built by the engine's host builder (the
same file format the reference writes); the oracle searches the same files. Ids, distances and
per-query counts must be identical, for single batches (one pass) and for a batch larger than the
resident warps (descent pass, order, level-0 pass)."""
import numpy as np
import pytest

import nmslib_b200 as nmslib
from nmslib_b200 import SPACES, _capi
from nmslib_b200.build import build
from oracle.oracle import OracleIndex

from conftest import ALGO_CODES

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    build()


def _compare(got, want, reps=1):
    ids, d, cnt, st = got
    oi, od, oc, ost = want
    np.testing.assert_array_equal(cnt, np.tile(oc, reps))
    np.testing.assert_array_equal(ids, np.tile(oi, (reps, 1)))
    np.testing.assert_array_equal(d.view(np.int32), np.tile(od, (reps, 1)).view(np.int32))
    np.testing.assert_array_equal(st, np.tile(ost, (reps, 1)))


@pytest.mark.parametrize("space", ["l2", "cosinesimil", "negdotprod"])
@pytest.mark.parametrize("dim,m", [(16, 24), (48, 8), (64, 8), (64, 24), (96, 16), (96, 32), (128, 32),
                                   (256, 8), (256, 24)])
def test_lean_shapes_match_oracle(tmp_path, space, dim, m):
    rng = np.random.default_rng(dim * 100 + m)
    n, nq = 3000, 300
    base = rng.standard_normal((n, dim)).astype(np.float32)
    q = rng.standard_normal((nq, dim)).astype(np.float32)
    path = str(tmp_path / f"lean_{space}_{dim}_{m}.hnsw")
    _capi.build_index(base, SPACES[space], m, 64, nthreads=0, out_path=path)
    idx = nmslib.init(method="hnsw", space=space)
    idx.loadIndex(path)
    orc = OracleIndex(path)
    for ef, k in ((10, 10), (64, 10), (40, 100)):
        idx.setQueryTimeParams({"efSearch": ef, "algoType": "v1merge"})
        want = orc.search(q, k=k, ef=ef, algo=ALGO_CODES["v1merge"])
        _compare(idx.knnQueryBatchArrays(q, k, stats=True), want)
    # more queries than resident warps: the split search
    reps = 20
    big = np.ascontiguousarray(np.tile(q, (reps, 1)))
    idx.setQueryTimeParams({"efSearch": 64, "algoType": "v1merge"})
    want = orc.search(q, k=10, ef=64, algo=ALGO_CODES["v1merge"])
    _compare(idx.knnQueryBatchArrays(big, 10, stats=True), want, reps)
