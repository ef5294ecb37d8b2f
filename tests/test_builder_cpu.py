"""The engine's host HNSW builder writes files that the reference format reader, the oracle and
the reference module all accept, with recall in the reference's range."""
import os

import numpy as np
import pytest

from nmslib_b200 import SPACES, _capi
from nmslib_b200.build import build
from nmslib_b200.datasets import mixture
from oracle.oracle import OracleIndex, bruteforce_fp64, normalize, recall, reference_module


@pytest.fixture(scope="module", autouse=True)
def _built():
    build()


@pytest.mark.parametrize("space,dim,m", [("l2", 128, 16), ("l2", 20, 8), ("cosinesimil", 100, 24),
                                         ("negdotprod", 96, 16)])
def test_builder_file_is_valid_and_searchable(tmp_path, space, dim, m):
    kind = {"l2": "gauss", "cosinesimil": "glove", "negdotprod": "absgauss"}[space]
    x = mixture(kind, 3_300, dim, 20, 5, 0.3)
    base, q = x[:3_000], x[3_000:]
    ids = (np.arange(3_000) * 7 + 3).astype(np.int32)
    p = str(tmp_path / "b.hnsw")
    _capi.build_index(base, SPACES[space], m, 100, ids=ids, nthreads=4, out_path=p)
    ix = OracleIndex(p)
    assert ix.info["maxM"] == m and ix.info["maxM0"] == 2 * m and ix.n == 3_000 and ix.dim == dim
    vecs, ext, l0, lev = ix.export()
    np.testing.assert_array_equal(ext, ids)
    assert (l0[:, 0] >= 1).all() and (l0[:, 0] <= 2 * m).all()
    assert lev.max() == ix.info["maxlevel"] and lev[ix.info["enterpoint"]] == ix.info["maxlevel"]
    if space == "cosinesimil":  # stored rows are the reference's float normalisation
        for i in range(0, 3_000, 97):
            np.testing.assert_array_equal(vecs[i], normalize(base[i]))
    else:
        np.testing.assert_array_equal(vecs, base)
    true_i, _ = bruteforce_fp64(base, q, 10, space, ids=ids)
    fi, fd, fc, _ = ix.search(q, k=10, ef=100)
    assert recall(fi, true_i, fc) >= 0.95
    ref = reference_module()
    if ref is not None:  # the reference loads the file and returns the oracle's distances
        r = ref.init(method="hnsw", space=space)
        r.loadIndex(p)
        r.setQueryTimeParams({"efSearch": 100})
        res = r.knnQueryBatch(q, k=10, num_threads=2)
        for row, (ri, rd) in enumerate(res):
            np.testing.assert_array_equal(rd, fd[row, : len(rd)])


def test_builder_empty_and_errors(tmp_path):
    p = str(tmp_path / "e.hnsw")
    _capi.build_index(np.zeros((0, 8), np.float32), SPACES["l2"], 16, 100, out_path=p)
    with open(p, "rb") as f:
        assert f.read(8) == b"\0" * 8  # regular-format header of an empty index
    with pytest.raises(ValueError):
        _capi.build_index(np.zeros((10, 8), np.float32), SPACES["l2"], 1, 100, out_path=p)
