"""The tensor-core brute-force k-NN against an exact float64 scan of the same stored vectors:
identical ids (ties by id) and distances within float rounding."""
import numpy as np
import pytest

import nmslib_b200 as nmslib
from nmslib_b200 import _capi
from nmslib_b200.build import build
from oracle.oracle import OracleIndex, dist, normalize

from conftest import golden_manifest, golden_path, load_golden

pytestmark = pytest.mark.gpu


def fp64_topk(name_or_path, queries, k, space):
    """Exact top-k over the index's stored vectors in float64: keys q.x (cosine: the query
    normalised as the engine normalises it; negdot) or 2 q.x - |x|^2 (l2); ties by node index."""
    ix = OracleIndex(name_or_path)
    vecs, ext, _, _ = ix.export()
    x = vecs.astype(np.float64)
    out_i, out_d = [], []
    for q in queries:
        qf = normalize(q) if space == "cosinesimil" else np.asarray(q, np.float32)
        qd = qf.astype(np.float64)
        dot = x @ qd
        key = 2 * dot - (x * x).sum(1) if space == "l2" else dot
        order = np.lexsort((np.arange(len(key)), -key))[:k]
        out_i.append(ext[order])
        if space == "l2":
            out_d.append((qd @ qd) - key[order])
        elif space == "cosinesimil":
            out_d.append(np.maximum(0, 1 - np.clip(key[order], -1, 1)))
        else:
            out_d.append(-key[order])
    return np.array(out_i), np.array(out_d)


def _index(name):
    build()
    idx = nmslib.init(method="hnsw", space=golden_manifest()[name]["space"])
    idx.loadIndex(golden_path(name))
    return idx


@pytest.mark.parametrize("name,k", [("tiny_l2_d20_sqids", 10), ("one_l2_d3", 3), ("tiny_cos_d48", 7),
                                    ("dup_l2_d16", 10), ("c1_l2_d128", 10), ("c1_l2_d128", 32),
                                    ("cos_d100", 10), ("cos_d100", 1), ("sift_l2_ties", 10),
                                    ("tiny_negdot_d7", 5)])
def test_bruteforce_matches_fp64(name, k):
    space = golden_manifest()[name]["space"]
    idx = _index(name)
    q = load_golden(name)["queries"]
    ids, d, cnt, st = idx.bruteForceBatchArrays(q, k, stats=True)
    n = idx.info["n"]
    want_i, want_d = fp64_topk(golden_path(name), q, min(k, n), space)
    np.testing.assert_array_equal(cnt, np.full(len(q), min(k, n)))
    np.testing.assert_array_equal(ids[:, : min(k, n)], want_i)
    np.testing.assert_allclose(d[:, : min(k, n)], want_d, rtol=2e-6, atol=2e-6)
    assert st[0] >= 1 and st[1] >= min(k, n) and st[2] == 0


@pytest.mark.parametrize("name,k,nq", [("negdot_d960", 10, 40), ("l1_d22", 10, 50), ("l1_d64", 32, 50),
                                       ("linf_d37", 10, 50), ("linf_d128", 5, 50)])
def test_exact_scan_matches_reference_distances(name, k, nq):
    """L1 / LInf (and any space with exact_scan=True) take the exact CUDA-core scan: every id and
    distance equals a full scan with the oracle's restatement of the reference's distance function
    (bit for bit), ordered by (distance, node)."""
    idx = _index(name)
    q = load_golden(name)["queries"][:nq]
    ids, d, cnt, st = idx.bruteForceBatchArrays(q, k, stats=True, exact_scan=True)
    ix = OracleIndex(golden_path(name))
    vecs, ext, _, _ = ix.export()
    dt = ix.info["dist_type"]
    n = len(vecs)
    for qi in range(len(q)):
        dd = np.array([dist(dt, q[qi], vecs[r]) for r in range(n)], np.float32)
        order = np.lexsort((np.arange(n), dd))[: min(k, n)]
        assert cnt[qi] == min(k, n)
        np.testing.assert_array_equal(ids[qi, : cnt[qi]], ext[order])
        np.testing.assert_array_equal(d[qi, : cnt[qi]], dd[order])
    assert st[0] == 0 and st[1] == n and st[2] == 0


@pytest.mark.parametrize("space,code,dim", [("l2", 0, 307), ("l2", 0, 320), ("cosinesimil", 1, 304),
                                            ("negdotprod", 2, 271)])
def test_exact_scan_wide_rows_tiled(tmp_path, space, code, dim):
    """The exact CUDA-core scan of the fused-multiply-add spaces (the register-tiled kernel): odd
    widths (16-element half block, 4-wide and scalar tails), a row count that ends inside a warp's
    pass, several chunks and a last query block of 4; every id and distance equals the oracle's full
    scan bit for bit. The same rows through the default tensor-core path (query K-blocks streamed,
    the rows being wider than 256) give the float64 top-k ids and distances within float rounding."""
    rng = np.random.default_rng(dim)
    n, nq, k = 4_333, 20, 12
    base = rng.standard_normal((n, dim)).astype(np.float32)
    q = rng.standard_normal((nq, dim)).astype(np.float32)
    p = str(tmp_path / f"wide_{space}_{dim}.hnsw")
    _capi.build_index(base, code, 4, 16, nthreads=0, out_path=p)
    idx = nmslib.init(method="hnsw", space=space)
    idx.loadIndex(p)
    ids, d, cnt, st = idx.bruteForceBatchArrays(q, k, stats=True, exact_scan=True)
    assert st[0] == 0 and st[1] == n and st[3] >= 2
    ti, td, tc, tst = idx.bruteForceBatchArrays(q, k, stats=True)
    assert tst[0] >= 1  # the tensor-core path
    want_i, want_d = fp64_topk(p, q, k, space)
    np.testing.assert_array_equal(tc, np.full(nq, k))
    np.testing.assert_array_equal(ti, want_i)
    np.testing.assert_allclose(td, want_d, rtol=2e-6, atol=2e-6)
    ix = OracleIndex(p)
    vecs, ext, _, _ = ix.export()
    dt = ix.info["dist_type"]
    for qi in range(nq):
        qv = normalize(q[qi]) if space == "cosinesimil" else q[qi]
        dd = np.array([dist(dt, qv, vecs[r]) for r in range(n)], np.float32)
        order = np.lexsort((np.arange(n), dd))[:k]
        assert cnt[qi] == k
        np.testing.assert_array_equal(ids[qi], ext[order])
        np.testing.assert_array_equal(d[qi], dd[order])


def _oracle_scan(p, q, k, cosine=False):
    ix = OracleIndex(p)
    vecs, ext, _, _ = ix.export()
    dt = ix.info["dist_type"]
    n = len(vecs)
    out = []
    for qi in range(len(q)):
        qv = normalize(q[qi]) if cosine else q[qi]
        dd = np.array([dist(dt, qv, vecs[r]) for r in range(n)], np.float32)
        order = np.lexsort((np.arange(n), dd))[:k]
        out.append((ext[order], dd[order]))
    return out


@pytest.mark.parametrize("k", [1, 32])
def test_exact_scan_tiled_k_extremes_and_ties(tmp_path, k):
    """4,333 rows that are copies of 37 distinct 288-wide vectors (every distance tied ~117 ways,
    across warps, chunks and query blocks): the tiled scan and the list merge keep the lowest
    rows of each tie, exactly as a full scan ordered by (distance, node) does."""
    rng = np.random.default_rng(k)
    distinct = rng.integers(-3, 4, (37, 288)).astype(np.float32)
    base = distinct[rng.integers(0, 37, 4_333)]
    q = np.concatenate([distinct[:5], rng.integers(-3, 4, (6, 288)).astype(np.float32)])
    p = str(tmp_path / f"ties_{k}.hnsw")
    _capi.build_index(base, 0, 4, 16, nthreads=0, out_path=p)
    idx = nmslib.init(method="hnsw", space="l2")
    idx.loadIndex(p)
    ids, d, cnt, st = idx.bruteForceBatchArrays(q, k, stats=True, exact_scan=True)
    assert st[0] == 0 and st[3] >= 2
    for qi, (want_i, want_d) in enumerate(_oracle_scan(p, q, k)):
        assert cnt[qi] == k
        np.testing.assert_array_equal(ids[qi, :k], want_i)
        np.testing.assert_array_equal(d[qi, :k], want_d)


def test_exact_scan_tiled_zero_cosine_query(tmp_path):
    """A zero query under cosine is not normalised (the search leaves it as is): every distance is
    1 - 0 = 1 and the k lowest rows come back."""
    rng = np.random.default_rng(3)
    base = rng.standard_normal((3_000, 300)).astype(np.float32)
    q = np.concatenate([np.zeros((1, 300), np.float32), rng.standard_normal((2, 300)).astype(np.float32)])
    p = str(tmp_path / "zero_cos.hnsw")
    _capi.build_index(base, 1, 4, 16, nthreads=0, out_path=p)
    idx = nmslib.init(method="hnsw", space="cosinesimil")
    idx.loadIndex(p)
    ids, d, cnt, st = idx.bruteForceBatchArrays(q, 10, stats=True, exact_scan=True)
    want = _oracle_scan(p, q, 10, cosine=True)
    for qi, (want_i, want_d) in enumerate(want):
        np.testing.assert_array_equal(ids[qi], want_i)
        np.testing.assert_array_equal(d[qi], want_d)
    np.testing.assert_array_equal(d[0], np.ones(10, np.float32))


def test_bruteforce_limits():
    idx = _index("c1_l2_d128")
    with pytest.raises(RuntimeError, match="k <= 32"):
        idx.bruteForceBatchArrays(load_golden("c1_l2_d128")["queries"][:4], 33)


def test_bruteforce_larger_cosine(tmp_path):
    """200K x 100 cosine (the C3 distribution): exact ids against float64 on a sample."""
    from nmslib_b200.datasets import mixture
    x = mixture("glove", 200_256, 100, 100, 3)
    base, q = x[:200_000], x[200_000:]
    p = str(tmp_path / "c3s.hnsw")
    _capi.build_index(base, 1, 8, 40, nthreads=0, out_path=p)
    idx = nmslib.init(method="hnsw", space="cosinesimil")
    idx.loadIndex(p)
    ids, d, cnt, st = idx.bruteForceBatchArrays(q, 10, stats=True)
    want_i, want_d = fp64_topk(p, q, 10, "cosinesimil")
    np.testing.assert_array_equal(ids, want_i)
    np.testing.assert_allclose(d, want_d, rtol=2e-6, atol=2e-6)


def _far_medium_near(n=40_000, dim=16, seed=5, nq=2560):
    """A base whose sampled tiles hold only far vectors, so the sample's threshold admits every
    other vector: more than the collection holds. Tile t (256 rows) is sampled when t % 9 == 0
    and t <= 135 (16 of the 157 tiles). Ten near vectors sit in tile 1. With 20 blocks of 128
    queries the full scan's work items span two tiles each, so each 64-entry list of a column
    quarter sees 128 candidate rows and overflows."""
    rng = np.random.default_rng(seed)
    u = rng.standard_normal((n, dim))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    tile = np.arange(n) // 256
    sampled = (tile % 9 == 0) & (tile <= 135)
    radius = np.where(sampled, 100.0, 10.0 + 5.0 * rng.random(n))
    radius[256:266] = 1.0 + 0.01 * np.arange(10)
    return (u * radius[:, None]).astype(np.float32), (0.01 * rng.standard_normal((nq, dim))).astype(np.float32)


def test_bruteforce_rescans_overflowed_queries(tmp_path):
    base, q = _far_medium_near()
    p = str(tmp_path / "fmn.hnsw")
    _capi.build_index(base, 0, 8, 40, nthreads=0, out_path=p)
    idx = nmslib.init(method="hnsw", space="l2")
    idx.loadIndex(p)
    ids, d, cnt, st = idx.bruteForceBatchArrays(q, 10, stats=True)
    want_i, want_d = fp64_topk(p, q, 10, "l2")
    np.testing.assert_array_equal(ids, want_i)
    np.testing.assert_array_equal(np.sort(ids, axis=1), np.tile(np.arange(256, 266), (len(q), 1)))
    np.testing.assert_allclose(d, want_d, rtol=2e-6, atol=2e-6)
    assert st[1] > 16384 and st[2] == len(q)


def test_bruteforce_capacity_error(tmp_path):
    """17000 identical vectors: every one stays within the error bound of the k-th, on every
    rescan. 4608 queries (36 blocks), so that the full scan's work items span two tiles and its
    lists can overflow."""
    base = np.tile(np.linspace(-1, 1, 8, dtype=np.float32), (17_000, 1))
    p = str(tmp_path / "same.hnsw")
    _capi.build_index(base, 0, 4, 10, nthreads=0, out_path=p)
    idx = nmslib.init(method="hnsw", space="l2")
    idx.loadIndex(p)
    with pytest.raises(RuntimeError, match="within the BF16 error bound"):
        idx.bruteForceBatchArrays(np.tile(base[:2] + 0.5, (2304, 1)), 10)


@pytest.mark.parametrize("k", [1, 10, 32])
def test_tensor_core_wide_rows_match_fp64(k):
    """960-wide negative dot products (the reference-built fixture) on the tensor cores with the
    query block's K-blocks streamed beside the base's: the float64 top-k ids, ties by id."""
    name = "negdot_d960"
    idx = _index(name)
    q = load_golden(name)["queries"]
    ids, d, cnt, st = idx.bruteForceBatchArrays(q, k, stats=True)
    assert st[0] >= 1
    want_i, want_d = fp64_topk(golden_path(name), q, k, "negdotprod")
    np.testing.assert_array_equal(ids[:, :k], want_i)
    np.testing.assert_allclose(d[:, :k], want_d, rtol=2e-6, atol=2e-6)


def test_exact_scan_then_tensor_path_on_one_index():
    """The exact scan first, then the tensor-core path, then the exact scan again on the same
    loaded index: each call prepares what it needs and gives its own path's results."""
    name = "c1_l2_d128"
    idx = _index(name)
    q = load_golden(name)["queries"][:30]
    want_i, want_d = fp64_topk(golden_path(name), q, 10, "l2")
    a = idx.bruteForceBatchArrays(q, 10, stats=True, exact_scan=True)
    b = idx.bruteForceBatchArrays(q, 10, stats=True)
    c = idx.bruteForceBatchArrays(q, 10, stats=True, exact_scan=True)
    assert a[3][0] == 0 and b[3][0] >= 1 and c[3][0] == 0
    np.testing.assert_array_equal(b[0], want_i)
    np.testing.assert_array_equal(a[0], c[0])
    np.testing.assert_array_equal(a[1].view(np.int32), c[1].view(np.int32))
