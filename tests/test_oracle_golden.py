"""The oracle (CPU restatement) against the reference's own outputs recorded in tests/golden."""
import numpy as np
import pytest

from conftest import ALGO_CODES, assert_same_results, golden_cases, golden_manifest, golden_path, load_golden
from oracle.oracle import OracleIndex, bruteforce_fp64, normalize, recall
from nmslib_b200.datasets import mixture


@pytest.mark.parametrize("name,si,k,ef,algo", golden_cases())
def test_oracle_matches_reference(name, si, k, ef, algo):
    ix = OracleIndex(golden_path(name))
    g = load_golden(name)
    ids, d, cnt, _ = ix.search(g["queries"], k=k, ef=ef, algo=ALGO_CODES[algo], nthreads=4)
    frac = assert_same_results(ids, d, cnt, g[f"ids_{si}"], g[f"dists_{si}"], g[f"counts_{si}"])
    assert frac >= 0.69  # the remainder differ only inside runs of equal distance


def test_cosine_normalisation_is_float_and_unfused():
    """The stored base rows of a cosine index are the reference's NormalizeVect output; the
    oracle's float reading reproduces all of them, the double reading does not."""
    x = mixture("glove", 4_500, 100, 100, 3)[:4_000]
    ix = OracleIndex(golden_path("cos_d100"))
    vecs, ext, _, _ = ix.export()
    raw = x[ext]
    ok_f = sum(bool((normalize(raw[i]) == vecs[i]).all()) for i in range(400))
    ok_d = sum(bool((normalize(raw[i], use_double=True) == vecs[i]).all()) for i in range(400))
    assert ok_f == 400
    assert ok_d < 400


def test_recall_c1_against_fp64():
    """C1 (10K x 128 l2, efSearch 100, k 10): recall@10 against exact FP64 kNN."""
    x = mixture("gauss", 11_000, 128, 32, 0, 0.3)
    ix = OracleIndex(golden_path("c1_l2_d128"))
    _, ext, _, _ = ix.export()
    g = load_golden("c1_l2_d128")
    true_i, _ = bruteforce_fp64(x[:10_000], g["queries"], 10, "l2")
    assert recall(g["ids_0"], true_i, g["counts_0"]) >= 0.99
    ids, _, cnt, _ = ix.search(g["queries"], k=10, ef=100)
    assert recall(ids, true_i, cnt) >= 0.99


def test_stats_are_consistent():
    ix = OracleIndex(golden_path("c1_l2_d128"))
    g = load_golden("c1_l2_d128")
    _, _, _, st = ix.search(g["queries"][:50], k=10, ef=100)
    d = ix.dim
    # bytes = rows gathered + neighbour lists; every distance reads one row
    assert (st[:, 3] >= st[:, 0] * 4 * d).all()
    assert (st[:, 1] >= 1).all()
