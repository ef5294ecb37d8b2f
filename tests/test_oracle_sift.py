"""The oracle's l2sqr_sift restatement against the reference's own results (fixtures made by
tests/golden/make_golden_sift.py with the reference module): regular graph file + objects file,
128 uint8 values per object, int distances.

The reference's result queue orders (distance, Object*) pairs (similarity_search/include/
knnqueue.h:29-81), so equal distances come out in object-address order. The objects of a regular
index are separate allocations made while loading <file>.dat, so that order is the allocator's,
not the algorithm's. The comparison is therefore exact for every distance, exact for the ids of
every distance below the k-th, and by count at the k-th distance: under SearchOld
(hnsw.cc:1078-1175) which of the items tied there stays in the queue also follows the addresses.
SearchV1Merge adds its first k items without eviction (hnsw.cc:1295-1297).
"""
import json
import os

import numpy as np
import pytest

from oracle.oracle import OracleSiftIndex

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ALGO = {"hybrid": 0, "old": 1, "v1merge": 2}


def _manifest():
    with open(os.path.join(HERE, "manifest_sift.json")) as f:
        return json.load(f)


def _cases():
    return [(name, si) for name, c in _manifest().items() for si in range(len(c["settings"]))]


def assert_same_up_to_address_ties(ids, dists, counts, want_ids, want_dists, want_counts):
    np.testing.assert_array_equal(counts, want_counts)
    for qi in range(len(counts)):
        c = counts[qi]
        d, i = dists[qi, :c], ids[qi, :c]
        wd, wi = want_dists[qi, :c], want_ids[qi, :c]
        np.testing.assert_array_equal(d, wd)  # ascending in both
        if c == 0:
            continue
        below = d < d[-1]
        np.testing.assert_array_equal(np.sort(i[below]), np.sort(wi[wd < wd[-1]]))
        assert len(set(i.tolist())) == c  # no duplicates


@pytest.mark.parametrize("name,si", _cases())
def test_sift_oracle_matches_reference(name, si):
    k, ef, algo = _manifest()[name]["settings"][si]
    g = np.load(os.path.join(HERE, name + ".npz"))
    ix = OracleSiftIndex(os.path.join(HERE, name + ".hnsw"))
    ids, dists, counts = ix.search(g["queries"], k, ef, ALGO[algo])
    assert_same_up_to_address_ties(ids, dists, counts, g[f"ids_{si}"], g[f"dists_{si}"], g[f"counts_{si}"])


def test_sift_oracle_exact_where_no_ties():
    """Without tied distances the oracle reproduces the reference's output exactly, order included."""
    g = np.load(os.path.join(HERE, "sift_u8_d128.npz"))
    ix = OracleSiftIndex(os.path.join(HERE, "sift_u8_d128.hnsw"))
    for si, (k, ef, algo) in enumerate(_manifest()["sift_u8_d128"]["settings"]):
        ids, dists, counts = ix.search(g["queries"], k, ef, ALGO[algo])
        np.testing.assert_array_equal(ids, g[f"ids_{si}"])
        np.testing.assert_array_equal(dists, g[f"dists_{si}"])


def test_sift_distance_is_the_integer_l2():
    """Every reported distance equals sum((q - x)^2) over the 128 uint8 values, in integers."""
    g = np.load(os.path.join(HERE, "sift_u8_tiny.npz"))
    ix = OracleSiftIndex(os.path.join(HERE, "sift_u8_tiny.hnsw"))
    ids, dists, counts = ix.search(g["queries"], 40, 5, 0)
    with open(os.path.join(HERE, "sift_u8_tiny.hnsw.dat"), "rb") as f:
        raw = f.read()
    n = int(np.frombuffer(raw[:8], np.uint64)[0])
    vecs = np.stack([np.frombuffer(raw[8 + i * 156 + 24: 8 + i * 156 + 152], np.uint8) for i in range(n)])
    for qi in range(len(counts)):
        for j in range(counts[qi]):
            diff = g["queries"][qi].astype(np.int64) - vecs[ids[qi, j]].astype(np.int64)
            assert dists[qi, j] == int((diff * diff).sum())


def test_sift_loader_rejects_mismatched_files(tmp_path):
    bad = tmp_path / "bad.dat"
    bad.write_bytes(np.array([3], np.uint64).tobytes())
    with pytest.raises(ValueError, match="objects file"):
        OracleSiftIndex(os.path.join(HERE, "sift_u8_tiny.hnsw"), str(bad))
    with pytest.raises(ValueError, match="not a regular index"):
        OracleSiftIndex(os.path.join(HERE, "c1_l2_d128.hnsw"), os.path.join(HERE, "sift_u8_tiny.hnsw.dat"))
    # a count far beyond what the file holds is refused before anything is sized from it
    huge = tmp_path / "huge.dat"
    huge.write_bytes(np.array([1 << 60], np.uint64).tobytes() + b"\0" * 200)
    with pytest.raises(ValueError, match="does not fit the file"):
        OracleSiftIndex(os.path.join(HERE, "sift_u8_tiny.hnsw"), str(huge))
