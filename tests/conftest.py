import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
ALGO_CODES = {"hybrid": 0, "old": 1, "v1merge": 2}


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def golden_manifest():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)


def golden_cases():
    """[(case, setting_index, k, ef, algo)] over every committed fixture."""
    out = []
    for name, m in golden_manifest().items():
        for si, (k, ef, algo) in enumerate(m["settings"]):
            out.append((name, si, k, ef, algo))
    return out


def golden_path(name):
    return os.path.join(GOLDEN, name + ".hnsw")


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def assert_same_results(ids_a, d_a, cnt_a, ids_b, d_b, cnt_b, rtol=0.0, max_tie_only_frac=1.0):
    """Result lists agree: counts equal; distances equal (bit-exact when rtol == 0) position by
    position; ids equal except that ids sharing one distance may come in any order (the reference
    orders equal distances by object address). Returns the fraction of queries whose id lists
    were identical."""
    np.testing.assert_array_equal(cnt_a, cnt_b)
    identical = 0
    for r in range(len(cnt_a)):
        c = int(cnt_a[r])
        da, db = d_a[r, :c], d_b[r, :c]
        if rtol == 0.0:
            np.testing.assert_array_equal(da.view(np.int32), db.view(np.int32), err_msg=f"query {r}")
        else:
            np.testing.assert_allclose(da, db, rtol=rtol, atol=0, err_msg=f"query {r}")
        ia, ib = ids_a[r, :c], ids_b[r, :c]
        if (ia == ib).all():
            identical += 1
            continue
        # same multiset of ids within every run of equal distances
        keys = da if rtol == 0.0 else db
        s = 0
        while s < c:
            e = s
            while e < c and keys[e] == keys[s]:
                e += 1
            assert sorted(ia[s:e].tolist()) == sorted(ib[s:e].tolist()), f"query {r}: ids differ beyond ties"
            s = e
    frac = identical / max(1, len(cnt_a))
    return frac
