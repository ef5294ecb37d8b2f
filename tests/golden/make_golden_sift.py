"""Generates the committed l2sqr_sift golden fixtures from the reference itself.

Run once, where the reference sources are available:

    make -C oracle ref                                 # oracle/_ref/nmslib*.so from the sources
    python tests/golden/make_golden_sift.py [case ...]  # all cases, or only the named ones

For every case it builds an HNSW index over 128-dimensional uint8 vectors in space
``l2sqr_sift`` (DENSE_UINT8_VECTOR data, int distances) with the reference's own
``createIndex`` (one index thread, so the build is reproducible), saves it with
``saveIndex(path, save_data=True)`` -- the regular graph file ``<case>.hnsw`` and the objects file
``<case>.hnsw.dat``, since the reference has no optimized layout for this space -- and records
the reference's ``knnQueryBatch`` output for several (k, efSearch, algoType) settings in
``<case>.npz`` (queries, ids, dists, counts; int32 distances). The cases are listed in
``manifest_sift.json``, apart from the float fixtures' manifest.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import reference_module  # noqa: E402


# name: (base rows uint8 [n, 128], queries uint8 [nq, 128], M, efC, [(k, ef, algoType)])
def cases():
    c = {}
    rng = np.random.default_rng(31)
    centres = rng.integers(0, 256, (40, 128))
    lab = rng.integers(0, 40, 2_050)
    x = np.clip(centres[lab] + rng.normal(0, 18, (2_050, 128)), 0, 255).astype(np.uint8)
    c["sift_u8_d128"] = (x[:2_000], x[2_000:], 8, 60,
                         [(10, 40, "hybrid"), (10, 1000, "hybrid"), (5, 30, "old"), (10, 200, "v1merge")])
    # four levels per coordinate and duplicated rows: integer distances tie everywhere
    rng = np.random.default_rng(32)
    y = (rng.integers(0, 4, (560, 128)) * 60).astype(np.uint8)
    base = np.repeat(y[:500], 3, axis=0)
    c["sift_u8_ties"] = (base, y[500:], 6, 40, [(10, 64, "hybrid"), (10, 64, "old"), (30, 300, "hybrid")])
    rng = np.random.default_rng(33)
    z = rng.integers(0, 256, (42, 128)).astype(np.uint8)
    c["sift_u8_tiny"] = (z[:30], z[30:], 4, 20, [(10, 10, "hybrid"), (40, 5, "hybrid")])
    return c


def main(only=None):
    ref = reference_module()
    if ref is None:
        raise SystemExit("reference module not built: run `make -C oracle ref` first")
    manifest = {}
    mpath = os.path.join(HERE, "manifest_sift.json")
    if only and os.path.exists(mpath):
        with open(mpath) as f:
            manifest = json.load(f)

    def new_index():
        return ref.init(method="hnsw", space="l2sqr_sift", data_type=ref.DataType.DENSE_UINT8_VECTOR,
                        dtype=ref.DistType.INT)

    for name, (base, queries, m, efc, settings) in cases().items():
        if only and name not in only:
            continue
        index = new_index()
        index.addDataPointBatch(base)
        index.createIndex({"M": m, "efConstruction": efc, "indexThreadQty": 1})
        path = os.path.join(HERE, name + ".hnsw")
        index.saveIndex(path, save_data=True)
        loaded = new_index()
        loaded.loadIndex(path, load_data=True)
        out = {"queries": queries}
        for si, (k, ef, algo) in enumerate(settings):
            loaded.setQueryTimeParams({"efSearch": ef, "algoType": algo})
            res = loaded.knnQueryBatch(queries, k=k, num_threads=1)
            ids_a = np.full((len(queries), k), -1, np.int32)
            d_a = np.full((len(queries), k), np.iinfo(np.int32).max, np.int32)
            cnt = np.zeros(len(queries), np.int32)
            for qi, (ri, rd) in enumerate(res):
                cnt[qi] = len(ri)
                ids_a[qi, : len(ri)] = ri
                d_a[qi, : len(rd)] = rd
            out[f"ids_{si}"], out[f"dists_{si}"], out[f"counts_{si}"] = ids_a, d_a, cnt
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        manifest[name] = {"space": "l2sqr_sift", "M": m, "efConstruction": efc,
                          "settings": [list(s) for s in settings], "n": int(len(base)), "dim": 128,
                          "nq": int(len(queries))}
        print(name, os.path.getsize(path), os.path.getsize(path + ".dat"), "bytes")
    with open(mpath, "w") as f:
        json.dump(manifest, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1:] or None)
