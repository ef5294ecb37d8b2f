"""Generates the committed golden fixtures from the reference itself.

Run once, where the reference sources are available:

    make -C oracle ref          # builds oracle/_ref/nmslib*.so from the reference sources
    python tests/golden/make_golden.py [case ...]   # all cases, or only the named ones

For every case it builds an HNSW index with the reference's own ``createIndex`` (single
index thread, so the build is reproducible), writes the reference's ``saveIndex`` file as
``<case>.hnsw``, and records the reference's ``knnQueryBatch`` output for several
(k, efSearch, algoType) settings in ``<case>.npz`` (queries, ids, dists, counts).
Index builds are not bit-reproducible across machines; the committed files are the fixtures.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from nmslib_b200.datasets import mixture  # noqa: E402
from oracle.oracle import reference_module  # noqa: E402

# name: (space, base rows, queries, M, efC, [(k, ef, algoType)], ids)
def cases():
    c = {}
    x = mixture("gauss", 11_000, 128, 32, 0, 0.3)
    c["c1_l2_d128"] = ("l2", x[:10_000], x[10_000:], 16, 200,
                       [(10, 100, "hybrid"), (10, 20, "hybrid"), (1, 10, "hybrid"), (100, 50, "hybrid"),
                        (10, 1000, "hybrid"), (10, 100, "old"), (10, 300, "v1merge")], None)
    x = mixture("sift", 5_500, 128, 100, 2)
    c["sift_l2_ties"] = ("l2", x[:5_000], x[5_000:], 16, 200,
                         [(10, 64, "hybrid"), (10, 256, "hybrid"), (10, 1000, "hybrid"), (100, 128, "hybrid")],
                         None)
    x = mixture("glove", 4_500, 100, 100, 3)
    c["cos_d100"] = ("cosinesimil", x[:4_000], x[4_000:], 24, 200,
                     [(10, 200, "hybrid"), (10, 1000, "hybrid"), (1, 16, "hybrid")], None)
    x = mixture("absgauss", 1_200, 960, 50, 4)
    c["negdot_d960"] = ("negdotprod", x[:1_000], x[1_000:], 16, 200,
                        [(1, 64, "hybrid"), (10, 512, "hybrid"), (100, 1024, "hybrid")], None)
    # small and ragged shapes: every tail path of the distance kernels, custom external ids
    x = mixture("gauss", 70, 20, 4, 11, 0.5)
    c["tiny_l2_d20_sqids"] = ("l2", x[:50], x[50:], 8, 50, [(10, 10, "hybrid"), (60, 5, "hybrid")],
                              np.arange(50) ** 2)
    x = mixture("gauss", 300, 7, 5, 12, 0.5)
    c["tiny_negdot_d7"] = ("negdotprod", x[:250], x[250:], 5, 40, [(5, 20, "hybrid"), (5, 1000, "hybrid")], None)
    x = mixture("glove", 240, 48, 6, 13)
    c["tiny_cos_d48"] = ("cosinesimil", x[:200], x[200:], 6, 40, [(7, 30, "hybrid"), (7, 30, "old")], None)
    x = mixture("gauss", 2, 3, 1, 14, 0.5)
    c["one_l2_d3"] = ("l2", x[:1], x[1:], 4, 10, [(3, 10, "hybrid")], None)
    # exact duplicates: every distance comes in triples, stressing tie order everywhere
    x = np.round(mixture("gauss", 140, 16, 3, 15, 0.6) * 4).astype(np.float32)
    base = np.repeat(x[:100], 3, axis=0)
    c["dup_l2_d16"] = ("l2", base, x[100:], 6, 60, [(10, 24, "hybrid"), (10, 24, "old"), (30, 200, "hybrid")],
                       None)
    # L1 / LInf (dist codes 5 / 6): dim 22 has a final 16-block, a 4-wide remainder and a
    # 2-element tail that L1 sums in double; dim 64 is whole 32-chunks; dim 37 has every part
    x = mixture("gauss", 1_050, 22, 20, 21, 0.4)
    c["l1_d22"] = ("l1", x[:1_000], x[1_000:], 8, 60, [(10, 40, "hybrid"), (10, 1000, "hybrid"), (5, 30, "old")],
                   None)
    x = mixture("gauss", 1_550, 64, 30, 22, 0.3)
    c["l1_d64"] = ("l1", x[:1_500], x[1_500:], 12, 100, [(10, 64, "hybrid"), (20, 200, "v1merge")], None)
    x = mixture("gauss", 1_050, 37, 20, 23, 0.4)
    c["linf_d37"] = ("linf", x[:1_000], x[1_000:], 8, 60, [(10, 50, "hybrid"), (10, 1000, "hybrid")], None)
    x = mixture("gauss", 1_550, 128, 30, 24, 0.3)
    c["linf_d128"] = ("linf", x[:1_500], x[1_500:], 12, 100, [(10, 64, "hybrid"), (1, 16, "hybrid")], None)
    return c


def main(only=None):
    ref = reference_module()
    if ref is None:
        raise SystemExit("reference module not built: run `make -C oracle ref` first")
    manifest = {}
    mpath = os.path.join(HERE, "manifest.json")
    if only and os.path.exists(mpath):  # regenerate only the named cases, keep the others
        with open(mpath) as f:
            manifest = json.load(f)
    for name, (space, base, queries, m, efc, settings, ids) in cases().items():
        if only and name not in only:
            continue
        index = ref.init(method="hnsw", space=space)
        if ids is None:
            index.addDataPointBatch(base)
        else:
            index.addDataPointBatch(base, ids=ids)
        index.createIndex({"M": m, "efConstruction": efc, "indexThreadQty": 1})
        path = os.path.join(HERE, name + ".hnsw")
        index.saveIndex(path)
        loaded = ref.init(method="hnsw", space=space)
        loaded.loadIndex(path)
        out = {"queries": queries}
        for si, (k, ef, algo) in enumerate(settings):
            loaded.setQueryTimeParams({"efSearch": ef, "algoType": algo})
            res = loaded.knnQueryBatch(queries, k=k, num_threads=1)
            ids_a = np.full((len(queries), k), -1, np.int32)
            d_a = np.full((len(queries), k), np.inf, np.float32)
            cnt = np.zeros(len(queries), np.int32)
            for qi, (ri, rd) in enumerate(res):
                cnt[qi] = len(ri)
                ids_a[qi, : len(ri)] = ri
                d_a[qi, : len(rd)] = rd
            out[f"ids_{si}"], out[f"dists_{si}"], out[f"counts_{si}"] = ids_a, d_a, cnt
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        manifest[name] = {"space": space, "M": m, "efConstruction": efc,
                          "settings": [list(s) for s in settings], "n": int(len(base)),
                          "dim": int(base.shape[1]), "nq": int(len(queries))}
        print(name, os.path.getsize(path), "bytes")
    with open(mpath, "w") as f:
        json.dump(manifest, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1:] or None)
