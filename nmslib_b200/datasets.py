"""Seeded synthetic workloads with the shapes and value distributions of the benchmark suite.

The public datasets the reference benchmarks on (SIFT1M, GloVe-100, GIST-like, Deep-like) are
not available offline, so each workload is drawn from a seeded Gaussian mixture that mimics
their value ranges:

* ``gauss``   — centres ~ N(0, 1), x = c[z] + sigma * N(0, 1)                      (plain l2)
* ``sift``    — centres round(clip(|N(0, 40)|, 0, 255)), x = clip(round(c[z] + N(0, 12)), 0, 255)
                stored as float32: integer-valued squared distances, so exact ties are common
* ``glove``   — per-dimension scale s_j ~ U(0.5, 2); centres ~ N(0, diag(s^2));
                x = c[z] + 0.5 * N(0, diag(s^2)); unit-normalised                  (cosine)
* ``absgauss``— centres ~ |N(0, 1)|, x = |c[z] + 0.5 * N(0, 1)|                   (negdot, wide)
* ``unit``    — centres ~ N(0, 1), x = c[z] + sigma * N(0, 1), unit-normalised    (serving)

Base rows and queries come from one draw of ``n_base + n_query`` rows, split in that order.
"""
from __future__ import annotations

import numpy as np

_CHUNK = 1 << 16


def mixture(kind: str, n: int, dim: int, n_centres: int, seed: int, sigma: float = 0.3) -> np.ndarray:
    rng = np.random.default_rng(seed)
    out = np.empty((n, dim), np.float32)
    if kind == "gauss" or kind == "unit":
        c = rng.standard_normal((n_centres, dim))
    elif kind == "sift":
        c = np.round(np.clip(np.abs(rng.normal(0.0, 40.0, (n_centres, dim))), 0, 255))
    elif kind == "glove":
        s = rng.uniform(0.5, 2.0, dim)
        c = rng.standard_normal((n_centres, dim)) * s
    elif kind == "absgauss":
        c = np.abs(rng.standard_normal((n_centres, dim)))
    else:
        raise ValueError(f"unknown mixture kind {kind!r}")
    for s0 in range(0, n, _CHUNK):
        m = min(_CHUNK, n - s0)
        z = rng.integers(0, n_centres, m)
        if kind == "gauss":
            x = c[z] + sigma * rng.standard_normal((m, dim))
        elif kind == "unit":
            x = c[z] + sigma * rng.standard_normal((m, dim))
            x /= np.linalg.norm(x, axis=1, keepdims=True)
        elif kind == "sift":
            x = np.clip(np.round(c[z] + rng.normal(0.0, 12.0, (m, dim))), 0, 255)
        elif kind == "glove":
            x = c[z] + 0.5 * rng.standard_normal((m, dim)) * s
            x /= np.linalg.norm(x, axis=1, keepdims=True)
        else:  # absgauss
            x = np.abs(c[z] + 0.5 * rng.standard_normal((m, dim)))
        out[s0:s0 + m] = x
    return out


# name -> (kind, n_base, n_query, dim, n_centres, seed, sigma, space, M)
WORKLOADS = {
    "c1_gauss10k_d128_l2": ("gauss", 10_000, 1_000, 128, 32, 0, 0.3, "l2", 16),
    "c2_sift1m_d128_l2": ("sift", 1_000_000, 10_000, 128, 1000, 2, 0.0, "l2", 16),
    "c3_glove1m_d100_cos": ("glove", 1_000_000, 10_000, 100, 100, 3, 0.0, "cosinesimil", 24),
    "c4_abs1m_d960_negdot": ("absgauss", 1_000_000, 8_000, 960, 500, 4, 0.0, "negdotprod", 16),
    "c5_unit5m_d96_l2": ("unit", 5_000_000, 200_000, 96, 2000, 5, 0.4, "l2", 32),
}


def workload(name: str, n_base: int | None = None, n_query: int | None = None):
    """(base, queries, space, M) for a named workload; sizes may be overridden (smaller cases
    keep the distribution and the seed)."""
    kind, nb, nq, dim, nc, seed, sigma, space, m = WORKLOADS[name]
    nb = nb if n_base is None else n_base
    nq = nq if n_query is None else n_query
    x = mixture(kind, nb + nq, dim, nc, seed, sigma)
    return x[:nb], x[nb:], space, m
