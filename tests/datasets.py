"""Seeded synthetic inputs with the shapes and distributions of the benchmark
configurations (the real datasets are not available; these stand in for them)."""
from __future__ import annotations

import numpy as np


def mixture(rng, n, centres, sigma):
    lab = rng.integers(0, len(centres), n)
    X = (centres[lab] + sigma * rng.standard_normal((n, centres.shape[1]))).astype(np.float32)
    return X, lab


def cfg1():
    """10,000 x 64 N(0,1) reference rows (seed 0), 2,000 queries (seed 1)."""
    X = np.random.default_rng(0).standard_normal((10000, 64)).astype(np.float32)
    Q = np.random.default_rng(1).standard_normal((2000, 64)).astype(np.float32)
    return X, Q


def cfg2a(n=1_000_000, m=100_000, d=128):
    """Gaussian mixture: 1,024 centres uniform in [-1,1]^d, sigma 0.1, equal
    weights; reference rows seed 2, queries seed 3."""
    C = np.random.default_rng(2).uniform(-1, 1, (1024, d))
    X, _ = mixture(np.random.default_rng(2), n, C, 0.1)
    Q, _ = mixture(np.random.default_rng(3), m, C, 0.1)
    return X, Q


def pixels(rng, n, d=784, classes=10, templates=None):
    """Integer pixels in [0,255] stored as float32, ~80% exact zeros, the
    nonzeros uniform on 1..255, clustered into 10 synthetic class templates."""
    if templates is None:
        templates = rng.random((classes, d)) < 0.2
    lab = rng.integers(0, classes, n)
    mask = templates[lab].copy()
    mask ^= rng.random((n, d)) < 0.03
    vals = rng.integers(1, 256, (n, d))
    return np.where(mask, vals, 0).astype(np.float32), lab, templates


def cfg2b(n=60_000, m=10_000):
    rng = np.random.default_rng(8)
    X, y, T = pixels(rng, n)
    Q, yq, _ = pixels(rng, m, templates=T)
    return X, Q, y


def cfg3(n=200_000, m=50_000, d=32):
    """10 centres N(0, 4I) in d=32 (seed 4), labels 0-9, within-class sigma 1."""
    rng = np.random.default_rng(4)
    cen = rng.normal(0, 2.0, (10, d))
    X, y = mixture(rng, n, cen, 1.0)
    Q, _ = mixture(np.random.default_rng(40), m, cen, 1.0)
    return X, y, Q


def cfg4(seed=5, problems=256, n_range=(1_000, 200_000), m_range=(100, 20_000),
         dims=(16, 32, 64, 128, 256), ks=(1, 5, 10, 50)):
    """Batched uneven problems: n_ref and n_query log-uniform over their
    ranges, d and k drawn from their sets, rows i.i.d. N(0,1) float32, and 1%
    of each problem's reference rows duplicated (ties).  Returns a list of
    (X, Q, k) in draw order."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(problems):
        n = int(round(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1])))))
        m = int(round(np.exp(rng.uniform(np.log(m_range[0]), np.log(m_range[1])))))
        d = int(rng.choice(dims))
        k = int(rng.choice(ks))
        X = rng.standard_normal((n, d)).astype(np.float32)
        dup = max(1, n // 100)
        dst = rng.choice(n, dup, replace=False)
        X[dst] = X[rng.integers(0, n, dup)]
        Q = rng.standard_normal((m, d)).astype(np.float32)
        out.append((X, Q, min(k, n)))
    return out


def cfg5(seed=6, pairs=64, points=8192, self_n=4096, self_d=64):
    """Point clouds for the differentiable kNN losses: `pairs` pairs of
    `points` x 3 clouds uniform on the unit sphere plus N(0, 0.01^2) noise,
    and one self_n x self_d N(0,1) matrix (self k-NN)."""
    rng = np.random.default_rng(seed)

    def cloud():
        v = rng.standard_normal((points, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        return (v + 0.01 * rng.standard_normal((points, 3))).astype(np.float32)

    clouds = [(cloud(), cloud()) for _ in range(pairs)]
    S = rng.standard_normal((self_n, self_d)).astype(np.float32)
    return clouds, S
