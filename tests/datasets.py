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
