"""Pin the CPU oracle against the reference's own outputs and known answers.

Fixtures in tests/golden were produced by tests/golden/make_golden.py from the
reference's CPU path (mlxlearn estimators, auto policy, no MLX).  The
known-answer cases restate the reference's tests (file:line cited per test).
"""
from __future__ import annotations

from fractions import Fraction

import numpy as np
import pytest

import oracle
from conftest import golden
from datasets import cfg1, mixture, pixels


def test_cfg1_against_reference_outputs():
    X, Q = cfg1()
    g = golden("knn_cfg1.npz")
    d, i = oracle.knn(X, Q, 5)
    np.testing.assert_array_equal(i, g["idx"])
    np.testing.assert_allclose(d, g["dist"], rtol=1e-12, atol=1e-12)
    assert d.dtype == np.float64 and i.dtype == np.int64


def test_self_query_with_duplicates_against_reference():
    X, _ = cfg1()
    Xs = X[:3000].copy()
    Xs[100:130] = Xs[:30]
    g = golden("knn_self_dups.npz")
    d, i = oracle.knn(Xs, Xs, 7, exclude_self=True)
    np.testing.assert_array_equal(i, g["idx"])
    np.testing.assert_allclose(d, g["dist"], rtol=1e-12, atol=1e-12)


def test_mixture128_against_reference():
    C = np.random.default_rng(2).uniform(-1, 1, (1024, 128))
    X, _ = mixture(np.random.default_rng(2), 50000, C, 0.1)
    Q, _ = mixture(np.random.default_rng(3), 256, C, 0.1)
    g = golden("knn_mixture128.npz")
    d, i = oracle.knn(X, Q, 10)
    np.testing.assert_array_equal(i, g["idx"])
    np.testing.assert_allclose(d, g["dist"], rtol=1e-12)


def test_pixels784_against_reference():
    rng = np.random.default_rng(7)
    X, y, T = pixels(rng, 8000)
    Q, _, _ = pixels(rng, 200, templates=T)
    g = golden("knn_pixels784.npz")
    d, i = oracle.knn(X, Q, 5)
    np.testing.assert_array_equal(i, g["idx"])
    np.testing.assert_allclose(d, g["dist"], rtol=1e-12)


def test_radius_against_reference():
    rng = np.random.default_rng(4)
    cen = rng.normal(0, 2.0, (10, 32))
    X, y = mixture(rng, 20000, cen, 1.0)
    Q, _ = mixture(np.random.default_rng(44), 500, cen, 1.0)
    Q[:5] += 40.0
    g = golden("radius_mixture32.npz")
    ip, ix, dd = oracle.radius(X, Q, float(g["radius"]))
    np.testing.assert_array_equal(ip, g["indptr"])
    np.testing.assert_array_equal(ix, g["indices"])
    np.testing.assert_array_equal(dd, g["dist"])  # canonical distances are bit-exact
    ip, ix, dd = oracle.radius(X, Q, float(g["radius"]), sort_results=True)
    np.testing.assert_array_equal(ix, g["sorted_indices"])
    np.testing.assert_array_equal(dd, g["sorted_dist"])
    assert (np.diff(ip)[:5] == 0).all()  # outliers have no neighbours


# ------------------------------------------------------------ known answers

def test_ties_break_on_training_index():
    # reference tests/parity/test_neighbors.py:48-54
    X = np.array([[1.0], [1.0], [1.0], [2.0]], dtype=np.float32)
    d, i = oracle.knn(X, np.array([[0.0]], np.float32), 3)
    np.testing.assert_array_equal(i, [[0, 1, 2]])
    np.testing.assert_allclose(d, [[1.0, 1.0, 1.0]])


@pytest.mark.parametrize("k", [1, 2])
def test_offset_seed251_distinct_distances(k):
    # reference tests/unit/test_neighbors_precision.py:42-70
    rng = np.random.default_rng(251)
    train = (rng.normal(size=(50_000, 32)) + 10_000).astype(np.float32)
    queries = (rng.normal(size=(256, 32)) + 10_000).astype(np.float32)
    sub, q = train[[1902, 43153]], queries[79:80]
    delta = sub.astype(np.float64) - q.astype(np.float64)
    sq = np.sum(delta * delta, axis=1)
    assert sq.astype(np.float32)[0] == sq.astype(np.float32)[1]
    _, i = oracle.knn(sub, q, k)
    np.testing.assert_array_equal(i, [[1]] if k == 1 else [[1, 0]])
    assert oracle.exact_compare(q[0], sub[1], sub[0]) < 0


def test_offset_seed251_k_boundary():
    # reference tests/unit/test_neighbors_precision.py:73-92
    rng = np.random.default_rng(251)
    train = (rng.normal(size=(50_000, 32)) + 10_000).astype(np.float32)
    queries = (rng.normal(size=(256, 32)) + 10_000).astype(np.float32)
    _, i4 = oracle.knn(train, queries[79:80], 4)
    _, i5 = oracle.knn(train, queries[79:80], 5)
    assert i4[0, 3] == 43153 and 1902 not in i4[0]
    assert i5[0, 4] == 1902


def test_genuinely_equal_distances_choose_smallest_indices():
    # reference tests/unit/test_neighbors_precision.py:95-106
    train = np.zeros((8, 32), dtype=np.float32)
    train[:4, :2] = [[1, 0], [-1, 0], [0, 1], [0, -1]]
    train[4:, 0] = 2
    for k in (1, 3):
        _, i = oracle.knn(train, np.zeros((1, 32), np.float32), k)
        np.testing.assert_array_equal(i, np.arange(k)[None, :])


def test_monotone_training_copied_rows():
    # reference tests/unit/test_neighbors_precision.py:108-118
    train = np.arange(8192 * 32, dtype=np.float32).reshape(8192, 32)
    queries = train[[0, 3, 4, 4096, 8191]].copy()
    d, i = oracle.knn(train, queries, 5)
    np.testing.assert_array_equal(i[:, 0], [0, 3, 4, 4096, 8191])
    np.testing.assert_array_equal(d[:, 0], 0)


def _fraction_key(q, x):
    return sum((Fraction(float(a)) - Fraction(float(b))) ** 2 for a, b in zip(q, x)) * 2**298


@pytest.mark.parametrize("seed", range(8))
def test_exact_key_matches_rational_arithmetic(seed):
    rng = np.random.default_rng(seed)
    d = int(rng.integers(1, 40))
    scale = float(10.0 ** rng.integers(-40, 36))
    q = (rng.standard_normal(d) * scale).astype(np.float32)
    x = (rng.standard_normal(d) * scale * float(10.0 ** rng.integers(-6, 6))).astype(np.float32)
    x[0] = np.float32(1.4e-45)  # smallest subnormal
    q[-1] = -np.float32(3.0e38)
    assert np.isfinite(q).all() and np.isfinite(x).all()
    assert oracle.exact_key(q, x) == _fraction_key(q, x)


def test_arbitrary_bit_patterns_order():
    # reference tests/unit/test_neighbors_cpu_native.py:51-177 (finite bit patterns)
    rng = np.random.default_rng(3)
    bits = rng.integers(0, 2**32, size=(64, 6), dtype=np.uint64).astype(np.uint32)
    bits &= ~np.uint32(0x40000000)  # clear the top exponent bit: finite values
    X = bits.view(np.float32)
    assert np.isfinite(X).all()
    q = X[0]
    keys = [_fraction_key(q, x) for x in X[1:]]
    order = sorted(range(len(keys)), key=lambda j: (keys[j], j))
    _, i = oracle.knn(X[1:], q[None, :], 10)
    np.testing.assert_array_equal(i[0], order[:10])


def test_exact_le_boundaries():
    q = np.array([0.0, 0.0], np.float32)
    x = np.array([3.0, 4.0], np.float32)
    assert oracle.exact_le(q, x, 25.0)
    assert not oracle.exact_le(q, x, np.nextafter(25.0, 0))
    assert oracle.exact_le(q, x, float("inf"))
    assert oracle.exact_le(q, q, 0.0)
    assert not oracle.exact_le(q, x, 0.0)


def test_oracle_matches_reference_native_scan():
    """Second checker: the reference's compiled exact scan, when oracle/_ref exists."""
    ref = oracle.ref_native()
    if ref is None:
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(11)
    X = rng.integers(-2, 3, size=(3000, 12)).astype(np.float32)  # lattice: many ties
    Q = rng.integers(-2, 3, size=(64, 12)).astype(np.float32) + 0.25
    rd = np.empty((64, 9)); ri = np.empty((64, 9), np.int64)
    ref.neighbors.query(X, Q, 9, False, 0, rd, ri)
    d, i = oracle.knn(X, Q, 9)
    np.testing.assert_array_equal(i, ri)
    np.testing.assert_allclose(d, rd, rtol=1e-12)
