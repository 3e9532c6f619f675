"""Radius search parity: exact membership, CSR layout, canonical distances.

Checked against the reference's own outputs (tests/golden) and the oracle,
bit-exact: indptr, indices and distances (the canonical float64 value is
deterministic)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import golden
from datasets import mixture

pytestmark = pytest.mark.gpu


def make_index(X):
    from mlxlearn_b200.index import build_index

    return build_index(X)


def csr(parts):
    from mlxlearn_b200.radius_result import join_batches

    return join_batches(parts)


def test_radius_matches_reference_fixture():
    rng = np.random.default_rng(4)
    cen = rng.normal(0, 2.0, (10, 32))
    X, y = mixture(rng, 20000, cen, 1.0)
    Q, _ = mixture(np.random.default_rng(44), 500, cen, 1.0)
    Q[:5] += 40.0
    g = golden("radius_mixture32.npz")
    r = float(g["radius"])
    index = make_index(X)
    ip, ix, dd = csr(index.query_radius_csr(Q, r))
    np.testing.assert_array_equal(ip, g["indptr"])
    np.testing.assert_array_equal(ix, g["indices"])
    np.testing.assert_array_equal(dd, g["dist"])
    ip, ix, dd = csr(index.query_radius_csr(Q, r, sort_results=True))
    np.testing.assert_array_equal(ix, g["sorted_indices"])
    np.testing.assert_array_equal(dd, g["sorted_dist"])


@pytest.mark.parametrize("n,d,m", [(3000, 8, 200), (5000, 32, 300), (2500, 130, 64),
                                   (40, 3, 40)])
def test_radius_matches_oracle(n, d, m, rng):
    X = rng.normal(size=(n, d)).astype(np.float32)
    Q = rng.normal(size=(m, d)).astype(np.float32)
    _, oi = oracle.knn(X, Q[:20], min(20, n))
    r = float(np.median(oracle.knn(X, Q[:20], min(20, n))[0][:, -1]))
    index = make_index(X)
    for sort in (False, True):
        op, oix, od = oracle.radius(X, Q, r, sort_results=sort)
        ip, ix, dd = csr(index.query_radius_csr(Q, r, sort_results=sort))
        np.testing.assert_array_equal(ip, op)
        np.testing.assert_array_equal(ix, oix)
        np.testing.assert_array_equal(dd, od)


def test_radius_exact_boundary_lattice(rng):
    """Integer lattice with radius exactly on many squared distances: the band
    must be resolved exactly (S <= R2 inclusive)."""
    X = rng.integers(-4, 5, size=(4000, 6)).astype(np.float32)
    Q = rng.integers(-4, 5, size=(100, 6)).astype(np.float32)
    index = make_index(X)
    for r in (0.0, 1.0, 2.0, np.sqrt(3.0), 3.0):
        op, oix, od = oracle.radius(X, Q, r)
        ip, ix, dd = csr(index.query_radius_csr(Q, r))
        np.testing.assert_array_equal(ip, op)
        np.testing.assert_array_equal(ix, oix)
        np.testing.assert_array_equal(dd, od)


def test_radius_self_exclusion_and_infinite_radius(rng):
    X = rng.normal(size=(600, 5)).astype(np.float32)
    X[10:20] = X[:10]
    index = make_index(X)
    op, oix, od = oracle.radius(X, X, 1.5, exclude_self=True)
    ip, ix, dd = csr(index.query_radius_csr(X, 1.5, exclude_self=True))
    np.testing.assert_array_equal(ip, op)
    np.testing.assert_array_equal(ix, oix)
    ip, ix, _ = csr(index.query_radius_csr(X[:30], np.inf, need_distance=False))
    assert (np.diff(ip) == 600).all()
    np.testing.assert_array_equal(ix[:600], np.arange(600))


def test_radius_empty_and_zero_neighbours(rng):
    X = rng.normal(size=(100, 4)).astype(np.float32)
    index = make_index(X)
    ip, ix, dd = csr(index.query_radius_csr(np.empty((0, 4), np.float32), 1.0))
    assert ip.tolist() == [0] and len(ix) == 0
    ip, ix, dd = csr(index.query_radius_csr(X[:5] + 100, 1.0))
    assert (ip == 0).all()
    with pytest.raises(ValueError, match="non-negative"):
        index.query_radius_csr(X, -1.0)
    with pytest.raises(TypeError):
        index.query_radius_csr(X, "1")


def test_radius_big_rows_sort(rng):
    """Rows longer than the shared-memory sort capacity take the global path."""
    X = rng.normal(size=(9000, 4)).astype(np.float32)
    Q = rng.normal(size=(3, 4)).astype(np.float32)
    index = make_index(X)
    op, oix, od = oracle.radius(X, Q, 3.0, sort_results=True)
    ip, ix, dd = csr(index.query_radius_csr(Q, 3.0, sort_results=True))
    assert np.diff(op).max() > 4096
    np.testing.assert_array_equal(ip, op)
    np.testing.assert_array_equal(ix, oix)
    np.testing.assert_array_equal(dd, od)


@pytest.mark.parametrize("sort", [True, False])
def test_radius_every_sort_stage_in_one_call(sort):
    """Row lengths from 3 to 7,330 in one call: rows of up to 256 entries
    are sorted by one warp each, up to 4,096 by one CTA each and longer rows
    by the global-memory sort; every stage runs, with rows on both sides of
    1,024 inside the CTA stage."""
    rng = np.random.default_rng(31)
    X = rng.normal(size=(9000, 4)).astype(np.float32)
    dirs = rng.normal(size=(48, 4))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    Q = (dirs * np.linspace(0, 5.5, 48)[:, None]).astype(np.float32)
    op, oix, od = oracle.radius(X, Q, 2.5, sort_results=sort)
    lens = np.diff(op)
    for lo, hi in ((2, 256), (257, 1024), (1025, 4096), (4097, 1 << 30)):
        assert ((lens >= lo) & (lens <= hi)).sum() >= 5
    index = make_index(X)
    ip, ix, dd = csr(index.query_radius_csr(Q, 2.5, sort_results=sort))
    np.testing.assert_array_equal(ip, op)
    np.testing.assert_array_equal(ix, oix)
    np.testing.assert_array_equal(dd, od)


@pytest.mark.parametrize("group", ["0", "1"])
def test_radius_row_grouping_both_ways(group, monkeypatch):
    """With grouped operand rows the fill pass lists operand rows; they are
    mapped to training rows and each row re-sorted by index (or by distance
    when asked), rows past the shared-memory sort included."""
    monkeypatch.setenv("B2K_GROUP_ROWS", group)
    C = np.random.default_rng(18).normal(0, 2.0, (12, 24))
    X, _ = mixture(np.random.default_rng(19), 24000, C, 1.0)
    Q, _ = mixture(np.random.default_rng(20), 400, C, 1.0)
    index = make_index(X)
    for r, sort in ((5.0, False), (5.0, True), (12.0, False), (12.0, True)):
        op, oix, od = oracle.radius(X, Q, r, sort_results=sort)
        ip, ix, dd = csr(index.query_radius_csr(Q, r, sort_results=sort))
        np.testing.assert_array_equal(ip, op)
        np.testing.assert_array_equal(ix, oix)
        np.testing.assert_array_equal(dd, od)
    assert np.diff(op).max() > 4096  # the r = 12 rows exceed the shared-memory sort
    ip, ix, dd = csr(index.query_radius_csr(Q, 5.0, need_distance=False))
    op, oix, _ = oracle.radius(X, Q, 5.0)
    np.testing.assert_array_equal(ip, op)
    np.testing.assert_array_equal(ix, oix)
    assert dd is None
    op, oix, od = oracle.radius(X, X, 4.0, exclude_self=True)
    ip, ix, dd = csr(index.query_radius_csr(X, 4.0, exclude_self=True))
    np.testing.assert_array_equal(ip, op)
    np.testing.assert_array_equal(ix, oix)
    np.testing.assert_array_equal(dd, od)


@pytest.mark.parametrize("cap", ["0", "4", "40"])
def test_radius_single_pass_overflow_and_counted_form(cap, monkeypatch):
    """The tcgen05 radius screen runs once into lists of a fixed capacity; a
    row whose count passes it in any list is answered again by the counted
    two-pass form on those rows alone and scattered into the CSR.  Capacity 0
    is the counted form for every row; 4 sends most rows (and every row past
    4 x 4 x 64 entries) through the sub-call, self-queries included (their
    excluded column follows the row into the sub-call); 40 only the long
    rows."""
    monkeypatch.setenv("B2K_RADIUS_CAP", cap)
    C = np.random.default_rng(21).normal(0, 2.0, (12, 24))
    X, _ = mixture(np.random.default_rng(22), 24000, C, 1.0)
    Q, _ = mixture(np.random.default_rng(23), 600, C, 1.0)
    Q[:3] += 30.0  # no neighbours
    index = make_index(X)
    for r, sort in ((5.0, False), (5.0, True), (12.0, False), (12.0, True)):
        op, oix, od = oracle.radius(X, Q, r, sort_results=sort)
        ip, ix, dd = csr(index.query_radius_csr(Q, r, sort_results=sort))
        np.testing.assert_array_equal(ip, op)
        np.testing.assert_array_equal(ix, oix)
        np.testing.assert_array_equal(dd, od)
    assert np.diff(op).max() > 4 * 4 * 64  # overflows any list layout at capacity 4
    ip, ix, dd = csr(index.query_radius_csr(Q, 12.0, need_distance=False))
    op, oix, _ = oracle.radius(X, Q, 12.0)
    np.testing.assert_array_equal(ip, op)
    np.testing.assert_array_equal(ix, oix)
    assert dd is None
    op, oix, od = oracle.radius(X, X, 4.0, exclude_self=True)
    ip, ix, dd = csr(index.query_radius_csr(X, 4.0, exclude_self=True))
    np.testing.assert_array_equal(ip, op)
    np.testing.assert_array_equal(ix, oix)
    np.testing.assert_array_equal(dd, od)
