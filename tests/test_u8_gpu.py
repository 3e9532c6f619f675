"""The exact u8 screen (tcgen05 kind::i8) for integer pixels.

When the index and the queries hold integers in [0, 255] only, AUTO answers
k <= 16 with exact integer products and a merge of the per-list top-k (no
certified band): indices and canonical float64 distances must equal the
oracle's bit for bit, ties in training-index order.  Data that do not
qualify (a fractional query, k > 16, an explicit u8 request on float data)
take the certified screens and stay exact.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from datasets import pixels

pytestmark = pytest.mark.gpu

MODE_U8 = 5


def make_index(X):
    from mlxlearn_b200.index import build_index

    return build_index(X)


def ints(rng, shape, hi=256):
    return rng.integers(0, hi, shape).astype(np.float32)


def check_u8(index, X, Q, k, **kw):
    d, i = index.query(Q, k, stats=True, **kw)
    assert index.last_stats["mode_used"] == MODE_U8
    od, oi = oracle.knn(X, Q, k, exclude_self=kw.get("exclude_self", False))
    np.testing.assert_array_equal(i, oi)
    np.testing.assert_array_equal(d, od)


@pytest.mark.parametrize("n,d,m,k", [(3000, 16, 130, 5), (20000, 100, 257, 16),
                                     (9001, 784, 64, 1), (60000, 784, 300, 5),
                                     (2048, 300, 2000, 8)])
def test_u8_matches_oracle(n, d, m, k):
    rng = np.random.default_rng(n + d)
    X, _, T = pixels(rng, n, d)
    Q, _, _ = pixels(rng, m, d, templates=T)
    check_u8(make_index(X), X, Q, k)


def test_u8_ties_duplicates_and_self_query():
    rng = np.random.default_rng(31)
    X = ints(rng, (5000, 32), hi=4)  # few distinct values: many equal distances
    X[1000:1100] = X[:100]
    index = make_index(X)
    Q = np.concatenate([X[:50], ints(rng, (150, 32), hi=4)])
    check_u8(index, X, Q, 16)
    check_u8(index, X, Q, 3)
    check_u8(index, X, X, 7, exclude_self=True)


def test_u8_self_query_with_offset_on_the_device():
    """A slice of the training rows as queries: q_offset places each query's
    own row, which the u8 screen excludes."""
    import torch

    rng = np.random.default_rng(34)
    X = ints(rng, (12000, 40), hi=8)
    X[6000:6040] = X[5000:5040]  # duplicates across the slice boundary
    index = make_index(X)
    Xd = torch.from_numpy(X).cuda()
    for lo in (0, 4990, 9000):
        dd, di = index.query_device(Xd[lo:lo + 3000], 9, exclude_self=True, q_offset=lo,
                                    stats=True)
        assert index.last_stats["mode_used"] == MODE_U8
        od, oi = oracle.knn(X, X[lo:lo + 3000], 9, exclude_self=True, q_offset=lo)
        np.testing.assert_array_equal(di.cpu().numpy(), oi)
        np.testing.assert_array_equal(dd.cpu().numpy(), od)


def test_u8_squared_distances_on_the_device():
    import torch

    rng = np.random.default_rng(32)
    X, _, T = pixels(rng, 8000, 64)
    Q, _, _ = pixels(rng, 300, 64, templates=T)
    index = make_index(X)
    d2, i2 = index.query_device(torch.from_numpy(Q).cuda(), 6, _squared=True, stats=True)
    assert index.last_stats["mode_used"] == MODE_U8
    od, oi = oracle.knn(X, Q, 6)
    np.testing.assert_array_equal(i2.cpu().numpy(), oi)
    # the exact integer squared distances (float64 sums of integer squares)
    diff = Q[:, None, :].astype(np.float64) - X[oi].astype(np.float64)
    np.testing.assert_array_equal(d2.cpu().numpy(), (diff * diff).sum(axis=2))
    np.testing.assert_array_equal(np.sqrt(d2.cpu().numpy()), od)


def test_u8_not_taken_for_other_data():
    rng = np.random.default_rng(33)
    X, _, T = pixels(rng, 6000, 48)
    index = make_index(X)
    Q, _, _ = pixels(rng, 200, 48, templates=T)
    Qf = Q.copy()
    Qf[7, 3] = 12.5  # one fractional coordinate: the certified screen runs
    d, i = index.query(Qf, 5, stats=True)
    assert index.last_stats["mode_used"] != MODE_U8
    od, oi = oracle.knn(X, Qf, 5)
    np.testing.assert_array_equal(i, oi)
    np.testing.assert_array_equal(d, od)
    d, i = index.query(Q, 17, stats=True)  # past the u8 screen's k
    assert index.last_stats["mode_used"] != MODE_U8
    od, oi = oracle.knn(X, Q, 17)
    np.testing.assert_array_equal(i, oi)
    Xf = X + 0.25  # float data: an explicit u8 request runs the certified screens
    findex = make_index(Xf)
    d, i = findex.query(Q, 5, mode="u8", stats=True)
    assert findex.last_stats["mode_used"] != MODE_U8
    od, oi = oracle.knn(Xf, Q, 5)
    np.testing.assert_array_equal(i, oi)
    np.testing.assert_array_equal(d, od)
