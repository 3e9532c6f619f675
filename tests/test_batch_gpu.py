"""Batched uneven problems (KnnBatch / b2k_batch_*) against the oracle.

Every problem of a batch must return exactly what a single-problem query
returns: indices bit-exact to the float64 + exact-tie oracle and the
oracle's canonical distances.  Problems mix widths (the concatenated operand
groups), heap widths (one screen launch each), a self-query, two problems on
one index, a problem below the bf16 screen's width (answered outside the
graph), and 1% duplicated rows (ties resolved to the smaller index).
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from datasets import cfg4

pytestmark = pytest.mark.gpu


def _problems(seed=5, count=24):
    probs = cfg4(seed=seed, problems=count, n_range=(1_000, 12_000), m_range=(50, 1_500))
    rng = np.random.default_rng(seed + 100)
    # below the tensor-core width: answered through the single-problem path
    Xs = rng.standard_normal((3000, 8)).astype(np.float32)
    probs.append((Xs, rng.standard_normal((300, 8)).astype(np.float32), 5))
    # wide rows: query tiles streamed with every block
    Xw = rng.standard_normal((2500, 320)).astype(np.float32)
    probs.append((Xw, rng.standard_normal((200, 320)).astype(np.float32), 10))
    return probs


def _build(probs, shared=(), self_query=None):
    import torch

    from mlxlearn_b200.index import build_index

    indexes = [build_index(X) for X, _, _ in probs]
    items, truth = [], []
    for i, (X, Q, k) in enumerate(probs):
        items.append((indexes[i], torch.from_numpy(Q).cuda(), k))
        truth.append((X, Q, k, False))
    for a in shared:  # a second query block on problem a's index
        X, _, k = probs[a]
        Q = np.random.default_rng(a).standard_normal((77, X.shape[1])).astype(np.float32)
        items.append((indexes[a], torch.from_numpy(Q).cuda(), k))
        truth.append((X, Q, k, False))
    if self_query is not None:
        X, _, k = probs[self_query]
        items.append((indexes[self_query], torch.from_numpy(X).cuda(), k, True))
        truth.append((X, X, k, True))
    return indexes, items, truth


def _check(results, truth):
    for (dist, idx), (X, Q, k, self_q) in zip(results, truth):
        rd, ri = oracle.knn(X, Q, k, exclude_self=self_q)
        gi = idx.cpu().numpy()
        assert np.array_equal(gi, ri), f"indices differ for n={X.shape[0]} d={X.shape[1]} k={k}"
        assert np.array_equal(dist.cpu().numpy(), rd)


def test_batch_matches_oracle_and_replays():
    import torch

    from mlxlearn_b200.batch import KnnBatch

    probs = _problems()
    indexes, items, truth = _build(probs, shared=[0], self_query=2)
    batch = KnnBatch(items)
    results = batch()
    st = batch.last_stats
    assert st["problems"] == len(items)
    assert st["graph_problems"] == len(items) - 1  # the d=8 problem runs outside the graph
    assert st["screen_launches"] >= 3
    _check(results, truth)
    # replay the graph on new queries written into the same buffers
    rng = np.random.default_rng(99)
    new_truth = []
    for (ix, Qd, k, *rest), (X, Q, _, self_q) in zip(items, truth):
        if self_q:
            new_truth.append((X, Q, k, True))
            continue
        Qn = rng.standard_normal(Q.shape).astype(np.float32)
        Qd.copy_(torch.from_numpy(Qn))
        new_truth.append((X, Qn, k, False))
    results = batch()
    _check(results, new_truth)
    batch.close()


def test_batch_autotune_same_answers():
    from mlxlearn_b200.batch import KnnBatch

    probs = _problems(seed=6, count=10)
    indexes, items, truth = _build(probs)
    batch = KnnBatch(items, autotune=True)
    results = batch()
    _check(results, truth)
    assert batch.last_stats["tune_ms"] >= 0.0
    batch.close()


def test_batch_ties_and_duplicates():
    import torch

    from mlxlearn_b200.batch import kneighbors_batch
    from mlxlearn_b200.index import build_index

    rng = np.random.default_rng(3)
    # every row duplicated 4x: each query's k nearest are tied groups
    base = rng.integers(-3, 4, (700, 24)).astype(np.float32)
    X = np.repeat(base, 4, axis=0)
    Q = rng.integers(-3, 4, (300, 24)).astype(np.float32)
    ix = build_index(X)
    res = kneighbors_batch([(ix, torch.from_numpy(Q).cuda(), 10),
                            (ix, torch.from_numpy(X[:500]).cuda(), 7)])
    _check(res, [(X, Q, 10, False), (X, X[:500], 7, False)])


def test_batch_rejects_bad_problems():
    import torch

    from mlxlearn_b200.batch import KnnBatch
    from mlxlearn_b200.index import build_index

    X = np.random.default_rng(0).standard_normal((100, 16)).astype(np.float32)
    ix = build_index(X)
    with pytest.raises(ValueError):
        KnnBatch([(ix, torch.zeros((5, 16), device="cuda"), 101)])
    with pytest.raises(ValueError):
        KnnBatch([(ix, torch.zeros((5, 8), device="cuda"), 3)])
    with pytest.raises(TypeError):
        KnnBatch([(ix, torch.zeros((5, 16)), 3)])


def test_empty_and_zero_row_problems():
    import torch

    from mlxlearn_b200.batch import KnnBatch
    from mlxlearn_b200.index import build_index

    X = np.random.default_rng(1).standard_normal((4000, 32)).astype(np.float32)
    ix = build_index(X)
    b = KnnBatch([])
    assert b() == []
    b.close()
    Q = np.random.default_rng(2).standard_normal((130, 32)).astype(np.float32)
    b = KnnBatch([(ix, torch.zeros((0, 32), device="cuda"), 3),
                  (ix, torch.from_numpy(Q).cuda(), 3)])
    res = b()
    assert res[0][1].shape == (0, 3)
    _check(res[1:], [(X, Q, 3, False)])
    b.close()
