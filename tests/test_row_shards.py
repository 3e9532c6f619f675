"""Reference-row shards merged in one process (CPU restatement of the device steps).

Checks the merge protocol itself: the answer over S row shards, after the
float64 merge, the flagging of cross-shard near ties and the exact resolve,
equals one oracle search over all rows (indices and distances bit-exact),
including exact duplicates that sit in different shards, a shard with fewer
rows than k, and self-exclusion.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

import oracle
from _row_shards_cpu import CpuRowShardOps, CpuShard, planted_rows
from mlxlearn_b200.sharding import merge_row_shards


class CountingOps(CpuRowShardOps):
    flagged = 0

    def merge(self, D, I, k, d, self_offset):
        out = super().merge(D, I, k, d, self_offset)
        self.flagged += int(out[2].sum())
        return out


@pytest.mark.parametrize("n_shards,k", [(2, 5), (3, 9)])
def test_row_shards_equal_one_search(n_shards, k):
    rng = np.random.default_rng(30 + n_shards)
    X, bounds = planted_rows(rng, 1200, 6, n_shards)
    Q = np.concatenate([rng.standard_normal((60, 6)), X[:10] + 1e-3, X[:5]]).astype(np.float32)
    parts = [(CpuShard(X[a:b]), int(a)) for a, b in zip(bounds[:-1], bounds[1:])]
    ops = CountingOps()
    d, i = merge_row_shards(parts, torch.from_numpy(Q), k, ops=ops)
    od, oi = oracle.knn(X, Q, k)
    np.testing.assert_array_equal(i.numpy(), oi)
    np.testing.assert_array_equal(d.numpy(), od)
    assert ops.flagged > 0  # the planted cross-shard duplicates took the exact path


def test_row_shards_self_exclusion_and_small_shard():
    rng = np.random.default_rng(41)
    X = rng.standard_normal((300, 4)).astype(np.float32)
    X[290:296] = X[:6]  # duplicates across the shard boundary
    bounds = [0, 7, 150, 300]  # the first shard holds fewer rows than k + 1
    parts = [(CpuShard(X[a:b]), a) for a, b in zip(bounds[:-1], bounds[1:])]
    d, i = merge_row_shards(parts, torch.from_numpy(X[:40]), 8, exclude_self=True, q_offset=0,
                            ops=CpuRowShardOps())
    od, oi = oracle.knn(X, X[:40], 8, exclude_self=True)
    np.testing.assert_array_equal(i.numpy(), oi)
    np.testing.assert_array_equal(d.numpy(), od)
    assert not np.any(i.numpy() == np.arange(40)[:, None])


def test_row_shards_reject_bad_k():
    X = np.zeros((10, 2), np.float32)
    parts = [(CpuShard(X[:5]), 0), (CpuShard(X[5:]), 5)]
    with pytest.raises(ValueError, match="n_neighbors must be <= 10"):
        merge_row_shards(parts, torch.zeros((1, 2)), 11, ops=CpuRowShardOps())
    with pytest.raises(ValueError, match="n_neighbors must be <= 9"):
        merge_row_shards(parts, torch.zeros((10, 2)), 10, exclude_self=True, ops=CpuRowShardOps())


@pytest.mark.parametrize("sort_results", [False, True])
def test_radius_row_shards_equal_one_search(sort_results):
    from _row_shards_cpu import oracle_radius_local
    from mlxlearn_b200.sharding import merge_radius_row_shards

    rng = np.random.default_rng(70)
    X, bounds = planted_rows(rng, 2000, 3, 3)
    Q = np.concatenate([rng.standard_normal((50, 3)), X[:10]]).astype(np.float32)
    parts = [(CpuShard(X[a:b]), int(a)) for a, b in zip(bounds[:-1], bounds[1:])]
    res = merge_radius_row_shards(parts, Q, 0.6, sort_results=sort_results,
                                  local=oracle_radius_local)
    ip, ii, dd = oracle.radius(X, Q, 0.6, sort_results=sort_results)
    np.testing.assert_array_equal(res.indptr, ip)
    np.testing.assert_array_equal(res.indices, ii)
    np.testing.assert_array_equal(res.distances, dd)
    # self-query: every row drops its own global index
    res = merge_radius_row_shards(parts, X[:100], 0.6, exclude_self=True, q_offset=0,
                                  sort_results=sort_results, local=oracle_radius_local)
    ip, ii, dd = oracle.radius(X, X[:100], 0.6, exclude_self=True, sort_results=sort_results)
    np.testing.assert_array_equal(res.indptr, ip)
    np.testing.assert_array_equal(res.indices, ii)
    np.testing.assert_array_equal(res.distances, dd)


def test_row_shards_lattice_ties():
    # integer lattice points: exact duplicates and equal distances everywhere,
    # spread over four shards; every tie breaks by global row
    rng = np.random.default_rng(95)
    X = rng.integers(-3, 4, size=(1600, 4)).astype(np.float32)
    Q = (rng.integers(-3, 4, size=(120, 4)) + 0.5).astype(np.float32)
    bounds = [0, 300, 800, 1100, 1600]
    parts = [(CpuShard(X[a:b]), a) for a, b in zip(bounds[:-1], bounds[1:])]
    ops = CountingOps()
    d, i = merge_row_shards(parts, torch.from_numpy(Q), 10, ops=ops)
    od, oi = oracle.knn(X, Q, 10)
    np.testing.assert_array_equal(i.numpy(), oi)
    np.testing.assert_array_equal(d.numpy(), od)
    assert ops.flagged > 0


@pytest.mark.parametrize("seed", range(6))
def test_row_shards_random_layouts(seed):
    # random shard counts and uneven boundaries, duplicates planted across
    # shards, self-queries on some seeds
    rng = np.random.default_rng(1000 + seed)
    n, d = int(rng.integers(200, 900)), int(rng.integers(2, 9))
    X = rng.normal(size=(n, d)).astype(np.float32)
    dup = rng.integers(0, n, size=12)
    X[rng.integers(0, n, size=12)] = X[dup]
    S = int(rng.integers(2, 7))
    cuts = np.sort(rng.choice(np.arange(1, n), size=S - 1, replace=False))
    bounds = [0, *cuts.tolist(), n]
    parts = [(CpuShard(X[a:b]), int(a)) for a, b in zip(bounds[:-1], bounds[1:])]
    k = int(rng.integers(1, 12))
    exclude = bool(seed % 2)
    Q = X[:50] if exclude else rng.normal(size=(50, d)).astype(np.float32)
    d_, i_ = merge_row_shards(parts, torch.from_numpy(np.ascontiguousarray(Q)), k,
                              exclude_self=exclude, q_offset=0, ops=CpuRowShardOps())
    od, oi = oracle.knn(X, Q, k, exclude_self=exclude)
    np.testing.assert_array_equal(i_.numpy(), oi)
    np.testing.assert_array_equal(d_.numpy(), od)
