"""Reference-row shards through the CUDA library (shards emulated in one process).

Each shard is its own device index over a contiguous range of the rows; the
merge (csrc/shards.cu: float64 k-way merge, flags for cross-shard near ties,
exact keys, exact resolve) must return one oracle search over all rows,
indices and distances bit-exact.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from _row_shards_cpu import planted_rows

pytestmark = pytest.mark.gpu


def _ops(mode=None):
    from mlxlearn_b200.sharding import RowShardOps

    class Ops(RowShardOps):
        flagged = 0

        def search(self, index, Q, k):
            return index.query_device(Q, k, mode=mode)

        def merge(self, D, I, k, d, self_offset):
            out = super().merge(D, I, k, d, self_offset)
            self.flagged += int(out[2].sum())
            return out

    return Ops()


def _parts(X, bounds):
    from mlxlearn_b200.index import build_index

    return [(build_index(X[a:b]), int(a)) for a, b in zip(bounds[:-1], bounds[1:])]


@pytest.mark.parametrize("n_shards,k,mode", [(2, 10, "bf16"), (3, 1, "fp32"), (5, 40, "bf16"),
                                             (4, 7, "exact")])
def test_row_shards_equal_one_search(n_shards, k, mode):
    import torch

    from mlxlearn_b200.sharding import merge_row_shards

    rng = np.random.default_rng(50 + n_shards)
    X, bounds = planted_rows(rng, 30000, 32, n_shards)
    Q = np.concatenate([rng.standard_normal((700, 32)), X[:20] + 1e-3, X[:10]]).astype(np.float32)
    ops = _ops(mode)
    d, i = merge_row_shards(_parts(X, bounds), torch.from_numpy(Q).cuda(), k, ops=ops)
    od, oi = oracle.knn(X, Q, k)
    np.testing.assert_array_equal(i.cpu().numpy(), oi)
    np.testing.assert_array_equal(d.cpu().numpy(), od)
    assert ops.flagged > 0  # the planted cross-shard duplicates took the exact path


def test_row_shards_exact_order_across_shards():
    # rows 1902 and 43153: float32 squared distances to query 79 round equal,
    # the exact order puts 43153 first; they sit in different shards here
    import torch

    from mlxlearn_b200.sharding import merge_row_shards

    rng = np.random.default_rng(251)
    train = (rng.normal(size=(50_000, 32)) + 10_000).astype(np.float32)
    queries = (rng.normal(size=(256, 32)) + 10_000).astype(np.float32)
    Q = np.repeat(queries[79:80], 3, axis=0)
    od, oi = oracle.knn(train, Q, 5)
    assert oi[0, 3] == 43153 and oi[0, 4] == 1902
    d, i = merge_row_shards(_parts(train, [0, 25000, 50000]), torch.from_numpy(Q).cuda(), 5,
                            ops=_ops())
    np.testing.assert_array_equal(i.cpu().numpy(), oi)
    np.testing.assert_array_equal(d.cpu().numpy(), od)


def test_row_shards_self_query():
    import torch

    from mlxlearn_b200.sharding import merge_row_shards

    rng = np.random.default_rng(60)
    X, bounds = planted_rows(rng, 12000, 24, 3)
    d, i = merge_row_shards(_parts(X, bounds), torch.from_numpy(X[:600]).cuda(), 6,
                            exclude_self=True, q_offset=0, ops=_ops())
    od, oi = oracle.knn(X, X[:600], 6, exclude_self=True)
    np.testing.assert_array_equal(i.cpu().numpy(), oi)
    np.testing.assert_array_equal(d.cpu().numpy(), od)
    assert not np.any(i.cpu().numpy() == np.arange(600)[:, None])


@pytest.mark.parametrize("sort_results", [False, True])
def test_radius_row_shards_equal_one_search(sort_results):
    from mlxlearn_b200.sharding import merge_radius_row_shards

    rng = np.random.default_rng(80)
    X, bounds = planted_rows(rng, 20000, 8, 3)
    Q = np.concatenate([rng.standard_normal((300, 8)), X[:20]]).astype(np.float32)
    res = merge_radius_row_shards(_parts(X, bounds), Q, 1.4, sort_results=sort_results)
    ip, ii, dd = oracle.radius(X, Q, 1.4, sort_results=sort_results)
    np.testing.assert_array_equal(res.indptr, ip)
    np.testing.assert_array_equal(res.indices, ii)
    np.testing.assert_array_equal(res.distances, dd)
    res = merge_radius_row_shards(_parts(X, bounds), X[:500], 1.4, exclude_self=True,
                                  q_offset=0, sort_results=sort_results)
    ip, ii, dd = oracle.radius(X, X[:500], 1.4, exclude_self=True, sort_results=sort_results)
    np.testing.assert_array_equal(res.indptr, ip)
    np.testing.assert_array_equal(res.indices, ii)
    np.testing.assert_array_equal(res.distances, dd)


def test_row_shards_lattice_ties():
    import torch

    from mlxlearn_b200.sharding import merge_row_shards

    rng = np.random.default_rng(96)
    X = rng.integers(-3, 4, size=(20000, 8)).astype(np.float32)
    Q = (rng.integers(-3, 4, size=(400, 8)) + 0.5).astype(np.float32)
    ops = _ops()
    d, i = merge_row_shards(_parts(X, [0, 4000, 11000, 15000, 20000]),
                            torch.from_numpy(Q).cuda(), 20, ops=ops)
    od, oi = oracle.knn(X, Q, 20)
    np.testing.assert_array_equal(i.cpu().numpy(), oi)
    np.testing.assert_array_equal(d.cpu().numpy(), od)
    assert ops.flagged > 0
