"""Query-sharded replicas on two gloo ranks (CPU).

The multi-GPU kneighbors path partitions a query batch into per-rank shards
against full index replicas; these tests run its host plumbing (row
broadcast, shard bounds, gather in query order, max-over-ranks timing) as two
processes on the gloo backend, with the oracle standing in for each rank's
local search, and check the gathered answer against one unsharded search.
"""
from __future__ import annotations

import os
import socket
import traceback

import numpy as np
import pytest

from mlxlearn_b200.sharding import shard_bounds


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, case, errq):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=60))
        _CASES[case](rank, world)
        dist.barrier()
        dist.destroy_process_group()
    except Exception:
        errq.put((rank, traceback.format_exc()))
        raise


def _case_knn(rank, world):
    import oracle
    from mlxlearn_b200.sharding import broadcast_rows, kneighbors_sharded

    rng = np.random.default_rng(11)
    X = rng.standard_normal((3000, 24)).astype(np.float32) if rank == 0 else None
    X = broadcast_rows(X, src=0)
    assert X.shape == (3000, 24) and X.dtype == np.float32
    Q = np.random.default_rng(12).standard_normal((513, 24)).astype(np.float32)

    def local(Qs, k, start):
        return oracle.knn(X, Qs, k, nthreads=2)

    d, i = kneighbors_sharded(local, Q, 7)
    rd, ri = oracle.knn(X, Q, 7, nthreads=2)
    assert np.array_equal(i, ri)
    assert np.array_equal(d, rd)
    # un-gathered form: this rank's rows only
    ds, is_, start = kneighbors_sharded(local, Q, 7, gather=False)
    a, b = shard_bounds(513, world, rank)
    assert start == a and np.array_equal(is_, ri[a:b])


def _case_self(rank, world):
    # kneighbors() on the training rows: each shard passes its first row as the
    # query offset so row j still skips index j.
    import oracle
    from mlxlearn_b200.sharding import broadcast_rows, kneighbors_sharded

    X = np.random.default_rng(5).standard_normal((801, 9)).astype(np.float32)
    X = broadcast_rows(X if rank == 0 else None)

    def local(Qs, k, start):
        return oracle.knn(X, Qs, k, exclude_self=True, q_offset=start, nthreads=2)

    d, i = kneighbors_sharded(local, X, 5)
    rd, ri = oracle.knn(X, X, 5, exclude_self=True, nthreads=2)
    assert np.array_equal(i, ri) and np.array_equal(d, rd)
    assert not np.any(i == np.arange(801)[:, None])


def _case_tiny(rank, world):
    # fewer queries than ranks: the empty shard still joins the gather
    import oracle
    from mlxlearn_b200.sharding import kneighbors_sharded

    X = np.random.default_rng(6).standard_normal((50, 3)).astype(np.float32)
    Q = X[:1] + 0.25

    def local(Qs, k, start):
        assert Qs.shape[0] > 0
        return oracle.knn(X, Qs, k, nthreads=1)

    d, i = kneighbors_sharded(local, Q, 4)
    rd, ri = oracle.knn(X, Q, 4, nthreads=1)
    assert np.array_equal(i, ri) and np.array_equal(d, rd)


def _case_timer(rank, world):
    import time

    from mlxlearn_b200.sharding import ShardTimer, max_over_ranks

    assert max_over_ranks(float(rank + 1)) == float(world)
    t = ShardTimer()
    t.start()
    time.sleep(0.05 if rank == 1 else 0.0)
    ms = t.stop(steps=1)
    # every rank reports the slowest rank's time
    assert ms >= 45.0, ms


def _case_rows(rank, world):
    # reference-row shards: each rank holds its own rows; one all-gather of the
    # per-shard lists plus the exact-key all-reduce give the all-rows answer
    import torch

    import oracle
    from _row_shards_cpu import CpuRowShardOps, CpuShard, planted_rows
    from mlxlearn_b200.sharding import kneighbors_row_sharded

    rng = np.random.default_rng(21)
    X, bounds = planted_rows(rng, 900, 5, world)
    Q = np.concatenate([rng.standard_normal((40, 5)), X[:8] + 1e-3, X[:4]]).astype(np.float32)
    a, b = int(bounds[rank]), int(bounds[rank + 1])
    d, i = kneighbors_row_sharded(CpuShard(X[a:b]), a, X.shape[0], torch.from_numpy(Q), 6,
                                  ops=CpuRowShardOps())
    od, oi = oracle.knn(X, Q, 6, nthreads=2)
    assert np.array_equal(i.numpy(), oi)
    assert np.array_equal(d.numpy(), od)
    # self-query over the sharded rows
    d, i = kneighbors_row_sharded(CpuShard(X[a:b]), a, X.shape[0], torch.from_numpy(X[:30]), 4,
                                  exclude_self=True, q_offset=0, ops=CpuRowShardOps())
    od, oi = oracle.knn(X, X[:30], 4, exclude_self=True, nthreads=2)
    assert np.array_equal(i.numpy(), oi) and np.array_equal(d.numpy(), od)


def _case_radius_rows(rank, world):
    import oracle
    from _row_shards_cpu import CpuShard, oracle_radius_local, planted_rows
    from mlxlearn_b200.sharding import radius_neighbors_row_sharded

    rng = np.random.default_rng(22)
    X, bounds = planted_rows(rng, 1500, 3, world)
    Q = np.concatenate([rng.standard_normal((30, 3)), X[:6]]).astype(np.float32)
    a, b = int(bounds[rank]), int(bounds[rank + 1])
    for sort_results in (False, True):
        res = radius_neighbors_row_sharded(CpuShard(X[a:b]), a, Q, 0.7,
                                           sort_results=sort_results, local=oracle_radius_local)
        ip, ii, dd = oracle.radius(X, Q, 0.7, sort_results=sort_results, nthreads=2)
        assert np.array_equal(res.indptr, ip) and np.array_equal(res.indices, ii)
        assert np.array_equal(res.distances, dd)
    # a rank with no entries for any query still joins both gathers
    res = radius_neighbors_row_sharded(CpuShard(X[a:b]), a, Q + 100.0, 0.1,
                                       local=oracle_radius_local)
    assert res.nnz == 0 and res.indptr.shape == (Q.shape[0] + 1,)


_CASES = {"knn": _case_knn, "self": _case_self, "tiny": _case_tiny, "timer": _case_timer,
          "rows": _case_rows, "radius_rows": _case_radius_rows}


def _run(case, world=2):
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    errq = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, errq)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
        p.join()
    errs = []
    while not errq.empty():
        errs.append(errq.get())
    assert not alive, f"ranks did not finish: {[p.pid for p in alive]}"
    assert not errs, "\n".join(f"rank {r}:\n{tb}" for r, tb in errs)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]


@pytest.mark.parametrize("m,world", [(0, 2), (1, 2), (513, 2), (100000, 8), (7, 3)])
def test_shard_bounds_partition(m, world):
    spans = [shard_bounds(m, world, r) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == m
    for (a0, b0), (a1, b1) in zip(spans, spans[1:]):
        assert b0 == a1
    sizes = [b - a for a, b in spans]
    assert max(sizes) - min(sizes) <= 1


def test_shard_bounds_rejects_bad_rank():
    with pytest.raises(ValueError):
        shard_bounds(10, 2, 2)
    with pytest.raises(ValueError):
        shard_bounds(-1, 2, 0)


@pytest.mark.parametrize("case", ["knn", "self", "tiny", "timer", "rows", "radius_rows"])
def test_gloo_two_ranks(case):
    _run(case)
