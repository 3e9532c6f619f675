"""b2k_knn_device_noalloc: the kNN entry point that allocates no memory.

It serves callers that may not allocate device memory during a query (their
GPU memory belongs to another allocator, or allocation's implicit
synchronisation is not allowed on their path).  Its scratch is a fixed array
inside the library.  These tests call it through the C ABI and compare its
output with the oracle (indices and canonical distances bit-exact, the
tolerance of the other kNN tests), on calls in a row that reuse the array the
previous call left behind, and on each branch it has: the screen with the
certified re-rank, the exhaustive scan for k > 64 or an out-of-range index,
the exhaustive redo for an out-of-range query coordinate, and the non-finite
query error.

This file is named so that pytest collects it last.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _noalloc(index, Q, k, exclude_self=False, q_offset=0, want_dist=True):
    """One call through the C ABI; returns (rc, dist or None, idx) on the host."""
    import torch

    from mlxlearn_b200 import _lib

    h = index._ensure_device()
    m = Q.shape[0]
    Qd = torch.from_numpy(np.ascontiguousarray(Q, dtype=np.float32)).cuda()
    ni = torch.full((m, k), -7, dtype=torch.int64, device="cuda")
    nd = torch.full((m, k), -7.0, dtype=torch.float64, device="cuda") if want_dist else None
    rc = _lib.load().b2k_knn_device_noalloc(
        h, _ptr(Qd), m, k, int(exclude_self), q_offset, None if nd is None else _ptr(nd),
        _ptr(ni), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return rc, (None if nd is None else nd.cpu().numpy()), ni.cpu().numpy()


def _check(index, X, Q, k, **kw):
    from mlxlearn_b200 import _lib

    rc, nd, ni = _noalloc(index, Q, k, **kw)
    assert rc == 0, _lib.last_error()
    od, oi = oracle.knn(X, Q, k, exclude_self=kw.get("exclude_self", False),
                       q_offset=kw.get("q_offset", 0))
    np.testing.assert_array_equal(ni, oi)
    np.testing.assert_array_equal(nd, od)


def test_noalloc_matches_oracle_on_consecutive_calls():
    from mlxlearn_b200.index import build_index

    rng = np.random.default_rng(5)
    X = rng.standard_normal((20000, 48)).astype(np.float32)
    X[500:520] = X[:20]  # exact duplicates: index tie rule
    index = build_index(X)
    # the second call reuses the array the first one wrote; a third with a
    # smaller k and a duplicated-row query checks the cleared counters again
    Q3 = np.concatenate([X[:20], rng.standard_normal((80, 48))]).astype(np.float32)
    for Q, k in [(rng.standard_normal((700, 48)).astype(np.float32), 10),
                 (rng.standard_normal((1500, 48)).astype(np.float32), 7),
                 (Q3, 3)]:
        _check(index, X, Q, k)


def test_noalloc_self_query_and_size_limit():
    from mlxlearn_b200 import _lib
    from mlxlearn_b200.index import build_index

    rng = np.random.default_rng(6)
    X = rng.standard_normal((3000, 16)).astype(np.float32)
    index = build_index(X)
    _check(index, X, X, 5, exclude_self=True)
    # a screened batch beyond the fixed scratch is rejected with a clear error
    rc, _, _ = _noalloc(index, np.zeros((100_000, 16), np.float32), 5, want_dist=False)
    assert rc == _lib.B2K_EINVAL
    assert "at most" in _lib.last_error()


@pytest.mark.parametrize("k", [65, 200])
def test_noalloc_exhaustive_scan_for_large_k(k):
    from mlxlearn_b200.index import build_index

    rng = np.random.default_rng(7)
    X = rng.standard_normal((4000, 24)).astype(np.float32)
    X[1000:1050] = X[:50]
    index = build_index(X)
    Q = np.concatenate([X[:30], rng.standard_normal((170, 24))]).astype(np.float32)
    _check(index, X, Q, k)
    # the exhaustive path needs only the status block, so batches past the
    # screened limit are accepted
    Qb = rng.standard_normal((12000, 24)).astype(np.float32)
    _check(index, X, Qb, k)


def test_noalloc_out_of_range_query_redo_and_index():
    from mlxlearn_b200.index import build_index

    rng = np.random.default_rng(8)
    X = rng.standard_normal((5000, 20)).astype(np.float32)
    index = build_index(X)
    Q = rng.standard_normal((300, 20)).astype(np.float32)
    Q[17, 3] = 1e-30  # nonzero and below 2^-60: outside the screen's safe range
    _check(index, X, Q, 8)
    # an index holding such a coordinate is never screened
    Xo = X.copy()
    Xo[9, 0] = 3e-25
    _check(build_index(Xo), Xo, Q, 8)


@pytest.mark.parametrize("k", [10, 70])
def test_noalloc_rejects_non_finite_queries(k):
    from mlxlearn_b200 import _lib
    from mlxlearn_b200.index import build_index

    rng = np.random.default_rng(9)
    X = rng.standard_normal((4000, 16)).astype(np.float32)
    index = build_index(X)
    Q = rng.standard_normal((200, 16)).astype(np.float32)
    Q[33, 5] = np.nan
    rc, _, _ = _noalloc(index, Q, k)
    assert rc == _lib.B2K_ENONFINITE
    assert "finite" in _lib.last_error()
    Q[33, 5] = np.inf
    rc, _, _ = _noalloc(index, Q, k)
    assert rc == _lib.B2K_ENONFINITE
    # the next call on the shared array is answered correctly
    Q[33, 5] = 0.5
    _check(index, X, Q, k)


def test_noalloc_rejects_overlapping_outputs():
    import torch

    from mlxlearn_b200 import _lib
    from mlxlearn_b200.index import build_index

    X = np.random.default_rng(10).standard_normal((1000, 8)).astype(np.float32)
    index = build_index(X)
    h = index._ensure_device()
    buf = torch.zeros(4096, dtype=torch.float64, device="cuda")
    Q = torch.zeros((64, 8), dtype=torch.float32, device="cuda")
    # distances and indices on the same memory
    rc = _lib.load().b2k_knn_device_noalloc(h, _ptr(Q), 64, 4, 0, 0, _ptr(buf), _ptr(buf),
                                            torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.B2K_EINVAL
    assert "overlap" in _lib.last_error()
