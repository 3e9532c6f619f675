"""b2k_knn_device_noalloc: the kNN entry point that allocates no memory.

It serves callers that may not allocate device memory during a query (their
GPU memory belongs to another allocator, or allocation's implicit
synchronisation is not allowed on their path).  Its scratch is a fixed array
inside the library.  This test calls it through the C ABI and compares its
output with the regular device entry point's, on two calls in a row (the
second call reuses the array the first one left behind).  The tolerance is
the one the other kNN tests use: indices and canonical distances bit-exact.

This file is named so that pytest collects it last.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_matches_regular_entry_point_twice():
    import torch

    from mlxlearn_b200 import _lib
    from mlxlearn_b200.index import build_index

    lib = _lib.load()
    rng = np.random.default_rng(5)
    X = rng.standard_normal((20000, 48)).astype(np.float32)
    X[500:520] = X[:20]  # exact duplicates: index tie rule
    index = build_index(X)
    h = index._ensure_device()
    stream = torch.cuda.current_stream().cuda_stream
    for call, (m, k) in enumerate([(700, 10), (1500, 7)]):
        Q = torch.from_numpy(rng.standard_normal((m, 48)).astype(np.float32)).cuda()
        ri = torch.empty((m, k), dtype=torch.int64, device="cuda")
        rd = torch.empty((m, k), dtype=torch.float64, device="cuda")
        rc = lib.b2k_knn_device(h, _ptr(Q), m, k, 0, 0, _lib.MODE_FP32, _ptr(rd), _ptr(ri),
                                stream, None)
        _lib.check(rc)
        ni = torch.full((m, k), -1, dtype=torch.int64, device="cuda")
        nd = torch.full((m, k), -1.0, dtype=torch.float64, device="cuda")
        rc = lib.b2k_knn_device_noalloc(h, _ptr(Q), m, k, 0, 0, _ptr(nd), _ptr(ni), stream)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        assert torch.equal(ni, ri), f"call {call}: indices differ"
        assert torch.equal(nd, rd), f"call {call}: distances differ"


def test_noalloc_self_query_and_size_limit():
    import torch

    from mlxlearn_b200 import _lib
    from mlxlearn_b200.index import build_index

    lib = _lib.load()
    rng = np.random.default_rng(6)
    X = rng.standard_normal((3000, 16)).astype(np.float32)
    index = build_index(X)
    h = index._ensure_device()
    stream = torch.cuda.current_stream().cuda_stream
    Xd = torch.from_numpy(X).cuda()
    m, k = 3000, 5
    ni = torch.empty((m, k), dtype=torch.int64, device="cuda")
    nd = torch.empty((m, k), dtype=torch.float64, device="cuda")
    rc = lib.b2k_knn_device_noalloc(h, _ptr(Xd), m, k, 1, 0, _ptr(nd), _ptr(ni), stream)
    assert rc == 0, _lib.last_error()
    rd, ri = index.query(X, k, exclude_self=True)
    np.testing.assert_array_equal(ni.cpu().numpy(), ri)
    np.testing.assert_array_equal(nd.cpu().numpy(), rd)
    # a batch beyond the fixed scratch is rejected with a clear error
    big = 100_000
    Qb = torch.zeros((big, 16), dtype=torch.float32, device="cuda")
    bi = torch.empty((big, k), dtype=torch.int64, device="cuda")
    rc = lib.b2k_knn_device_noalloc(h, _ptr(Qb), big, k, 0, 0, None, _ptr(bi), stream)
    assert rc == _lib.B2K_EINVAL
    assert "at most" in _lib.last_error()
