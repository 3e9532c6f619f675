"""The C-ABI library loads, exports every declared symbol, and fails loudly
without a GPU (no CPU fallback).  Runs on CPU."""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np
import pytest

from conftest import HAS_GPU, REPO

HEADER = os.path.join(REPO, "include", "b200knn.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"B2K_API\s+[\w\s\*]*?\b(b2k_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from mlxlearn_b200 import _build, _lib

    if not os.path.exists(_lib.LIB_PATH):
        _build.build()
    return _lib.load()


def test_library_exports_every_declared_symbol(lib):
    syms = declared_symbols()
    assert len(syms) >= 10
    for name in syms:
        assert hasattr(lib, name), name


def test_binding_covers_every_declared_symbol():
    from mlxlearn_b200 import _lib

    missing = set(declared_symbols()) - set(_lib.SIGNATURES)
    assert not missing, missing


def test_version_and_last_error(lib):
    assert lib.b2k_version() >= 100
    assert isinstance(lib.b2k_last_error(), bytes)


def test_invalid_arguments_rejected_before_device_use(lib):
    from mlxlearn_b200 import _lib

    h = ctypes.c_void_p()
    X = np.zeros((0, 3), np.float32)
    rc = lib.b2k_index_create(X.ctypes.data, 0, 3, 0, ctypes.byref(h))
    assert rc == _lib.B2K_EINVAL
    assert b"nonempty" in lib.b2k_last_error()
    rc = lib.b2k_index_create(None, 10, 3, 0, None)
    assert rc == _lib.B2K_EINVAL


def test_shard_merge_rejects_bad_shapes(lib):
    # the row-shard merge checks its shapes before touching any device memory
    from mlxlearn_b200 import _lib

    assert lib.b2k_shard_merge(None, None, 17, 4, 3, 3, 8, -1, None, None, None,
                               None) == _lib.B2K_EINVAL
    assert b"shard count" in lib.b2k_last_error()
    assert lib.b2k_shard_merge(None, None, 2, 4, 3, 5, 8, -1, None, None, None,
                               None) == _lib.B2K_EINVAL  # k_in < k
    assert lib.b2k_shard_merge(None, None, 2, 4, 258, 257, 8, -1, None, None, None,
                               None) == _lib.B2K_EINVAL  # k above 256
    assert lib.b2k_shard_merge(None, None, 2, 0, 3, 3, 8, -1, None, None, None,
                               None) == _lib.B2K_OK      # no queries: nothing to do
    assert lib.b2k_shard_merge(None, None, 2, 4, 3, 3, 8, -1, None, None, None,
                               None) == _lib.B2K_EINVAL  # NULL buffers
    assert lib.b2k_shard_resolve(None, None, 2, 4, 3, 3, -1, None, 5, None, None, None,
                                 None) == _lib.B2K_EINVAL  # more flagged rows than queries
    assert lib.b2k_shard_keys(None, 0, None, None, 2, 4, 3, None, 0, None,
                              None) == _lib.B2K_EINVAL     # no index


def test_injected_allocation_failure(lib, monkeypatch):
    from mlxlearn_b200 import _lib

    monkeypatch.setenv("B2K_FAULT", "alloc")
    X = np.ones((10, 3), np.float32)
    h = ctypes.c_void_p()
    rc = lib.b2k_index_create(X.ctypes.data, 10, 3, 0, ctypes.byref(h))
    assert rc == _lib.B2K_ENOMEM
    assert b"injected" in lib.b2k_last_error()
    with pytest.raises(MemoryError):
        _lib.check(rc)


@pytest.mark.skipif(HAS_GPU, reason="checks the no-GPU behaviour")
def test_no_gpu_raises_instead_of_cpu_fallback():
    from mlxlearn_b200.exceptions import BackendExecutionError
    from mlxlearn_b200.index import build_index

    X = np.random.default_rng(0).standard_normal((50, 4)).astype(np.float32)
    index = build_index(X)
    with pytest.raises(BackendExecutionError, match="no CUDA device|sm_100"):
        index.query(X[:3], 2)


def test_status_mapping():
    from mlxlearn_b200 import _lib
    from mlxlearn_b200.exceptions import BackendExecutionError

    with pytest.raises(ValueError):
        _lib.check(_lib.B2K_EINVAL)
    with pytest.raises(BackendExecutionError):
        _lib.check(_lib.B2K_ETIMEOUT)
