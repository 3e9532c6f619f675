"""Failure detection, exercised without faulting the GPU.

* Bounded waits.  Every wait of the tcgen05 screen polls at most a limit
  (2^26 by default; B2K_SPIN_LIMIT sets it).  With a limit of one poll the
  first wait that is not already satisfied gives up: the kernel records the
  timeout in the call's status word, waits (with the full limit) for the
  bulk copies and tensor-core operations it issued itself, frees its TMEM
  and returns; the kernels after it see the status and leave the outputs
  alone; the call raises BackendExecutionError (the reference's exception
  for a backend failure, src/mlxlearn/_common/base.py:57-80).  The same
  index then answers the next call correctly: the context stays usable.
* Host-side injection (B2K_FAULT): a launch failure and a timeout reported
  by the status read; the index stays usable afterwards.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from datasets import mixture

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def data():
    from mlxlearn_b200.index import build_index

    C = np.random.default_rng(60).uniform(-1, 1, (32, 32))
    X, _ = mixture(np.random.default_rng(61), 20000, C, 0.2)
    Q, _ = mixture(np.random.default_rng(62), 600, C, 0.2)
    od, oi = oracle.knn(X, Q, 10)
    return build_index(X), X, Q, od, oi


def _answers_correctly(index, Q, od, oi):
    dist, idx = index.query(Q, 10, mode="bf16")
    np.testing.assert_array_equal(idx, oi)
    np.testing.assert_array_equal(dist, od)


def test_screen_wait_limit_gives_a_timeout_status(data, monkeypatch):
    from mlxlearn_b200.exceptions import BackendExecutionError

    index, X, Q, od, oi = data
    _answers_correctly(index, Q, od, oi)  # the operand is built before the limit is set
    monkeypatch.setenv("B2K_SPIN_LIMIT", "1")
    with pytest.raises(BackendExecutionError, match="bounded device wait"):
        index.query(Q, 10, mode="bf16")
    # the radius screen (count pass) gives up the same way
    with pytest.raises(BackendExecutionError, match="bounded device wait"):
        index.query_radius_csr(Q, 1.0)
    monkeypatch.delenv("B2K_SPIN_LIMIT")
    _answers_correctly(index, Q, od, oi)
    ip, ix, dd = oracle.radius(X, Q[:50], 1.0)
    part = index.query_radius_csr(Q[:50], 1.0)[0]
    np.testing.assert_array_equal(part.indptr, ip)
    np.testing.assert_array_equal(part.indices, ix)


@pytest.mark.parametrize("fault,match", [("launch", "injected kernel launch failure"),
                                         ("timeout", "bounded device wait")])
def test_injected_host_faults(data, monkeypatch, fault, match):
    from mlxlearn_b200.exceptions import BackendExecutionError

    index, X, Q, od, oi = data
    monkeypatch.setenv("B2K_FAULT", fault)
    with pytest.raises(BackendExecutionError, match=match):
        index.query(Q, 10, mode="bf16")
    monkeypatch.delenv("B2K_FAULT")
    _answers_correctly(index, Q, od, oi)
