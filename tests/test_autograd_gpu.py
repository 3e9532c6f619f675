"""Differentiable kNN distances: the hand-written backward against FP64 central
finite differences (indices fixed, inputs away from ties) and against torch
autograd through gathered distances.  The reference has no differentiable kNN,
so these checks are the whole parity story for the backward (forward indices
are the exact search's)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _gathered(Q, X, idx, squared):
    diff = Q[:, None, :] - X[idx]
    s = (diff * diff).sum(-1)
    return s if squared else s.sqrt()


@pytest.mark.parametrize("squared", [True, False])
def test_backward_matches_fp64_finite_differences(squared):
    import torch

    from mlxlearn_b200.autograd import knn_distances

    rng = np.random.default_rng(21)
    Qn = rng.normal(size=(30, 5))
    Xn = rng.normal(size=(60, 5))
    Q = torch.tensor(Qn, dtype=torch.float32, device="cuda", requires_grad=True)
    X = torch.tensor(Xn, dtype=torch.float32, device="cuda", requires_grad=True)
    W = torch.tensor(rng.normal(size=(30, 3)), dtype=torch.float32, device="cuda")
    d, idx = knn_distances(Q, X, 3, squared=squared)
    _, oi = oracle.knn(Xn.astype(np.float32), Qn.astype(np.float32), 3)
    np.testing.assert_array_equal(idx.cpu().numpy(), oi)
    (d * W).sum().backward()
    # FP64 central differences of the same function with the indices held fixed
    q64, x64 = Qn.astype(np.float32).astype(np.float64), Xn.astype(np.float32).astype(np.float64)
    I, w = idx.cpu().numpy(), W.cpu().numpy().astype(np.float64)

    def f(q, x):
        s = ((q[:, None, :] - x[I]) ** 2).sum(-1)
        return float(((s if squared else np.sqrt(s)) * w).sum())

    h = 1e-6
    gq = np.zeros_like(q64)
    for i in range(q64.shape[0]):
        for j in range(q64.shape[1]):
            a, b = q64.copy(), q64.copy()
            a[i, j] += h
            b[i, j] -= h
            gq[i, j] = (f(a, x64) - f(b, x64)) / (2 * h)
    gx = np.zeros_like(x64)
    for i in range(x64.shape[0]):
        for j in range(x64.shape[1]):
            a, b = x64.copy(), x64.copy()
            a[i, j] += h
            b[i, j] -= h
            gx[i, j] = (f(q64, a) - f(q64, b)) / (2 * h)
    np.testing.assert_allclose(Q.grad.cpu().numpy(), gq, rtol=1e-4, atol=1e-5)
    np.testing.assert_allclose(X.grad.cpu().numpy(), gx, rtol=1e-4, atol=1e-5)


def test_chamfer_matches_torch_autograd_and_is_deterministic():
    import torch

    from mlxlearn_b200.autograd import chamfer_loss, knn_distances

    rng = np.random.default_rng(6)

    def cloud(n):
        v = rng.normal(size=(n, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        return (v + rng.normal(0, 0.01, size=(n, 3))).astype(np.float32)

    A = torch.tensor(cloud(8192), device="cuda", requires_grad=True)
    B = torch.tensor(cloud(8192), device="cuda", requires_grad=True)
    loss = chamfer_loss(A, B)
    loss.backward()
    ga, gb = A.grad.clone(), B.grad.clone()
    # reference: torch autograd through gathered distances with the same indices
    _, iab = knn_distances(A.detach(), B.detach(), 1)
    _, iba = knn_distances(B.detach(), A.detach(), 1)
    A2 = A.detach().clone().requires_grad_(True)
    B2 = B.detach().clone().requires_grad_(True)
    ref = _gathered(A2, B2, iab, True).sum() + _gathered(B2, A2, iba, True).sum()
    ref.backward()
    torch.testing.assert_close(loss, ref, rtol=1e-5, atol=1e-5)
    torch.testing.assert_close(ga, A2.grad, rtol=1e-5, atol=1e-6)
    torch.testing.assert_close(gb, B2.grad, rtol=1e-5, atol=1e-6)
    A.grad = None
    B.grad = None
    chamfer_loss(A, B).backward()
    assert torch.equal(A.grad, ga) and torch.equal(B.grad, gb)


def test_self_knn_embedding_loss():
    import torch

    from mlxlearn_b200.autograd import knn_distances

    rng = np.random.default_rng(60)
    E = torch.tensor(rng.normal(size=(4096, 64)).astype(np.float32), device="cuda",
                     requires_grad=True)
    d, idx = knn_distances(E, None, 8)
    assert not (idx == torch.arange(4096, device="cuda")[:, None]).any()
    _, oi = oracle.knn(E.detach().cpu().numpy(), E.detach().cpu().numpy(), 8, exclude_self=True)
    np.testing.assert_array_equal(idx.cpu().numpy(), oi)
    d.mean().backward()
    E2 = E.detach().clone().requires_grad_(True)
    _gathered(E2, E2, idx, False).mean().backward()
    torch.testing.assert_close(E.grad, E2.grad, rtol=1e-4, atol=1e-7)
