"""Many small problems in one call (b2k_knn_segments) and the batched Chamfer.

Each segment pair must give exactly the oracle's answer for that problem:
indices bit-exact (ties to the smaller index) and canonical float64
distances; the batched Chamfer loss and its gradients must equal the per-pair
``chamfer_loss``.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _run(Qs, Xs, k, exclude_self=False):
    import torch

    from mlxlearn_b200.autograd import knn_segments

    Q = torch.from_numpy(np.concatenate(Qs)).cuda()
    X = torch.from_numpy(np.concatenate(Xs)).cuda()
    dist, idx = knn_segments(Q, X, [len(q) for q in Qs], [len(x) for x in Xs], k,
                             exclude_self=exclude_self)
    return dist.double().cpu().numpy(), idx.cpu().numpy()


def _check(Qs, Xs, k, dist, idx, exclude_self=False):
    r = 0
    for Qp, Xp in zip(Qs, Xs):
        m = len(Qp)
        if m == 0:
            continue
        od, oi = oracle.knn(Xp, Qp, k, exclude_self=exclude_self)
        np.testing.assert_array_equal(idx[r:r + m], oi)
        # the float32 output of the autograd path holds the canonical distance rounded
        np.testing.assert_allclose(dist[r:r + m], od, rtol=1e-6, atol=0)
        r += m


@pytest.mark.parametrize("d,k", [(3, 1), (3, 8), (8, 5), (16, 13), (5, 29), (32, 4), (64, 8),
                                 (50, 20)])
def test_uneven_segments_match_oracle(d, k):
    rng = np.random.default_rng(100 + d + k)
    sizes = [(int(rng.integers(1, 700)), int(rng.integers(k, 2500))) for _ in range(9)]
    sizes[3] = (0, 200)  # a segment without queries
    Qs = [rng.standard_normal((m, d)).astype(np.float32) for m, _ in sizes]
    Xs = [rng.standard_normal((n, d)).astype(np.float32) for _, n in sizes]
    dist, idx = _run(Qs, Xs, k)
    _check(Qs, Xs, k, dist, idx)


def test_ties_and_self_exclusion():
    rng = np.random.default_rng(7)
    # integer lattice points with many duplicates: ties everywhere
    Xs = [np.repeat(rng.integers(-2, 3, (300, 3)), 3, axis=0).astype(np.float32)
          for _ in range(4)]
    dist, idx = _run(Xs, Xs, 6, exclude_self=True)
    _check(Xs, Xs, 6, dist, idx, exclude_self=True)
    r = 0
    for Xp in Xs:
        assert not np.any(idx[r:r + len(Xp)] == np.arange(len(Xp))[:, None])
        r += len(Xp)


def test_out_of_range_coordinates_take_the_exact_path():
    rng = np.random.default_rng(8)
    Xs = [rng.standard_normal((500, 3)).astype(np.float32) * 1e-19 for _ in range(2)]
    Qs = [rng.standard_normal((70, 3)).astype(np.float32) * 1e-19 for _ in range(2)]
    dist, idx = _run(Qs, Xs, 3)
    _check(Qs, Xs, 3, dist, idx)


def test_rejects_bad_segments():
    import torch

    from mlxlearn_b200.autograd import knn_segments

    Q = torch.zeros((10, 3), device="cuda")
    X = torch.zeros((10, 3), device="cuda")
    with pytest.raises(ValueError):
        knn_segments(Q, X, [5, 5], [9, 1], 2)       # k > rows of the second segment
    with pytest.raises(ValueError):
        knn_segments(Q, X, [4, 5], [5, 5], 1)       # sizes do not add up
    from mlxlearn_b200.exceptions import BackendExecutionError
    with pytest.raises(BackendExecutionError):
        knn_segments(torch.zeros((4, 80), device="cuda"), torch.zeros((4, 80), device="cuda"),
                     [4], [4], 1)                   # d > 64


def test_chamfer_batch_equals_per_pair_loss():
    import torch

    from mlxlearn_b200.autograd import chamfer_loss, chamfer_loss_batch

    rng = np.random.default_rng(6)

    def cloud(n):
        v = rng.normal(size=(n, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        return (v + rng.normal(0, 0.01, size=(n, 3))).astype(np.float32)

    pairs = [(cloud(int(rng.integers(500, 3000))), cloud(int(rng.integers(500, 3000))))
             for _ in range(6)]
    A = [torch.tensor(a, device="cuda", requires_grad=True) for a, _ in pairs]
    B = [torch.tensor(b, device="cuda", requires_grad=True) for _, b in pairs]
    loss = chamfer_loss_batch(A, B)
    loss.backward()
    A2 = [a.detach().clone().requires_grad_(True) for a in A]
    B2 = [b.detach().clone().requires_grad_(True) for b in B]
    ref = sum(chamfer_loss(a, b) for a, b in zip(A2, B2))
    ref.backward()
    torch.testing.assert_close(loss, ref, rtol=1e-6, atol=1e-6)
    for a, a2 in zip(A, A2):
        torch.testing.assert_close(a.grad, a2.grad, rtol=1e-6, atol=1e-7)
    for b, b2 in zip(B, B2):
        torch.testing.assert_close(b.grad, b2.grad, rtol=1e-6, atol=1e-7)


def test_chamfer_batch_stacked_tensors():
    import torch

    from mlxlearn_b200.autograd import chamfer_loss, chamfer_loss_batch

    rng = np.random.default_rng(9)
    A = torch.tensor(rng.normal(size=(5, 1000, 3)).astype(np.float32), device="cuda",
                     requires_grad=True)
    B = torch.tensor(rng.normal(size=(5, 1300, 3)).astype(np.float32), device="cuda",
                     requires_grad=True)
    loss = chamfer_loss_batch(A, B)
    loss.backward()
    A2 = A.detach().clone().requires_grad_(True)
    B2 = B.detach().clone().requires_grad_(True)
    ref = sum(chamfer_loss(A2[i], B2[i]) for i in range(5))
    ref.backward()
    torch.testing.assert_close(loss, ref, rtol=1e-6, atol=1e-6)
    torch.testing.assert_close(A.grad, A2.grad, rtol=1e-6, atol=1e-7)
    torch.testing.assert_close(B.grad, B2.grad, rtol=1e-6, atol=1e-7)


def test_small_knn_distances_take_the_direct_scan_and_match_the_index_path():
    # a self-kNN of 3,000 x 64 is below the direct-scan limit; its answer must
    # equal the oracle's, exactly as the index path's does
    import torch

    from mlxlearn_b200.autograd import knn_distances

    rng = np.random.default_rng(12)
    X = rng.standard_normal((3000, 64)).astype(np.float32)
    Xt = torch.from_numpy(X).cuda().requires_grad_()
    d, i = knn_distances(Xt, None, 8)
    od, oi = oracle.knn(X, X, 8, exclude_self=True)
    np.testing.assert_array_equal(i.cpu().numpy(), oi)
    np.testing.assert_allclose(d.detach().double().cpu().numpy(), od, rtol=1e-6, atol=0)
    d.mean().backward()
    assert torch.isfinite(Xt.grad).all()
