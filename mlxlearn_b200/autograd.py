"""Differentiable kNN distances (torch.autograd.Function).

Indices come from the exact search and are held fixed; the outputs are the
selected distances, differentiable with respect to both the query and the
reference coordinates.  The backward is the hand-written CUDA kernel
``b2k_knn_backward`` (deterministic scatter-add, no float atomics).  The
reference library has no differentiable kNN; this exists for point-set losses
such as a Chamfer term.
"""
from __future__ import annotations

import torch

from . import _lib

__all__ = ["knn_distances", "chamfer_loss", "KnnDistances"]


def _device_index(X: torch.Tensor):
    """A temporary exact index over a CUDA float32 tensor (copied)."""
    from .index import NeighborIndex

    return NeighborIndex.from_device(X)


class KnnDistances(torch.autograd.Function):
    """distances[i, j] = ||Q[i] - X[idx[i, j]]|| (or its square), idx exact."""

    @staticmethod
    def forward(ctx, Q, X, k, exclude_self, squared):
        if not (Q.is_cuda and X.is_cuda):
            raise TypeError("knn_distances expects CUDA tensors")
        Qc = Q.detach().to(torch.float32).contiguous()
        Xc = X.detach().to(torch.float32).contiguous()
        index = _device_index(Xc)
        try:
            dist64, idx = index.query_device(Qc, int(k), exclude_self=bool(exclude_self))
        finally:
            index.close()
        e = dist64.to(torch.float32)
        out = dist64.square().to(torch.float32) if squared else e
        ctx.save_for_backward(Qc, Xc, idx, e)
        ctx.squared = bool(squared)
        ctx.q_dtype, ctx.x_dtype = Q.dtype, X.dtype
        return out.to(Q.dtype), idx

    @staticmethod
    def backward(ctx, grad_out, grad_idx):
        Qc, Xc, idx, e = ctx.saved_tensors
        m, d = Qc.shape
        n = Xc.shape[0]
        k = idx.shape[1]
        g = grad_out.detach().to(torch.float32).contiguous()
        want_q, want_x = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        dQ = torch.empty_like(Qc) if want_q else None
        dX = torch.empty_like(Xc) if want_x else None
        stream = torch.cuda.current_stream(Qc.device).cuda_stream
        rc = _lib.load().b2k_knn_backward(
            Qc.data_ptr(), m, Xc.data_ptr(), n, d, k, idx.data_ptr(), g.data_ptr(),
            e.data_ptr(), int(ctx.squared), None if dQ is None else dQ.data_ptr(),
            None if dX is None else dX.data_ptr(), stream)
        _lib.check(rc, "b2k_knn_backward")
        return (None if dQ is None else dQ.to(ctx.q_dtype),
                None if dX is None else dX.to(ctx.x_dtype), None, None, None)


def knn_distances(Q, X=None, k=1, *, exclude_self=False, squared=False):
    """Selected distances ``[m, k]`` and exact indices ``[m, k]``; with
    ``X=None`` the queries are the reference rows and each row's own index is
    excluded (``exclude_self`` is then implied)."""
    if X is None:
        X = Q
        exclude_self = True
    return KnnDistances.apply(Q, X, k, exclude_self, squared)


def chamfer_loss(A, B):
    """Symmetric k=1 Chamfer term: sum of squared nearest distances both ways."""
    dab, _ = knn_distances(A, B, 1, squared=True)
    dba, _ = knn_distances(B, A, 1, squared=True)
    return dab.sum() + dba.sum()
