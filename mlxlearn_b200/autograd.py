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

__all__ = ["knn_distances", "chamfer_loss", "KnnDistances", "knn_segments",
           "chamfer_loss_batch", "KnnSegmentDistances"]


# Below this many (query, reference) pairs a direct scan (b2k_knn_segments)
# costs less than building and querying a temporary index.
_DIRECT_PAIRS = 1 << 27


def _segments_forward(Qc, Xc, q_sizes, x_sizes, k, exclude_self):
    """float64 distances and int64 indices (within each reference segment)."""
    import numpy as np

    qo = np.zeros(len(q_sizes) + 1, dtype=np.int64)
    np.cumsum(np.asarray(q_sizes, dtype=np.int64), out=qo[1:])
    xo = np.zeros(len(x_sizes) + 1, dtype=np.int64)
    np.cumsum(np.asarray(x_sizes, dtype=np.int64), out=xo[1:])
    if qo[-1] != Qc.shape[0] or xo[-1] != Xc.shape[0]:
        raise ValueError("segment sizes must add up to the row counts")
    rows, d = Qc.shape
    idx = torch.empty((rows, k), dtype=torch.int64, device=Qc.device)
    dist64 = torch.empty((rows, k), dtype=torch.float64, device=Qc.device)
    stream = torch.cuda.current_stream(Qc.device).cuda_stream
    _lib.check(_lib.load().b2k_knn_segments(
        Qc.data_ptr(), Xc.data_ptr(), d, qo.ctypes.data, xo.ctypes.data, len(q_sizes), k,
        int(bool(exclude_self)), dist64.data_ptr(), idx.data_ptr(), stream),
        "b2k_knn_segments")
    return dist64, idx


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
        m, n, d = Qc.shape[0], Xc.shape[0], Qc.shape[1]
        if d <= 64 and int(k) <= 29 and m * n <= _DIRECT_PAIRS:
            # small problem: one direct exact scan, no temporary index
            dist64, idx = _segments_forward(Qc, Xc, (m,), (n,), int(k), bool(exclude_self))
        else:
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


def _offsets(sizes):
    import numpy as np

    off = np.zeros(len(sizes) + 1, dtype=np.int64)
    np.cumsum(np.asarray(sizes, dtype=np.int64), out=off[1:])
    return off


class KnnSegmentDistances(torch.autograd.Function):
    """Selected distances of many small problems given as segments of two
    tensors (``b2k_knn_segments``); indices are within each reference segment."""

    @staticmethod
    def forward(ctx, Q, X, q_sizes, x_sizes, k, exclude_self, squared):
        if not (Q.is_cuda and X.is_cuda):
            raise TypeError("knn_segments expects CUDA tensors")
        Qc = Q.detach().to(torch.float32).contiguous()
        Xc = X.detach().to(torch.float32).contiguous()
        k = int(k)
        dist64, idx = _segments_forward(Qc, Xc, q_sizes, x_sizes, k, exclude_self)
        xo = _offsets(x_sizes)
        # global reference rows for the backward
        starts = torch.as_tensor(xo[:-1], device=Qc.device)
        seg = torch.repeat_interleave(torch.arange(len(q_sizes), device=Qc.device),
                                      torch.as_tensor(q_sizes, device=Qc.device))
        gidx = idx + starts[seg].unsqueeze(1)
        e = dist64.to(torch.float32)
        out = dist64.square().to(torch.float32) if squared else e
        ctx.save_for_backward(Qc, Xc, gidx, e)
        ctx.squared = bool(squared)
        ctx.q_dtype, ctx.x_dtype = Q.dtype, X.dtype
        ctx.mark_non_differentiable(idx)
        return out.to(Q.dtype), idx

    @staticmethod
    def backward(ctx, grad_out, grad_idx):
        Qc, Xc, gidx, e = ctx.saved_tensors
        m, d = Qc.shape
        n = Xc.shape[0]
        k = gidx.shape[1]
        g = grad_out.detach().to(torch.float32).contiguous()
        want_q, want_x = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        dQ = torch.empty_like(Qc) if want_q else None
        dX = torch.empty_like(Xc) if want_x else None
        stream = torch.cuda.current_stream(Qc.device).cuda_stream
        rc = _lib.load().b2k_knn_backward(
            Qc.data_ptr(), m, Xc.data_ptr(), n, d, k, gidx.data_ptr(), g.data_ptr(),
            e.data_ptr(), int(ctx.squared), None if dQ is None else dQ.data_ptr(),
            None if dX is None else dX.data_ptr(), stream)
        _lib.check(rc, "b2k_knn_backward")
        return (None if dQ is None else dQ.to(ctx.q_dtype),
                None if dX is None else dX.to(ctx.x_dtype), None, None, None, None, None)


def knn_segments(Q, X, q_sizes, x_sizes, k=1, *, exclude_self=False, squared=False):
    """Distances ``[rows, k]`` and indices (within each reference segment) of
    many small problems at once: problem p is the p-th block of ``q_sizes[p]``
    rows of ``Q`` against the p-th block of ``x_sizes[p]`` rows of ``X``
    (d <= 64, k <= 29)."""
    return KnnSegmentDistances.apply(Q, X, tuple(int(v) for v in q_sizes),
                                     tuple(int(v) for v in x_sizes), k, exclude_self, squared)


def chamfer_loss_batch(As, Bs):
    """Sum over pairs of the symmetric k=1 Chamfer term of ``chamfer_loss``,
    with one search and one backward call for all pairs (clouds of d <= 64).
    ``As`` and ``Bs`` are lists of ``[n_i, d]`` tensors, or two ``[P, n, d]``
    tensors of equally sized clouds (cheaper: no per-cloud gradient tensors)."""
    if torch.is_tensor(As) and torch.is_tensor(Bs) and As.dim() == 3 and Bs.dim() == 3:
        P, na, d = As.shape
        nb = Bs.shape[1]
        if Bs.shape[0] != P or Bs.shape[2] != d:
            raise ValueError("As and Bs must hold the same number of clouds of one width")
        Q = torch.cat([As, Bs], dim=1).reshape(-1, d)
        X = torch.cat([Bs, As], dim=1).reshape(-1, d)
        q_sizes = [na, nb] * P
        x_sizes = [nb, na] * P
    else:
        if len(As) != len(Bs):
            raise ValueError("As and Bs must hold the same number of clouds")
        Q = torch.cat([t for a, b in zip(As, Bs) for t in (a, b)])
        X = torch.cat([t for a, b in zip(As, Bs) for t in (b, a)])
        q_sizes = [t.shape[0] for a, b in zip(As, Bs) for t in (a, b)]
        x_sizes = [t.shape[0] for a, b in zip(As, Bs) for t in (b, a)]
    d2, _ = knn_segments(Q, X, q_sizes, x_sizes, 1, squared=True)
    return d2.sum()
