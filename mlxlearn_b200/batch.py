"""Many independent kNN problems in one planned device run.

``KnnBatch`` takes problems of uneven size (each its own fitted
``NeighborIndex``, a CUDA query block and a k) and answers all of them with
one CUDA graph: a batched query preparation, persistent tcgen05 screen
launches over a device work queue, one batched certify and one batched
exhaustive-scan launch (``b2k_batch_create`` in include/b200knn.h).  Results
are identical to calling ``NeighborIndex.query_device`` per problem.

The reference has no batched API (mlxlearn answers one problem per call,
src/mlxlearn/_kernels/distance.py:242-270); this is the multi-problem form of
the same contract: float64 distances and int64 indices in (distance, index)
order with ties to the smaller index.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence, Tuple

from . import _lib
from .index import NeighborIndex

__all__ = ["KnnBatch", "kneighbors_batch"]


class KnnBatch:
    """A planned batch.  ``problems`` holds ``(index, queries, k)`` or
    ``(index, queries, k, exclude_self)`` tuples; ``queries`` are CUDA float32
    tensors ``[m, d]`` on the index's device.  The query tensors are read in
    place on every run: write new queries into them and call the batch again.
    ``autotune`` times the tuning candidates on this batch at construction
    (cached per process).
    """

    def __init__(self, problems: Sequence[tuple], *, autotune: bool = False,
                 return_distance: bool = True):
        import torch

        self._handle = None
        self.queries: List = []
        self.dist: List[Optional[object]] = []
        self.idx: List = []
        self._indexes: List[NeighborIndex] = []
        arr = (_lib.Problem * max(1, len(problems)))()
        for i, prob in enumerate(problems):
            index, Q, k = prob[0], prob[1], int(prob[2])
            exclude_self = bool(prob[3]) if len(prob) > 3 else False
            if not isinstance(index, NeighborIndex):
                raise TypeError(f"problem {i}: expected a NeighborIndex")
            if not (isinstance(Q, torch.Tensor) and Q.is_cuda and Q.dim() == 2):
                raise TypeError(f"problem {i}: queries must be a 2-D CUDA tensor")
            if Q.dtype != torch.float32 or not Q.is_contiguous():
                raise ValueError(f"problem {i}: queries must be contiguous float32")
            if Q.shape[1] != index.n_features:
                raise ValueError(f"problem {i}: queries must have {index.n_features} columns")
            m = int(Q.shape[0])
            index._check_query(m, k, exclude_self)
            h = index._ensure_device()
            idx = torch.empty((m, k), dtype=torch.int64, device=Q.device)
            dist = (torch.empty((m, k), dtype=torch.float64, device=Q.device)
                    if return_distance else None)
            arr[i] = _lib.Problem(h.value if hasattr(h, "value") else h, Q.data_ptr(), m, k,
                                  int(exclude_self), 0,
                                  None if dist is None else dist.data_ptr(), idx.data_ptr())
            self.queries.append(Q)
            self.dist.append(dist)
            self.idx.append(idx)
            self._indexes.append(index)
        self._problems = arr
        lib = _lib.load()
        h = ctypes.c_void_p()
        stream = torch.cuda.current_stream().cuda_stream
        flags = _lib.BATCH_AUTOTUNE if autotune else 0
        _lib.check(lib.b2k_batch_create(arr, len(problems), flags, stream, ctypes.byref(h)),
                   "b2k_batch_create")
        self._handle = h
        self.last_stats = None

    def run(self):
        """Launch one run on the current torch stream (asynchronous)."""
        import torch

        _lib.check(_lib.load().b2k_batch_run(self._handle, torch.cuda.current_stream().cuda_stream),
                   "b2k_batch_run")

    def finish(self) -> dict:
        """Wait for the last run; answers problems outside the graph; stats."""
        import torch

        st = _lib.BatchStats()
        _lib.check(_lib.load().b2k_batch_finish(
            self._handle, torch.cuda.current_stream().cuda_stream, ctypes.byref(st)),
            "b2k_batch_finish")
        self.last_stats = st.as_dict()
        return self.last_stats

    def __call__(self) -> List[Tuple[Optional[object], object]]:
        self.run()
        self.finish()
        return list(zip(self.dist, self.idx))

    def close(self):
        if self._handle is not None and _lib._lib is not None:
            _lib._lib.b2k_batch_destroy(self._handle)
        self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def kneighbors_batch(problems: Sequence[tuple], *, return_distance: bool = True):
    """One-shot batch: ``[(dist, idx), ...]`` per problem (torch tensors)."""
    b = KnnBatch(problems, return_distance=return_distance)
    try:
        return b()
    finally:
        b.close()
