"""Multi-GPU kneighbors: index replicas, query shards, max-over-ranks timing.

One process per GPU (torchrun).  Every rank holds a full replica of the
fitted rows; a query batch is cut into contiguous shards, one per rank, and
each rank answers its shard with no collective on the data path.  The only
exchanges are host plumbing around the search: the training rows are
broadcast once from the rank that holds them, and the per-shard answers are
gathered back in query order.  The reference has no multi-device path; this
module only partitions the work the single-device entry points already do,
so answers are identical to one ``kneighbors`` over the whole batch.

All exchanges go through ``torch.distributed`` on whatever backend the
caller initialised (NCCL on GPUs, gloo on CPU); tensors are moved to the
backend's device here.
"""
from __future__ import annotations

from typing import Callable, Optional, Tuple

import numpy as np

__all__ = ["shard_bounds", "broadcast_rows", "max_over_ranks", "kneighbors_sharded",
           "ShardTimer"]

_DTYPES = {0: np.float32, 1: np.float64, 2: np.int64, 3: np.int32}
_CODES = {np.dtype(v): k for k, v in _DTYPES.items()}


def shard_bounds(m: int, world: int, rank: int) -> Tuple[int, int]:
    """Half-open row range of ``rank``'s shard of an ``m``-row batch.

    Shards are contiguous and differ in size by at most one row; the first
    ``m % world`` ranks take the extra row.  Ranks beyond ``m`` get an empty
    shard."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of size {world}")
    if m < 0:
        raise ValueError("row count must be non-negative")
    base, extra = divmod(m, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def _device_for(dist) -> str:
    import torch

    backend = dist.get_backend()
    if backend == "nccl":
        return f"cuda:{torch.cuda.current_device()}"
    return "cpu"


def broadcast_rows(X: Optional[np.ndarray], src: int = 0) -> np.ndarray:
    """Broadcast a 2-D array from ``src`` to every rank (others pass None).

    Shape and dtype travel first, so non-source ranks need not know them."""
    import torch
    import torch.distributed as dist

    dev = _device_for(dist)
    rank = dist.get_rank()
    if rank == src:
        if X is None or X.ndim != 2:
            raise ValueError("the source rank must pass a 2-D array")
        arr = np.ascontiguousarray(X)
        if arr.dtype not in _CODES:
            raise TypeError(f"unsupported dtype {arr.dtype}")
        meta = torch.tensor([arr.shape[0], arr.shape[1], _CODES[arr.dtype]], dtype=torch.int64,
                            device=dev)
    else:
        meta = torch.zeros(3, dtype=torch.int64, device=dev)
    dist.broadcast(meta, src)
    n, d, code = (int(v) for v in meta.cpu())
    dtype = _DTYPES[code]
    if rank == src:
        buf = torch.from_numpy(arr).to(dev)
    else:
        buf = torch.empty((n, d), dtype=getattr(torch, np.dtype(dtype).name), device=dev)
    dist.broadcast(buf, src)
    return buf.cpu().numpy()


def max_over_ranks(value: float) -> float:
    """The largest ``value`` any rank passed (every rank gets it)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=_device_for(dist))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _gather_rows(part: np.ndarray, m: int, world: int, width: int, dtype) -> np.ndarray:
    """All-gather contiguous row shards (sizes from ``shard_bounds``) into [m, width]."""
    import torch
    import torch.distributed as dist

    dev = _device_for(dist)
    rows = shard_bounds(m, world, 0)[1] - shard_bounds(m, world, 0)[0]
    tdt = getattr(torch, np.dtype(dtype).name)
    padded = torch.zeros((rows, width), dtype=tdt, device=dev)
    if part.shape[0]:
        padded[: part.shape[0]] = torch.from_numpy(np.ascontiguousarray(part, dtype=dtype)).to(dev)
    bufs = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(bufs, padded)
    out = np.empty((m, width), dtype=dtype)
    for r in range(world):
        a, b = shard_bounds(m, world, r)
        out[a:b] = bufs[r][: b - a].cpu().numpy()
    return out


def kneighbors_sharded(query: Callable[[np.ndarray, int, int], Tuple[np.ndarray, np.ndarray]],
                       Q: np.ndarray, k: int, *, gather: bool = True):
    """Answer ``Q`` with each rank searching its own shard.

    ``query(Q_shard, k, start) -> (dist [s, k] float64, idx [s, k] int64)``
    is the rank's local search (normally ``NeighborIndex.query`` on its
    replica); ``start`` is the shard's first row in ``Q``, which a self-query
    passes on as the query offset so each row still skips its own index.
    Every rank must pass the same ``Q`` and ``k``.  With ``gather`` every
    rank receives the full ``[m, k]`` answer in query order; without it each
    rank returns only its shard and the shard's first row."""
    import torch.distributed as dist

    world, rank = dist.get_world_size(), dist.get_rank()
    m = int(Q.shape[0])
    a, b = shard_bounds(m, world, rank)
    if b > a:
        d, i = query(Q[a:b], k, a)
        d = np.asarray(d, dtype=np.float64)
        i = np.asarray(i, dtype=np.int64)
    else:
        d = np.empty((0, k), np.float64)
        i = np.empty((0, k), np.int64)
    if d.shape != (b - a, k) or i.shape != (b - a, k):
        raise ValueError(f"local query returned shapes {d.shape}, {i.shape}; "
                         f"expected {(b - a, k)}")
    if not gather:
        return d, i, a
    return _gather_rows(d, m, world, k, np.float64), _gather_rows(i, m, world, k, np.int64)


class ShardTimer:
    """Device time of a block of steps, as the max over ranks.

    ``start()`` / ``stop()`` bracket the steps with a barrier and a device
    synchronize on both sides; ``stop`` returns milliseconds per step, the
    max over ranks.  On CPU (gloo) the host clock stands in for CUDA events.
    """

    def __init__(self, stream=None):
        self.stream = stream
        self._ev = None
        self._t0 = None

    def _sync(self):
        import torch
        import torch.distributed as dist

        if dist.is_initialized():
            dist.barrier()
        if torch.cuda.is_available():
            torch.cuda.synchronize()

    def start(self):
        import time

        import torch

        self._sync()
        if torch.cuda.is_available():
            s = self.stream or torch.cuda.current_stream()
            self._ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            self._ev[0].record(s)
        else:
            self._t0 = time.perf_counter()

    def stop(self, steps: int) -> float:
        import time

        import torch
        import torch.distributed as dist

        if self._ev is not None:
            s = self.stream or torch.cuda.current_stream()
            self._ev[1].record(s)
            self._sync()
            ms = self._ev[0].elapsed_time(self._ev[1])
        else:
            self._sync()
            ms = 1000.0 * (time.perf_counter() - self._t0)
        ms /= max(1, steps)
        if dist.is_initialized() and dist.get_world_size() > 1:
            ms = max_over_ranks(ms)
        return ms
