"""Multi-GPU kneighbors: query shards over index replicas, or reference-row
shards with an exact merge; max-over-ranks timing.

One process per GPU (torchrun).  Query shards: every rank holds a full
replica of the fitted rows; a query batch is cut into contiguous shards, one
per rank, and each rank answers its shard with no collective on the data
path (the training rows are broadcast once, the answers gathered back in
query order).  Row shards (``kneighbors_row_sharded``): every rank holds a
contiguous range of the fitted rows and answers the whole batch with its own
exact top-k; one all-gather of those lists (16 bytes per candidate) and a
device merge give the answer over all rows, with exact 640-bit keys
exchanged only for the rare queries whose candidates from different shards
sit within float64 rounding of each other.  The reference has no
multi-device path; both forms return exactly what one ``kneighbors`` over
the whole batch and all rows returns.

All exchanges go through ``torch.distributed`` on whatever backend the
caller initialised (NCCL on GPUs, gloo on CPU); tensors are moved to the
backend's device here.
"""
from __future__ import annotations

from typing import Callable, Optional, Tuple

import numpy as np

__all__ = ["shard_bounds", "broadcast_rows", "max_over_ranks", "kneighbors_sharded",
           "kneighbors_row_sharded", "merge_row_shards", "radius_neighbors_row_sharded",
           "merge_radius_row_shards", "RowShardOps", "ShardTimer"]

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


class RowShardOps:
    """The device steps of a row-shard query, through the CUDA library.

    Tensors are CUDA tensors on the current device; every step runs on the
    current torch stream.  (Tests swap in a CPU restatement to check the
    exchange protocol on gloo ranks.)"""

    def search(self, index, Q, k):
        """This shard's exact top-k of every query: float64 [m, k], int64 [m, k]."""
        return index.query_device(Q, k)

    def merge(self, D, I, k, d, self_offset):
        import torch

        from . import _lib

        S, m, k_in = I.shape
        out_d = torch.empty((m, k), dtype=torch.float64, device=I.device)
        out_i = torch.empty((m, k), dtype=torch.int64, device=I.device)
        flags = torch.empty((m,), dtype=torch.int32, device=I.device)
        st = torch.cuda.current_stream(I.device).cuda_stream
        _lib.check(_lib.load().b2k_shard_merge(D.data_ptr(), I.data_ptr(), S, m, k_in, k, d,
                                               self_offset, out_d.data_ptr(), out_i.data_ptr(),
                                               flags.data_ptr(), st), "b2k_shard_merge")
        return out_d, out_i, flags

    def keys(self, index, row_offset, Q, I, flagged, keys):
        import torch

        from . import _lib

        S, m, k_in = I.shape
        st = torch.cuda.current_stream(I.device).cuda_stream
        _lib.check(_lib.load().b2k_shard_keys(index._ensure_device(), row_offset, Q.data_ptr(),
                                              I.data_ptr(), S, m, k_in, flagged.data_ptr(),
                                              flagged.numel(), keys.data_ptr(), st),
                   "b2k_shard_keys")

    def resolve(self, D, I, k, self_offset, flagged, keys, out_d, out_i):
        import torch

        from . import _lib

        S, m, k_in = I.shape
        st = torch.cuda.current_stream(I.device).cuda_stream
        _lib.check(_lib.load().b2k_shard_resolve(D.data_ptr(), I.data_ptr(), S, m, k_in, k,
                                                 self_offset, flagged.data_ptr(), flagged.numel(),
                                                 keys.data_ptr(), out_d.data_ptr(),
                                                 out_i.data_ptr(), st), "b2k_shard_resolve")


_KEY_LIMBS = 10


def _shard_lists(index, row_offset, Q, k_in, ops):
    """One shard's answer padded to k_in columns, rows made global (-1 = none)."""
    import torch

    n = int(index.n_samples)
    m = int(Q.shape[0])
    D = torch.full((m, k_in), float("inf"), dtype=torch.float64, device=Q.device)
    I = torch.full((m, k_in), -1, dtype=torch.int64, device=Q.device)
    kl = min(k_in, n)
    if kl > 0 and m > 0:
        d, i = ops.search(index, Q, kl)
        D[:, :kl] = d
        I[:, :kl] = i + row_offset
    return D, I


def _check_row_shard_args(k, n_total, exclude_self, q_offset, m):
    limit = n_total - (1 if exclude_self else 0)
    if k < 1:
        raise ValueError(f"Expected n_neighbors > 0. Got {k}")
    if k > limit:
        raise ValueError(f"n_neighbors must be <= {limit}, got {k}.")
    if exclude_self and (q_offset < 0 or q_offset + m > n_total):
        raise ValueError("exclude_self requires the query matrix to be the training matrix")


def merge_row_shards(parts, Q, k: int, *, exclude_self: bool = False, q_offset: int = 0,
                     ops: Optional[RowShardOps] = None):
    """The row-shard answer with every shard in this process.

    ``parts`` lists ``(index, row_offset)`` in row order: index ``s`` holds
    global rows ``[row_offset, row_offset + index.n_samples)``.  Returns float64
    distances and int64 global rows [m, k], identical to one search over all
    rows.  The same merge as ``kneighbors_row_sharded``, with stacking in
    place of the collectives."""
    import torch

    ops = ops or RowShardOps()
    n_total = sum(int(ix.n_samples) for ix, _ in parts)
    m, d = int(Q.shape[0]), int(Q.shape[1])
    _check_row_shard_args(k, n_total, exclude_self, q_offset, m)
    k_in = k + (1 if exclude_self else 0)
    lists = [_shard_lists(ix, off, Q, k_in, ops) for ix, off in parts]
    D = torch.stack([a for a, _ in lists])
    I = torch.stack([b for _, b in lists])
    self_offset = q_offset if exclude_self else -1
    out_d, out_i, flags = ops.merge(D, I, k, d, self_offset)
    flagged = torch.nonzero(flags).flatten().to(torch.int64)
    if flagged.numel():
        keys = torch.zeros((flagged.numel(), len(parts) * k_in, _KEY_LIMBS), dtype=torch.int64,
                           device=I.device)
        for ix, off in parts:
            ops.keys(ix, off, Q, I, flagged, keys)
        ops.resolve(D, I, k, self_offset, flagged, keys, out_d, out_i)
    return out_d, out_i


def kneighbors_row_sharded(index, row_offset: int, n_total: int, Q, k: int, *,
                           exclude_self: bool = False, q_offset: int = 0,
                           ops: Optional[RowShardOps] = None):
    """Answer ``Q`` over rows spread across the ranks.

    Rank ``r`` passes its own ``index`` over global rows
    ``[row_offset, row_offset + index.n_samples)`` (ranks hold consecutive ranges in
    rank order, together ``n_total`` rows) and the same query tensor ``Q``
    as every other rank.  Every rank returns the float64 distances and int64
    global rows [m, k] of one search over all rows.  Collectives: one
    all-gather of each rank's [m, k] lists, plus one all-reduce of exact keys
    when some query has candidates from different shards within float64
    rounding of each other (every rank takes the same branch)."""
    import torch
    import torch.distributed as dist

    ops = ops or RowShardOps()
    world = dist.get_world_size()
    m, d = int(Q.shape[0]), int(Q.shape[1])
    _check_row_shard_args(k, n_total, exclude_self, q_offset, m)
    k_in = k + (1 if exclude_self else 0)
    D_s, I_s = _shard_lists(index, row_offset, Q, k_in, ops)
    Ds = [torch.empty_like(D_s) for _ in range(world)]
    Is = [torch.empty_like(I_s) for _ in range(world)]
    dist.all_gather(Ds, D_s.contiguous())
    dist.all_gather(Is, I_s.contiguous())
    D, I = torch.stack(Ds), torch.stack(Is)
    self_offset = q_offset if exclude_self else -1
    out_d, out_i, flags = ops.merge(D, I, k, d, self_offset)
    flagged = torch.nonzero(flags).flatten().to(torch.int64)
    if flagged.numel():  # the same on every rank: the inputs are
        keys = torch.zeros((flagged.numel(), world * k_in, _KEY_LIMBS), dtype=torch.int64,
                           device=I.device)
        ops.keys(index, row_offset, Q, I, flagged, keys)
        dist.all_reduce(keys)  # each entry has exactly one owner
        ops.resolve(D, I, k, self_offset, flagged, keys, out_d, out_i)
    return out_d, out_i


def _local_radius(index, Q, radius, need_distance, sort_results):
    from .radius_result import RadiusCSR, join_batches

    return RadiusCSR(*join_batches(index.query_radius_csr(Q, radius, need_distance=need_distance,
                                                         sort_results=sort_results)))


def _radius_part(index, row_offset, Q, radius, need, exclude_self, q_offset, local):
    """One shard's entries as (query row, global row, distance) arrays."""
    part = (local or _local_radius)(index, Q, radius, need, False)
    rows = part.row_ids()
    idx = np.asarray(part.indices, dtype=np.int64) + int(row_offset)
    dd = (np.asarray(part.distances, dtype=np.float64) if need
          else np.zeros(len(idx), np.float64))
    if exclude_self:
        keep = idx != rows + int(q_offset)
        rows, idx, dd = rows[keep], idx[keep], dd[keep]
    return rows, idx, dd


def _assemble_radius(rows, idx, dd, m, sort_results, return_distance):
    """Per query row: ascending global index, or (float64 distance, index) --
    the single-index path's sort key, so the result is identical."""
    from .radius_result import RadiusCSR

    order = np.lexsort((idx, dd, rows)) if sort_results else np.lexsort((idx, rows))
    indptr = np.zeros(m + 1, np.int64)
    np.cumsum(np.bincount(rows, minlength=m), out=indptr[1:])
    return RadiusCSR(indptr, idx[order], dd[order] if return_distance else None)


def merge_radius_row_shards(parts, Q: np.ndarray, radius: float, *, return_distance: bool = True,
                            sort_results: bool = False, exclude_self: bool = False,
                            q_offset: int = 0, local: Optional[Callable] = None):
    """``radius_neighbors_row_sharded`` with every shard in this process:
    ``parts`` lists ``(index, row_offset)``."""
    Q = np.ascontiguousarray(Q, dtype=np.float32)
    need = bool(return_distance or sort_results)
    got = [_radius_part(ix, off, Q, radius, need, exclude_self, q_offset, local)
           for ix, off in parts]
    return _assemble_radius(np.concatenate([g[0] for g in got]),
                            np.concatenate([g[1] for g in got]),
                            np.concatenate([g[2] for g in got]), int(Q.shape[0]), sort_results,
                            return_distance)


def radius_neighbors_row_sharded(index, row_offset: int, Q: np.ndarray, radius: float, *,
                                 return_distance: bool = True, sort_results: bool = False,
                                 exclude_self: bool = False, q_offset: int = 0,
                                 local: Optional[Callable] = None):
    """Radius neighbourhoods over rows spread across the ranks, as one CSR.

    Rank ``r`` passes its own ``index`` over global rows
    ``[row_offset, row_offset + index.n_samples)`` and the same host query
    array ``Q``.  Every rank returns the ``RadiusCSR`` of one search over all
    rows: each rank answers with its rows (global indices), the per-rank
    entries are all-gathered (counts first, then padded arrays), and each
    query row is reassembled in ascending global index, or in (float64
    distance, index) order with ``sort_results``.  With ``exclude_self``
    query row ``j`` drops global row ``q_offset + j``.
    ``local(index, Q, radius, need_distance, sort_results)`` replaces the
    local search (default: ``index.query_radius_csr``)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size()
    dev = _device_for(dist)
    Q = np.ascontiguousarray(Q, dtype=np.float32)
    need = bool(return_distance or sort_results)
    rows, idx, dd = _radius_part(index, row_offset, Q, radius, need, exclude_self, q_offset,
                                 local)
    cnt = torch.tensor([len(idx)], dtype=torch.int64, device=dev)
    cnts = [torch.empty_like(cnt) for _ in range(world)]
    dist.all_gather(cnts, cnt)
    sizes = [int(c.item()) for c in cnts]
    width = max(max(sizes), 1)
    payload = np.zeros((3, width), np.float64)  # rows and indices exact below 2^53
    payload[0, :len(idx)] = rows
    payload[1, :len(idx)] = idx
    payload[2, :len(idx)] = dd
    mine = torch.from_numpy(payload).to(dev)
    bufs = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(bufs, mine)
    allp = np.concatenate([b.cpu().numpy()[:, :sz] for b, sz in zip(bufs, sizes)], axis=1)
    return _assemble_radius(allp[0].astype(np.int64), allp[1].astype(np.int64), allp[2],
                            int(Q.shape[0]), sort_results, return_distance)


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
