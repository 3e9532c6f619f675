"""Radius neighbourhoods as CSR batches, fed from the search's device result.

``b2k_radius`` leaves one batch of neighbourhoods on the GPU: row offsets
(int64 ``[m + 1]``), training indices (int64, ascending within a row, or in
``(distance, index)`` order when sorting was asked for) and float64
distances.  :class:`RadiusCSR` wraps that device result:

* the host arrays are copied out only when first read, each with one DMA
  into page-locked memory (no pageable staging copy);
* ``votes`` and ``mean`` reduce the neighbourhoods on the device while the
  result is still there, so a classifier's ``predict`` never downloads them.

The field and method names are the ones mlxlearn's estimators read from a
batch, so the reference's own estimator code consumes these objects
unchanged: the CSR fields ``indptr``/``indices``/``distances`` with
``n_query``, ``nnz``, ``lengths()``, ``row_ids()`` (reference
src/mlxlearn/_kernels/radius_result.py:33-55), and ``votes(codes, n_classes,
weighted)`` / ``mean(targets, weighted)``, which the reference calls on every
batch that is not its own CSR class (src/mlxlearn/_kernels/radius_reduce.py:75-94).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

__all__ = ["RadiusCSR", "join_batches", "ragged_rows", "neighbour_graph", "sparse_graph"]


def _page_locked(count: int, dtype) -> np.ndarray:
    """A host array in page-locked memory (torch's caching host allocator,
    so repeated batches reuse the same blocks)."""
    import torch

    tdtype = {np.dtype(np.int64): torch.int64, np.dtype(np.float64): torch.float64}[np.dtype(dtype)]
    return torch.empty(int(count), dtype=tdtype, pin_memory=True).numpy()


class RadiusCSR:
    """One batch of radius neighbourhoods in CSR form.

    Built either around a device result (``from_device``; the library's
    handle is released when the batch is dropped or ``release()`` is called)
    or from host arrays (the row-shard reassembly builds its batches that
    way).
    """

    __slots__ = ("route", "_indptr", "_indices", "_dist", "_handle", "_device", "_m", "_nnz",
                 "_has_dist", "__weakref__")

    def __init__(self, indptr, indices, distances=None, route: str = "cuda"):
        self.route = route
        self._indptr = np.asarray(indptr, dtype=np.int64)
        self._indices = np.asarray(indices, dtype=np.int64)
        self._dist = None if distances is None else np.asarray(distances, dtype=np.float64)
        self._handle = None
        self._device = None
        self._m = len(self._indptr) - 1
        self._nnz = int(self._indptr[-1] - self._indptr[0]) if self._m >= 0 else 0
        self._has_dist = distances is not None

    @classmethod
    def from_device(cls, handle, m: int, *, device: int, distances: bool) -> "RadiusCSR":
        """Take ownership of a ``b2k_radius_result`` handle of ``m`` rows."""
        self = cls.__new__(cls)
        self.route = "cuda"
        self._indptr = self._indices = self._dist = None
        self._handle = handle
        self._device = int(device)
        self._m = int(m)
        nnz = ctypes.c_int64()
        _lib.check(_lib.load().b2k_radius_result_nnz(handle, ctypes.byref(nnz)),
                   "b2k_radius_result_nnz")
        self._nnz = int(nnz.value)
        self._has_dist = bool(distances)
        return self

    # ------------------------------------------------------------ lifetime
    def release(self) -> None:
        """Free the device result (host arrays already read stay valid)."""
        h, self._handle = self._handle, None
        if h is not None and _lib._lib is not None:
            _lib._lib.b2k_radius_result_release(h)

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def _download(self) -> None:
        if self._indptr is not None:
            return
        if self._handle is None:
            raise RuntimeError("the device result of this batch was released before it was read")
        indptr = _page_locked(self._m + 1, np.int64)
        indices = _page_locked(self._nnz, np.int64)
        dist = _page_locked(self._nnz, np.float64) if self._has_dist else None
        _lib.check(_lib.load().b2k_radius_result_fetch(
            self._handle, indptr.ctypes.data, indices.ctypes.data,
            None if dist is None else dist.ctypes.data), "b2k_radius_result_fetch")
        self._indptr, self._indices, self._dist = indptr, indices, dist

    # ------------------------------------------------------------- fields
    @property
    def indptr(self) -> np.ndarray:
        self._download()
        return self._indptr

    @property
    def indices(self) -> np.ndarray:
        self._download()
        return self._indices

    @property
    def distances(self) -> np.ndarray | None:
        if not self._has_dist:
            return None
        self._download()
        return self._dist

    @property
    def n_query(self) -> int:
        return self._m

    @property
    def nnz(self) -> int:
        return self._nnz

    def lengths(self) -> np.ndarray:
        """Neighbours per query row (int64)."""
        ip = self.indptr
        return ip[1:] - ip[:-1]

    def row_ids(self) -> np.ndarray:
        """The query row of every stored neighbour (int64 ``[nnz]``)."""
        return np.arange(self._m, dtype=np.int64).repeat(self.lengths())

    # ---------------------------------------------------- device reductions
    def _reduce(self, values, kind: str, n_classes: int, weighted: bool):
        import torch

        if self._handle is None:
            raise RuntimeError("device reductions need a batch whose device result is held "
                               "(query_radius_csr(..., raw=True))")
        if weighted and not self._has_dist:
            raise ValueError("distance weights require distances")
        dev = torch.device("cuda", self._device)
        if kind == "votes":
            vals = (values if isinstance(values, torch.Tensor) and values.is_cuda
                    else torch.from_numpy(np.ascontiguousarray(values, dtype=np.int32)))
            vals = vals.to(device=dev, dtype=torch.int32).contiguous()
            out = torch.empty((self._m, n_classes), dtype=torch.float64, device=dev)
        else:
            vals = (values if isinstance(values, torch.Tensor) and values.is_cuda
                    else torch.from_numpy(np.ascontiguousarray(values, dtype=np.float64)))
            vals = vals.to(device=dev, dtype=torch.float64).contiguous()
            out = torch.empty(self._m, dtype=torch.float64, device=dev)
        counts = torch.empty(self._m, dtype=torch.int64, device=dev)
        if self._m:
            lib = _lib.load()
            stream = torch.cuda.current_stream(dev).cuda_stream
            if kind == "votes":
                rc = lib.b2k_radius_result_class_votes(
                    self._handle, vals.data_ptr(), int(n_classes), int(bool(weighted)),
                    out.data_ptr(), counts.data_ptr(), stream)
            else:
                rc = lib.b2k_radius_result_means(self._handle, vals.data_ptr(),
                                                 int(bool(weighted)), out.data_ptr(),
                                                 counts.data_ptr(), stream)
            _lib.check(rc, "radius reduction")
        return out.cpu().numpy(), counts.cpu().numpy()

    def votes(self, codes, n_classes: int, weighted: bool):
        """Per-row class votes (float64 ``[m, n_classes]``: weight 1, or 1/d
        with a row's zero distances taking their 0/1 indicator) and neighbour
        counts, summed on the device in ascending training-index order."""
        return self._reduce(codes, "votes", int(n_classes), weighted)

    def predict_codes(self, codes, n_classes: int):
        """Per-row first maximum of the class counts (ties -> smallest code,
        0 for an empty row) and the neighbour counts, computed on the device
        without downloading the votes; uniform weights only."""
        import torch

        if self._handle is None:
            raise RuntimeError("device reductions need a batch whose device result is held "
                               "(query_radius_csr(..., raw=True))")
        dev = torch.device("cuda", self._device)
        vals = (codes if isinstance(codes, torch.Tensor) and codes.is_cuda
                else torch.from_numpy(np.ascontiguousarray(codes, dtype=np.int32)))
        vals = vals.to(device=dev, dtype=torch.int32).contiguous()
        pred = torch.empty(self._m, dtype=torch.int64, device=dev)
        counts = torch.empty(self._m, dtype=torch.int64, device=dev)
        if self._m:
            stream = torch.cuda.current_stream(dev).cuda_stream
            rc = _lib.load().b2k_radius_result_class_predict(
                self._handle, vals.data_ptr(), int(n_classes), pred.data_ptr(),
                counts.data_ptr(), stream)
            _lib.check(rc, "radius prediction")
        return pred.cpu().numpy(), counts.cpu().numpy()

    def mean(self, targets, weighted: bool):
        """Per-row (1/d-weighted) mean of float64 targets, NaN for empty rows,
        and neighbour counts."""
        return self._reduce(targets, "mean", 0, weighted)


def join_batches(parts) -> tuple[np.ndarray, np.ndarray, np.ndarray | None]:
    """The batches of one query as a single host CSR ``(indptr, indices,
    distances or None)``; a single batch is returned without copying."""
    parts = list(parts)
    if not parts:
        return np.zeros(1, np.int64), np.empty(0, np.int64), None
    if len(parts) == 1:
        p = parts[0]
        return p.indptr, p.indices, p.distances
    m = sum(p.n_query for p in parts)
    nnz = sum(p.nnz for p in parts)
    with_dist = all(p.distances is not None for p in parts)
    indptr = np.empty(m + 1, np.int64)
    indices = np.empty(nnz, np.int64)
    dist = np.empty(nnz, np.float64) if with_dist else None
    indptr[0] = 0
    row = pos = 0
    for p in parts:
        ip = p.indptr
        indptr[row + 1:row + 1 + p.n_query] = ip[1:] - ip[0] + pos
        indices[pos:pos + p.nnz] = p.indices
        if with_dist:
            dist[pos:pos + p.nnz] = p.distances
        row += p.n_query
        pos += p.nnz
    return indptr, indices, dist


def _split_rows(indptr: np.ndarray, values: np.ndarray) -> np.ndarray:
    """Object array whose i-th entry is row i of a CSR value array (a view)."""
    m = len(indptr) - 1
    out = np.empty(max(m, 0), dtype=object)
    if m > 0:
        for i, row in enumerate(np.split(values, indptr[1:-1] - indptr[0])):
            out[i] = row
    return out


def ragged_rows(parts, *, return_distance: bool):
    """scikit-learn's ragged ``radius_neighbors`` output: object arrays of
    int64 index rows (and float64 distance rows first, when asked)."""
    indptr, indices, dist = join_batches(parts)
    rows = _split_rows(indptr, indices)
    if not return_distance:
        return rows
    return _split_rows(indptr, dist), rows


def sparse_graph(indptr, indices, values, shape):
    """A CSR neighbour graph in the container type scikit-learn's
    ``sparse_interface`` setting selects (``csr_matrix`` unless it is
    ``"sparray"``)."""
    from scipy import sparse
    from sklearn import get_config

    kind = sparse.csr_array if get_config().get("sparse_interface") == "sparray" else \
        sparse.csr_matrix
    return kind((values, indices, indptr), shape=shape)


def neighbour_graph(parts, n_samples_fit: int, *, mode: str):
    """``radius_neighbors_graph``: 1.0 per neighbour (``connectivity``) or its
    distance (``distance``)."""
    indptr, indices, dist = join_batches(parts)
    values = np.ones(len(indices)) if mode == "connectivity" else dist
    return sparse_graph(indptr, indices, values, (len(indptr) - 1, int(n_samples_fit)))
