"""CSR radius results and the conversions scikit-learn's API needs.

Mirrors ``mlxlearn._kernels.radius_result`` (reference
src/mlxlearn/_kernels/radius_result.py:33-147): one ``RadiusCSR`` per query
batch with exact per-row counts, rows in query order, training indices
ascending within a row (or ``(distance, index)`` order when sorting was
requested) and float64 distances when requested.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

INDEX_DTYPE = np.int64

__all__ = ["RadiusCSR", "concatenate", "csr_to_objects", "to_ragged", "to_graph"]


@dataclass(frozen=True, slots=True)
class RadiusCSR:
    indptr: np.ndarray            # int64[n_query + 1]
    indices: np.ndarray           # int64[nnz]
    distances: np.ndarray | None  # float64[nnz] or None
    route: str = "cuda"

    @property
    def n_query(self) -> int:
        return len(self.indptr) - 1

    @property
    def nnz(self) -> int:
        return int(self.indptr[-1]) if len(self.indptr) else 0

    def lengths(self) -> np.ndarray:
        return np.diff(self.indptr)

    def row_ids(self) -> np.ndarray:
        return np.repeat(np.arange(self.n_query, dtype=INDEX_DTYPE), self.lengths())


def csr_to_objects(indptr: np.ndarray, values: np.ndarray) -> np.ndarray:
    bounds = np.asarray(indptr).tolist()
    count = len(bounds) - 1
    if count <= 0:
        return np.empty(0, dtype=object)
    rows = map(values.__getitem__, map(slice, bounds[:-1], bounds[1:]))
    return np.fromiter(rows, dtype=object, count=count)


def concatenate(parts: list[RadiusCSR]) -> RadiusCSR:
    if len(parts) == 1:
        return parts[0]
    if not parts:
        raise ValueError("no results to concatenate")
    offsets = np.cumsum([0] + [p.nnz for p in parts[:-1]])
    indptr = np.concatenate([parts[0].indptr[:1]] + [
        p.indptr[1:] + off for p, off in zip(parts, offsets, strict=True)])
    indices = np.concatenate([p.indices for p in parts])
    distances = (None if parts[0].distances is None
                 else np.concatenate([p.distances for p in parts]))
    return RadiusCSR(indptr.astype(INDEX_DTYPE, copy=False), indices, distances, parts[0].route)


def to_ragged(parts: list[RadiusCSR], *, return_distance: bool):
    """scikit-learn's ragged output: object arrays of 1-d int64 / float64 rows."""
    if not parts:
        empty = np.empty(0, dtype=object)
        return (empty, np.empty(0, dtype=object)) if return_distance else empty
    joined = concatenate(parts)
    indices = csr_to_objects(joined.indptr, joined.indices)
    if not return_distance:
        return indices
    return csr_to_objects(joined.indptr, joined.distances), indices


def to_graph(parts: list[RadiusCSR], n_samples_fit: int, *, mode: str):
    """scikit-learn's CSR neighbour graph, without object arrays."""
    from scipy import sparse
    from sklearn import get_config as get_sklearn_config

    joined = concatenate(parts)
    data = np.ones(joined.nnz) if mode == "connectivity" else joined.distances
    graph = sparse.csr_array((data, joined.indices, joined.indptr),
                             shape=(joined.n_query, int(n_samples_fit)))
    if get_sklearn_config().get("sparse_interface", "spmatrix") == "spmatrix":
        graph = sparse.csr_matrix(graph)
    return graph
