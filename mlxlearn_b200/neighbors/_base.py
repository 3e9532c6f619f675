"""Shared neighbour-estimator machinery on the CUDA index.

Mirrors ``mlxlearn.neighbors._base`` (reference
src/mlxlearn/neighbors/_base.py:84-785): capability checks, validation,
``kneighbors`` / ``kneighbors_graph`` / ``radius_neighbors`` /
``radius_neighbors_graph``, distance weights.  The numerical work is the
CUDA library's (``mlxlearn_b200.index``); there is no CPU or scikit-learn
fallback: a capability mismatch raises, a device failure raises
``BackendExecutionError``.
"""
from __future__ import annotations

from numbers import Integral, Real

import numpy as np
from sklearn.utils.validation import check_is_fitted, validate_data

from ..exceptions import SparseInputError, UnsupportedInputError, UnsupportedParameterError
from ..index import build_index
from ..radius_result import neighbour_graph, ragged_rows, sparse_graph

__all__ = ["NeighborsMixin", "RadiusMixin", "SUPPORTED_METRICS", "compute_weights"]

#: Metrics whose squared form is what the engine computes (reference _base.py:49-53).
SUPPORTED_METRICS = ("euclidean", "l2", "minkowski")
_SUPPORTED_ALGORITHMS = ("auto", "brute")
_FLT_MAX = float(np.finfo(np.float32).max)


def _require_dense(X, estimator, operation="fit"):
    from scipy import sparse

    if sparse.issparse(X):
        raise SparseInputError(
            f"{estimator}.{operation} received sparse input; the CUDA neighbour path is "
            "dense-only. Convert with X.toarray().")


def _check_float32_range(X):
    """float64 values outside float32's range are a capability limit
    (reference _base.py:200-201, parity/test_neighbors_fp32.py:89-99)."""
    arr = np.asarray(X) if not hasattr(X, "dtype") else X
    if getattr(arr, "dtype", None) is not None and arr.dtype.kind == "f" and arr.dtype.itemsize > 4:
        finite = np.isfinite(arr)
        if np.any(np.abs(arr[finite]) > _FLT_MAX):
            raise UnsupportedInputError(
                "Input contains finite values outside the float32 range; the CUDA neighbour "
                "path computes on float32 coordinates.", reason="float32-overflow")


class NeighborsMixin:
    """``fit`` and ``kneighbors`` on the CUDA brute-force engine."""

    # ----------------------------------------------------------- validation
    def _check_params(self):
        name = type(self).__name__
        if self.algorithm not in _SUPPORTED_ALGORITHMS:
            raise UnsupportedParameterError(
                f"{name} implements algorithm in {_SUPPORTED_ALGORITHMS} (brute force) on the "
                f"CUDA path; got algorithm={self.algorithm!r}.",
                parameter="algorithm", value=self.algorithm)
        if self.metric not in SUPPORTED_METRICS:
            raise UnsupportedParameterError(
                f"{name} implements metric in {SUPPORTED_METRICS} on the CUDA path; got "
                f"metric={self.metric!r}.", parameter="metric", value=self.metric)
        if self.metric == "minkowski" and self.p != 2:
            raise UnsupportedParameterError(
                f"{name} implements metric='minkowski' only at p=2 (Euclidean) on the CUDA "
                f"path; got p={self.p!r}.", parameter="p", value=self.p)
        if getattr(self, "metric_params", None):
            raise UnsupportedParameterError(
                f"{name} does not implement metric_params on the CUDA path; got "
                f"{self.metric_params!r}. It will not ignore it and return unweighted "
                "Euclidean distances.", parameter="metric_params", value=self.metric_params)
        weights = getattr(self, "weights", "uniform")
        if callable(weights):
            raise UnsupportedParameterError(
                f"{name} does not implement a callable weights function on the CUDA path.",
                parameter="weights", value=weights)
        nn = getattr(self, "n_neighbors", None)
        if nn is not None and (not isinstance(nn, Integral) or isinstance(nn, bool) or nn < 1):
            raise ValueError(f"n_neighbors must be an int in the range [1, inf); got {nn!r}")
        radius = getattr(self, "radius", None)
        if radius is not None and (not isinstance(radius, Real) or radius < 0):
            raise ValueError(f"radius must be a float in the range [0, inf); got {radius!r}")

    def _fit_neighbors(self, X, y=None, *, target=None):
        name = type(self).__name__
        self._check_params()
        _require_dense(X, name)
        _check_float32_range(X)
        if target is None:
            Xc = validate_data(self, X, accept_sparse=False, dtype=np.float32, order="C",
                               ensure_min_samples=1, reset=True)
            yc = None
        else:
            Xc, yc = validate_data(self, X, y, accept_sparse=False, dtype=np.float32,
                                   order="C", ensure_min_samples=1, multi_output=False,
                                   y_numeric=target == "regression", reset=True)
            if target == "classification":
                from sklearn.utils.multiclass import check_classification_targets

                check_classification_targets(yc)
        self._index_ = build_index(Xc)
        self._index_._ensure_device()
        self.n_samples_fit_ = int(Xc.shape[0])
        self.effective_metric_ = "euclidean"
        self.effective_metric_params_ = {}
        self._fit_method = "brute"
        self.execution_backend_ = "cuda"
        self.execution_policy_ = "fixed"
        self._last_query_backend = None
        return yc

    @property
    def last_query_backend_(self):
        if getattr(self, "_last_query_backend", None) is None:
            raise AttributeError("last_query_backend_")
        return self._last_query_backend

    @property
    def _fit_X(self):
        return self._index_.X

    def _resolve_n_neighbors(self, n_neighbors, query_is_train):
        """scikit-learn's exact messages (reference _base.py:466-488)."""
        if n_neighbors is None:
            n_neighbors = self.n_neighbors
        if not isinstance(n_neighbors, Integral):
            raise TypeError(f"n_neighbors does not take {type(n_neighbors)} value, "
                            "enter integer value")
        if n_neighbors <= 0:
            raise ValueError(f"Expected n_neighbors > 0. Got {n_neighbors}")
        limit = self.n_samples_fit_ - int(query_is_train)
        if n_neighbors > limit:
            inequality = ("n_neighbors < n_samples_fit" if query_is_train
                          else "n_neighbors <= n_samples_fit")
            raise ValueError(f"Expected {inequality}, but n_neighbors = {n_neighbors}, "
                             f"n_samples_fit = {self.n_samples_fit_}")
        return int(n_neighbors)

    def _validate_query(self, X, operation):
        _require_dense(X, type(self).__name__, operation)
        _check_float32_range(X)
        return validate_data(self, X, accept_sparse=False, dtype=np.float32, order="C",
                             reset=False)

    def _prepare_neighbor_query(self, X, n_neighbors=None):
        query_is_train = X is None
        k = self._resolve_n_neighbors(n_neighbors, query_is_train)
        Q = self._index_.training_data if query_is_train else self._validate_query(X, "kneighbors")
        return Q, k, query_is_train

    # ------------------------------------------------------------ kneighbors
    def kneighbors(self, X=None, n_neighbors=None, return_distance=True):
        """k nearest training rows: float64 distances (ascending) and int64
        indices ordered by (distance, index); X=None excludes each row itself."""
        check_is_fitted(self, "_index_")
        Q, k, query_is_train = self._prepare_neighbor_query(X, n_neighbors)
        dist, idx = self._index_.query(Q, k, return_distance=return_distance,
                                       exclude_self=query_is_train)
        self._last_query_backend = "cuda"
        return (dist, idx) if return_distance else idx

    def kneighbors_graph(self, X=None, n_neighbors=None, mode="connectivity"):
        """Sparse ``[n_queries, n_samples_fit]`` graph with one stored entry
        per selected neighbour: 1.0 (``connectivity``) or the distance
        (``distance``); X=None excludes each row itself (the contract of
        reference _base.py:426-444)."""
        check_is_fitted(self, "_index_")
        _check_graph_mode(mode)
        want_dist = mode == "distance"
        dist, idx = self._index_query_for_graph(X, n_neighbors, want_dist)
        m, k = idx.shape
        # every row holds exactly k entries, so the row offsets are k * row
        offsets = k * np.arange(m + 1, dtype=np.int64)
        weights = dist.reshape(-1) if want_dist else np.full(m * k, 1.0)
        return sparse_graph(offsets, idx.reshape(-1), weights, (m, self.n_samples_fit_))

    def _index_query_for_graph(self, X, n_neighbors, want_dist):
        if want_dist:
            return self.kneighbors(X, n_neighbors, return_distance=True)
        return None, self.kneighbors(X, n_neighbors, return_distance=False)

    def __getstate__(self):
        state = dict(self.__dict__)
        return state

    def __setstate__(self, state):
        self.__dict__.update(state)


class RadiusMixin:
    """``radius_neighbors`` and ``radius_neighbors_graph`` (reference _base.py:541-696)."""

    def _radius_query(self, X):
        """The query rows of a radius call and whether they are the training rows."""
        check_is_fitted(self, "_index_")
        query_is_train = X is None
        if query_is_train:
            return self._index_.training_data, True
        from scipy import sparse

        if sparse.issparse(X):
            X = X.toarray()
        return self._validate_query(X, "radius_neighbors"), False

    def _radius_parts(self, X, radius, *, need_distance, sort_results):
        value = self.radius if radius is None else radius
        Q, query_is_train = self._radius_query(X)
        parts = self._index_.query_radius_csr(Q, value, need_distance=need_distance,
                                              exclude_self=query_is_train,
                                              sort_results=sort_results)
        self._last_query_backend = "cuda"
        return parts

    def radius_neighbors(self, X=None, radius=None, return_distance=True, sort_results=False):
        """Every training row within ``radius`` (inclusive, exact) of each query,
        as scikit-learn's ragged object arrays."""
        if sort_results and not return_distance:
            raise ValueError("return_distance must be True if sort_results is True.")
        parts = self._radius_parts(X, radius, need_distance=return_distance,
                                   sort_results=sort_results)
        return ragged_rows(parts, return_distance=return_distance)

    def radius_neighbors_graph(self, X=None, radius=None, mode="connectivity",
                               sort_results=False):
        _check_graph_mode(mode)
        distance = mode == "distance"
        parts = self._radius_parts(X, radius, need_distance=distance,
                                   sort_results=distance and sort_results)
        return neighbour_graph(parts, self.n_samples_fit_, mode=mode)


def _check_graph_mode(mode):
    if mode not in ("connectivity", "distance"):
        raise ValueError('Unsupported mode, must be one of "connectivity", '
                         f'or "distance" but got "{mode}" instead')


def compute_weights(dist, weights):
    """``1/d`` weights; rows with a zero distance use its 0/1 indicator
    (reference _base.py:752-785)."""
    if weights in (None, "uniform"):
        return None
    if weights != "distance":
        raise ValueError("weights not recognized: should be 'uniform' or 'distance', "
                         f"got {weights!r}")
    if dist is None:
        raise ValueError("weights='distance' requires neighbor distances.")
    with np.errstate(divide="ignore"):
        w = 1.0 / np.asarray(dist, dtype=np.float64)
    coincident = np.isinf(w)
    rows = np.any(coincident, axis=1)
    if np.any(rows):
        w[rows] = coincident[rows].astype(np.float64)
    if np.any(np.all(w == 0, axis=1)):
        raise ValueError("All neighbors of some sample are getting zero weights. Please modify "
                         "'weights' to avoid this case if you are using a user-defined function.")
    return w
