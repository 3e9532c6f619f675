"""The five neighbour estimators (reference src/mlxlearn/neighbors/
_unsupervised.py, _classification.py, _regression.py, _radius.py): same
constructors, parameters, fitted attributes, methods and error messages."""
from __future__ import annotations

import warnings

import numpy as np
from sklearn.base import BaseEstimator, ClassifierMixin, RegressorMixin
from sklearn.utils.validation import check_is_fitted

from ._base import NeighborsMixin, RadiusMixin, compute_weights

__all__ = ["NearestNeighbors", "KNeighborsClassifier", "KNeighborsRegressor",
           "RadiusNeighborsClassifier", "RadiusNeighborsRegressor"]


class NearestNeighbors(RadiusMixin, NeighborsMixin, BaseEstimator):
    """Unsupervised exact Euclidean neighbour search on a B200.

    Parameters follow ``sklearn.neighbors.NearestNeighbors``; ``algorithm`` is
    ``"auto"`` or ``"brute"``, ``metric`` Euclidean (``minkowski`` at ``p=2``).
    Neighbours are ordered by exact distance of the float32 coordinates, then
    by training index.
    """

    def __init__(self, *, n_neighbors=5, radius=1.0, algorithm="auto", leaf_size=30,
                 metric="minkowski", p=2, metric_params=None, n_jobs=None):
        self.n_neighbors = n_neighbors
        self.radius = radius
        self.algorithm = algorithm
        self.leaf_size = leaf_size
        self.metric = metric
        self.p = p
        self.metric_params = metric_params
        self.n_jobs = n_jobs

    def fit(self, X, y=None):
        self._fit_neighbors(X, None)
        return self


class KNeighborsClassifier(NeighborsMixin, ClassifierMixin, BaseEstimator):
    """k-nearest-neighbours classifier; a tied vote goes to the smallest class
    code (the class that sorts first in ``classes_``)."""

    def __init__(self, n_neighbors=5, *, weights="uniform", algorithm="auto", leaf_size=30,
                 p=2, metric="minkowski", metric_params=None, n_jobs=None):
        self.n_neighbors = n_neighbors
        self.weights = weights
        self.algorithm = algorithm
        self.leaf_size = leaf_size
        self.p = p
        self.metric = metric
        self.metric_params = metric_params
        self.n_jobs = n_jobs

    def fit(self, X, y):
        y = self._fit_neighbors(X, y, target="classification")
        self.classes_, encoded = np.unique(y, return_inverse=True)
        self._y = encoded.astype(np.intp, copy=False)
        self.outputs_2d_ = False
        return self

    def _votes(self, X):
        """Search and vote on the GPU; one host transfer of the result
        (reference _classification.py:126-186)."""
        import torch

        from .. import _lib

        if self.weights not in (None, "uniform", "distance"):
            raise ValueError("weights not recognized: should be 'uniform' or 'distance', "
                             f"got {self.weights!r}")
        weighted = self.weights == "distance"
        Q, k, query_is_train = self._prepare_neighbor_query(X)
        dev = torch.device("cuda", self._index_.device)
        codes = self.__dict__.get("_codes_dev")
        if codes is None:
            codes = torch.from_numpy(self._y.astype(np.int32)).to(dev)
            self.__dict__["_codes_dev"] = codes
        Qd = torch.from_numpy(np.ascontiguousarray(Q)).to(dev)
        dist, idx = self._index_.query_device(Qd, k, return_distance=weighted,
                                              exclude_self=query_is_train)
        m, n_classes = idx.shape[0], len(self.classes_)
        votes = torch.empty((m, n_classes), dtype=torch.float64, device=dev)
        pred = torch.empty(m, dtype=torch.int64, device=dev)
        rc = _lib.load().b2k_class_votes(
            idx.data_ptr(), None if dist is None else dist.data_ptr(), m, k, codes.data_ptr(),
            n_classes, int(weighted), votes.data_ptr(), pred.data_ptr(),
            torch.cuda.current_stream(dev).cuda_stream)
        _lib.check(rc, "b2k_class_votes")
        self._last_query_backend = "cuda"
        return votes.cpu().numpy(), pred.cpu().numpy()

    def predict(self, X):
        check_is_fitted(self, "_index_")
        _, pred = self._votes(X)
        return self.classes_.take(pred)

    def predict_proba(self, X):
        check_is_fitted(self, "_index_")
        votes, _ = self._votes(X)
        return votes / votes.sum(axis=1, keepdims=True)

    def __getstate__(self):
        state = dict(self.__dict__)
        state.pop("_codes_dev", None)  # device copy of the labels, rebuilt lazily
        return state


class KNeighborsRegressor(NeighborsMixin, RegressorMixin, BaseEstimator):
    """k-nearest-neighbours regressor (mean, or 1/d-weighted mean, of the
    neighbours' targets)."""

    def __init__(self, n_neighbors=5, *, weights="uniform", algorithm="auto", leaf_size=30,
                 p=2, metric="minkowski", metric_params=None, n_jobs=None):
        self.n_neighbors = n_neighbors
        self.weights = weights
        self.algorithm = algorithm
        self.leaf_size = leaf_size
        self.p = p
        self.metric = metric
        self.metric_params = metric_params
        self.n_jobs = n_jobs

    def fit(self, X, y):
        y = self._fit_neighbors(X, y, target="regression")
        self._y = np.array(y, dtype=np.float64, copy=True)
        return self

    def predict(self, X):
        check_is_fitted(self, "_index_")
        need_distance = self.weights == "distance"
        if need_distance:
            dist, idx = self.kneighbors(X, return_distance=True)
        else:
            dist, idx = None, self.kneighbors(X, return_distance=False)
        neighbors = self._y[idx]
        w = compute_weights(dist, self.weights)
        if w is None:
            return np.mean(neighbors, axis=1)
        return np.sum(neighbors * w, axis=1) / np.sum(w, axis=1)


def _resolve_outlier_label(outlier_label, classes, encoded_y):
    """``outlier_label_`` as scikit-learn sets it for one output
    (reference src/mlxlearn/neighbors/_radius.py:346-380)."""
    if outlier_label is None:
        return None
    if isinstance(outlier_label, str) and outlier_label == "most_frequent":
        counts = np.bincount(encoded_y, minlength=len(classes))
        return [classes[int(counts.argmax())]]

    def arraylike(value):
        return ((hasattr(value, "__len__") or hasattr(value, "shape")
                 or hasattr(value, "__array__")) and not isinstance(value, (str, bytes)))

    if arraylike(outlier_label):
        if len(outlier_label) != 1:
            raise ValueError(f"The length of outlier_label: {outlier_label} is inconsistent "
                             "with the output length: 1")
        label = list(outlier_label)[0]
    else:
        label = outlier_label
    if arraylike(label):
        raise TypeError(f"The outlier_label of classes {classes} is supposed to be a scalar, "
                        f"got {label}.")
    if np.append(classes, label).dtype != classes.dtype:
        raise TypeError(f"The dtype of outlier_label {label} is inconsistent with "
                        f"classes {classes} in y.")
    return [label]


class RadiusNeighborsClassifier(RadiusMixin, NeighborsMixin, ClassifierMixin, BaseEstimator):
    """Every training row within ``radius`` votes; an empty neighbourhood is
    handled by ``outlier_label`` (``None`` raises, as in scikit-learn)."""

    n_neighbors = None

    def __init__(self, radius=1.0, *, weights="uniform", algorithm="auto", leaf_size=30,
                 p=2, metric="minkowski", outlier_label=None, metric_params=None, n_jobs=None):
        self.radius = radius
        self.weights = weights
        self.algorithm = algorithm
        self.leaf_size = leaf_size
        self.p = p
        self.metric = metric
        self.outlier_label = outlier_label
        self.metric_params = metric_params
        self.n_jobs = n_jobs

    def fit(self, X, y):
        y = self._fit_neighbors(X, y, target="classification")
        self.classes_, encoded = np.unique(y, return_inverse=True)
        self._y = encoded.astype(np.intp, copy=False)
        self.outputs_2d_ = False
        self.outlier_label_ = _resolve_outlier_label(self.outlier_label, self.classes_, self._y)
        return self

    def _codes_device(self):
        """The training rows' class codes on the index's device (cached)."""
        import torch

        codes = self.__dict__.get("_codes_dev")
        if codes is None:
            codes = torch.from_numpy(self._y.astype(np.int32)).to(
                torch.device("cuda", self._index_.device))
            self.__dict__["_codes_dev"] = codes
        return codes

    def _check_weights(self):
        if self.weights not in (None, "uniform", "distance"):
            raise ValueError("weights not recognized: should be 'uniform' or 'distance', "
                             f"got {self.weights!r}")
        return self.weights == "distance"

    def _outliers(self, counts, stacklevel):
        """Rows without neighbours; raises without an outlier label, and
        returns the label's column in ``classes_`` (or None, with the
        reference's warning at the user's call) when there are some."""
        outliers = np.flatnonzero(counts == 0)
        if outliers.size > 0 and self.outlier_label_ is None:
            raise ValueError("No neighbors found for test samples "
                             f"{outliers!r}, you can try using larger radius, giving a label "
                             "for outliers, or considering removing them from your dataset.")
        match = None
        if outliers.size > 0:
            label = self.outlier_label_[0]
            found = np.flatnonzero(self.classes_ == label)
            if found.size == 1:
                match = int(found[0])
            else:
                warnings.warn(f"Outlier label {label} is not in training classes. All class "
                              "probabilities of outliers will be assigned with 0.",
                              stacklevel=stacklevel)
        return outliers, match

    def _proba(self, X):
        weighted = self._check_weights()
        Q, query_is_train = self._radius_query(X)
        # votes reduced on the device from the device neighbourhoods
        votes, counts = self._index_.query_radius_reduce(
            Q, self.radius, codes=self._codes_device(), n_classes=len(self.classes_),
            weighted=weighted, exclude_self=query_is_train)
        self._last_query_backend = "cuda"
        outliers, match = self._outliers(counts, stacklevel=4)  # user -> predict* -> _proba
        if match is not None:
            votes[outliers, match] = 1.0
        normalizer = votes.sum(axis=1)[:, None]
        normalizer[normalizer == 0.0] = 1.0
        votes /= normalizer
        return votes

    def predict(self, X):
        check_is_fitted(self, "_index_")
        if self._check_weights():
            proba = self._proba(X)
            labels = self.classes_.take(proba.argmax(axis=1))
            empty = np.all(proba == 0.0, axis=1)
            if np.any(empty):
                labels = np.array(labels, copy=True)
                labels[empty] = self.outlier_label_[0]
            return labels
        # uniform weights: the counts are integers, so the argmax of the
        # normalised votes is the argmax of the counts, taken on the device;
        # a row with neighbours is never all-zero, an outlier row takes the
        # outlier label either way
        Q, query_is_train = self._radius_query(X)
        pred, counts = self._index_.query_radius_predict(
            Q, self.radius, codes=self._codes_device(), n_classes=len(self.classes_),
            exclude_self=query_is_train)
        self._last_query_backend = "cuda"
        outliers, _ = self._outliers(counts, stacklevel=3)  # user -> predict
        labels = self.classes_.take(pred)
        if outliers.size > 0:
            labels = np.array(labels, copy=True)
            labels[outliers] = self.outlier_label_[0]
        return labels

    def predict_proba(self, X):
        check_is_fitted(self, "_index_")
        return self._proba(X)

    def __getstate__(self):
        state = dict(self.__dict__)
        state.pop("_codes_dev", None)  # device copy of the labels, rebuilt lazily
        return state


class RadiusNeighborsRegressor(RadiusMixin, NeighborsMixin, RegressorMixin, BaseEstimator):
    """Mean (or 1/d-weighted mean) of the targets within ``radius``; a query
    with no neighbour predicts NaN and warns, as in scikit-learn."""

    n_neighbors = None

    def __init__(self, radius=1.0, *, weights="uniform", algorithm="auto", leaf_size=30,
                 p=2, metric="minkowski", metric_params=None, n_jobs=None):
        self.radius = radius
        self.weights = weights
        self.algorithm = algorithm
        self.leaf_size = leaf_size
        self.p = p
        self.metric = metric
        self.metric_params = metric_params
        self.n_jobs = n_jobs

    def fit(self, X, y):
        y_arr = np.asarray(y)
        yc = self._fit_neighbors(X, y, target="regression")
        self._y = np.array(yc, dtype=np.float64, copy=True)
        self._y_out_dtype_ = np.float32 if y_arr.dtype == np.float32 else np.float64
        return self

    def predict(self, X):
        import torch

        check_is_fitted(self, "_index_")
        if self.weights not in (None, "uniform", "distance"):
            raise ValueError("weights not recognized: should be 'uniform' or 'distance', "
                             f"got {self.weights!r}")
        weighted = self.weights == "distance"
        targets = self.__dict__.get("_targets_dev")
        if targets is None:
            targets = torch.from_numpy(self._y).to(torch.device("cuda", self._index_.device))
            self.__dict__["_targets_dev"] = targets
        Q, query_is_train = self._radius_query(X)
        pred, counts = self._index_.query_radius_reduce(
            Q, self.radius, targets=targets, weighted=weighted, exclude_self=query_is_train)
        self._last_query_backend = "cuda"
        if np.any(counts == 0):
            warnings.warn("One or more samples have no neighbors within specified radius; "
                          "predicting NaN.", stacklevel=2)
        return pred.astype(self._y_out_dtype_, copy=False)

    def __getstate__(self):
        state = dict(self.__dict__)
        state.pop("_targets_dev", None)  # device copy of the targets, rebuilt lazily
        return state
