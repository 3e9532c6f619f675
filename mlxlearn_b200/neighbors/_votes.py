"""Vote and mean reductions over neighbour sets.

kNN votes follow the reference's host path (src/mlxlearn/neighbors/
_classification.py:150-163): per-query class totals of 1 or 1/d weights,
accumulated in neighbour order; ``argmax`` then picks the first maximum, i.e.
ties go to the smallest class code.  Radius votes/means follow
src/mlxlearn/_kernels/radius_reduce.py:19-94 (``bincount`` in ascending
training-index order, so the result does not depend on batching).
"""
from __future__ import annotations

import numpy as np

from ..radius_result import RadiusCSR


def class_votes(idx: np.ndarray, codes: np.ndarray, n_classes: int,
                weights: np.ndarray | None) -> np.ndarray:
    votes = np.zeros((len(idx), n_classes), dtype=np.float64)
    rows = np.arange(len(idx))[:, None]
    np.add.at(votes, (rows, codes[idx]), 1.0 if weights is None else weights)
    return votes


def _distance_weights(result: RadiusCSR, rows: np.ndarray) -> np.ndarray:
    dist = result.distances
    if dist is None:
        raise ValueError("distance weights require distances")
    zero = dist == 0.0
    with np.errstate(divide="ignore"):
        weights = 1.0 / dist
    if zero.any():
        coincident = np.bincount(rows[zero], minlength=result.n_query) > 0
        on_row = coincident[rows]
        weights[on_row] = zero[on_row]
    return weights


def radius_votes(result: RadiusCSR, codes: np.ndarray, n_classes: int, *, weighted: bool):
    nq = result.n_query
    lengths = result.lengths().astype(np.int64, copy=False)
    rows = result.row_ids()
    keys = rows * n_classes + np.asarray(codes)[result.indices]
    if weighted:
        votes = np.bincount(keys, weights=_distance_weights(result, rows),
                            minlength=nq * n_classes).astype(np.float64, copy=False)
    else:
        votes = np.bincount(keys, minlength=nq * n_classes).astype(np.float64)
    return votes.reshape(nq, n_classes), lengths


def radius_mean(result: RadiusCSR, targets: np.ndarray, *, weighted: bool):
    nq = result.n_query
    lengths = result.lengths().astype(np.int64, copy=False)
    rows = result.row_ids()
    values = np.asarray(targets, dtype=np.float64)[result.indices]
    if weighted:
        w = _distance_weights(result, rows)
        num = np.bincount(rows, weights=values * w, minlength=nq)
        den = np.bincount(rows, weights=w, minlength=nq)
    else:
        num = np.bincount(rows, weights=values, minlength=nq)
        den = lengths.astype(np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        pred = num / den
    pred[lengths == 0] = np.nan
    return pred, lengths
