"""Vote and mean reductions over neighbour sets.

kNN votes run on the GPU (csrc/votes.cu, b2k_class_votes).  Radius votes/means follow
src/mlxlearn/_kernels/radius_reduce.py:19-94 (``bincount`` in ascending
training-index order, so the result does not depend on batching).
"""
from __future__ import annotations

import numpy as np

from ..radius_result import RadiusCSR


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
