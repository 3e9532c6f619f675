"""Neighbour estimators on the B200 engine (the API of ``mlxlearn.neighbors``,
reference src/mlxlearn/neighbors/__init__.py:1-22)."""
from ._estimators import (
    KNeighborsClassifier,
    KNeighborsRegressor,
    NearestNeighbors,
    RadiusNeighborsClassifier,
    RadiusNeighborsRegressor,
)

__all__ = ["NearestNeighbors", "KNeighborsClassifier", "KNeighborsRegressor",
           "RadiusNeighborsClassifier", "RadiusNeighborsRegressor"]
