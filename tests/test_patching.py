"""The scikit-learn patching shell (CPU: no estimator is fitted here).

Mirrors the reference's patching tests in spirit: names resolve bare or
dotted, unknown names raise in both directions, patching is idempotent and
restores the original class, and a third-party replacement is never
discarded.
"""
from __future__ import annotations

import warnings

import pytest

from mlxlearn_b200 import patching


@pytest.fixture(autouse=True)
def _clean():
    patching.unpatch_sklearn()
    yield
    patching.unpatch_sklearn()


def test_patch_and_unpatch_all():
    import sklearn.neighbors as skn

    original = skn.KNeighborsClassifier
    patching.patch_sklearn()
    assert skn.KNeighborsClassifier.__module__.startswith("mlxlearn_b200")
    assert patching.is_patched()
    assert len(patching.patched_estimators()) == 5
    patching.patch_sklearn()  # idempotent
    patching.unpatch_sklearn()
    assert skn.KNeighborsClassifier is original
    assert not patching.is_patched()


def test_names_resolve_and_unknown_names_raise():
    import sklearn.neighbors as skn

    patching.patch_sklearn("NearestNeighbors")
    patching.patch_sklearn(["sklearn.neighbors.RadiusNeighborsRegressor"])
    assert patching.is_patched(["NearestNeighbors", "RadiusNeighborsRegressor"])
    assert not patching.is_patched("KNeighborsRegressor")
    m = patching.get_patch_map()
    assert m["sklearn.neighbors.NearestNeighbors"]["patched"]
    assert m["sklearn.neighbors.KNeighborsRegressor"]["original"] is None
    with pytest.raises(ValueError, match="Available"):
        patching.patch_sklearn("SVC")
    with pytest.raises(ValueError, match="Available"):
        patching.unpatch_sklearn("SVC")
    patching.unpatch_sklearn("NearestNeighbors")
    assert skn.NearestNeighbors.__module__.startswith("sklearn")


def test_third_party_replacement_is_kept():
    import sklearn.neighbors as skn

    patching.patch_sklearn("KNeighborsRegressor")

    class Other:
        pass

    skn.KNeighborsRegressor = Other
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        patching.patch_sklearn("KNeighborsRegressor")
        patching.unpatch_sklearn("KNeighborsRegressor")
    assert skn.KNeighborsRegressor is Other
    assert len([x for x in w if issubclass(x.category, patching.PatchWarning)]) == 2
    from sklearn.neighbors._regression import KNeighborsRegressor as Original

    skn.KNeighborsRegressor = Original
