"""The reference's own estimators on the B200 index: the drop-in boundary.

mlx-learn's estimator layer (installed from the reference into baseline/_ref
by ``make -C oracle refpkg``) is bound to the B200 ``NeighborIndex`` exactly
as INTEGRATION.md shows, by replacing ``mlxlearn.neighbors._base.build_index``
(the only constructor its estimators call, reference
src/mlxlearn/neighbors/_base.py:367-370).  Every other line of the reference's
estimators runs unchanged: kneighbors, kneighbors_graph, the classifier's
policy query and host votes (_classification.py:126-159), the radius methods
and the radius classifier's ``votes_of_parts`` (radius_reduce.py:75-84), which
reduces our batches on the device.

GPU tests compare with the golden fixtures the reference's own CPU path
produced (tests/golden/make_golden.py).  The CPU test checks the interface
alone, with a test-only index whose answers come from the oracle.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden
from datasets import mixture

refpkg = pytest.importorskip("oracle.refpkg")


@pytest.fixture
def ref_neighbors(monkeypatch):
    ref = refpkg.import_reference()
    if ref is None:
        pytest.skip("reference package not installed (make -C oracle refpkg)")
    import mlxlearn.neighbors._base as base

    from mlxlearn_b200.index import build_index

    monkeypatch.setattr(base, "build_index", build_index)
    return ref.neighbors


def radius_data():
    rng = np.random.default_rng(4)
    cen = rng.normal(0, 2.0, (10, 32))
    X, y = mixture(rng, 20000, cen, 1.0)
    Q, _ = mixture(np.random.default_rng(44), 500, cen, 1.0)
    Q[:5] += 40.0
    return X, y, Q


# ------------------------------------------------------------------- GPU

@pytest.mark.gpu
def test_reference_nearest_neighbors_on_b200(ref_neighbors):
    from mlxlearn_b200.index import NeighborIndex

    X = np.random.default_rng(0).standard_normal((10000, 64)).astype(np.float32)
    Q = np.random.default_rng(1).standard_normal((2000, 64)).astype(np.float32)
    nn = ref_neighbors.NearestNeighbors(n_neighbors=5, algorithm="brute",
                                        metric="euclidean").fit(X)
    assert isinstance(nn._index_, NeighborIndex)
    d, i = nn.kneighbors(Q)
    g = golden("knn_cfg1.npz")
    np.testing.assert_array_equal(i, g["idx"])
    np.testing.assert_allclose(d, g["dist"], rtol=1e-6, atol=1e-6)
    assert i.dtype == np.int64 and d.dtype == np.float64
    assert nn._index_.last_query_backend == "cuda"

    # graphs: the reference's own builder over our indices and distances
    G = nn.kneighbors_graph(Q[:300], mode="distance")
    np.testing.assert_array_equal(G.indices, g["idx"][:300].ravel())
    np.testing.assert_allclose(G.data, g["dist"][:300].ravel(), rtol=1e-6, atol=1e-6)
    C = nn.kneighbors_graph(Q[:300])
    np.testing.assert_array_equal(C.indices, g["idx"][:300].ravel())
    assert np.all(C.data == 1.0)


@pytest.mark.gpu
def test_reference_self_query_on_b200(ref_neighbors):
    X = np.random.default_rng(0).standard_normal((10000, 64)).astype(np.float32)[:3000].copy()
    X[100:130] = X[:30]
    nn = ref_neighbors.NearestNeighbors(n_neighbors=7, algorithm="brute").fit(X)
    d, i = nn.kneighbors()
    g = golden("knn_self_dups.npz")
    np.testing.assert_array_equal(i, g["idx"])
    np.testing.assert_allclose(d, g["dist"], rtol=1e-6, atol=1e-6)


@pytest.mark.gpu
def test_reference_kneighbors_classifier_and_regressor_on_b200(ref_neighbors):
    X, y, Q = radius_data()
    g = golden("predict_mixture32.npz")
    clf = ref_neighbors.KNeighborsClassifier(n_neighbors=9, weights="distance").fit(X, y)
    np.testing.assert_array_equal(clf.predict(Q), g["cls"])
    np.testing.assert_allclose(clf.predict_proba(Q), g["proba"], rtol=1e-12, atol=1e-12)
    reg = ref_neighbors.KNeighborsRegressor(n_neighbors=9).fit(X, y.astype(np.float64) * 0.5)
    np.testing.assert_allclose(reg.predict(Q), g["reg"], rtol=1e-12, atol=1e-12)
    assert clf._index_.last_query_backend == "cuda"


@pytest.mark.gpu
def test_reference_radius_classifier_on_b200(ref_neighbors):
    X, y, Q = radius_data()
    g = golden("radius_mixture32.npz")
    r = float(g["radius"])
    est = ref_neighbors.RadiusNeighborsClassifier(radius=r, outlier_label="most_frequent")
    est.fit(X, y)
    # predict / predict_proba: the reference's votes_of_parts calls our
    # batches' device votes
    np.testing.assert_array_equal(est.predict(Q), g["pred"])
    np.testing.assert_allclose(est.predict_proba(Q), g["proba"], rtol=1e-12, atol=1e-12)
    rd, ri = est.radius_neighbors(Q)
    lens = np.array([len(a) for a in ri], np.int64)
    np.testing.assert_array_equal(np.concatenate([[0], np.cumsum(lens)]), g["indptr"])
    np.testing.assert_array_equal(np.concatenate(ri), g["indices"])
    np.testing.assert_allclose(np.concatenate(rd), g["dist"], rtol=1e-6, atol=1e-6)
    sd, si = est.radius_neighbors(Q, sort_results=True)
    np.testing.assert_array_equal(np.concatenate(si), g["sorted_indices"])
    G = est.radius_neighbors_graph(Q, mode="distance")
    np.testing.assert_array_equal(G.indptr, g["indptr"])
    np.testing.assert_array_equal(G.indices, g["indices"])
    reg = ref_neighbors.RadiusNeighborsRegressor(radius=r).fit(X, y.astype(np.float64))
    with pytest.warns(UserWarning):  # the five far queries have no neighbour
        pr = reg.predict(Q)
    cnt = lens.astype(np.float64)
    want = np.full(len(Q), np.nan)
    ok = cnt > 0
    sums = np.add.reduceat(y[g["indices"]].astype(np.float64), g["indptr"][:-1][ok])
    want[ok] = sums / cnt[ok]
    np.testing.assert_allclose(pr[ok], want[ok], rtol=1e-12)
    assert np.all(np.isnan(pr[~ok]))


# ------------------------------------------------------------------- CPU

def test_reference_estimators_accept_the_index_interface(monkeypatch):
    """The reference's estimator layer drives the B200 index's seam methods
    (build_index arguments, _query_policy, query with _policy, last backend);
    a test-only subclass answers with the oracle so no GPU is needed."""
    ref = refpkg.import_reference()
    if ref is None:
        pytest.skip("reference package not installed (make -C oracle refpkg)")
    import mlxlearn.neighbors._base as base

    import oracle
    from mlxlearn_b200 import index as b200

    calls = []

    class OracleAnswers(b200.NeighborIndex):
        def query(self, Q, k, *, return_distance=True, exclude_self=False,
                  query_block_size=None, train_block_size=None, _policy=None, **kw):
            calls.append(("query", _policy))
            d, i = oracle.knn(self.training_data, Q, k, exclude_self=exclude_self)
            self.last_query_backend = "cuda"
            return (d if return_distance else None), i

    def build(X, **kw):
        calls.append(("build", tuple(sorted(kw))))
        ix = b200.build_index(X, **kw)
        ix.__class__ = OracleAnswers
        return ix

    monkeypatch.setattr(base, "build_index", build)
    rng = np.random.default_rng(5)
    X = rng.normal(size=(400, 6)).astype(np.float32)
    y = rng.integers(0, 3, size=400)
    Q = rng.normal(size=(50, 6)).astype(np.float32)
    nn = ref.neighbors.NearestNeighbors(n_neighbors=4).fit(X)
    d, i = nn.kneighbors(Q)
    od, oi = oracle.knn(X, Q, 4)
    np.testing.assert_array_equal(i, oi)
    np.testing.assert_array_equal(d, od)
    clf = ref.neighbors.KNeighborsClassifier(n_neighbors=5).fit(X, y)
    pred = clf.predict(Q)
    _, oi5 = oracle.knn(X, Q, 5)
    votes = np.zeros((len(Q), 3))
    np.add.at(votes, (np.arange(len(Q))[:, None], y[oi5]), 1.0)
    np.testing.assert_array_equal(pred, votes.argmax(axis=1))
    assert ("query", (b200.HOST_ARRAY_ROUTE, None)) in calls
    assert any(c[0] == "build" for c in calls)
    assert isinstance(clf._index_, b200.NeighborIndex)
