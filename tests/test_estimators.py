"""Estimator API: parity with the reference's outputs (GPU) and its
validation / error behaviour (CPU)."""
from __future__ import annotations

import pickle
import warnings

import numpy as np
import pytest

from conftest import golden
from datasets import mixture, pixels
from mlxlearn_b200.exceptions import (
    SparseInputError,
    UnsupportedInputError,
    UnsupportedParameterError,
)
from mlxlearn_b200.neighbors import (
    KNeighborsClassifier,
    KNeighborsRegressor,
    NearestNeighbors,
    RadiusNeighborsClassifier,
    RadiusNeighborsRegressor,
)

gpu = pytest.mark.gpu


def radius_data():
    rng = np.random.default_rng(4)
    cen = rng.normal(0, 2.0, (10, 32))
    X, y = mixture(rng, 20000, cen, 1.0)
    Q, _ = mixture(np.random.default_rng(44), 500, cen, 1.0)
    Q[:5] += 40.0
    return X, y, Q


# ------------------------------------------------------------------ CPU side

@pytest.mark.parametrize("kw,param", [({"metric": "manhattan"}, "metric"),
                                      ({"metric": "minkowski", "p": 1}, "p"),
                                      ({"metric_params": {"w": 1}}, "metric_params"),
                                      ({"algorithm": "kd_tree"}, "algorithm")])
def test_capability_errors_raise_before_any_device_use(kw, param):
    X = np.random.default_rng(0).random((10, 3))
    with pytest.raises(UnsupportedParameterError) as e:
        NearestNeighbors(**kw).fit(X)
    assert e.value.parameter == param
    assert isinstance(e.value, ValueError)


def test_callable_weights_and_sparse_and_overflow_rejected():
    from scipy import sparse

    X = np.random.default_rng(0).random((10, 3))
    y = np.arange(10) % 2
    with pytest.raises(UnsupportedParameterError):
        KNeighborsClassifier(weights=lambda d: d).fit(X, y)
    with pytest.raises(SparseInputError, match="sparse"):
        NearestNeighbors().fit(sparse.csr_matrix(X))
    big = X.copy()
    big[0, 0] = 1e300
    with pytest.raises(UnsupportedInputError):
        NearestNeighbors().fit(big)


def test_sklearn_estimator_protocol():
    from sklearn.base import clone

    est = KNeighborsClassifier(n_neighbors=7, weights="distance")
    c = clone(est)
    assert c.get_params()["n_neighbors"] == 7 and c.get_params()["weights"] == "distance"
    assert NearestNeighbors().get_params()["radius"] == 1.0


# ------------------------------------------------------------------ GPU side

def test_radius_outlier_rules_on_the_host():
    # the outlier rules shared by predict and predict_proba, without a search:
    # no label raises the reference's error, a label among the classes gives
    # its column, a label outside them warns at the caller and gives none
    clf = RadiusNeighborsClassifier(radius=1.0)
    clf.classes_ = np.array([3, 5, 9])
    counts = np.array([2, 0, 1, 0])
    clf.outlier_label_ = None
    with pytest.raises(ValueError, match=r"No neighbors found for test samples array\(\[1, 3\]\)"):
        clf._outliers(counts, stacklevel=2)
    clf.outlier_label_ = [5]
    outliers, match = clf._outliers(counts, stacklevel=2)
    np.testing.assert_array_equal(outliers, [1, 3])
    assert match == 1
    clf.outlier_label_ = [4]
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        outliers, match = clf._outliers(counts, stacklevel=2)
    assert match is None and len(w) == 1
    assert "Outlier label 4 is not in training classes" in str(w[0].message)
    assert w[0].filename == __file__
    # no outliers: nothing raised or warned, whatever the label
    clf.outlier_label_ = None
    outliers, match = clf._outliers(np.array([1, 2]), stacklevel=2)
    assert outliers.size == 0 and match is None


@gpu
def test_classifier_regressor_match_reference_predictions():
    X, y, Q = radius_data()
    g = golden("predict_mixture32.npz")
    clf = KNeighborsClassifier(n_neighbors=9, weights="distance").fit(X, y)
    np.testing.assert_array_equal(clf.predict(Q), g["cls"])
    np.testing.assert_allclose(clf.predict_proba(Q), g["proba"], rtol=1e-12, atol=1e-12)
    reg = KNeighborsRegressor(n_neighbors=9).fit(X, y.astype(np.float64) * 0.5)
    np.testing.assert_allclose(reg.predict(Q), g["reg"], rtol=1e-12)
    assert clf.last_query_backend_ == "cuda"


@gpu
def test_pixel_classifier_matches_reference():
    rng = np.random.default_rng(7)
    X, y, T = pixels(rng, 8000)
    Q, _, _ = pixels(rng, 200, templates=T)
    g = golden("knn_pixels784.npz")
    clf = KNeighborsClassifier(n_neighbors=5).fit(X, y)
    d, i = clf.kneighbors(Q)
    np.testing.assert_array_equal(i, g["idx"])
    np.testing.assert_array_equal(clf.predict(Q), g["pred"])


@gpu
def test_radius_classifier_matches_reference():
    X, y, Q = radius_data()
    g = golden("radius_mixture32.npz")
    r = float(g["radius"])
    clf = RadiusNeighborsClassifier(radius=r, outlier_label="most_frequent").fit(X, y)
    np.testing.assert_array_equal(clf.predict(Q), g["pred"])
    np.testing.assert_allclose(clf.predict_proba(Q), g["proba"], rtol=1e-12, atol=1e-12)
    rd, ri = clf.radius_neighbors(Q)
    assert rd.dtype == object and ri.dtype == object and len(ri) == len(Q)
    np.testing.assert_array_equal(np.concatenate(ri), g["indices"])
    np.testing.assert_array_equal(np.concatenate(rd), g["dist"])
    with pytest.raises(ValueError, match="No neighbors found"):
        RadiusNeighborsClassifier(radius=r).fit(X, y).predict(Q)


@gpu
def test_radius_classifier_device_predict_equals_proba_argmax():
    # uniform weights: predict takes each row's first maximum of its class
    # counts on the device; it must equal the argmax of predict_proba (the
    # reference's route) including ties (lattice points, many equal counts),
    # outliers whose label is or is not a class, and 40 classes (two passes)
    rng = np.random.default_rng(41)
    X = rng.integers(-3, 4, size=(3000, 3)).astype(np.float32)
    y = rng.integers(0, 40, size=3000)
    Q = np.concatenate([rng.integers(-3, 4, size=(300, 3)).astype(np.float32),
                        np.full((4, 3), 50.0, np.float32)])
    for label, in_classes in ((7, True), (99, False)):
        clf = RadiusNeighborsClassifier(radius=1.0, outlier_label=label).fit(X, y)
        with warnings.catch_warnings(record=True) as w:
            warnings.simplefilter("always")
            pred = clf.predict(Q)
            proba = clf.predict_proba(Q)
        want = clf.classes_.take(proba.argmax(axis=1))
        empty = np.all(proba == 0.0, axis=1)
        want[empty] = label
        np.testing.assert_array_equal(pred, want)
        assert (pred[-4:] == label).all()
        msgs = [str(x.message) for x in w if "not in training classes" in str(x.message)]
        assert len(msgs) == (0 if in_classes else 2)  # predict and predict_proba
        if not in_classes:
            assert all(x.filename == __file__ for x in w
                       if "not in training classes" in str(x.message))
        # rows with tied top counts exist, so the tie rule is exercised
        top = np.sort(proba[:-4], axis=1)
        assert (top[:, -1] == top[:, -2]).any()
    # string labels and self-queries (X=None) through the same route
    names = np.array([f"c{v:02d}" for v in y])
    clf = RadiusNeighborsClassifier(radius=1.0, outlier_label="most_frequent").fit(X, names)
    proba = clf.predict_proba(None)
    np.testing.assert_array_equal(clf.predict(None), clf.classes_.take(proba.argmax(axis=1)))


@gpu
def test_radius_regressor_nan_and_warning():
    X, y, Q = radius_data()
    reg = RadiusNeighborsRegressor(radius=6.25).fit(X, y.astype(np.float64))
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        pred = reg.predict(Q)
    counts = np.array([len(r) for r in reg.radius_neighbors(Q, return_distance=False)])
    assert np.isnan(pred[:5]).all()
    np.testing.assert_array_equal(np.isnan(pred), counts == 0)
    assert any("no neighbors" in str(x.message) for x in w)


@gpu
def test_kneighbors_self_query_graph_and_errors(rng):
    X = rng.normal(size=(1500, 4)).astype(np.float32)
    nn = NearestNeighbors(n_neighbors=3).fit(X)
    d, i = nn.kneighbors()
    assert not np.any(i == np.arange(1500)[:, None])
    from sklearn.neighbors import NearestNeighbors as SkNN

    sd, si = SkNN(n_neighbors=3, algorithm="brute").fit(X.astype(np.float64)).kneighbors()
    np.testing.assert_array_equal(i, si)
    np.testing.assert_allclose(d, sd, rtol=1e-6, atol=1e-6)
    G = nn.kneighbors_graph(X[:10], mode="distance")
    assert G.shape == (10, 1500) and G.nnz == 30
    with pytest.raises(ValueError, match="Expected n_neighbors <= n_samples_fit"):
        nn.kneighbors(X[:2], n_neighbors=1501)
    with pytest.raises(ValueError, match="Expected n_neighbors < n_samples_fit"):
        nn.kneighbors(n_neighbors=1500)
    with pytest.raises(ValueError, match="Expected n_neighbors > 0"):
        nn.kneighbors(X[:2], n_neighbors=0)
    with pytest.raises(TypeError, match="does not take"):
        nn.kneighbors(X[:2], n_neighbors=2.5)
    Gr = nn.radius_neighbors_graph(X[:10], radius=0.5, mode="connectivity")
    assert Gr.shape == (10, 1500)
    with pytest.raises(ValueError, match="return_distance must be True"):
        nn.radius_neighbors(X[:2], return_distance=False, sort_results=True)


@gpu
def test_pickle_roundtrip(rng):
    X = rng.normal(size=(800, 6)).astype(np.float32)
    y = (X[:, 0] > 0).astype(int)
    clf = KNeighborsClassifier(n_neighbors=4).fit(X, y)
    before = clf.predict(X[:50])
    clone = pickle.loads(pickle.dumps(clf))
    np.testing.assert_array_equal(clone.predict(X[:50]), before)


@gpu
@pytest.mark.parametrize("weighted", [False, True])
def test_device_radius_reductions_equal_reference_reductions(weighted):
    # the device reductions sum each row in the order numpy's bincount does,
    # so they must equal the reference's own host reductions
    # (src/mlxlearn/_kernels/radius_reduce.py:36-72) over the downloaded CSR
    # exactly; queries that coincide with training rows exercise the
    # zero-distance rule
    import torch

    from mlxlearn_b200.index import build_index
    from mlxlearn_b200.radius_result import join_batches
    from oracle import refpkg

    ref = refpkg.import_reference()
    if ref is None:
        pytest.skip("reference package not installed (make -C oracle refpkg)")
    from mlxlearn._kernels.radius_reduce import reduce_mean_csr, reduce_votes_csr
    from mlxlearn._kernels.radius_result import RadiusCSR as RefCSR

    rng = np.random.default_rng(31)
    X = rng.normal(size=(6000, 8)).astype(np.float32)
    Q = np.concatenate([X[:40], rng.normal(size=(400, 8)).astype(np.float32)])
    labels = rng.integers(0, 7, size=6000)
    targets = rng.normal(size=6000)
    ix = build_index(X)
    r = 1.9
    csr = RefCSR(*join_batches(ix.query_radius_csr(Q, r, need_distance=True)))
    hv, hc = reduce_votes_csr(csr, labels, 7, weighted=weighted)
    hm, _ = reduce_mean_csr(csr, targets, weighted=weighted)
    dev = torch.device("cuda", 0)
    dv, dc = ix.query_radius_reduce(Q, r, codes=torch.from_numpy(labels.astype(np.int32)).to(dev),
                                    n_classes=7, weighted=weighted)
    dm, _ = ix.query_radius_reduce(Q, r, targets=torch.from_numpy(targets).to(dev),
                                   weighted=weighted, query_block_size=97)
    np.testing.assert_array_equal(dv, hv)
    np.testing.assert_array_equal(dc, hc)
    np.testing.assert_array_equal(np.isnan(dm), np.isnan(hm))
    np.testing.assert_array_equal(dm[~np.isnan(dm)], hm[~np.isnan(hm)])


@gpu
@pytest.mark.parametrize("weighted", [False, True])
def test_device_radius_reductions_many_classes_and_long_rows(weighted):
    # 40 classes (two 32-class passes of the device reduction) and rows of up
    # to a few hundred entries; each class's float64 sum in entry order is
    # np.bincount's, each mean's numerator and denominator a sequential
    # (cumulative) sum; queries equal to training rows take the zero rule
    import torch

    from mlxlearn_b200.index import build_index
    from mlxlearn_b200.radius_result import join_batches

    rng = np.random.default_rng(37)
    X = rng.normal(size=(5000, 4)).astype(np.float32)
    Q = np.concatenate([X[:30], rng.normal(size=(300, 4)).astype(np.float32)])
    labels = rng.integers(0, 40, size=5000)
    targets = rng.normal(size=5000)
    ix = build_index(X)
    r = 0.9
    ip, ii, dd = join_batches(ix.query_radius_csr(Q, r, need_distance=True))
    lens = np.diff(ip)
    assert lens.max() > 200 and (lens == 0).any()
    hv = np.zeros((len(Q), 40))
    hm = np.full(len(Q), np.nan)
    for q in range(len(Q)):
        a, b = ip[q], ip[q + 1]
        if b == a:
            continue
        d = dd[a:b]
        if weighted:
            w = (d == 0).astype(np.float64) if (d == 0).any() else 1.0 / d
        else:
            w = np.ones(b - a)
        hv[q] = np.bincount(labels[ii[a:b]], weights=w, minlength=40)
        y = targets[ii[a:b]]
        num = np.cumsum(y * w)[-1] if weighted else np.cumsum(y)[-1]
        den = np.cumsum(w)[-1] if weighted else float(b - a)
        hm[q] = num / den
    dev = torch.device("cuda", 0)
    dv, dc = ix.query_radius_reduce(Q, r, codes=torch.from_numpy(labels.astype(np.int32)).to(dev),
                                    n_classes=40, weighted=weighted)
    dm, _ = ix.query_radius_reduce(Q, r, targets=torch.from_numpy(targets).to(dev),
                                   weighted=weighted)
    np.testing.assert_array_equal(dc, lens)
    np.testing.assert_array_equal(dv, hv)
    np.testing.assert_array_equal(np.isnan(dm), np.isnan(hm))
    np.testing.assert_array_equal(dm[~np.isnan(dm)], hm[~np.isnan(hm)])


@gpu
def test_radius_estimators_pickle(rng):
    X, y, Q = radius_data()
    clf = RadiusNeighborsClassifier(radius=6.25, outlier_label="most_frequent").fit(X, y)
    before = clf.predict(Q[:200])
    np.testing.assert_array_equal(pickle.loads(pickle.dumps(clf)).predict(Q[:200]), before)
    reg = RadiusNeighborsRegressor(radius=6.25, weights="distance").fit(X, y.astype(np.float64))
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        p0 = reg.predict(Q[:200])
        p1 = pickle.loads(pickle.dumps(reg)).predict(Q[:200])
    np.testing.assert_array_equal(np.isnan(p0), np.isnan(p1))
    np.testing.assert_array_equal(p0[~np.isnan(p0)], p1[~np.isnan(p1)])


@gpu
def test_distance_weights_zero_distance_rule_matches_sklearn():
    # queries that coincide with training rows: only the zero-distance
    # neighbours vote (weights = indicator of zero distances), the rule of
    # scikit-learn's distance weights that the reference follows
    from sklearn.neighbors import KNeighborsClassifier as SkC
    from sklearn.neighbors import KNeighborsRegressor as SkR

    rng = np.random.default_rng(77)
    X = rng.normal(size=(3000, 6)).astype(np.float32)
    y = rng.integers(0, 4, size=3000)
    t = rng.normal(size=3000)
    Q = np.concatenate([X[:40], rng.normal(size=(40, 6)).astype(np.float32)])
    ours = KNeighborsClassifier(n_neighbors=7, weights="distance").fit(X, y)
    ref = SkC(n_neighbors=7, weights="distance", algorithm="brute").fit(X, y)
    np.testing.assert_array_equal(ours.predict(Q), ref.predict(Q))
    # zero-distance rows: the indicator weights, exactly; elsewhere scikit-learn
    # weighs by float32 distances (its arithmetic for float32 input), this
    # engine by the canonical float64 ones, hence the float32-level tolerance
    p, rp = ours.predict_proba(Q), ref.predict_proba(Q)
    np.testing.assert_array_equal(p[:40], rp[:40])
    np.testing.assert_allclose(p[40:], rp[40:], rtol=1e-6, atol=1e-7)
    ours_r = KNeighborsRegressor(n_neighbors=7, weights="distance").fit(X, t)
    ref_r = SkR(n_neighbors=7, weights="distance", algorithm="brute").fit(X, t)
    pr, rpr = ours_r.predict(Q), ref_r.predict(Q)
    np.testing.assert_array_equal(pr[:40], rpr[:40])
    np.testing.assert_allclose(pr[40:], rpr[40:], rtol=1e-6, atol=1e-7)
    # the first 40 queries are training rows: their prediction is that row's label
    np.testing.assert_array_equal(ours.predict(Q[:40]), y[:40])
