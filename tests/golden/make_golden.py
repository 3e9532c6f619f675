"""Generate golden fixtures from the reference's own CPU path.

Run in a container that has the reference tree (read-only) at /root/reference:

    make -C oracle ref            # compiles the reference's CPU extensions into oracle/_ref
    python tests/golden/make_golden.py

The reference package is copied to a temporary directory (its tree is
read-only), the compiled extensions from oracle/_ref are placed beside its
sources, and mlxlearn's own estimators are run.  MLX is not installed, so the
reference's automatic policy runs its CPU engines (NeighborIndex ->
CPUIndex / native C++ / radius engines).  Outputs are written as small .npz
files next to this script; tests read only those files.
"""
from __future__ import annotations

import glob
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("MLXLEARN_REFERENCE", "/root/reference")
sys.path.insert(0, os.path.join(REPO, "tests"))
from datasets import mixture, pixels  # noqa: E402


def import_reference():
    tmp = tempfile.mkdtemp(prefix="mlxlearn_ref_")
    shutil.copytree(os.path.join(REF, "src"), os.path.join(tmp, "src"))
    kernels = os.path.join(tmp, "src", "mlxlearn", "_kernels")
    for so in glob.glob(os.path.join(REPO, "oracle", "_ref", "*.so")):
        shutil.copy(so, kernels)
    sys.path.insert(0, os.path.join(tmp, "src"))
    import mlxlearn  # noqa: F401
    from mlxlearn import neighbors
    from mlxlearn._kernels import neighbors_cpu, radius_cpu

    assert neighbors_cpu._native_query is not None, "reference native kNN not loaded"
    assert radius_cpu.AVAILABLE, "reference native radius engine not loaded"
    return neighbors


def main():
    nb = import_reference()
    out = {}

    # config 1: NearestNeighbors(n_neighbors=5, brute, euclidean), 10000x64 / 2000x64
    X = np.random.default_rng(0).standard_normal((10000, 64)).astype(np.float32)
    Q = np.random.default_rng(1).standard_normal((2000, 64)).astype(np.float32)
    est = nb.NearestNeighbors(n_neighbors=5, algorithm="brute", metric="euclidean").fit(X)
    d, i = est.kneighbors(Q)
    np.savez_compressed(os.path.join(HERE, "knn_cfg1.npz"), dist=d, idx=i)
    out["cfg1"] = i.shape

    # self-query (X=None) on a small slice, with duplicated rows
    Xs = X[:3000].copy()
    Xs[100:130] = Xs[:30]
    est = nb.NearestNeighbors(n_neighbors=7, algorithm="brute").fit(Xs)
    d, i = est.kneighbors()
    np.savez_compressed(os.path.join(HERE, "knn_self_dups.npz"), dist=d, idx=i)

    # config 2a subset: Gaussian mixture 1024 centres in [-1,1]^128, sigma 0.1.
    # A 50,000-row slice keeps the reference CPU run short; 256 queries.
    C = np.random.default_rng(2).uniform(-1, 1, (1024, 128))
    X2, _ = mixture(np.random.default_rng(2), 50000, C, 0.1)
    Q2, _ = mixture(np.random.default_rng(3), 256, C, 0.1)
    est = nb.NearestNeighbors(n_neighbors=10, algorithm="brute").fit(X2)
    d, i = est.kneighbors(Q2)
    np.savez_compressed(os.path.join(HERE, "knn_mixture128.npz"), dist=d, idx=i)

    # config 2b subset: integer pixels 784-d, k=5 (8,000 rows, 200 queries)
    rng = np.random.default_rng(7)
    Xp, yp, T = pixels(rng, 8000)
    Qp, _, _ = pixels(rng, 200, templates=T)
    est = nb.KNeighborsClassifier(n_neighbors=5).fit(Xp, yp)
    d, i = est.kneighbors(Qp)
    pred = est.predict(Qp)
    np.savez_compressed(os.path.join(HERE, "knn_pixels784.npz"), dist=d, idx=i, pred=pred)

    # config 3 subset: radius classifier, 10-class mixture in d=32 (20,000 rows, 500 queries)
    rng = np.random.default_rng(4)
    cen = rng.normal(0, 2.0, (10, 32))
    Xr, yr = mixture(rng, 20000, cen, 1.0)
    Qr, _ = mixture(np.random.default_rng(44), 500, cen, 1.0)
    Qr[:5] += 40.0  # guaranteed outliers (no neighbours)
    r = 6.25  # empirical median 50th-neighbour distance of this sample
    est = nb.RadiusNeighborsClassifier(radius=r, outlier_label="most_frequent").fit(Xr, yr)
    rd, ri = est.radius_neighbors(Qr)
    lens = np.array([len(a) for a in ri], np.int64)
    indptr = np.concatenate([[0], np.cumsum(lens)])
    pred = est.predict(Qr)
    proba = est.predict_proba(Qr)
    sd, si = est.radius_neighbors(Qr, sort_results=True)
    np.savez_compressed(
        os.path.join(HERE, "radius_mixture32.npz"), indptr=indptr,
        indices=np.concatenate(ri), dist=np.concatenate(rd), pred=pred, proba=proba,
        sorted_indices=np.concatenate(si), sorted_dist=np.concatenate(sd), radius=r)

    # kNN classifier / regressor predictions on the same mixture
    clf = nb.KNeighborsClassifier(n_neighbors=9, weights="distance").fit(Xr, yr)
    reg = nb.KNeighborsRegressor(n_neighbors=9).fit(Xr, yr.astype(np.float64) * 0.5)
    np.savez_compressed(os.path.join(HERE, "predict_mixture32.npz"),
                        cls=clf.predict(Qr), proba=clf.predict_proba(Qr), reg=reg.predict(Qr))
    print("wrote fixtures", out)


if __name__ == "__main__":
    main()
