"""kNN parity of the CUDA library against the oracle and the reference's outputs.

Indices must be bit-exact.  Distances are checked two ways: bit-exact against
the oracle's canonical float64 value, and within atol=rtol=1e-6 of the
reference's own outputs (the tolerance of its parity helper,
tests/_helpers.py:73-120 of mlx-learn).
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import golden
from datasets import cfg1, mixture, pixels

pytestmark = pytest.mark.gpu

MODES = ["bf16", "tf32", "fp32", "exact"]


def make_index(X, **kw):
    from mlxlearn_b200.index import build_index

    return build_index(X, **kw)


def check(dist, idx, ref_dist, ref_idx, *, exact_dist=None):
    np.testing.assert_array_equal(idx, ref_idx)
    np.testing.assert_allclose(dist, ref_dist, rtol=1e-6, atol=1e-6)
    if exact_dist is not None:
        np.testing.assert_array_equal(dist, exact_dist)


@pytest.mark.parametrize("mode", MODES)
def test_cfg1_matches_reference_and_oracle(mode):
    X, Q = cfg1()
    g = golden("knn_cfg1.npz")
    od, oi = oracle.knn(X, Q, 5)
    dist, idx = make_index(X).query(Q, 5, mode=mode)
    check(dist, idx, g["dist"], g["idx"], exact_dist=od)
    assert dist.dtype == np.float64 and idx.dtype == np.int64


@pytest.mark.parametrize("mode", MODES)
def test_self_query_with_duplicates(mode):
    X, _ = cfg1()
    Xs = X[:3000].copy()
    Xs[100:130] = Xs[:30]
    g = golden("knn_self_dups.npz")
    dist, idx = make_index(Xs).query(Xs, 7, exclude_self=True, mode=mode)
    check(dist, idx, g["dist"], g["idx"])
    assert not np.any(idx == np.arange(len(Xs))[:, None])


@pytest.mark.parametrize("mode", ["bf16", "tf32", "fp32"])
def test_mixture128_subset(mode):
    C = np.random.default_rng(2).uniform(-1, 1, (1024, 128))
    X, _ = mixture(np.random.default_rng(2), 50000, C, 0.1)
    Q, _ = mixture(np.random.default_rng(3), 256, C, 0.1)
    g = golden("knn_mixture128.npz")
    index = make_index(X)
    dist, idx = index.query(Q, 10, mode=mode, stats=True)
    check(dist, idx, g["dist"], g["idx"])
    st = index.last_stats
    assert st["fallback_rows"] == 0, st


@pytest.mark.parametrize("mode", ["bf16", "tf32", "fp32"])
def test_pixels784_subset(mode):
    rng = np.random.default_rng(7)
    X, y, T = pixels(rng, 8000)
    Q, _, _ = pixels(rng, 200, templates=T)
    g = golden("knn_pixels784.npz")
    dist, idx = make_index(X).query(Q, 5, mode=mode)
    check(dist, idx, g["dist"], g["idx"])


@pytest.mark.parametrize("mode", MODES)
def test_ties_break_on_training_index(mode):
    X = np.array([[1.0], [1.0], [1.0], [2.0]], dtype=np.float32)
    dist, idx = make_index(X).query(np.array([[0.0]], dtype=np.float32), 3, mode=mode)
    np.testing.assert_array_equal(idx, [[0, 1, 2]])
    np.testing.assert_allclose(dist, [[1.0, 1.0, 1.0]])


@pytest.mark.parametrize("mode", MODES)
def test_offset_seed251_exact_order(mode):
    """Rows 1902 and 43153: float32 squared distances round equal, exact order differs
    (reference tests/unit/test_neighbors_precision.py:42-92)."""
    rng = np.random.default_rng(251)
    train = (rng.normal(size=(50_000, 32)) + 10_000).astype(np.float32)
    queries = (rng.normal(size=(256, 32)) + 10_000).astype(np.float32)
    q = queries[79:80]
    sub = train[[1902, 43153]]
    _, i2 = make_index(sub).query(q, 2, mode=mode)
    np.testing.assert_array_equal(i2, [[1, 0]])
    od, oi = oracle.knn(train, np.repeat(q, 65, axis=0), 5)
    assert oi[0, 3] == 43153 and oi[0, 4] == 1902
    dist, idx = make_index(train).query(np.repeat(q, 65, axis=0), 5, mode=mode)
    np.testing.assert_array_equal(idx, oi)
    np.testing.assert_array_equal(dist, od)


@pytest.mark.parametrize("mode", MODES)
def test_equal_distances_choose_smallest_indices(mode):
    train = np.zeros((8, 32), dtype=np.float32)
    train[:4, :2] = [[1, 0], [-1, 0], [0, 1], [0, -1]]
    train[4:, 0] = 2
    query = np.zeros((1, 32), dtype=np.float32)
    for k in (1, 3):
        dist, idx = make_index(train).query(query, k, mode=mode)
        np.testing.assert_array_equal(idx, np.arange(k)[None, :])


@pytest.mark.parametrize("mode", MODES)
def test_monotone_copied_rows(mode):
    train = np.arange(8192 * 32, dtype=np.float32).reshape(8192, 32)
    queries = train[[0, 3, 4, 4096, 8191]].copy()
    od, oi = oracle.knn(train, queries, 5)
    dist, idx = make_index(train).query(queries, 5, mode=mode)
    np.testing.assert_array_equal(idx, oi)
    np.testing.assert_array_equal(idx[:, 0], [0, 3, 4, 4096, 8191])
    np.testing.assert_array_equal(dist[:, 0], 0)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("n,d,m,k", [(512, 16, 31, 7), (5000, 24, 96, 9), (300, 12, 16, 64),
                                     (40, 3, 40, 1), (3000, 130, 257, 33), (1000, 700, 19, 5)])
def test_random_shapes_match_oracle(mode, n, d, m, k, rng):
    X = rng.normal(size=(n, d)).astype(np.float32)
    Q = rng.normal(size=(m, d)).astype(np.float32)
    od, oi = oracle.knn(X, Q, k)
    dist, idx = make_index(X).query(Q, k, mode=mode)
    np.testing.assert_array_equal(idx, oi)
    np.testing.assert_array_equal(dist, od)


@pytest.mark.parametrize("mode", ["bf16", "fp32"])
def test_lattice_ties_and_duplicates(mode, rng):
    """Integer lattice points: many exactly equal distances with different coordinates."""
    X = rng.integers(-3, 4, size=(6000, 8)).astype(np.float32)
    Q = rng.integers(-3, 4, size=(300, 8)).astype(np.float32) + 0.5
    od, oi = oracle.knn(X, Q, 20)
    dist, idx = make_index(X).query(Q, 20, mode=mode)
    np.testing.assert_array_equal(idx, oi)


def test_empty_query_and_k_limits(rng):
    X = rng.normal(size=(20, 3)).astype(np.float32)
    index = make_index(X)
    dist, idx = index.query(np.empty((0, 3), np.float32), 4)
    assert idx.shape == (0, 4) and dist.shape == (0, 4)
    X6 = rng.normal(size=(6, 3)).astype(np.float32)
    i6 = make_index(X6)
    with pytest.raises(ValueError, match="n_neighbors must be <= 6"):
        i6.query(X6, 7)
    with pytest.raises(ValueError, match="n_neighbors must be <= 5"):
        i6.query(X6, 6, exclude_self=True)


def test_blocking_is_invariant(rng):
    X = rng.normal(size=(300, 5)).astype(np.float32)
    Q = rng.normal(size=(37, 5)).astype(np.float32)
    index = make_index(X)
    ref = index.query(Q, 4)
    for qb in (1, 2, 7, 8, 37):
        d, i = index.query(Q, 4, query_block_size=qb)
        np.testing.assert_array_equal(i, ref[1])
        np.testing.assert_array_equal(d, ref[0])


def test_repeat_calls_bitwise_identical(rng):
    X = rng.normal(size=(20000, 48)).astype(np.float32)
    Q = rng.normal(size=(500, 48)).astype(np.float32)
    index = make_index(X)
    a = index.query(Q, 10)
    b = index.query(Q, 10)
    np.testing.assert_array_equal(a[1], b[1])
    np.testing.assert_array_equal(a[0], b[0])


def test_index_owns_its_copy(rng):
    X = rng.normal(size=(500, 8)).astype(np.float32)
    Q = rng.normal(size=(20, 8)).astype(np.float32)
    index = make_index(X)
    before = index.query(Q, 3)
    X[:] = 0
    after = index.query(Q, 3)
    np.testing.assert_array_equal(before[1], after[1])


def test_device_query_matches_host(rng):
    import torch

    X = rng.normal(size=(4000, 64)).astype(np.float32)
    Q = rng.normal(size=(300, 64)).astype(np.float32)
    index = make_index(X)
    hd, hi = index.query(Q, 8)
    dd, di = index.query_device(torch.from_numpy(Q).cuda(), 8)
    np.testing.assert_array_equal(di.cpu().numpy(), hi)
    np.testing.assert_array_equal(dd.cpu().numpy(), hd)


@pytest.mark.parametrize("reorder", ["0", "1"])
@pytest.mark.parametrize("mode", ["bf16", "fp32"])
def test_query_grouping_both_ways(mode, reorder, monkeypatch):
    """Queries are grouped by nearest pivot before the screen (results are
    written back to the original rows); both orders give the oracle's answer."""
    monkeypatch.setenv("B2K_REORDER", reorder)
    C = np.random.default_rng(12).uniform(-1, 1, (64, 40))
    X, _ = mixture(np.random.default_rng(13), 20000, C, 0.15)
    Q, _ = mixture(np.random.default_rng(14), 5000, C, 0.15)
    index = make_index(X)
    od, oi = oracle.knn(X, Q, 12)
    dist, idx = index.query(Q, 12, mode=mode)
    np.testing.assert_array_equal(idx, oi)
    np.testing.assert_array_equal(dist, od)
    od, oi = oracle.knn(X, X, 6, exclude_self=True)
    dist, idx = index.query(X, 6, exclude_self=True, mode=mode)
    np.testing.assert_array_equal(idx, oi)
    np.testing.assert_array_equal(dist, od)


@pytest.mark.parametrize("mode", ["bf16", "fp32"])
def test_full_lists_are_compacted_not_rescanned(mode):
    # k = 50 over 120k i.i.d. rows: a list admits ~k (1 + ln(n / k)) entries
    # while its k-th value settles, more than one list holds; full lists drop
    # what is above the running threshold instead of sending the row to the
    # exhaustive scan.
    rng = np.random.default_rng(17)
    X = rng.standard_normal((120_000, 64)).astype(np.float32)
    Q = rng.standard_normal((300, 64)).astype(np.float32)
    od, oi = oracle.knn(X, Q, 50)
    ix = make_index(X)
    dist, idx = ix.query(Q, 50, mode=mode, stats=True)
    np.testing.assert_array_equal(idx, oi)
    np.testing.assert_array_equal(dist, od)
    assert ix.last_stats["fallback_rows"] == 0


def test_non_finite_inputs_are_rejected():
    # checked on the device after the upload: NaN / inf in the training rows
    # or the queries raise ValueError, and the index stays usable
    rng = np.random.default_rng(23)
    X = rng.standard_normal((3000, 32)).astype(np.float32)
    bad = X.copy()
    bad[1234, 5] = np.inf
    with pytest.raises(ValueError, match="finite"):
        make_index(bad).query(X[:4], 3)
    ix = make_index(X)
    Q = X[:50].copy()
    Q[17, 3] = np.nan
    with pytest.raises(ValueError, match="finite"):
        ix.query(Q, 3)
    with pytest.raises(ValueError, match="finite"):
        ix.query_radius_csr(Q, 1.0)
    import torch

    for mode in ("bf16", "fp32", "exact"):
        with pytest.raises(ValueError, match="finite"):
            ix.query_device(torch.from_numpy(Q).cuda(), 3, mode=mode)
    od, oi = oracle.knn(X, X[:50], 3)
    dist, idx = ix.query(X[:50], 3)
    np.testing.assert_array_equal(idx, oi)


def test_uncertified_bf16_rows_get_an_fp32_second_pass():
    # reference rows on the unit sphere with 1e-5 radial jitter, queries next
    # to its centre: the squared distances spread ~2e-5 around 1, well inside
    # the bf16 bound (~1e-4: bf16 operands, fp32 tensor-core accumulation of
    # the norm column), so every row lands in the bf16 certify band and no
    # query can be certified there; the fp32 bound (~2e-7) leaves a few
    # candidates per query, so the fp32 pass certifies them without the
    # exhaustive scan
    rng = np.random.default_rng(41)
    v = rng.standard_normal((4000, 32))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    X = (v * (1.0 + 1e-5 * rng.standard_normal((4000, 1)))).astype(np.float32)
    Q = (1e-7 * rng.standard_normal((96, 32))).astype(np.float32)
    od, oi = oracle.knn(X, Q, 40)
    ix = make_index(X)
    dist, idx = ix.query(Q, 40, mode="bf16", stats=True)
    np.testing.assert_array_equal(idx, oi)
    np.testing.assert_array_equal(dist, od)
    st = ix.last_stats
    assert st["second_pass_rows"] > 0, st
    assert st["fallback_rows"] == 0, st
    # self-query: the second pass keeps each row's own index excluded
    import torch

    # (k = 60 > the 49 other near-centre rows, so the k-th lies on the sphere)
    Xs = np.concatenate([Q[:50], X]).astype(np.float32)
    ixs = make_index(Xs)
    d2, i2 = ixs.query_device(torch.from_numpy(Xs[:50]).cuda(), 60, mode="bf16",
                              exclude_self=True, q_offset=0, stats=True)
    assert ixs.last_stats["second_pass_rows"] > 0, ixs.last_stats
    o2d, o2i = oracle.knn(Xs, Xs[:50], 60, exclude_self=True)
    np.testing.assert_array_equal(i2.cpu().numpy(), o2i)


@pytest.mark.parametrize("k", [64, 65, 200])
def test_k_across_the_screen_limit(k, rng):
    """k up to 64 runs the screens; larger k takes the exhaustive exact scan.
    Both give the oracle's answer, for host and device queries and a
    self-query; k equal to every row of a small index too."""
    import torch

    X = rng.normal(size=(6000, 24)).astype(np.float32)
    Q = rng.normal(size=(150, 24)).astype(np.float32)
    index = make_index(X)
    od, oi = oracle.knn(X, Q, k)
    dist, idx = index.query(Q, k)
    np.testing.assert_array_equal(idx, oi)
    np.testing.assert_array_equal(dist, od)
    dd, di = index.query_device(torch.from_numpy(Q).cuda(), k)
    np.testing.assert_array_equal(di.cpu().numpy(), oi)
    np.testing.assert_array_equal(dd.cpu().numpy(), od)
    od, oi = oracle.knn(X, X[:100], k, exclude_self=True)
    dd, di = index.query_device(torch.from_numpy(X[:100]).cuda(), k, exclude_self=True,
                                q_offset=0)
    np.testing.assert_array_equal(di.cpu().numpy(), oi)
    np.testing.assert_array_equal(dd.cpu().numpy(), od)
    small = make_index(X[:k])
    od, oi = oracle.knn(X[:k], Q[:7], k)
    dist, idx = small.query(Q[:7], k)
    np.testing.assert_array_equal(idx, oi)
    np.testing.assert_array_equal(dist, od)


@pytest.mark.parametrize("mode", ["bf16", "tf32"])
@pytest.mark.parametrize("group,seed", [("0", "1"), ("1", "0"), ("1", "1")])
def test_row_grouping_both_ways(group, seed, mode, monkeypatch):
    """The bf16 operand's rows are grouped by nearest pivot (the screen's
    lists hold operand rows, certify maps them back to training rows, a
    self-query excludes its row's operand column), and a seeding pass over
    each query tile's home window starts the lists from published k-th
    values; every combination gives the oracle's answer, ties between
    duplicated rows and self-queries included."""
    import torch

    monkeypatch.setenv("B2K_GROUP_ROWS", group)
    monkeypatch.setenv("B2K_SEED", seed)
    C = np.random.default_rng(15).uniform(-1, 1, (128, 48))
    X, _ = mixture(np.random.default_rng(16), 30000, C, 0.1)
    X[20000:20060] = X[:60]  # exact duplicates: ties resolved by training index
    Q, _ = mixture(np.random.default_rng(17), 3000, C, 0.1)
    Q[:20] = X[:20]
    index = make_index(X)
    for k in (1, 10, 40):
        od, oi = oracle.knn(X, Q, k)
        dist, idx = index.query(Q, k, mode=mode, stats=True)
        np.testing.assert_array_equal(idx, oi)
        np.testing.assert_array_equal(dist, od)
        assert index.last_stats["fallback_rows"] == 0
        assert index.last_stats["mode_used"] == (2 if mode == "bf16" else 4)
    Xd = torch.from_numpy(X).cuda()
    for lo in (0, 19990):
        od, oi = oracle.knn(X, X[lo:lo + 3000], 9, exclude_self=True, q_offset=lo)
        dd, di = index.query_device(Xd[lo:lo + 3000], 9, exclude_self=True, q_offset=lo,
                                    mode=mode)
        np.testing.assert_array_equal(di.cpu().numpy(), oi)
        np.testing.assert_array_equal(dd.cpu().numpy(), od)
