"""weight_declustering through the engine's weights pass (btk_predict_weights) against the oracle and the
reference's own tests (python/tests/test_estimation.py weight declustering; crates/estimation/src/batch.rs:
1283-1325).

The oracle side restates batch.rs:76-125: each target's list from the oracle's search, its kriging weights
from the oracle's krige (krige.rs:83-95, weights spread over coincident clusters), summed per sample in
target order and scaled to the number of samples. The engine's weights come from its FP64 dense-LU pass, so
they agree with the oracle's to rounding (1e-10 relative); its own sums are reproducible to the bit.
"""

import numpy as np
import pytest

import boitata_b200 as bt
from boitata_b200 import _native as N

pytestmark = pytest.mark.gpu

MODEL = bt.Variogram([("spherical", 1.0, 40.0)], nugget=0.0)
SEARCH = bt.Search(radius=50, max_samples=16)


def clustered():
    """A 10 x 10 grid of samples at 10 m, 60 more clustered in [15, 30]^2, and a copy of the first."""
    grid = np.array([(x, y) for x in range(5, 100, 10) for y in range(5, 100, 10)], float)
    cluster = np.random.default_rng(3).uniform(15, 30, (60, 2))
    xy = np.vstack([grid, cluster, grid[:1]])
    return grid, xy, np.sin(xy[:, 0] / 15) + xy[:, 1] / 50


def oracle_declustering(oracle, xy, z, targets, passes, vg, kind="ordinary", kparam=0.0):
    """batch.rs:76-125 and estimation.rs:1509-1585 on the oracle: (weights per sample, declustered mean)."""
    locs = np.column_stack([xy, np.zeros(len(xy))]) if xy.shape[1] == 2 else xy
    _, first = np.unique(locs + 0.0, axis=0, return_index=True)
    keep = np.sort(first)
    kl, kz = locs[keep], z[keep]
    t3 = np.column_stack([targets, np.zeros(len(targets))]) if targets.shape[1] == 2 else targets
    per_target = [None] * len(t3)
    left = np.arange(len(t3))
    for s in passes:
        if len(left) == 0:
            break
        ref = oracle.estimate_many(t3[left], kl, kz, s, vg, kind=kind, kparam=kparam)
        for j, t in enumerate(left):
            if ref["status"][j] != 0:
                continue
            lst = [i for i in ref["neighbors"][j] if i >= 0]
            st, _, w = oracle.krige(kind, t3[t], kl[lst], kz[lst], vg, kparam=kparam)
            assert st == 0
            per_target[t] = (lst, w)
        left = np.array([t for t in left if per_target[t] is None], dtype=np.int64)
    sums = np.zeros(len(kl))
    for entry in per_target:
        if entry is not None:
            for i, w in zip(*entry):
                sums[i] += w
    total = 0.0
    for w in sums:
        total += w
    sums = sums * (len(kl) / total)
    where = {tuple(r): k for k, r in enumerate(kl + 0.0)}
    owner = np.array([where[tuple(r)] for r in locs + 0.0])
    shared = np.bincount(owner, minlength=len(kl))
    weights = sums[owner] / shared[owner] * (len(locs) / len(kl))
    mean = 0.0
    for w, v in zip(weights, z):
        mean += w * v
    return weights, mean / len(locs)


def test_downweights_clusters_and_shares_duplicates(oracle):
    grid, xy, z = clustered()
    targets = bt.BlockModel((0, 0, 0), (2, 2, 1), (50, 50, 1))
    with pytest.warns(UserWarning):
        d = bt.weight_declustering(xy, z, targets, estimator=bt.OrdinaryKriging(MODEL, SEARCH))
    assert d.weights.sum() == pytest.approx(len(xy))
    assert d.weights[100:160].mean() < 0.5 * d.weights[:100].mean()
    assert d.weights[0] == d.weights[-1]
    assert d.mean == pytest.approx(np.average(z, weights=d.weights))
    assert np.isnan(d.cell_size)
    cent = oracle.centroids((0.0, 0.0, 0.0), (2.0, 2.0, 1.0), (50, 50, 1), (0.0, 0.0, 0.0))
    w, mean = oracle_declustering(oracle, xy, z, cent[:, :2], [SEARCH], MODEL)
    np.testing.assert_allclose(d.weights, w, rtol=1e-10, atol=1e-12)
    assert d.mean == pytest.approx(mean, rel=1e-10)


@pytest.mark.parametrize("kind", ["ordinary", "simple"])
def test_passes_and_kinds_match_the_oracle(oracle, kind):
    _, xy, z = clustered()
    xy, z = xy[:-1], z[:-1]
    rng = np.random.default_rng(8)
    targets = rng.uniform(-20, 120, (3000, 2))
    passes = [bt.Search(radius=12, max_samples=8, min_samples=3), bt.Search(radius=60, max_samples=12)]
    est = (bt.OrdinaryKriging(MODEL, passes) if kind == "ordinary"
           else bt.SimpleKriging(MODEL, passes, mean=float(z.mean())))
    d = bt.weight_declustering(xy, z, targets, estimator=est)
    w, mean = oracle_declustering(oracle, xy, z, targets, passes, MODEL, kind=kind,
                                  kparam=0.0 if kind == "ordinary" else float(z.mean()))
    np.testing.assert_allclose(d.weights, w, rtol=1e-10, atol=1e-12)
    assert d.mean == pytest.approx(mean, rel=1e-10)
    again = bt.weight_declustering(xy, z, targets, estimator=est)
    np.testing.assert_array_equal(again.weights, d.weights)  # the sums do not depend on the launch
    assert est._samples is None  # the estimator given is not fitted


def test_uniform_on_a_regular_grid():
    """batch.rs:1283-1291: samples on a regular grid under targets that cover their cells evenly."""
    g = np.array([(x, y) for x in range(5, 100, 10) for y in range(5, 100, 10)], float)
    z = np.cos(g[:, 0] / 20) + g[:, 1] / 40
    targets = bt.BlockModel((0, 0, 0), (1, 1, 1), (100, 100, 1))
    for est in (bt.OrdinaryKriging(MODEL, SEARCH), bt.SimpleKriging(MODEL, SEARCH, mean=float(z.mean()))):
        w = bt.weight_declustering(g, z, targets, estimator=est).weights
        assert abs(w.sum() - 100.0) < 1e-9
        assert np.all(np.abs(w - 1.0) < 0.15), w


def test_weights_entry_point_lists_and_errors(oracle):
    _, xy, z = clustered()
    xy, z = xy[:-1], z[:-1]
    est = bt.OrdinaryKriging(MODEL, SEARCH).fit(xy, z)
    t = np.array([[50.0, 50.0, 0.0], [900.0, 900.0, 0.0], [20.0, 22.0, 0.0]])
    m, k = len(t), SEARCH.max_samples
    value, status = np.full(m, np.nan), np.zeros(m, dtype=np.int8)
    idx, w = np.zeros((m, k), dtype=np.int64), np.full((m, k), 7.0)
    o = N.OutputsC(value.ctypes.data, None, None, None, status.ctypes.data)
    ctx = est._ctx
    import ctypes

    ctx.check(ctx._lib.btk_predict_weights(ctx.handle, m, t.ctypes.data, N.ORDINARY, 0.0, N.FP64, None,
                                           ctypes.byref(o), idx.ctypes.data, w.ctypes.data), "weights")
    ref = oracle.estimate_many(t, np.column_stack([xy, np.zeros(len(xy))]), z, SEARCH, MODEL)
    assert status[1] == N.ST_SEARCH_FAILED and np.all(idx[1] == -1) and np.all(w[1] == 0.0)
    for j in (0, 2):
        lst = [i for i in ref["neighbors"][j] if i >= 0]
        assert idx[j, : len(lst)].tolist() == lst and np.all(idx[j, len(lst):] == -1)
        assert w[j].sum() == pytest.approx(1.0, abs=1e-12)  # ordinary kriging weights sum to one
        assert np.dot(w[j, : len(lst)], z[lst]) == pytest.approx(value[j], abs=1e-10)
    with pytest.raises(bt.InvalidInput, match="no target was estimated"):
        bt.weight_declustering(xy, z, [[900.0, 900.0]], estimator=bt.OrdinaryKriging(MODEL, SEARCH))


def weights_at(est, t):
    """btk_predict_weights at targets t (m x 3): (status, idx, weights)."""
    import ctypes

    m, k = len(t), est.searches[0].max_samples
    value, status = np.full(m, np.nan), np.zeros(m, dtype=np.int8)
    idx, w = np.zeros((m, k), dtype=np.int64), np.zeros((m, k))
    o = N.OutputsC(value.ctypes.data, None, None, None, status.ctypes.data)
    t = np.ascontiguousarray(t, dtype=np.float64)
    ctx = est._ctx
    ctx.check(ctx._lib.btk_predict_weights(ctx.handle, m, t.ctypes.data, est._kind, est._kparam, N.FP64, None,
                                           ctypes.byref(o), idx.ctypes.data, w.ctypes.data), "weights")
    return status, idx, w


def test_weights_of_coincident_clusters_and_blocks(oracle):
    """Per-system weights against the oracle's krige (krige.rs:83-95: the coincident guard merges samples
    within 1e-6 m and spreads the cluster's weight evenly) and block_krige (block.rs:120-198)."""
    rng = np.random.default_rng(12)
    xy = rng.uniform(0, 100, (120, 2))
    xy = np.vstack([xy, xy[:15] + [3e-7, 0.0]])  # near-duplicates: kept at fit, merged by the guard
    z = np.sin(xy[:, 0] / 15) + xy[:, 1] / 50
    locs = np.column_stack([xy, np.zeros(len(xy))])
    t = np.column_stack([rng.uniform(0, 100, (300, 2)), np.zeros(300)])
    est = bt.OrdinaryKriging(MODEL, SEARCH).fit(xy, z)
    status, idx, w = weights_at(est, t)
    merged = 0
    for j in range(len(t)):
        lst = idx[j][idx[j] >= 0].tolist()
        st, _, ref = oracle.krige("ordinary", t[j], locs[lst], z[lst], MODEL)
        assert (status[j] == N.ST_OK) == (st == 0)
        if st == 0:
            np.testing.assert_allclose(w[j, : len(lst)], ref, rtol=0, atol=1e-10 * (1 + np.abs(ref).max()))
            merged += any(i >= 120 for i in lst)
    assert merged > 20  # the guard's path was taken
    blk = bt.BlockKriging(MODEL, SEARCH, size=(10, 10), discretization=(3, 3, 1)).fit(xy[:120], z[:120])
    with blk._support(None):
        status, idx, w = weights_at(blk, t)
    off = oracle.block_offsets((10.0, 10.0, 1.0), (3, 3, 1))
    for j in range(len(t)):
        lst = idx[j][idx[j] >= 0].tolist()
        st, _, ref = oracle.block_krige(t[j], off, locs[lst], z[lst], MODEL)
        assert (status[j] == N.ST_OK) == (st == 0)
        if st == 0:
            np.testing.assert_allclose(w[j, : len(lst)], ref, rtol=0, atol=1e-10 * (1 + np.abs(ref).max()))


def test_lowers_clustered_samples_and_the_bias():
    """batch.rs:1293-1306: a 10 x 10 grid at 10 m plus 60 samples on a spiral where the field is high; over
    targets covering the square, the clustered samples weigh less than half the grid's and the declustered
    mean lies within a quarter of the naive mean's bias from the field's true mean."""
    field = lambda x, y: np.sin(x / 15.0) + y / 40.0  # noqa: E731
    i = np.arange(100)
    grid = np.column_stack([(i % 10) * 10.0 + 5.0, (i // 10) * 10.0 + 5.0])
    k = np.arange(60)
    a, r = k * 2.4, 1.0 + np.sqrt(k) * 1.5
    spiral = np.column_stack([23.0 + r * np.cos(a), 85.0 + r * np.sin(a)])
    xy = np.vstack([grid, spiral])
    z = field(xy[:, 0], xy[:, 1])
    c = np.arange(10_000)
    cover = np.column_stack([(c % 100) + 0.5, (c // 100) + 0.5])
    truth = field(cover[:, 0], cover[:, 1]).mean()
    naive = z.mean()
    vg = bt.Variogram([("spherical", 1.0, 40.0)])
    d = bt.weight_declustering(xy, z, cover, estimator=bt.OrdinaryKriging(vg, bt.Search(radius=50, max_samples=16)))
    assert abs(d.weights.sum() - 160.0) < 1e-9
    assert d.weights[100:].mean() < 0.5 * d.weights[:100].mean()
    assert abs(d.mean - truth) < 0.25 * abs(naive - truth)
