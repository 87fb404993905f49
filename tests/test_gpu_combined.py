"""Options combined on one call, each against the oracle composed the way the reference composes them:
passes with calibration and the diagnostics table (crates/py/src/estimation.rs:1600-1742 with by_pass,
batch.rs:132-147), block kriging with a calibrated search and its diagnostics, mixed-precision indicator
kriging with an efficiency target, and a persisted block-kriging estimator predicting a rotated model."""

import numpy as np
import pytest
from conftest import close
from test_gpu_parity import assert_same_estimates, centroids

import boitata_b200 as bt
from boitata_b200 import workloads as W

pytestmark = pytest.mark.gpu


def by_pass(oracle, targets, coords, values, searches, vg, **kw):
    """The oracle's estimate_many per pass over the targets earlier passes left (batch.rs:132-147)."""
    out = None
    left = np.arange(len(targets))
    for p, s in enumerate(searches):
        r = oracle.estimate_many(targets[left], coords, values, s, vg, neighbors=False, diagnostics=True, **kw)
        if out is None:
            out = {k: v.copy() for k, v in r.items()}
            out["pass"] = np.where(np.isfinite(r["value"]), 1.0, np.nan)
        else:
            got = np.isfinite(r["value"])
            for k in r:
                out[k][left[got]] = r[k][got]
            out["pass"][left[got]] = p + 1
        left = np.nonzero(~np.isfinite(out["value"]))[0]
        if len(left) == 0:
            break
    return out


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-6)])
def test_calibrated_passes_with_diagnostics(oracle, precision, tol):
    w = W.c1()
    tight = bt.Search(ranges=(90.0, 90.0, 30.0), max_samples=24, min_samples=6, target_slope=0.85)
    wide = bt.Search(ranges=(300.0, 300.0, 100.0), max_samples=24, min_samples=2, target_slope=0.85)
    rng = np.random.default_rng(31)
    t = np.vstack([centroids(oracle, w, 7), rng.uniform(-100, 1100, (400, 3)) * [1, 1, 0.2]])
    est = bt.OrdinaryKriging(w.variogram, [tight, wide], precision=precision).fit(w.coords, w.values)
    d = est.predict(t, diagnostics=True)
    ref = by_pass(oracle, t, w.coords, w.values, [tight, wide], w.variogram)
    fin = np.isfinite(ref["value"])
    assert np.array_equal(fin, np.isfinite(d["value"]))
    assert {1.0, 2.0} <= set(d["pass"][fin])
    np.testing.assert_array_equal(d["pass"][fin], ref["pass"][fin])
    np.testing.assert_array_equal(d["n_samples"][fin], ref["n_used"][fin])
    np.testing.assert_array_equal(d["target_met"][fin], ref["target_met"][fin])
    for key in ("value", "variance", "lagrange"):
        assert np.all(close(d[key][fin], ref[key][fin], tol)), key
    assert np.all(close(d["negative_weight_sum"][fin], ref["negative_weight_sum"][fin], 1e-10))


def test_block_kriging_with_a_calibrated_search_and_diagnostics(oracle):
    w = W.c1()
    s = bt.Search(ranges=(300.0, 300.0, 100.0), max_samples=40, min_samples=4, target_efficiency=0.3)
    size, disc = (20.0, 20.0, 10.0), (3, 3, 2)
    t = centroids(oracle, w, 17)
    bk = bt.BlockKriging(w.variogram, s, size, discretization=disc).fit(w.coords, w.values)
    ref = oracle.estimate_block(t, w.coords, w.values, s, w.variogram, oracle.block_offsets(size, disc))
    assert_same_estimates(bk.predict_full(t), ref, 1e-10)
    d = bk.predict(t, diagnostics=True)
    fin = np.isfinite(ref["value"])
    sv = bk.support_variance()
    np.testing.assert_array_equal(d["support_variance"][fin], sv)
    met = d["target_met"] == 1
    assert met.any() and np.all(d["efficiency"][met] >= 0.3 - 1e-9)


def test_mixed_indicator_kriging_with_an_efficiency_target(oracle):
    w = W.c3()
    s = bt.Search(radius=150.0, min_samples=4, max_samples=64, target_efficiency=0.2)
    t = centroids(oracle, w, 11)
    ik = bt.IndicatorKriging(w.variogram, s, 1.0, precision="mixed").fit(w.coords, w.values)
    ref = oracle.estimate_many(t, w.coords, w.values, s, w.variogram, kind="indicator", kparam=1.0,
                               neighbors=False)
    assert_same_estimates(ik.predict_full(t), ref, 1e-6)


def test_persisted_block_estimator_predicts_a_rotated_model(tmp_path):
    w = W.c2()
    g = bt.Geometry((120.0, 80.0, 40.0), (5.0, 5.0, 6.25), (24, 20, 12), rotation=(30.0, 0.0, 0.0))
    bk = bt.BlockKriging(w.variogram, w.search, g.size, discretization=(3, 3, 2)).fit(w.coords, w.values)
    path = tmp_path / "bk.parquet"
    bk.to_parquet(path)
    back = bt.BlockKriging.from_parquet(path)
    a, b = bk.predict_full(g), back.predict_full(g)
    for k in ("value", "variance", "lagrange", "n_used", "status"):
        np.testing.assert_array_equal(a[k], b[k])
    assert back.support_variance(g) == bk.support_variance(g)
