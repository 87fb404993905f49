"""Calibrated searches (target_slope / target_efficiency; crates/py/src/estimation.rs:846-895 with
kriging_algebra.rs:336-412 and the round-robin order of search.rs:913-936) against the oracle: estimates,
variances and n_used to 1e-10 (FP64) or 1e-6 (mixed), equal status and target_met; and the properties of the
reference's test (python/tests/test_estimation.py:510-538) on seeded synthetic data of its shape."""

import numpy as np
import pytest
from conftest import close
from test_gpu_parity import assert_same_estimates, centroids

from boitata_b200 import BlockKriging, IndicatorKriging, OrdinaryKriging, Search, SimpleKriging, Structure, Variogram
from boitata_b200 import workloads as W

pytestmark = pytest.mark.gpu


def assert_met(d, ref):
    fin = np.isfinite(ref["value"])
    np.testing.assert_array_equal(d["target_met"][fin], ref["target_met"][fin])
    assert np.all(np.isnan(d["target_met"][~fin]))


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-6)])
@pytest.mark.parametrize("cal", [{"target_slope": 0.9}, {"target_efficiency": 0.4}, {"target_slope": 0.97}])
def test_calibrated_ordinary_kriging_c1(oracle, precision, tol, cal):
    w = W.c1()
    s = Search(ranges=(300.0, 300.0, 100.0), max_samples=48, min_samples=3, **cal)
    rng = np.random.default_rng(21)
    t = np.vstack([centroids(oracle, w, 11), rng.uniform(-200, 1200, (300, 3)) * [1, 1, 0.2]])
    ok = OrdinaryKriging(w.variogram, s, precision=precision).fit(w.coords, w.values)
    got = ok.predict_full(t)
    ref = oracle.estimate_many(t, w.coords, w.values, s, w.variogram, neighbors=False, diagnostics=True)
    used = ref["n_used"][np.isfinite(ref["value"])]
    assert np.any(used < 48) and np.any(used == 48)  # both outcomes occur
    assert_same_estimates(got, ref, tol)
    assert_met(ok.predict(t, diagnostics=True), ref)


@pytest.mark.parametrize("search", [
    dict(radius=250.0, octant=True, max_per_sector=4, max_samples=32),
    dict(radius=250.0, sectors=6, max_per_sector=5, max_samples=30, min_sectors=2),
])
def test_calibration_takes_the_sectors_in_turn_c2(oracle, search):
    w = W.c2()
    s = Search(**search, target_slope=0.9)
    cent = centroids(oracle, w)
    t = cent[np.random.default_rng(4).choice(len(cent), 2000, replace=False)]
    ok = OrdinaryKriging(w.variogram, s).fit(w.coords, w.values)
    ref = oracle.estimate_many(t, w.coords, w.values, s, w.variogram, neighbors=False, diagnostics=True)
    assert_same_estimates(ok.predict_full(t), ref, 1e-10)
    assert_met(ok.predict(t, diagnostics=True), ref)


def test_calibrated_simple_indicator_and_block_kriging(oracle):
    w = W.c3()
    t = centroids(oracle, w, 13)
    s = Search(radius=150.0, min_samples=4, max_samples=64, target_efficiency=0.35)
    sk = SimpleKriging(w.variogram, s, mean=1.0).fit(w.coords, w.values)
    ref = oracle.estimate_many(t, w.coords, w.values, s, w.variogram, kind="simple", kparam=1.0, neighbors=False)
    assert_same_estimates(sk.predict_full(t), ref, 1e-10)
    s = Search(radius=150.0, min_samples=4, max_samples=64, target_slope=0.9)
    ik = IndicatorKriging(w.variogram, s, 1.2).fit(w.coords, w.values)
    ref = oracle.estimate_many(t, w.coords, w.values, s, w.variogram, kind="indicator", kparam=1.2,
                               neighbors=False)
    assert_same_estimates(ik.predict_full(t), ref, 1e-10)
    size, disc = (20.0, 20.0, 10.0), (3, 3, 2)
    bk = BlockKriging(w.variogram, s, size, discretization=disc).fit(w.coords, w.values)
    ref = oracle.estimate_block(t, w.coords, w.values, s, w.variogram, oracle.block_offsets(size, disc))
    assert_same_estimates(bk.predict_full(t), ref, 1e-10)


def test_calibrated_cross_validation(oracle):
    w = W.c1()
    s = Search(ranges=(300.0, 300.0, 100.0), max_samples=32, min_samples=2, target_slope=0.9)
    cv = OrdinaryKriging(w.variogram, s).fit(w.coords, w.values).cross_validate()
    ref = oracle.estimate_many(None, w.coords, w.values, s, w.variogram, loo=True, neighbors=False)
    fin = np.isfinite(ref["value"])
    assert np.array_equal(fin, np.isfinite(cv.estimate))
    assert np.all(close(cv.estimate[fin], ref["value"][fin], 1e-10))
    assert np.all(close(cv.variance[fin], ref["variance"][fin], 1e-10))


def test_calibrated_search_takes_the_fewest_samples_that_reach_the_target():
    # test_estimation.py:510-530 on seeded data of its shape.
    rng = np.random.default_rng(8)
    coords = rng.uniform(0, 100, (200, 2))
    values = np.sin(coords[:, 0] / 15) + np.cos(coords[:, 1] / 25) + rng.normal(0, 0.2, 200)
    model = Variogram([Structure("spherical", 1.0, 40.0)], nugget=0.1)
    targets = rng.uniform(0, 100, (300, 2))
    plain = Search(radius=60, max_samples=24, min_samples=2)
    calibrated = Search(radius=60, max_samples=24, min_samples=2, target_slope=0.9)
    full = OrdinaryKriging(model, plain).fit(coords, values).predict(targets, diagnostics=True)
    d = OrdinaryKriging(model, calibrated).fit(coords, values).predict(targets, diagnostics=True)
    assert np.isnan(full["target_met"]).all()
    met = d["target_met"] == 1
    assert met.any() and np.all(d["slope"][met] >= 0.9)
    np.testing.assert_array_equal(d["n_samples"][~met], full["n_samples"][~met])
    assert np.all(d["n_samples"] <= full["n_samples"]) and d["n_samples"].mean() < full["n_samples"].mean()
    fewer = OrdinaryKriging(model, Search(radius=60, max_samples=24, min_samples=2, target_slope=0.5))
    assert fewer.fit(coords, values).predict(targets, diagnostics=True)["n_samples"].mean() < d["n_samples"].mean()
    sk = SimpleKriging(model, Search(radius=60, target_efficiency=0.5), mean=1.0).fit(coords, values)
    s = sk.predict(targets, diagnostics=True)
    assert np.all(s["efficiency"][s["target_met"] == 1] >= 0.5 - 1e-12)
