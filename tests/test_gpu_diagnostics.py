"""The diagnostics table (predict(..., diagnostics=True), crates/py/src/estimation.rs:1046-1105) against the
oracle's restatement of neighborhood_stats (neighborhood.rs:66-98) and Estimate's derived columns
(krige.rs:44-75), and the properties the reference's own diagnostics tests assert
(python/tests/test_estimation.py:349-388, 491-507, 204-218), on seeded synthetic data of their shapes."""

import numpy as np
import pytest
from conftest import close
from test_gpu_parity import centroids

from boitata_b200 import (BlockKriging, BlockModel, Geometry, IndicatorKriging, OrdinaryKriging, Search,
                          SimpleKriging, Structure, Variogram)
from boitata_b200 import workloads as W
from boitata_b200.estimation import hole_codes

pytestmark = pytest.mark.gpu

COLUMNS = ["value", "variance", "efficiency", "slope", "n_samples", "pass", "n_holes", "n_other_domain",
           "mean_distance", "negative_weight_sum", "lagrange", "support_variance", "estimate_variance",
           "max_samples_reached", "target_met"]


def plane(seed, n=80):
    rng = np.random.default_rng(seed)
    xy = rng.uniform(0, 100, (n, 2))
    v = np.sin(xy[:, 0] / 20) + rng.normal(0, 0.1, n)
    return xy, v


def assert_matches_oracle(d, ref, tol, max_samples):
    fin = np.isfinite(ref["value"])
    assert np.array_equal(fin, np.isfinite(d["value"]))
    for key in ("value", "variance", "lagrange"):
        assert np.all(close(d[key][fin], ref[key][fin], tol)), key
    for key in ("negative_weight_sum", "mean_distance"):
        assert np.all(close(d[key][fin], ref[key][fin], 1e-10)), (key, np.max(np.abs(d[key][fin] - ref[key][fin])))
    np.testing.assert_array_equal(d["n_holes"][fin], ref["n_holes"][fin])
    np.testing.assert_array_equal(d["n_samples"][fin], ref["n_used"][fin])
    np.testing.assert_array_equal(d["max_samples_reached"][fin], (ref["n_within"][fin] >= max_samples) * 1.0)
    sv = ref["support"][fin]
    assert np.all(close(d["support_variance"][fin], sv, 1e-12))
    cov = sv - ref["variance"][fin] - ref["lagrange"][fin]
    assert np.all(close(d["efficiency"][fin], (sv - ref["variance"][fin]) / sv, tol))
    assert np.all(close(d["estimate_variance"][fin], cov - ref["lagrange"][fin], tol))
    for key in COLUMNS:
        assert np.all(np.isnan(d[key][~fin])), key
    assert np.all(np.isnan(d["target_met"]))
    np.testing.assert_array_equal(d["n_other_domain"][fin], 0.0)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-6)])
@pytest.mark.parametrize("labelled", [False, True])
def test_diagnostics_match_the_oracle_c1(oracle, precision, tol, labelled):
    w = W.c1()
    coords = np.vstack([w.coords, w.coords[:40] + [3e-7, 0.0, 0.0]])  # coincident pairs: spread weights
    values = np.concatenate([w.values, w.values[:40] * 1.5])
    labels = [f"H{i // 7}" if i % 11 else None for i in range(len(coords))] if labelled else None
    codes = hole_codes(labels) if labelled else None
    rng = np.random.default_rng(5)
    t = np.vstack([centroids(oracle, w, 13), rng.uniform(-200, 1200, (300, 3)) * [1, 1, 0.2]])
    ok = OrdinaryKriging(w.variogram, w.search, precision=precision).fit(coords, values, holes=labels)
    d = ok.predict(t, diagnostics=True)
    assert d.column_names == COLUMNS
    ref = oracle.estimate_many(t, coords, values, w.search, w.variogram, holes=codes, neighbors=False,
                               diagnostics=True)
    assert_matches_oracle(d, ref, tol, w.search.max_samples)
    assert np.any(ref["negative_weight_sum"] < 0)


@pytest.mark.parametrize("kind", ["simple", "indicator"])
def test_diagnostics_of_simple_and_indicator_kriging(oracle, kind):
    w = W.c3()
    t = centroids(oracle, w, 17)
    est = (SimpleKriging(w.variogram, w.search, mean=1.0) if kind == "simple"
           else IndicatorKriging(w.variogram, w.search, 1.2)).fit(w.coords, w.values)
    d = est.predict(t, diagnostics=True)
    ref = oracle.estimate_many(t, w.coords, w.values, w.search, w.variogram, kind=kind,
                               kparam=1.0 if kind == "simple" else 1.2, neighbors=False, diagnostics=True)
    assert_matches_oracle(d, ref, 1e-10, w.search.max_samples)


@pytest.mark.parametrize("vg,max_samples", [(None, 100), ("power", 40)])
def test_diagnostics_through_the_dense_lu(oracle, vg, max_samples):
    w = W.c1()
    v = w.variogram if vg is None else Variogram([Structure("power", 0.02, 100.0, exponent=1.5)], nugget=0.1)
    s = Search(ranges=(300.0, 300.0, 100.0), max_samples=max_samples, min_samples=1)
    t = centroids(oracle, w, 29)
    d = OrdinaryKriging(v, s).fit(w.coords, w.values).predict(t, diagnostics=True)
    ref = oracle.estimate_many(t, w.coords, w.values, s, v, neighbors=False, diagnostics=True)
    assert_matches_oracle(d, ref, 1e-10, max_samples)


def test_diagnostics_table_properties():
    # test_estimation.py:349-376: column order, slope > 0, efficiency <= 1, exact at data.
    xy, v = plane(1)
    grid = BlockModel(Geometry((0.0, 0.0, 0.0), (10.0, 10.0, 1.0), (10, 10, 1)))
    ok = OrdinaryKriging(Variogram([Structure("spherical", 1.0, 40.0)]), Search(radius=60, max_samples=12))
    d = ok.fit(xy, v).predict(grid, diagnostics=True)
    assert d.column_names == COLUMNS and d.num_rows == 100
    assert np.all(d["slope"] > 0) and np.all(d["efficiency"] <= 1 + 1e-9)
    at = ok.predict(xy[:3], diagnostics=True)
    np.testing.assert_allclose(at["slope"], 1.0)
    np.testing.assert_allclose(at["efficiency"], 1.0)
    assert d.to_pyarrow().num_rows == 100 and list(d.to_pandas().columns) == COLUMNS


def test_neighbourhood_columns():
    # test_estimation.py:491-505 on seeded data of its shape: holes of three samples each.
    xy, v = plane(2, 120)
    model = Variogram([Structure("spherical", 1.0, 30.0)], nugget=0.1)
    holes = np.arange(len(v)) // 3
    ok = OrdinaryKriging(model, Search(radius=30, max_samples=8)).fit(xy, v, holes=holes)
    d = ok.predict(np.random.default_rng(3).uniform(0, 100, (200, 2)), diagnostics=True)
    f = np.isfinite(d["value"])
    assert f.sum() > 150
    assert np.all((d["n_holes"][f] >= 1) & (d["n_holes"][f] <= d["n_samples"][f]))
    assert np.all((d["mean_distance"][f] > 0) & (d["mean_distance"][f] <= 30))
    assert np.all(d["negative_weight_sum"][f] <= 0) and np.any(d["negative_weight_sum"][f] < 0)
    assert np.isfinite(d["lagrange"][f]).all()
    np.testing.assert_array_equal(d["max_samples_reached"][f], d["n_samples"][f] == 8)
    np.testing.assert_array_equal(d["support_variance"][f], model.total_sill())
    covariance = d["support_variance"] - d["variance"] - d["lagrange"]
    np.testing.assert_allclose(covariance[f] / d["estimate_variance"][f], d["slope"][f], rtol=1e-12)


def test_pass_column():
    # test_estimation.py:204-218: the pass that filled each target.
    xy, v = plane(4, 60)
    model = Variogram([Structure("spherical", 1.0, 40.0)])
    tight, wide = Search(radius=8, max_samples=8, min_samples=3), Search(radius=60, max_samples=8, min_samples=3)
    grid = np.random.default_rng(5).uniform(0, 100, (300, 2))
    first = OrdinaryKriging(model, tight).fit(xy, v).predict(grid)
    second = OrdinaryKriging(model, wide).fit(xy, v).predict(grid)
    d = OrdinaryKriging(model, [tight, wide]).fit(xy, v).predict(grid, diagnostics=True)
    np.testing.assert_array_equal(d["pass"], np.where(np.isfinite(first), 1.0, np.where(np.isfinite(second), 2.0,
                                                                                      np.nan)))
    np.testing.assert_array_equal(d["value"], np.where(np.isfinite(first), first, second))
    assert {1.0, 2.0} <= set(d["pass"][np.isfinite(d["pass"])])


def test_block_diagnostics_use_the_block_support_variance(oracle):
    w = W.c1()
    size, disc = (20.0, 20.0, 10.0), (3, 3, 2)
    t = centroids(oracle, w, 23)
    bk = BlockKriging(w.variogram, w.search, size, discretization=disc).fit(w.coords, w.values)
    d = bk.predict(t, diagnostics=True)
    ref = oracle.estimate_block(t, w.coords, w.values, w.search, w.variogram, oracle.block_offsets(size, disc))
    fin = np.isfinite(ref["value"])
    assert np.all(close(d["value"][fin], ref["value"][fin], 1e-10))
    np.testing.assert_array_equal(d["support_variance"][fin], bk.support_variance())
    assert np.all(close(d["efficiency"][fin], (bk.support_variance() - ref["variance"][fin]) / bk.support_variance(),
                        1e-10))
    assert np.all(d["negative_weight_sum"][fin] <= 0)
