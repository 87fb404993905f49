"""Fitted estimators through to_parquet / from_parquet and pickle predict bit for bit as the saved ones
(python/tests/test_persist.py:209-247 on seeded data of their shape); the file is a table of the samples."""

import pickle

import numpy as np
import pyarrow.parquet as pq
import pytest

import boitata_b200 as bt
from boitata_b200 import workloads as W

pytestmark = pytest.mark.gpu

rng = np.random.default_rng(12)
coords = rng.uniform(0, 100, (300, 3)) * [1.0, 1.0, 0.3]
values = np.exp(rng.normal(0, 0.7, 300))
holes = np.arange(300) // 6
targets = rng.uniform(0, 100, (500, 3)) * [1.0, 1.0, 0.3]
model = bt.Variogram([bt.Structure("spherical", 0.8, 40.0), bt.Structure("exponential", 0.3, 90.0)], nugget=0.05,
                     rotation=(20.0, 5.0, 0.0), ratios=(0.6, 0.3))
search = bt.Search(35.0, max_samples=16, min_samples=2, octant=True, max_per_sector=3)


def estimators():
    return [
        (bt.OrdinaryKriging(model, [search, search.scaled(2.5, min_samples=1)]), {}),
        (bt.OrdinaryKriging(model, bt.Search(40.0, max_samples=24, max_per_hole=3, target_slope=0.9)),
         {"holes": holes}),
        (bt.SimpleKriging(model, search, mean=1.2), {"error_variance": np.full(300, 0.01)}),
        (bt.IndicatorKriging(model, search, 1.0), {}),
        (bt.BlockKriging(model, search, (10.0, 10.0, 5.0), discretization=(2, 2, 2)), {}),
        (bt.OrdinaryKriging(bt.Variogram([bt.Structure("power", 0.01, 10.0, exponent=1.5)], nugget=0.1),
                            bt.Search(40.0, max_samples=96)), {}),
        (bt.OrdinaryKriging(model, search, precision="mixed"), {}),
    ]


def same(a, b):
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("estimator, extra", estimators(), ids=lambda o: type(o).__name__)
def test_estimator_round_trip_predicts_bit_identically(estimator, extra, tmp_path):
    path = tmp_path / "model.parquet"
    estimator.to_parquet(path)
    unfitted = type(estimator).from_parquet(path)
    estimator.fit(coords, values, **extra)
    same(unfitted.fit(coords, values, **extra).predict(targets, return_variance=True),
         estimator.predict(targets, return_variance=True))
    estimator.to_parquet(path)
    for back in (type(estimator).from_parquet(path), pickle.loads(pickle.dumps(estimator))):
        assert type(back) is type(estimator) and back.precision == estimator.precision
        same(back.predict(targets, return_variance=True), estimator.predict(targets, return_variance=True))
        a, b = estimator.cross_validate(), back.cross_validate()
        same((a.estimate, a.variance), (b.estimate, b.variance))


def test_estimator_file_is_a_table_of_samples(tmp_path):
    path = tmp_path / "ok.parquet"
    bt.OrdinaryKriging(model, search).fit(coords, values, holes=holes).to_parquet(path)
    table = pq.read_table(path)
    assert table.column_names == ["x", "y", "z", "value", "hole", "error_variance", "domain"]
    assert table.num_rows == 300
    assert table.column("domain").null_count == 300 and table.column("hole").null_count == 0
    np.testing.assert_array_equal(table.column("value").to_numpy(), values)
    with pytest.raises(bt.InvalidInput, match="expected a SimpleKriging"):
        bt.SimpleKriging.from_parquet(path)


def test_reloaded_c1_estimator_matches_the_saved_one(tmp_path):
    w = W.c1()
    ok = bt.OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    path = tmp_path / "c1.parquet"
    ok.to_parquet(path)
    back = bt.OrdinaryKriging.from_parquet(path)
    a, b = ok.predict_full(w.geometry), back.predict_full(w.geometry)
    for k in ("value", "variance", "lagrange", "n_used", "status"):
        np.testing.assert_array_equal(a[k], b[k])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_runs_are_reproducible_across_contexts(precision):
    """Two estimators fitted alike give the same bits: the grid keeps each cell in sample order, so the
    leave-one-out walk and its tiles do not depend on the order atomics land in."""
    a, b = (bt.OrdinaryKriging(model, search, precision=precision).fit(coords, values) for _ in range(2))
    ca, cb = a.cross_validate(), b.cross_validate()
    same((ca.estimate, ca.variance), (cb.estimate, cb.variance))
    big = rng.uniform(0, 100, (5000, 3)) * [1.0, 1.0, 0.3]  # Morton-ordered caller targets
    same(a.predict(big, return_variance=True), b.predict(big, return_variance=True))


def test_estimator_with_domains_round_trips(tmp_path):
    """Domains travel as the fitted labels in the envelope and a code column (crates/py/src/estimation.rs:
    1110-1145); the reloaded estimator predicts each target in its domain as the saved one does."""
    labels = np.where(coords[:, 0] < 50.0, "north", "south")
    tl = np.where(targets[:, 0] < 50.0, "north", "south")
    est = bt.OrdinaryKriging(model, search).fit(coords, values, domains=labels)
    path = tmp_path / "zoned.parquet"
    est.to_parquet(path)
    table = pq.read_table(path)
    assert table.column("domain").null_count == 0
    for back in (bt.OrdinaryKriging.from_parquet(path), pickle.loads(pickle.dumps(est))):
        same(back.predict(targets, return_variance=True, domains=tl),
             est.predict(targets, return_variance=True, domains=tl))
        a, b = est.cross_validate(folds=4), back.cross_validate(folds=4)
        same((a.estimate, a.variance), (b.estimate, b.variance))
        with pytest.raises(bt.InvalidInput, match="needs domains too"):
            back.predict(targets)
