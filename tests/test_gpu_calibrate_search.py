"""calibrate_search through the engine: the reference's calibration tests (python/tests/test_estimation.py:
1055-1206) with their known answers and properties.

Each scenario's scores reduce the engine's own diagnostics and cross-validation, so these tests pin the
table's definitions (block variance without the nugget, a slope of one for simple kriging with a unique
neighbourhood, the ordering and choice of the suggested cells, domain restriction) on top of predictions
that the parity tests compare with the oracle. The reference's cutoff recoveries (Hermite anamorphosis),
soft domains and inverse-distance case are outside this engine and left out.
"""

import numpy as np
import pytest

import boitata_b200 as bt

pytestmark = pytest.mark.gpu


def scattered():
    """150 points in a 100 x 100 square with a smooth trend, a spherical model of range 40, radius 50."""
    r = np.random.default_rng(3)
    xy = r.uniform(0, 100, (150, 2))
    z = np.sin(xy[:, 0] / 15) + xy[:, 1] / 50
    return xy, z, bt.Variogram([("spherical", 1.0, 40.0)], nugget=0.0), bt.Search(radius=50, max_samples=16)


def gaussian_field(n=300, seed=11):
    """n points in a 200 m square with a Gaussian field of covariance 0.2 nugget + 0.8 spherical (60 m)."""
    g = np.random.default_rng(seed)
    at = g.uniform(0, 200, (n, 2))
    h = np.linalg.norm(at[:, None] - at[None], axis=-1) / 60.0
    cov = 0.8 * np.where(h < 1.0, 1.0 - h * (1.5 - 0.5 * h * h), 0.0) + np.where(h == 0, 0.2, 0.0)
    field = bt.Variogram([("spherical", 0.8, 60.0)], nugget=0.2)
    return field, at, np.linalg.cholesky(cov) @ g.standard_normal(n)


def cell_weights(xy, cell):
    """Declustering weights by cell counts (each sample 1 / its cell's count, scaled to a mean of 1)."""
    keys = [tuple(k) for k in np.floor(xy / cell).astype(int)]
    count = {}
    for k in keys:
        count[k] = count.get(k, 0) + 1
    w = np.array([1.0 / count[k] for k in keys])
    return w * len(w) / w.sum()


BLOCKS = bt.BlockModel(origin=(5.0, 5.0), size=(10, 10), count=(20, 20))


def test_block_variance_excludes_the_nugget():
    xy, z, _, _ = scattered()
    one = bt.Search(radius=1e4, max_samples=4)
    nugget = bt.BlockKriging(bt.Variogram([], nugget=1.0), one, size=(10, 10)).fit(xy, z)
    assert bt.calibrate_search(nugget, [one], BLOCKS, cross_validation=False)["block_variance"][0] == 0.0
    # a 60 m segment of 400 nodes under 0.4 nugget + spherical (1.0, 100 m): C(B,B) = c - mean gamma
    c0, c, a, length = 0.4, 1.0, 100.0, 60.0
    segment = bt.Variogram([("spherical", c, a)], nugget=c0)
    kriging = bt.BlockKriging(segment, one, size=(length, 1.0), discretization=(400, 1, 1)).fit(xy, z)
    gamma_bar = c * (length / (2 * a) - length ** 3 / (20 * a ** 3))
    table = bt.calibrate_search(kriging, [one], [[50.0, 50.0]], cross_validation=False)
    assert table["block_variance"][0] == pytest.approx(c - gamma_bar, abs=1e-4)


def test_simple_kriging_with_a_unique_neighbourhood_has_slope_one():
    xy, z, model, _ = scattered()
    unique = bt.Search(radius=1e6, max_samples=len(z))
    sk = bt.SimpleKriging(model, unique, mean=float(z.mean())).fit(xy, z)
    inside = bt.BlockModel(origin=(5.0, 5.0), size=(10, 10), count=(10, 10))
    table = bt.calibrate_search(sk, [unique], inside, cross_validation=False)
    assert table["slope_mean"][0] == 1.0 and table["slope_p10"][0] == 1.0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_more_samples_raise_the_slope_and_smooth_the_estimates(precision):
    field, at, z = gaussian_field()
    search = bt.Search(radius=50, max_samples=16)
    kriging = bt.BlockKriging(field, search, size=(10, 10), discretization=(3, 3, 1), precision=precision).fit(at, z)
    scenarios = [bt.Search(radius=1e4, max_samples=n) for n in (2, 4, 8, 16)]
    table = bt.calibrate_search(kriging, scenarios, BLOCKS)
    assert np.all(np.diff(table["slope_mean"]) > 0), table["slope_mean"]
    assert np.all(np.diff(table["variance_ratio"]) < 0), table["variance_ratio"]
    assert np.all(np.diff(table["model_variance_ratio"]) < 0), table["model_variance_ratio"]
    np.testing.assert_array_equal(table["scenario"], np.arange(4))


def test_scores_are_deterministic():
    field, at, z = gaussian_field()
    z = np.exp(z)
    weights = cell_weights(at, 20.0)
    search = bt.Search(radius=50, max_samples=16)
    kriging = bt.BlockKriging(field, search, size=(10, 10)).fit(at, z)
    passes = [bt.Search(radius=12, max_samples=8, min_samples=4), bt.Search(radius=1e4, max_samples=8)]

    def run():
        return bt.calibrate_search(kriging, [search, passes], BLOCKS, folds=5, weights=weights)

    first, second = run(), run()
    assert first.column_names == second.column_names
    for name in first.column_names:
        np.testing.assert_array_equal(first[name], second[name])
    assert {"cv_rmse", "cv_slope", "global_bias", "negative_weight_sum"} <= set(first.column_names)
    assert first["first_pass"][1] < 1.0 and first["estimated"][1] == 1.0
    assert all(np.isfinite(first[name]).all() for name in first.column_names)


def test_suggests_the_cheapest_search_reaching_the_slope():
    field, at, z = gaussian_field()
    holes = np.arange(len(z)) // 3
    search = bt.Search(radius=50, max_samples=16)
    kriging = bt.BlockKriging(field, search, size=(10, 10), discretization=(3, 3, 1)).fit(at, z, holes=holes)
    base = bt.Search(radius=30, max_samples=8)
    grid = {"max_samples": [16, 4, 8], "factors": [2, 1], "min_holes": [None, 3]}
    best, table = bt.calibrate_search(kriging, [base], BLOCKS, cross_validation=False, suggest=grid,
                                      target_slope=0.8)
    np.testing.assert_array_equal(table["max_samples"], np.repeat([4, 8, 16], 4))
    np.testing.assert_array_equal(table["factor"], np.tile(np.repeat([1, 2], 2), 3))
    np.testing.assert_array_equal(table["min_holes"], np.tile([np.nan, 3], 6))
    qualifies = (table["slope_mean"] >= 0.8) & (table["estimated"] == table["estimated"].max())
    reached = np.flatnonzero(qualifies)
    assert len(reached) and best is not None
    first = reached[0]
    assert (best.max_samples, best.radius) == (table["max_samples"][first], 30 * table["factor"][first])
    assert not qualifies[:first].any()
    plain = bt.calibrate_search(kriging, [best], BLOCKS, cross_validation=False)
    assert plain["slope_mean"][0] == table["slope_mean"][first]
    none, _ = bt.calibrate_search(kriging, [base], BLOCKS, cross_validation=False, suggest={"max_samples": [4]},
                                  target_slope=1.5)
    assert none is None
    passes, _ = bt.calibrate_search(kriging, [[base, bt.Search(radius=1e4)]], BLOCKS, cross_validation=False,
                                    suggest={"factors": [1]}, target_slope=0)
    assert [p.max_samples for p in passes] == [8, 8]
    empty, table = bt.calibrate_search(kriging, [bt.Search(radius=1, min_samples=4)], BLOCKS,
                                       cross_validation=False, suggest={"min_holes": [1]})
    assert empty is None and table["estimated"][0] == 0.0
    with pytest.raises(bt.InvalidInput, match="one scenario"):
        bt.calibrate_search(kriging, [base, base], BLOCKS, suggest={})
    with pytest.raises(bt.InvalidInput, match="suggest takes"):
        bt.calibrate_search(kriging, [base], BLOCKS, suggest={"radius": [10]})


def test_cross_validates_block_kriging_at_points():
    xy, z, model, search = scattered()
    kriging = bt.BlockKriging(model, search, size=(10, 10)).fit(xy, z)
    table = bt.calibrate_search(kriging, [search], BLOCKS)
    cv = bt.OrdinaryKriging(model, search).fit(xy, z).cross_validate()
    assert table["cv_rmse"][0] == pytest.approx(cv.rmse, rel=1e-12)
    assert table["cv_slope"][0] == pytest.approx(cv.slope, rel=1e-9)
    assert table["cv_mean_error"][0] == pytest.approx(cv.mean_error, rel=1e-9)


def test_calibration_errors():
    xy, z, model, search = scattered()
    kriging = bt.BlockKriging(model, search, size=(10, 10)).fit(xy, z)
    with pytest.raises(ValueError, match="sequence of scenarios"):
        bt.calibrate_search(kriging, search, BLOCKS)
    with pytest.raises(ValueError, match="HermiteAnamorphosis"):
        bt.calibrate_search(kriging, [search], BLOCKS, cutoffs=[1.0])
    with pytest.raises(ValueError, match="weights for"):
        bt.calibrate_search(kriging, [search], BLOCKS, weights=np.ones(3))
    with pytest.raises(ValueError, match="no target"):
        bt.calibrate_search(kriging, [bt.Search(radius=1, min_samples=3)], [[500.0, 500.0]])


def test_calibration_by_domain_matches_the_domain_alone():
    xy, z, model, search = scattered()
    zone = np.where(xy[:, 0] + 0.3 * xy[:, 1] < 50, "MS", "SM")
    grid = np.stack(np.meshgrid(np.arange(0, 100, 4.0), np.arange(0, 100, 4.0)), -1).reshape(-1, 2)
    grid_zone = np.where(grid[:, 0] + 0.3 * grid[:, 1] < 50, "MS", "SM")
    weights = cell_weights(xy, 20.0)
    scenarios = [bt.Search(radius=30, max_samples=8), [bt.Search(radius=30, max_samples=16), bt.Search(radius=80)]]
    at, inside = grid[grid_zone == "MS"], zone == "MS"
    passes = [bt.Search(radius=30, max_samples=16), bt.Search(radius=80, max_samples=8)]
    kriging = bt.OrdinaryKriging(model, passes).fit(xy, z, domains=zone)
    by_domain = bt.calibrate_search(kriging, scenarios, at, weights=weights, domains="MS")
    alone = bt.OrdinaryKriging(model, search).fit(xy[inside], z[inside])
    reference = bt.calibrate_search(alone, scenarios, at, weights=weights[inside])
    assert by_domain.column_names == reference.column_names
    for name in by_domain.column_names:
        np.testing.assert_allclose(by_domain[name], reference[name], rtol=1e-12, atol=1e-15, err_msg=name)
    table = bt.calibrate_search(kriging, [bt.Search(radius=30, max_samples=16)], grid, domains=grid_zone)
    assert np.all(table["estimated"] == 1.0)
    with pytest.raises(bt.InvalidInput, match="predict needs domains"):
        bt.calibrate_search(kriging, [bt.Search(radius=30, max_samples=16)], grid)
