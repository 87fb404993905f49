"""Known answers of the reference's estimation tests, run through the engine's call surface.

The reference's Python tests (python/tests/test_estimation.py) hold a few
cases whose answer follows from the kriging equations alone: exact
interpolation at the data without a nugget, the simple-kriging mean far from
the data, the variance of a pure-nugget block, a one-node block equal to the
point estimate. They pin the engine's end-to-end results (search, assembly,
solve, epilogue) without an oracle. Both precisions are held to the answer.
"""

import numpy as np
import pytest

import boitata_b200 as bt

pytestmark = pytest.mark.gpu

FORMS = [("fp64", 1e-8), ("mixed", 1e-6)]


def scattered():
    """150 points in a 100 x 100 square with a smooth trend, a spherical model of range 40, radius 50."""
    r = np.random.default_rng(3)
    xy = r.uniform(0, 100, (150, 2))
    z = np.sin(xy[:, 0] / 15) + xy[:, 1] / 50
    return xy, z, bt.Variogram([("spherical", 1.0, 40.0)], nugget=0.0), bt.Search(radius=50, max_samples=16)


@pytest.mark.parametrize("precision,tol", FORMS)
def test_ordinary_kriging_is_exact_at_the_data(precision, tol):
    xy, z, vg, s = scattered()
    est, var = bt.OrdinaryKriging(vg, s, precision=precision).fit(xy, z).predict(xy, return_variance=True)
    np.testing.assert_allclose(est, z, atol=tol)
    np.testing.assert_allclose(var, 0.0, atol=tol)


def test_variance_grows_away_from_the_data():
    xy, z, vg, s = scattered()
    near = bt.OrdinaryKriging(vg, s).fit(xy, z).predict(xy[:1] + [0.5, 0.0], return_variance=True)[1][0]
    far = bt.OrdinaryKriging(vg, bt.Search(radius=400)).fit(xy, z).predict([[200.0, 200.0]],
                                                                          return_variance=True)[1][0]
    assert 0.0 < near < far


def test_too_few_neighbours_leave_the_target_unestimated():
    xy, z, vg, _ = scattered()
    got = bt.OrdinaryKriging(vg, bt.Search(radius=5, min_samples=3)).fit(xy, z).predict([[500.0, 500.0]])
    assert np.isnan(got[0])


@pytest.mark.parametrize("precision,tol", FORMS)
def test_simple_kriging_takes_the_mean_beyond_the_range(precision, tol):
    # Every sample lies beyond the range (40) of (400, 400): all covariances to the target vanish.
    xy, z, vg, _ = scattered()
    sk = bt.SimpleKriging(vg, bt.Search(radius=1000), mean=7.0, precision=precision).fit(xy, z)
    assert sk.predict([[400.0, 400.0]])[0] == pytest.approx(7.0, abs=tol)


def test_a_pure_nugget_block_has_the_variance_of_a_mean_of_sixteen():
    # C(B, B) and C(B, x) vanish for a pure nugget: equal weights 1/16, variance -mu = 1/16.
    xy, z, _, s = scattered()
    d = bt.BlockKriging(bt.Variogram([], nugget=1.0), s, size=(10, 10)).fit(xy, z).predict([[50.0, 50.0]],
                                                                                           diagnostics=True)
    assert d["variance"][0] == pytest.approx(1.0 / 16, abs=1e-12)


def test_a_one_node_block_is_the_point_estimate():
    # One sample at distance 50: the point variance is 2 gamma(50), and a block discretized by one node equals
    # the point.
    vg = bt.Variogram([("spherical", 0.7, 100.0)], nugget=0.3)
    one = bt.Search(radius=1e4, max_samples=1)
    at, z = [[50.0, 0.0]], [1.0]
    point = bt.OrdinaryKriging(vg, one).fit(at, z).predict([[0.0, 0.0]], diagnostics=True)
    block = bt.BlockKriging(vg, one, size=(10, 10, 10), discretization=(1, 1, 1)).fit(at, z).predict(
        [[0.0, 0.0]], diagnostics=True)
    h = 0.5
    gamma50 = 0.3 + 0.7 * (1.5 * h - 0.5 * h ** 3)
    assert point["variance"][0] == pytest.approx(2 * gamma50, abs=1e-9)
    assert block["variance"][0] == pytest.approx(point["variance"][0], abs=1e-9)
    assert point["value"][0] == pytest.approx(1.0) and block["value"][0] == pytest.approx(1.0)


@pytest.mark.parametrize("octant", [False, True])
def test_max_samples_beyond_the_data_takes_them_all(oracle, octant):
    """max_samples far above the 40 samples (the reference's 'take them all' idiom): every target takes all
    40; with octants and a max_samples of 100, the per-octant cap the reference derives from it (13) still
    limits each octant, list for list as the oracle's tree."""
    r = np.random.default_rng(3)
    xyz = r.uniform(0, 100, (40, 3))
    vg = bt.Variogram([("spherical", 1.0, 40.0)])
    z = r.normal(size=40)
    every = bt.Search(radius=500, max_samples=1 << 40, octant=octant)
    d = bt.OrdinaryKriging(vg, every).fit(xyz, z).predict(xyz[:5] + 1.0, diagnostics=True)
    assert np.all(np.asarray(d["n_samples"]) == 40)
    capped = bt.Search(radius=500, max_samples=100, octant=octant)
    ok = bt.OrdinaryKriging(vg, capped).fit(xyz, z)
    targets = r.uniform(-20, 120, (60, 3))
    idx, cnt, good = ok.neighbors(targets)
    tree = oracle.Tree(xyz, capped, vg)
    for t, target in enumerate(targets):
        want_ok, want = tree.neighbors(target)
        assert idx[t, : cnt[t]].tolist() == want and bool(good[t]) == want_ok, t
    ref = oracle.estimate_many(targets, xyz, z, capped, vg, neighbors=False)
    np.testing.assert_allclose(ok.predict(targets), ref["value"], rtol=1e-10, atol=1e-10)


def test_ranges_select_the_same_neighbours_as_radius_and_ratios():
    r = np.random.default_rng(5)
    xyz, z, at = r.uniform(0, 100, (300, 3)), r.normal(size=300), r.uniform(10, 90, (80, 3))
    vg = bt.Variogram([("spherical", 1.0, 40.0)])
    by_ratios = bt.Search(radius=60, rotation=(30, 10, 0), ratios=(0.5, 0.25), max_samples=12, octant=True)
    by_ranges = bt.Search(ranges=(60, 30, 15), rotation=(30, 10, 0), max_samples=12, octant=True)
    a, b = (bt.OrdinaryKriging(vg, s).fit(xyz, z).predict(at, diagnostics=True) for s in (by_ratios, by_ranges))
    for key in ("value", "n_samples", "mean_distance"):
        np.testing.assert_array_equal(a[key], b[key])


@pytest.mark.parametrize("precision,tol", FORMS)
def test_block_kriging_of_a_constant_is_the_constant(precision, tol):
    xy, _, vg, s = scattered()
    bk = bt.BlockKriging(vg, s, size=(10, 10), precision=precision).fit(xy, np.full(len(xy), 3.0))
    np.testing.assert_allclose(bk.predict([[50.0, 50.0], [5.0, 95.0]]), 3.0, atol=tol)


def test_indicator_kriging_gives_probabilities():
    xy, z, vg, s = scattered()
    ik = bt.IndicatorKriging(vg, s, threshold=float(np.median(z))).fit(xy, z)
    p = ik.predict(np.random.default_rng(4).uniform(0, 100, (50, 2)))
    assert np.all((p >= -1e-9) & (p <= 1 + 1e-9))


def test_near_duplicates_share_their_weight_whatever_the_neighbourhood_size():
    # 64 samples take the warp kernels, 65 the dense LU: both merge the pair 1e-9 m apart.
    lattice = np.array([[x, y] for x in range(0, 100, 11) for y in range(0, 100, 11)], float)
    xy = np.vstack([[[50.5, 50.5], [50.5 + 1e-9, 50.5]], lattice])
    z = np.r_[1.0, 5.0, np.sin(lattice[:, 0] / 17.0) + 3.0]
    vg = bt.Variogram([("spherical", 1.0, 50.0)])
    out = [bt.OrdinaryKriging(vg, bt.Search(radius=1e3, max_samples=n)).fit(xy, z).predict([[52.0, 51.0]])[0]
           for n in (64, 65)]
    assert np.all(np.isfinite(out))


def test_measurement_error_blends_a_datum_with_its_neighbours():
    # With error variance e at datum 0, its estimate there is the LOO estimate moved towards the datum by
    # k = var_loo / (var_loo + e); zero error variances change nothing.
    xy, z, vg, _ = scattered()
    xy, z = xy[:20], z[:20]
    wide = bt.Search(radius=500, max_samples=50)
    plain = bt.OrdinaryKriging(vg, wide).fit(xy, z)
    zero = bt.OrdinaryKriging(vg, wide).fit(xy, z, error_variance=np.zeros(20))
    grid = np.random.default_rng(6).uniform(0, 100, (50, 2))
    np.testing.assert_array_equal(plain.predict(grid), zero.predict(grid))
    loo = plain.cross_validate()
    e = np.where(np.arange(20) == 0, 0.2, 0.0)
    noisy = bt.OrdinaryKriging(vg, wide).fit(xy, z, error_variance=e)
    k = loo.variance[0] / (loo.variance[0] + 0.2)
    assert noisy.predict(xy[:1])[0] == pytest.approx(loo.estimate[0] + k * (z[0] - loo.estimate[0]), abs=1e-9)


def test_block_kriging_follows_a_rotated_model():
    # A block model rotated 90 degrees with 50 x 5 blocks krigs as 5 x 50 blocks at the same centres.
    r = np.random.default_rng(0)
    xy, z = r.uniform(0, 100, (40, 2)), r.normal(size=40)
    s = bt.Search(radius=500, max_samples=40)
    vg = bt.Variogram([("spherical", 1.0, 20.0)])
    model = bt.BlockModel((0, 0, 0), (50, 5, 1), (1, 1, 1), rotation=(90, 0, 0))
    rotated = bt.BlockKriging(vg, s, (50, 5, 1)).fit(xy, z).predict(model)
    plain = bt.BlockKriging(vg, s, (5, 50, 1)).fit(xy, z).predict(model.coords[:, :2])
    assert rotated == pytest.approx(plain)


def test_cross_validation_summary():
    xy, z, vg, s = scattered()
    cv = bt.OrdinaryKriging(vg, s).fit(xy, z).cross_validate()
    assert cv.estimate.shape == z.shape
    assert abs(cv.mean_error) < 0.1 and cv.correlation > 0.8
    assert np.isfinite(cv.standardized_squared_error)


@pytest.mark.parametrize("rule", [
    bt.Search(radius=50, max_samples=4, octant=True, max_per_sector=1),
    bt.Search(radius=50, max_samples=6, sectors=6, max_per_sector=1, max_empty_sectors=2),
    bt.Search(radius=50, max_samples=6, max_per_hole=2, min_holes=3),
], ids=["octant", "sectors", "holes"])
def test_cross_validation_searches_as_if_the_sample_were_absent(rule):
    xy, z, vg, _ = scattered()
    holes = [f"DH{i // 5}" for i in range(len(xy))]
    cv = bt.OrdinaryKriging(vg, rule).fit(xy, z, holes=holes).cross_validate()
    for i in range(0, len(xy), 7):
        rest = np.arange(len(xy)) != i
        alone = bt.OrdinaryKriging(vg, rule).fit(xy[rest], z[rest], holes=list(np.array(holes)[rest]))
        np.testing.assert_allclose(cv.estimate[i], alone.predict(xy[i:i + 1])[0], rtol=1e-9, atol=1e-12)


def test_shared_locations_keep_the_first_and_name_their_holes():
    xy = np.array([[0.0, 0.0], [10.0, 0.0], [0.0, 0.0], [0.0, 10.0]])
    v = np.array([1.0, 2.0, 5.0, 3.0])
    vg, s = bt.Variogram([("spherical", 1.0, 30.0)]), bt.Search(radius=50, max_samples=8)
    with pytest.warns(UserWarning, match="holes DH1, DH3 at"):
        ok = bt.OrdinaryKriging(vg, s).fit(xy, v, holes=["DH1", "DH2", "DH3", "DH4"])
    np.testing.assert_array_equal(ok.cross_validate().actual, [1.0, 2.0, 3.0])
    assert np.isfinite(ok.predict([[2.0, 2.0]])).all()
    with pytest.warns(UserWarning, match="rows 0, 2"):
        sgs = bt.SGS(vg, s).fit(xy, v)
    assert np.isfinite(sgs.simulate([[2.0, 2.0], [5.0, 5.0]], n=2, seed=1).mean).all()


def test_neighbourhood_diagnostics():
    xy, z, vg, _ = scattered()
    holes = np.arange(len(z)) // 3
    ok = bt.OrdinaryKriging(vg, bt.Search(radius=30, max_samples=8)).fit(xy, z, holes=holes)
    d = ok.predict(np.random.default_rng(8).uniform(0, 100, (200, 2)), diagnostics=True)
    assert {"n_holes", "mean_distance", "negative_weight_sum", "lagrange", "max_samples_reached"} <= set(
        d.column_names)
    assert np.all((d["n_holes"] >= 1) & (d["n_holes"] <= d["n_samples"]))
    assert np.all((d["mean_distance"] > 0) & (d["mean_distance"] <= 30))
    assert np.all(d["negative_weight_sum"] <= 0) and np.any(d["negative_weight_sum"] < 0)
    assert np.isfinite(d["lagrange"]).all()
    np.testing.assert_array_equal(d["max_samples_reached"], d["n_samples"] == 8)
    np.testing.assert_array_equal(d["support_variance"], 1.0)
    cov = d["support_variance"] - d["variance"] - d["lagrange"]
    np.testing.assert_allclose(cov / d["estimate_variance"], d["slope"], rtol=1e-12)


def test_plane_sectors_cap_each_sector():
    r = np.random.default_rng(7)
    xyz, z = r.uniform(0, 100, (400, 3)), r.normal(size=400)
    vg = bt.Variogram([("spherical", 1.0, 40.0)])
    s = bt.Search(radius=60, max_samples=48, sectors=4, max_per_sector=3, rotation=(30, 0, 0), ratios=(0.5, 0.2))
    d = bt.OrdinaryKriging(vg, s).fit(xyz, z).predict(r.uniform(20, 80, (50, 3)), diagnostics=True)
    assert np.all(np.asarray(d["n_samples"]) <= 12)


def test_min_sectors_leaves_a_one_sided_target_to_the_next_pass():
    g = np.random.default_rng(5)
    east = np.column_stack([g.uniform(10, 60, 200), g.uniform(-25, 25, 200)])
    holes = np.arange(200) // 5
    flat = np.full(200, 3.0)
    vg = bt.Variogram([("spherical", 1.0, 40.0)])
    outside, inside = np.array([[-10.0, 0.0]]), np.array([[35.0, 0.0]])
    one_sided, fallback = bt.Search(radius=100, octant=True, min_sectors=3), bt.Search(radius=100)
    for s in (one_sided, bt.Search(radius=100, octant=True, max_empty_sectors=1)):
        ok = bt.OrdinaryKriging(vg, [s, fallback]).fit(east, flat, holes=holes)
        assert ok.predict(outside, diagnostics=True)["pass"][0] == 2.0
        assert ok.predict(inside, diagnostics=True)["pass"][0] == 1.0
    assert np.isnan(bt.OrdinaryKriging(vg, one_sided).fit(east, flat).predict(outside)[0])
    rules = bt.Search(radius=100, octant=True, max_per_sector=3, min_sectors=4, max_empty_sectors=1, min_holes=4)
    d = bt.OrdinaryKriging(vg, rules).fit(east, flat, holes=holes).predict(g.uniform(15, 55, (40, 2)),
                                                                          diagnostics=True)
    done = np.isfinite(d["value"])
    assert done.any()
    np.testing.assert_allclose(d["value"][done], 3.0, atol=1e-10)
    assert (d["n_holes"][done] >= 4).all() and (d["n_samples"][done] <= 12).all()


def test_min_holes_needs_that_many_holes():
    xy, z, vg, _ = scattered()
    holes = np.arange(150) // 50
    at = np.random.default_rng(9).uniform(0, 100, (60, 2))
    for need, estimated in ((3, True), (4, False)):
        s = bt.Search(radius=500, max_samples=150, min_holes=need)
        d = bt.OrdinaryKriging(vg, s).fit(xy, z, holes=holes).predict(at, diagnostics=True)
        assert np.isfinite(d["value"]).all() == estimated
    few = bt.Search(radius=500, max_samples=4, max_per_hole=1, min_holes=3)
    d = bt.OrdinaryKriging(vg, few).fit(xy, z, holes=holes).predict(at, diagnostics=True)
    assert np.isfinite(d["value"]).all() and (d["n_holes"] >= 3).all()


def test_passes_reach_further_targets():
    """Search.passes of a 10 m search that needs 3 samples: targets beyond the first pass's reach take the
    second (the pass column of the diagnostics)."""
    xy, z, vg, _ = scattered()
    grid = np.random.default_rng(12).uniform(-50, 150, (200, 2))
    ok = bt.OrdinaryKriging(vg, bt.Search.passes(bt.Search(radius=10, min_samples=3))).fit(xy, z)
    d = ok.predict(grid, diagnostics=True)
    assert {1.0, 2.0} <= set(np.asarray(d["pass"]).tolist())
    by_hand = bt.OrdinaryKriging(vg, [bt.Search(radius=r, min_samples=3) for r in (10, 20, 30)]).fit(xy, z)
    np.testing.assert_array_equal(ok.predict(grid), by_hand.predict(grid))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_with_search_keeps_the_samples(precision):
    """with_search (crates/py/src/estimation.rs:1742-1756): the same passes give the same predictions and
    k-fold estimates; another search gives others; the estimator's type, holes and error variances stay."""
    xy, z, vg, s = scattered()
    passes = [s, bt.Search(radius=200, max_samples=4)]
    holes = np.arange(len(z)) // 5
    ok = bt.OrdinaryKriging(vg, passes, precision=precision).fit(xy, z, holes=holes)
    targets = np.random.default_rng(13).uniform(-50, 150, (300, 2))
    same = ok.with_search(passes)
    assert type(same) is bt.OrdinaryKriging and same.precision == precision
    np.testing.assert_array_equal(same.predict(targets), ok.predict(targets))
    np.testing.assert_array_equal(same.cross_validate(folds=5).estimate, ok.cross_validate(folds=5).estimate)
    other = ok.with_search(bt.Search(radius=50, max_samples=4)).predict(targets)
    assert not np.array_equal(other, ok.predict(targets), equal_nan=True)
    np.testing.assert_array_equal(ok.predict(targets), same.predict(targets))
    one = bt.Search(radius=500, max_samples=150, min_holes=30)
    d = ok.with_search(one).predict(targets[:20], diagnostics=True)
    assert (d["n_holes"] == 30).all()
    sk = bt.SimpleKriging(vg, s, mean=0.5, precision=precision).fit(xy, z, error_variance=np.full(len(z), 0.1))
    again = sk.with_search(s)
    assert type(again) is bt.SimpleKriging
    np.testing.assert_array_equal(again.predict(targets), sk.predict(targets))
    with pytest.raises(bt.InvalidInput):
        sk.with_search(bt.Search(radius=50, target_slope=0.9))


def test_block_model_in_the_plane():
    """BlockModel(origin=(5, 5), size=(10, 10), count=(20, 20)) (the reference's 2-D form, containers.rs:808-811:
    origin z 0, size z 1, one layer): 400 centroids at 10, 20, ..., 200 (origin is the corner), x fastest, on
    the z = 0.5 plane; estimated on the plane of the 2-D data."""
    b = bt.BlockModel(origin=(5.0, 5.0), size=(10, 10), count=(20, 20))
    c = np.asarray(b.coords)
    assert c.shape == (400, 3)
    np.testing.assert_array_equal(c[:, 0], np.tile(np.arange(20) * 10.0 + 10.0, 20))
    np.testing.assert_array_equal(c[:, 1], np.repeat(np.arange(20) * 10.0 + 10.0, 20))
    np.testing.assert_array_equal(c[:, 2], 0.5)
    xy, z, vg, s = scattered()
    ok = bt.OrdinaryKriging(vg, s).fit(xy, z)
    # A one-layer model's centroids take the elevation of 2-D data (crates/py/src/estimation.rs:960-992).
    np.testing.assert_array_equal(ok.predict(b), ok.predict(c[:, :2]))
    assert not np.array_equal(ok.predict(b), ok.predict(c), equal_nan=True)


def test_search_passes_fill_what_earlier_passes_left():
    """A target the tight pass leaves unestimated takes the wide pass's estimate, bit for bit
    (estimation.py:337-355 over the passes)."""
    xy, z, vg, _ = scattered()
    grid = np.column_stack([np.repeat(np.arange(0, 150, 5.0), 30), np.tile(np.arange(0, 150, 5.0), 30)])
    tight, wide = bt.Search(radius=10, min_samples=4), bt.Search(radius=80, min_samples=2)
    first = bt.OrdinaryKriging(vg, tight).fit(xy, z).predict(grid)
    second = bt.OrdinaryKriging(vg, wide).fit(xy, z).predict(grid)
    ok = bt.OrdinaryKriging(vg, [tight, wide]).fit(xy, z)
    d = ok.predict(grid, diagnostics=True)
    np.testing.assert_array_equal(d["pass"], np.where(np.isfinite(first), 1.0, np.where(np.isfinite(second), 2.0,
                                                                                          np.nan)))
    np.testing.assert_array_equal(d["value"], np.where(np.isfinite(first), first, second))
    assert {1.0, 2.0} <= set(np.asarray(d["pass"])[np.isfinite(d["pass"])].tolist())
    assert np.isfinite(ok.cross_validate().estimate).all()
    with pytest.raises(bt.InvalidInput):
        bt.OrdinaryKriging(vg, [])


def test_k_fold_keeps_holes_whole():
    """cross_validate(folds=4) with 5 samples a hole: each fold is the estimate of an estimator fitted
    without that fold's holes, bit for bit; five folds are worse than leave-one-out."""
    xy, z, vg, s = scattered()
    holes = np.arange(len(z)) // 5
    cv = bt.OrdinaryKriging(vg, s).fit(xy, z, holes=holes).cross_validate(folds=4)
    expected = np.empty(len(z))
    for fold in range(4):
        test = holes % 4 == fold
        expected[test] = bt.OrdinaryKriging(vg, s).fit(xy[~test], z[~test]).predict(xy[test])
    np.testing.assert_array_equal(cv.estimate, expected)
    ok = bt.OrdinaryKriging(vg, s).fit(xy, z)
    np.testing.assert_array_equal(ok.cross_validate(folds=len(z)).estimate, ok.cross_validate().estimate)
    five = ok.cross_validate(folds=5)
    assert np.isfinite(five.estimate).all() and five.rmse > ok.cross_validate().rmse


def test_a_shared_contact_location_keeps_each_domains_sample():
    """Two samples at one location in two domains: each domain keeps its own, so a target there takes the
    sample of its domain (hard boundaries; the reference's test of this uses an infinite soft distance)."""
    xy, z, vg, _ = scattered()
    zone = np.where(xy[:, 0] < 50, "MS", "SM")
    both = np.vstack([xy, [[50.0, 50.0], [50.0, 50.0]]])
    labels = np.r_[zone, ["SM", "MS"]]
    data = np.r_[z, 5.0, -5.0]
    ok = bt.OrdinaryKriging(vg, bt.Search(radius=30)).fit(both, data, domains=labels)
    at = ok.predict([[50.0, 50.0]] * 2, domains=["MS", "SM"])
    np.testing.assert_allclose(at, [-5.0, 5.0], atol=1e-8)
    near = ok.predict([[50.5, 50.0]] * 2, domains=["MS", "SM"], diagnostics=True)
    assert np.isfinite(near["value"]).all() and near["value"][0] < near["value"][1]
    assert np.isfinite(ok.cross_validate().estimate[-2:]).all()


def test_column_names_match_arrays():
    """fit(PointSet, "grade", holes="hole", domain_column="zone") and predict(BlockModel,
    domain_column="zone") give the estimates of the same arrays, bit for bit; a PointSet target at the
    data returns the data."""
    xy, z, vg, s = scattered()
    holes = np.arange(len(z)) // 3
    zone = np.where(xy[:, 0] < 50, 1, 2)
    samples = bt.PointSet(xy, {"grade": z, "hole": holes, "zone": zone})
    grid = bt.BlockModel(origin=(0, 0), size=(10, 10), count=(10, 10))
    blocks = grid.with_column("zone", np.where(np.asarray(grid.coords)[:, 0] < 50, 1, 2))
    ok = bt.OrdinaryKriging(vg, s)
    arrays = ok.fit(xy, z, holes=holes, domains=zone).predict(grid, domains=blocks["zone"])
    names = ok.fit(samples, "grade", holes="hole", domain_column="zone").predict(blocks, domain_column="zone")
    np.testing.assert_array_equal(names, arrays)
    assert np.isfinite(arrays).all()
    plain = bt.OrdinaryKriging(vg, s).fit(samples, "grade")
    est = plain.predict(grid)
    assert est.shape == (100,)
    np.testing.assert_array_equal(grid.with_column("ok", est)["ok"], est)
    np.testing.assert_allclose(plain.predict(bt.PointSet(xy[:3])), z[:3], atol=1e-8)
    d = plain.predict(bt.PointSet(xy[:3]), diagnostics=True)
    np.testing.assert_allclose(d["slope"], 1.0)


def test_simple_kriging_needs_a_sill_and_ordinary_takes_the_power_model():
    xy, z, _, _ = scattered()
    power = bt.Variogram([("power", 1.0, 1.5)])
    with pytest.raises(bt.InvalidInput, match="simple kriging needs a variogram with a sill"):
        bt.SimpleKriging(power, bt.Search(radius=1000), mean=1.0)
    assert np.isfinite(bt.OrdinaryKriging(power, bt.Search(radius=1000)).fit(xy, z).predict([[50.0, 50.0]])[0])


@pytest.mark.parametrize("missing", [None, np.nan])
def test_missing_hole_ids_count_as_their_own_hole(missing):
    """Untagged samples (None or NaN hole ids) are holes of their own: a min_holes search gives the
    estimates of the estimator fitted without holes."""
    xy, z, vg, _ = scattered()
    holes = np.array([missing] * len(z), dtype=object)
    targets = xy[:3] + 1.0
    est = bt.OrdinaryKriging(vg, bt.Search(radius=200, max_samples=12, min_holes=2))
    out = est.fit(xy, z, holes=holes).predict(targets)
    np.testing.assert_array_equal(out, est.fit(xy, z).predict(targets))
    tagged = est.fit(xy, z, holes=np.r_[np.arange(len(z) - 1), np.nan]).predict(targets)
    np.testing.assert_array_equal(tagged, out)
