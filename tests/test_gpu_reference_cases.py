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
