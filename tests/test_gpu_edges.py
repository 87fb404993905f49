"""Edge cases of the call surface against the oracle: no targets, one sample, a target beyond every sample,
cross-validation of two samples, a mix of 2-D and 3-D inputs, in both precisions."""

import numpy as np
import pytest
from conftest import close

import boitata_b200 as bt
from boitata_b200 import _native as N

pytestmark = pytest.mark.gpu

FORMS = [("fp64", 1e-10), ("mixed", 1e-6)]
VG = bt.Variogram([bt.Structure("spherical", 0.9, 150.0)], nugget=0.1)


@pytest.mark.parametrize("precision,tol", FORMS)
def test_no_targets(precision, tol):
    xy = np.random.default_rng(1).uniform(0, 100, (40, 3))
    ok = bt.OrdinaryKriging(VG, bt.Search(radius=80), precision=precision).fit(xy, xy[:, 0])
    for targets in (np.zeros((0, 3)), np.zeros((0, 2))):
        v, s = ok.predict(targets, return_variance=True)
        assert v.shape == s.shape == (0,)
        full = ok.predict_full(targets)
        assert all(len(full[k]) == 0 for k in ("value", "variance", "lagrange", "n_used", "status"))
        assert ok.predict(targets, diagnostics=True).num_rows == 0


@pytest.mark.parametrize("precision,tol", FORMS)
def test_one_sample_and_a_target_out_of_reach(oracle, precision, tol):
    xyz = np.array([[10.0, 20.0, 5.0]])
    s = bt.Search(radius=50.0, max_samples=8)
    ok = bt.OrdinaryKriging(VG, s, precision=precision).fit(xyz, [3.5])
    targets = np.array([[10.0, 20.0, 5.0], [30.0, 20.0, 5.0], [500.0, 500.0, 5.0]])
    got = ok.predict_full(targets)
    ref = oracle.estimate_many(targets, xyz, np.array([3.5]), s, VG)
    np.testing.assert_array_equal(np.isfinite(got["value"]), np.isfinite(ref["value"]))
    assert np.isfinite(got["value"][:2]).all() and np.isnan(got["value"][2])
    assert got["status"][2] == N.ST_SEARCH_FAILED
    fin = np.isfinite(ref["value"])
    assert np.all(close(got["value"][fin], ref["value"][fin], tol))
    assert np.all(close(got["variance"][fin], ref["variance"][fin], tol))
    assert got["value"][1] == pytest.approx(3.5)  # one sample: weight 1


@pytest.mark.parametrize("precision,tol", FORMS)
def test_cross_validation_of_two_samples(oracle, precision, tol):
    xyz = np.array([[0.0, 0.0, 0.0], [40.0, 0.0, 0.0]])
    vals = np.array([1.0, 2.0])
    s = bt.Search(radius=100.0, max_samples=4)
    cv = bt.OrdinaryKriging(VG, s, precision=precision).fit(xyz, vals).cross_validate()
    ref = oracle.estimate_many(xyz, xyz, vals, s, VG, loo=True)
    np.testing.assert_allclose(cv.estimate, [2.0, 1.0])
    assert np.all(close(cv.variance, ref["variance"], tol))


@pytest.mark.parametrize("precision,tol", FORMS)
def test_planar_inputs_are_the_3d_inputs_at_zero_elevation(precision, tol):
    rng = np.random.default_rng(4)
    xy = rng.uniform(0, 200, (300, 2))
    v = np.sin(xy[:, 0] / 30) + xy[:, 1] / 100
    t = rng.uniform(0, 200, (500, 2))
    s = bt.Search(radius=60.0, max_samples=12, octant=True)
    flat = bt.OrdinaryKriging(VG, s, precision=precision).fit(xy, v).predict_full(t)
    full = bt.OrdinaryKriging(VG, s, precision=precision).fit(np.column_stack([xy, np.zeros(300)]), v)
    three = full.predict_full(np.column_stack([t, np.zeros(500)]))
    for k in ("value", "variance", "n_used", "status"):
        np.testing.assert_array_equal(flat[k], three[k])
