"""Block kriging (BlockKriging, btk_set_support) against the oracle's block_krige_points
(crates/estimation/src/block.rs:120-198 as crates/py/src/estimation.rs:775-784 runs it): estimates,
variances and Lagrange multipliers to 1e-10 (FP64) or 1e-6 (mixed) in the reference's convention, equal
status and n_used; C(B,B); and a one-point discretization is point kriging to the bit."""

import numpy as np
import pytest
from test_gpu_parity import assert_same_estimates

from boitata_b200 import BlockKriging, BlockModel, Geometry, OrdinaryKriging
from boitata_b200 import workloads as W

pytestmark = pytest.mark.gpu


def block_targets(oracle, g, step):
    return oracle.centroids(g.origin, g.size, g.count, g.rotation)[::step]


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-6)])
def test_block_kriging_matches_the_oracle_c1(oracle, precision, tol):
    w = W.c1()
    coords = np.vstack([w.coords, w.coords[:40] + [3e-7, 0.0, 0.0]])  # pairs inside the 1e-6 m guard
    values = np.concatenate([w.values, w.values[:40] * 1.5])
    size, disc = (20.0, 20.0, 10.0), (4, 4, 1)
    t = block_targets(oracle, w.geometry, 7)
    bk = BlockKriging(w.variogram, w.search, size, discretization=disc, precision=precision)
    bk.fit(coords, values)
    got = bk.predict_full(t)
    ref = oracle.estimate_block(t, coords, values, w.search, w.variogram, oracle.block_offsets(size, disc))
    assert_same_estimates(got, ref, tol)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-6)])
def test_block_kriging_of_a_rotated_block_model_c2(oracle, precision, tol):
    w = W.c2()
    g = Geometry((120.0, 80.0, 40.0), (5.0, 5.0, 6.25), (24, 20, 12), rotation=(30.0, 0.0, 0.0))
    size, disc = g.size, (3, 3, 2)
    bk = BlockKriging(w.variogram, w.search, size, discretization=disc, precision=precision)
    bk.fit(w.coords, w.values)
    got = bk.predict_full(g)
    cent = block_targets(oracle, g, 1)
    ref = oracle.estimate_block(cent, w.coords, w.values, w.search, w.variogram,
                                oracle.block_offsets(size, disc, g.rotation))
    assert_same_estimates(got, ref, tol)
    sv = bk.support_variance(g)
    st, one, _ = oracle.block_krige(cent[0], oracle.block_offsets(size, disc, g.rotation), w.coords[:3],
                                    w.values[:3], w.variogram)
    assert abs(sv - one["support"]) <= 1e-12 * (1 + abs(sv))


def test_one_point_block_is_point_kriging_to_the_bit():
    w = W.c2()
    g = Geometry((100.0, 100.0, 60.0), (2.5, 2.5, 3.125), (30, 30, 10))
    ok = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    bk = BlockKriging(w.variogram, w.search, g.size, discretization=(1, 1, 1)).fit(w.coords, w.values)
    a, b = ok.predict_full(g), bk.predict_full(BlockModel(g))
    for k in ("value", "variance", "lagrange", "n_used", "status"):
        np.testing.assert_array_equal(a[k], b[k])
    assert bk.support_variance() == w.variogram.total_sill()


def test_point_predictions_after_a_block_run_are_point_support():
    w = W.c1()
    t = np.array([[500.0, 500.0, 100.0], [123.0, 456.0, 78.0]])
    ok = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    before = ok.predict_full(t)
    bk = BlockKriging(w.variogram, w.search, (20.0, 20.0, 10.0)).fit(w.coords, w.values)
    bk.predict_full(t)
    cv = bk.cross_validate()  # point support, as the reference's cross-validation runs
    cv_ok = ok.cross_validate()
    np.testing.assert_array_equal(np.asarray(cv.estimate), np.asarray(cv_ok.estimate))
    after = ok.predict_full(t)
    np.testing.assert_array_equal(after["value"], before["value"])
