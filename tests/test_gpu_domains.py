"""Hard domains and k-fold cross-validation on the GPU against the oracle.

Hard domains (crates/estimation/src/search.rs:269-288, batch.rs:15-38): a
target takes only its own domain's samples; neighbour lists are the
oracle's index for index, and estimates agree to 1e-10 (FP64) or 1e-6
(mixed). k-fold (batch.rs:197-243): each sample kriged from a fit of the
samples outside its fold, holes kept whole, each in its own domain.
"""

import numpy as np
import pytest
from test_gpu_parity import assert_same_estimates
from test_oracle_pins import batch_grid, batch_samples, batch_search, domain_of, spherical_40

from boitata_b200 import OrdinaryKriging, SimpleKriging
from boitata_b200 import workloads as W
from boitata_b200.errors import InvalidInput

pytestmark = pytest.mark.gpu

LABELS = ["oxide", "transition", "fresh"]


def zoned_c1():
    """c1's samples and block centroids in three domains split by x (labels as strings)."""
    from oracle import oracle

    w = W.c1()
    g = w.geometry
    cent = oracle.centroids(g.origin, g.size, g.count, g.rotation)[::3]
    zone = lambda p: np.digitize(p[:, 0] + 0.2 * p[:, 1], [400.0, 800.0])  # noqa: E731
    return w, cent, zone(w.coords), zone(cent)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-6)])
def test_hard_domains_match_the_oracle(oracle, precision, tol):
    w, cent, sdom, tdom = zoned_c1()
    labels = [LABELS[d] for d in sdom]
    est = OrdinaryKriging(w.variogram, w.search, precision=precision).fit(w.coords, w.values, domains=labels)
    tl = [LABELS[d] for d in tdom]
    idx, cnt, good = est.neighbors(cent[:2000], domains=tl[:2000])
    lists = oracle.estimate_many(cent[:2000], w.coords, w.values, w.search, w.variogram, domains=sdom,
                                 target_domains=tdom[:2000])["neighbors"]
    for t in range(2000):
        want = [i for i in lists[t] if i >= 0]
        assert idx[t, : cnt[t]].tolist() == want, t
        assert all(sdom[i] == tdom[t] for i in want)
    got = est.predict_full(cent, domains=tl)
    ref = oracle.estimate_many(cent, w.coords, w.values, w.search, w.variogram, domains=sdom, target_domains=tdom,
                               neighbors=False)
    assert_same_estimates(got, ref, tol)
    cv = est.cross_validate()
    ref_cv = oracle.estimate_many(None, w.coords, w.values, w.search, w.variogram, loo=True, domains=sdom,
                                  neighbors=False)
    fin = np.isfinite(ref_cv["value"])
    assert np.array_equal(fin, np.isfinite(cv.estimate))
    scale = 1 + np.maximum(np.abs(cv.estimate[fin]), np.abs(ref_cv["value"][fin]))
    assert np.all(np.abs(cv.estimate[fin] - ref_cv["value"][fin]) <= tol * scale)


def test_domains_are_the_reference_calls():
    w, cent, sdom, tdom = zoned_c1()
    est = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values, domains=[LABELS[d] for d in sdom])
    with pytest.raises(InvalidInput, match="needs domains too"):
        est.predict(cent[:10])
    # One label for every target; a domain without samples leaves its targets unestimated.
    one = est.predict(cent[:50], domains="fresh")
    assert np.isfinite(one).any()
    assert np.all(np.isnan(est.predict(cent[:50], domains="unknown")))
    plain = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    with pytest.raises(InvalidInput, match="takes none"):
        plain.predict(cent[:10], domains="fresh")


def test_hard_domains_are_separate_estimations():
    # batch.rs:1047-1075 on the engine: each domain alone gives the same bits as the zoned estimator.
    xyz, v = batch_samples()
    targets = batch_grid()
    dom = np.array([domain_of(p) for p in xyz])
    tdom = np.array([domain_of(p) for p in targets])
    s, vg = batch_search(2, 30.0), spherical_40()
    est = OrdinaryKriging(vg, s).fit(xyz, v, domains=dom)
    hard = est.predict_full(targets, domains=tdom)
    hard_cv = est.cross_validate()
    for d in range(3):
        own, at = dom == d, tdom == d
        alone = OrdinaryKriging(vg, s).fit(xyz[own], v[own])
        np.testing.assert_array_equal(alone.predict_full(targets[at])["value"], hard["value"][at])
        np.testing.assert_array_equal(alone.cross_validate().estimate, hard_cv.estimate[own])


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-6)])
def test_k_fold_matches_the_oracle(oracle, precision, tol):
    """k-fold with holes kept whole, measurement errors and domains, k = 2, 5 and 13."""
    w = W.c2(holes=8)
    labels = [f"DH{i // 125:03d}" for i in range(len(w.coords))]
    rng = np.random.default_rng(4)
    err = rng.uniform(0.0, 0.05, len(w.coords))
    dom = (w.coords[:, 2] < 150.0).astype(int)
    est = OrdinaryKriging(w.variogram, w.search, precision=precision).fit(w.coords, w.values, holes=labels,
                                                                        error_variance=err, domains=dom)
    from boitata_b200.estimation import hole_codes

    codes = hole_codes(labels)
    for k in (2, 5, 13):
        got = est.cross_validate(folds=k)
        ref = oracle.k_fold(k, w.coords, w.values, w.search, w.variogram, err=err, holes=codes, domains=dom)
        fin = np.isfinite(ref["value"])
        assert np.array_equal(fin, np.isfinite(got.estimate)), k
        scale = 1 + np.maximum(np.abs(got.estimate[fin]), np.abs(ref["value"][fin]))
        assert np.all(np.abs(got.estimate[fin] - ref["value"][fin]) <= tol * scale), k
        scale = 1 + np.maximum(np.abs(got.variance[fin]), np.abs(ref["variance"][fin]))
        assert np.all(np.abs(got.variance[fin] - ref["variance"][fin]) <= tol * scale), k


def test_k_fold_with_one_sample_per_fold_is_leave_one_out():
    # batch.rs:349-372 on the engine.
    xyz, v = batch_samples()
    s, vg = batch_search(4, 30.0), spherical_40()
    est = SimpleKriging(vg, s, mean=0.5).fit(xyz, v)
    loo, folds = est.cross_validate(), est.cross_validate(folds=len(xyz))
    np.testing.assert_array_equal(loo.estimate, folds.estimate)
    np.testing.assert_array_equal(loo.variance, folds.variance)
    with pytest.raises(InvalidInput):
        est.cross_validate(folds=1)
