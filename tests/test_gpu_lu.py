"""The dense LU path (crates/estimation/src/krige.rs:127-201, krige_lu) against the oracle: systems of more than
64 samples, and variograms with a power structure (not stationary, kernel.rs:31), whose bordered matrix is
not positive definite. Neighbour lists identical; estimates, variances and Lagrange multipliers to 1e-10
(FP64) or 1e-6 (mixed, whose n > 64 systems are solved in FP64) in the reference's convention; equal status
and n_used."""

import numpy as np
import pytest
from test_gpu_parity import assert_same_estimates, assert_same_neighbors, centroids

from boitata_b200 import BlockKriging, IndicatorKriging, OrdinaryKriging, Search, SimpleKriging, Structure, Variogram
from boitata_b200 import workloads as W
from boitata_b200.errors import InvalidInput

pytestmark = pytest.mark.gpu

ST = {0: 0, 1: 1, 2: 2, 4: 4}  # oracle status -> engine status (ok, search failed, singular, invalid)


def power_variogram():
    return Variogram([Structure("power", 0.02, 100.0, exponent=1.5)], nugget=0.1, ratios=(1.0, 1.0 / 3.0))


def power_nested():
    return Variogram([Structure("spherical", 0.5, 120.0), Structure("power", 0.3, 400.0, exponent=0.8)],
                     nugget=0.05, rotation=(30.0, 10.0, 0.0), ratios=(0.75, 0.5))


def with_pairs(w, k=40):
    """c1's samples plus k copies 3e-7 m away (inside the 1e-6 m coincidence guard, coincident.rs:11-15)."""
    coords = np.vstack([w.coords, w.coords[:k] + [3e-7, 0.0, 0.0]])
    values = np.concatenate([w.values, w.values[:k] * 1.5])
    return coords, values


@pytest.mark.parametrize("max_samples", [65, 96, 128])
def test_search_beyond_64_matches_the_oracle(oracle, max_samples):
    w = W.c1()
    s = Search(ranges=(300.0, 300.0, 100.0), max_samples=max_samples, min_samples=1)
    rng = np.random.default_rng(max_samples)
    targets = np.vstack([centroids(oracle, w, 29), rng.uniform(-200, 1200, (300, 3)) * [1, 1, 0.2]])
    ok = OrdinaryKriging(w.variogram, s).fit(w.coords, w.values)
    assert_same_neighbors(ok, oracle, w.coords, s, w.variogram, targets)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-6)])
@pytest.mark.parametrize("max_samples", [96, 128])
def test_more_than_64_samples_match_krige_lu(oracle, precision, tol, max_samples):
    w = W.c1()
    coords, values = with_pairs(w)
    s = Search(ranges=(300.0, 300.0, 100.0), max_samples=max_samples, min_samples=1)
    rng = np.random.default_rng(7)
    targets = np.vstack([centroids(oracle, w, 11), rng.uniform(-200, 1200, (300, 3)) * [1, 1, 0.2]])
    ok = OrdinaryKriging(w.variogram, s, precision=precision).fit(coords, values)
    got = ok.predict_full(targets)
    ref = oracle.estimate_many(targets, coords, values, s, w.variogram, neighbors=False)
    assert np.count_nonzero(ref["n_used"] > 64) > len(targets) // 2  # most systems take the LU
    assert np.count_nonzero((ref["n_used"] > 32) & (ref["n_used"] <= 64)) > 0  # and the warp kernels the rest
    assert_same_estimates(got, ref, tol)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-6)])
def test_simple_and_indicator_kriging_beyond_64(oracle, precision, tol):
    w = W.c1()
    s = Search(ranges=(300.0, 300.0, 100.0), max_samples=100, min_samples=1)
    targets = centroids(oracle, w, 17)
    sk = SimpleKriging(w.variogram, s, mean=1.0, precision=precision).fit(w.coords, w.values)
    ref = oracle.estimate_many(targets, w.coords, w.values, s, w.variogram, kind="simple", kparam=1.0,
                               neighbors=False)
    assert_same_estimates(sk.predict_full(targets), ref, tol)
    ik = IndicatorKriging(w.variogram, s, 1.2, precision=precision).fit(w.coords, w.values)
    ref = oracle.estimate_many(targets, w.coords, w.values, s, w.variogram, kind="indicator", kparam=1.2,
                               neighbors=False)
    assert_same_estimates(ik.predict_full(targets), ref, tol)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("vg", [power_variogram, power_nested])
def test_power_model_matches_krige_lu(oracle, precision, vg):
    w = W.c1()
    v = vg()
    coords, values = with_pairs(w)
    s = Search(ranges=(300.0, 300.0, 100.0), max_samples=48, min_samples=1)
    rng = np.random.default_rng(3)
    targets = np.vstack([centroids(oracle, w, 13), rng.uniform(-200, 1200, (300, 3)) * [1, 1, 0.2]])
    ok = OrdinaryKriging(v, s, precision=precision).fit(coords, values)
    ref = oracle.estimate_many(targets, coords, values, s, v, neighbors=False)
    assert_same_estimates(ok.predict_full(targets), ref, 1e-10)  # the power path is FP64 in both forms
    ik = IndicatorKriging(v, s, 1.0, precision=precision).fit(coords, values)
    ref = oracle.estimate_many(targets, coords, values, s, v, kind="indicator", kparam=1.0, neighbors=False)
    assert_same_estimates(ik.predict_full(targets), ref, 1e-10)


def test_power_model_with_128_samples_and_cross_validation(oracle):
    w = W.c1()
    v = power_variogram()
    s = Search(ranges=(300.0, 300.0, 100.0), max_samples=128, min_samples=1)
    targets = centroids(oracle, w, 23)
    ok = OrdinaryKriging(v, s).fit(w.coords, w.values)
    ref = oracle.estimate_many(targets, w.coords, w.values, s, v, neighbors=False)
    assert_same_estimates(ok.predict_full(targets), ref, 1e-10)
    cv = OrdinaryKriging(v, w.search).fit(w.coords, w.values).cross_validate()
    ref = oracle.estimate_many(None, w.coords, w.values, w.search, v, loo=True, neighbors=False)
    fin = np.isfinite(ref["value"])
    assert np.array_equal(fin, np.isfinite(cv.estimate))
    tol = lambda a, b: np.abs(a - b) <= 1e-10 * (1 + np.maximum(np.abs(a), np.abs(b)))  # noqa: E731
    assert np.all(tol(cv.estimate[fin], ref["value"][fin]))
    assert np.all(tol(cv.variance[fin], ref["variance"][fin]))


def test_simple_kriging_with_a_power_structure_is_invalid(oracle):
    w = W.c1()
    v = power_variogram()
    with pytest.raises(InvalidInput):
        SimpleKriging(v, w.search, mean=1.0)
    # Per-target kinds reach the solve: check_simple (krige.rs:117-124) fails the simple-kriging targets.
    targets = centroids(oracle, w, 31)
    kinds = np.where(np.arange(len(targets)) % 4 == 0, "simple", "ordinary")
    got = OrdinaryKriging(v, w.search).fit(w.coords, w.values).predict_kinds(targets, kinds, mean=1.0)
    for kind in ("ordinary", "simple"):
        sel = kinds == kind
        ref = oracle.estimate_many(targets[sel], w.coords, w.values, w.search, v, kind=kind, kparam=1.0,
                                   neighbors=False)
        sub = {k: x[sel] for k, x in got.items()}
        assert np.array_equal(sub["status"] & 0x0F, np.vectorize(ST.get)(ref["status"]).astype(np.int8))
        if kind == "simple":
            assert np.all(ref["status"] == 4) and np.all(np.isnan(sub["value"]))
        else:
            assert_same_estimates(sub, ref, 1e-10)


@pytest.mark.parametrize("vg", [None, power_variogram])
def test_block_kriging_through_the_lu(oracle, vg):
    w = W.c1()
    v = w.variogram if vg is None else vg()
    s = Search(ranges=(300.0, 300.0, 100.0), max_samples=100 if vg is None else 40, min_samples=1)
    size, disc = (20.0, 20.0, 10.0), (3, 3, 2)
    t = centroids(oracle, w, 19)
    bk = BlockKriging(v, s, size, discretization=disc).fit(w.coords, w.values)
    ref = oracle.estimate_block(t, w.coords, w.values, s, v, oracle.block_offsets(size, disc))
    assert_same_estimates(bk.predict_full(t), ref, 1e-10)


@pytest.mark.parametrize("max_samples", [129, 200, 400])
def test_systems_beyond_128_samples_match_krige_lu(oracle, max_samples):
    """Beyond 128 samples the LU's matrix lives in global memory (krige_lu has no upper limit): lists, and
    OK / SK estimates with coincident pairs, against the oracle; FP64 in both precisions."""
    w = W.c1()
    coords, values = with_pairs(w)
    s = Search(ranges=(400.0, 400.0, 150.0), max_samples=max_samples, min_samples=1, max_per_hole=60)
    holes = np.arange(len(coords)) // 7
    rng = np.random.default_rng(max_samples)
    targets = np.vstack([centroids(oracle, w, 97), rng.uniform(-200, 1200, (60, 3)) * [1, 1, 0.2]])
    ok = OrdinaryKriging(w.variogram, s, precision="mixed").fit(coords, values, holes=holes)
    idx, cnt, good = ok.neighbors(targets)
    ref = oracle.estimate_many(targets, coords, values, s, w.variogram, holes=ok._holes)
    for t in range(len(targets)):
        assert idx[t, : cnt[t]].tolist() == [i for i in ref["neighbors"][t] if i >= 0], t
    assert np.count_nonzero(ref["n_used"] > 128) > len(targets) // 2
    assert_same_estimates(ok.predict_full(targets), ref, 1e-10)
    sk = SimpleKriging(w.variogram, s, mean=1.0).fit(coords, values, holes=holes)
    ref = oracle.estimate_many(targets, coords, values, s, w.variogram, holes=ok._holes, kind="simple", kparam=1.0,
                               neighbors=False)
    assert_same_estimates(sk.predict_full(targets), ref, 1e-10)


def test_more_than_1024_samples_is_refused():
    w = W.c1()
    s = Search(ranges=(300.0, 300.0, 100.0), max_samples=1025, min_samples=1)
    with pytest.raises(Exception, match="1024"):
        OrdinaryKriging(w.variogram, s).fit(w.coords, w.values).predict_full(w.coords[:4])
