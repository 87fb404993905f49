"""Parity of the CUDA engine with the oracle (the reference path restated).

Neighbour lists must be identical, index for index and in order; estimates
and variances agree to 1e-10 (FP64 form) or 1e-6 (mixed form) in the
reference's convention |a - b| <= tol (1 + max(|a|, |b|)); the NaN pattern
and the per-target status must be equal.
"""

import numpy as np
import pytest
from conftest import close

from boitata_b200 import (BlockModel, Geometry, IndicatorKriging, OrdinaryKriging, Search, SimpleKriging, Structure,
                          Variogram)
from boitata_b200 import workloads as W

pytestmark = pytest.mark.gpu

ST = {0: 0, 1: 1, 2: 2}  # oracle status -> engine status (ok, search failed, singular)


def assert_same_neighbors(ok, oracle, coords, search, vg, targets):
    idx, cnt, good = ok.neighbors(targets)
    tree = oracle.Tree(coords, search, vg)
    for t, target in enumerate(targets):
        want_ok, want = tree.neighbors(target)
        got = idx[t, : cnt[t]].tolist()
        assert got == want, f"target {t} at {target}: {got} != {want}"
        assert bool(good[t]) == want_ok


def assert_same_estimates(got, ref, tol):
    fin = np.isfinite(ref["value"])
    assert np.array_equal(fin, np.isfinite(got["value"]))
    st = got["status"] & 0x0F
    assert np.array_equal(st, np.vectorize(ST.get)(ref["status"]).astype(np.int8))
    assert np.all(close(got["value"][fin], ref["value"][fin], tol)), np.max(
        np.abs(got["value"][fin] - ref["value"][fin]))
    assert np.all(close(got["variance"][fin], ref["variance"][fin], tol))
    assert np.all(close(got["lagrange"][fin], ref["lagrange"][fin], tol))
    assert np.array_equal(got["n_used"][fin], ref["n_used"][fin])


def centroids(oracle, w, step=1):
    g = w.geometry
    return oracle.centroids(g.origin, g.size, g.count, g.rotation)[::step]


def test_search_matches_oracle_c1(oracle):
    w = W.c1()
    rng = np.random.default_rng(11)
    targets = np.vstack([centroids(oracle, w, 13), rng.uniform(-200, 1200, (500, 3)) * [1, 1, 0.2]])
    ok = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    assert_same_neighbors(ok, oracle, w.coords, w.search, w.variogram, targets)


def test_search_matches_oracle_c2_octant(oracle):
    w = W.c2()
    rng = np.random.default_rng(12)
    cent = centroids(oracle, w)
    targets = np.vstack([cent[rng.choice(len(cent), 3000, replace=False)], [[-50.0, -50.0, 300.0], [250, 250, 125]]])
    ok = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    assert_same_neighbors(ok, oracle, w.coords, w.search, w.variogram, targets)


@pytest.mark.parametrize("octant", [False, True])
def test_search_ties_far_from_the_origin(oracle, octant):
    # search.rs:1272-1333: a lattice at UTM-sized coordinates with exact ties.
    x0, y0, z0 = 612_345.0, 7_654_321.0, 850.0
    i = np.arange(9 * 9 * 12)
    coords = np.column_stack([x0 + (i % 9) * 10.0, y0 + (i // 9 % 9) * 10.0, z0 - (i // 81) * 2.5])
    k = np.arange(80)
    targets = np.column_stack([x0 + (k % 9) * 5.0, y0 + (k // 9) * 10.0, z0 - (k % 5) * 5.0])
    vg = Variogram([Structure("spherical", 1.0, 100.0)])
    for rot in [None, (0.0, 0.0), (90.0, 0.0), (45.0, 30.0)]:
        for radius in [10.0, 20.0, 25.0, 40.0]:
            kw = {} if rot is None else dict(rotation=(rot[0], rot[1], 0.0), ratios=(0.5, 0.25))
            s = Search(radius=radius, max_samples=16, min_samples=1, octant=octant, **kw)
            ok = OrdinaryKriging(vg, s).fit(coords, np.zeros(len(coords)))
            assert_same_neighbors(ok, oracle, coords, s, vg, targets)


def test_planar_data_search_quadrants(oracle):
    # search.rs:1440-1456: 2D data balance quadrants.
    i = np.arange(400)
    coords = np.column_stack([(i % 20) * 1.0, (i // 20) * 1.0])
    vg = Variogram([Structure("spherical", 1.0, 50.0)])
    rng = np.random.default_rng(5)
    targets = np.column_stack([rng.uniform(-3, 23, 300), rng.uniform(-3, 23, 300), np.zeros(300)])
    for kw in [{}, dict(rotation=(35.0, 0.0, 0.0), ratios=(0.5, 0.5))]:
        s = Search(radius=100.0, max_samples=24, octant=True, **kw)
        ok = OrdinaryKriging(vg, s).fit(coords, np.zeros(400))
        assert_same_neighbors(ok, oracle, np.column_stack([coords, np.zeros(400)]), s, vg, targets)


def test_leave_one_out_search_matches_oracle(oracle):
    w = W.c1()
    ok = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    idx, cnt, good = ok.neighbors(None, loo=True)
    tree = oracle.Tree(w.coords, w.search, w.variogram)
    for i in range(len(w.coords)):
        want_ok, want = tree.neighbors(w.coords[i], left_out=i)
        assert idx[i, : cnt[i]].tolist() == want


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-6)])
def test_predict_c1_block_model(oracle, precision, tol):
    w = W.c1()
    targets = centroids(oracle, w)
    ok = OrdinaryKriging(w.variogram, w.search, precision=precision).fit(w.coords, w.values)
    got = ok.predict_full(targets)
    ref = oracle.estimate_many(targets, w.coords, w.values, w.search, w.variogram, neighbors=False)
    assert_same_estimates(got, ref, tol)
    on_device = ok.predict_full(w.geometry)
    for k in ("value", "variance", "lagrange"):
        np.testing.assert_array_equal(on_device[k], got[k])


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-6)])
def test_predict_c2_octant_subset(oracle, precision, tol):
    w = W.c2()
    rng = np.random.default_rng(3)
    cent = centroids(oracle, w)
    targets = cent[rng.choice(len(cent), 20000, replace=False)]
    ok = OrdinaryKriging(w.variogram, w.search, precision=precision).fit(w.coords, w.values)
    got = ok.predict_full(targets)
    ref = oracle.estimate_many(targets, w.coords, w.values, w.search, w.variogram, neighbors=False)
    assert_same_estimates(got, ref, tol)


def test_predict_c2_model_200k_blocks(oracle):
    """Both forms over 200,000 blocks of the 3.2M-block c2 model (every 16th cell, the whole model's
    geometry on the device) against the oracle: FP64 at 1e-10, mixed at 1e-6, per result."""
    w = W.c2()
    cells = np.arange(0, w.geometry.cells(), 16)
    targets = centroids(oracle, w)[cells]
    ref = oracle.estimate_many(targets, w.coords, w.values, w.search, w.variogram, neighbors=False)
    est = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    for precision, tol in (("fp64", 1e-10), ("mixed", 1e-6)):
        got = est.predict_full(w.geometry, precision=precision)
        assert_same_estimates({k: v[cells] for k, v in got.items()}, ref, tol)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-6)])
def test_predict_up_to_64_samples(oracle, precision, tol):
    w = W.c3()
    targets = centroids(oracle, w, 7)
    ok = OrdinaryKriging(w.variogram, w.search, precision=precision).fit(w.coords, w.values)
    got = ok.predict_full(targets)
    ref = oracle.estimate_many(targets, w.coords, w.values, w.search, w.variogram, neighbors=False)
    assert_same_estimates(got, ref, tol)
    assert np.max(got["n_used"]) == 64 and np.min(got["n_used"][got["status"] == 0]) < 33


@pytest.mark.parametrize("kind", ["simple", "indicator"])
def test_simple_and_indicator_kriging(oracle, kind):
    w = W.c1()
    targets = centroids(oracle, w, 11)
    est = (SimpleKriging(w.variogram, w.search, mean=1.2) if kind == "simple"
           else IndicatorKriging(w.variogram, w.search, 1.5)).fit(w.coords, w.values)
    got = est.predict_full(targets)
    ref = oracle.estimate_many(targets, w.coords, w.values, w.search, w.variogram, kind=kind,
                               kparam=1.2 if kind == "simple" else 1.5, neighbors=False)
    assert_same_estimates(got, ref, 1e-10)


def test_cross_validation_matches_oracle(oracle):
    w = W.c1()
    for precision, tol in [("fp64", 1e-10), ("mixed", 1e-6)]:
        cv = OrdinaryKriging(w.variogram, w.search, precision=precision).fit(w.coords, w.values).cross_validate()
        ref = oracle.estimate_many(None, w.coords, w.values, w.search, w.variogram, loo=True, neighbors=False)
        fin = np.isfinite(ref["value"])
        assert np.array_equal(fin, np.isfinite(cv.estimate))
        assert np.all(close(cv.estimate[fin], ref["value"][fin], tol))
        assert np.all(close(cv.variance[fin], ref["variance"][fin], tol))


def pair_and_lattice(n, gap):
    """coincident.rs:127-141: a near-coincident pair at (10, 10) then lattice samples."""
    s = [(10.0, 10.0, 1.0), (10.0 + gap, 10.0, 5.0)]
    k = 0
    while len(s) < n:
        x, y = (k % 9) * 7.0 - 20.0, (k // 9) * 7.0 - 20.0
        if abs(x - 10.0) + abs(y - 10.0) > 1.0:
            s.append((x, y, 3.0 + np.sin(k * 0.3)))
        k += 1
    a = np.array(s)
    return a[:, :2], a[:, 2]


# Gaps up to 1e-6 m are merged by the coincident guard and agree to 1e-10.
# At 1e-5 m the pair stays two samples; with no nugget the system's
# condition number is about 1e7, so two FP64 evaluation orders agree only to
# about 1e-16 * 1e7: that case is held to 1e-7.
@pytest.mark.parametrize("gap,tol", [(1e-12, 1e-10), (1e-7, 1e-10), (1e-6, 1e-10), (1e-5, 1e-7)])
def test_coincident_samples_krige_as_one(oracle, gap, tol):
    vg = Variogram([Structure("spherical", 1.0, 50.0)])
    xy, z = pair_and_lattice(60, gap)
    t = np.array([[12.0, 11.0], [10.0, 10.0], [-5.0, 3.0], [30.0, 30.0]])
    for kind, kp in [("ordinary", 0.0), ("simple", 3.0), ("indicator", 2.0)]:
        s = Search(radius=1000.0, max_samples=60)
        est = {"ordinary": lambda: OrdinaryKriging(vg, s), "simple": lambda: SimpleKriging(vg, s, mean=3.0),
               "indicator": lambda: IndicatorKriging(vg, s, 2.0)}[kind]().fit(xy, z)
        got = est.predict_full(t)
        xyz = np.column_stack([xy, np.zeros(len(xy))])
        ref = oracle.estimate_many(np.column_stack([t, np.zeros(4)]), xyz, z, s, vg, kind=kind, kparam=kp,
                                   neighbors=False)
        assert_same_estimates(got, ref, tol)


def test_singular_systems_are_flagged(oracle):
    vg = Variogram([Structure("gaussian", 1.0, 100.0)])
    rng = np.random.default_rng(1)
    base = rng.uniform(0, 100, (30, 3))
    coords = np.vstack([base, base[:10] + 1e-4])
    vals = rng.uniform(size=40)
    s = Search(radius=1000.0, max_samples=40)
    targets = rng.uniform(0, 100, (20, 3))
    got = OrdinaryKriging(vg, s).fit(coords, vals).predict_full(targets)
    ref = oracle.estimate_many(targets, coords, vals, s, vg, neighbors=False)
    assert np.array_equal(got["status"] & 0x0F, ref["status"].astype(np.int8))
    assert np.sum(got["status"] == 2) >= 5


def test_reference_python_properties():
    # python/tests/test_estimation.py:7-35
    rng = np.random.default_rng(3)
    coords = rng.uniform(0, 100, (150, 2))
    values = np.sin(coords[:, 0] / 15) + coords[:, 1] / 50
    model = Variogram([("spherical", 1.0, 40.0)], nugget=0.0)
    search = Search(radius=50, max_samples=16)
    est, var = OrdinaryKriging(model, search).fit(coords, values).predict(coords, return_variance=True)
    np.testing.assert_allclose(est, values, atol=1e-8)
    np.testing.assert_allclose(var, 0.0, atol=1e-8)
    ok = OrdinaryKriging(model, Search(radius=5, min_samples=3)).fit(coords, values)
    assert np.isnan(ok.predict([[500.0, 500.0]])[0])
    sk = SimpleKriging(model, Search(radius=1000), mean=7.0).fit(coords, values)
    assert sk.predict([[400.0, 400.0]])[0] == pytest.approx(7.0)
    near = coords[:1] + [0.5, 0.0]
    wide = OrdinaryKriging(model, Search(radius=400)).fit(coords, values)
    assert OrdinaryKriging(model, search).fit(coords, values).predict(near, return_variance=True)[1][0] < \
        wide.predict(np.array([[200.0, 200.0]]), return_variance=True)[1][0]


def test_geometry_centroids_are_the_reference_ones(oracle):
    g = Geometry((1000.0, 2000.0, 100.0), (5.0, 7.5, 2.5), (13, 9, 7), rotation=(30.0, 10.0, 5.0))
    ours = BlockModel(g).centroids()
    ref = oracle.centroids(g.origin, g.size, g.count, g.rotation)
    np.testing.assert_array_equal(ours, ref)


def test_passes_fill_what_earlier_passes_left(oracle):
    # python/tests/test_estimation.py search passes; batch.rs:132-147
    rng = np.random.default_rng(3)
    coords = rng.uniform(0, 100, (150, 2))
    values = np.sin(coords[:, 0] / 15) + coords[:, 1] / 50
    model = Variogram([("spherical", 1.0, 40.0)])
    grid = np.column_stack([np.repeat(np.arange(0, 150, 5.0), 30), np.tile(np.arange(0, 150, 5.0), 30)])
    tight, wide = Search(radius=10, min_samples=4), Search(radius=80, min_samples=2)
    first = OrdinaryKriging(model, tight).fit(coords, values).predict(grid)
    both = OrdinaryKriging(model, [tight, wide]).fit(coords, values).predict_full(grid)
    filled = np.isfinite(first)
    np.testing.assert_array_equal(both["value"][filled], first[filled])
    assert np.all(both["pass"][filled] == 1)
    later = ~filled & np.isfinite(both["value"])
    assert later.any() and np.all(both["pass"][later] == 2)
    second = OrdinaryKriging(model, wide).fit(coords, values).predict(grid)
    np.testing.assert_array_equal(both["value"][later], second[later])


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-6)])
def test_ordinary_and_simple_kriging_in_one_launch(oracle, precision, tol):
    # c3: uneven neighbour counts (4-64) with simple kriging (mean 1.0) on every 10th target.
    w = W.c3()
    targets = centroids(oracle, w, 3)
    kinds = np.where(np.arange(len(targets)) % 10 == 0, "simple", "ordinary")
    est = OrdinaryKriging(w.variogram, w.search, precision=precision).fit(w.coords, w.values)
    got = est.predict_kinds(targets, kinds, mean=1.0)
    for kind in ("ordinary", "simple"):
        sel = kinds == kind
        ref = oracle.estimate_many(targets[sel], w.coords, w.values, w.search, w.variogram, kind=kind, kparam=1.0,
                                   neighbors=False)
        assert_same_estimates({k: v[sel] for k, v in got.items()}, ref, tol)


def cond_tolerance(oracle, w, ref, targets, t, floor):
    """The tolerance of target t's FP64 estimate: max(floor, eps cond |w|_2 |z|_2 / (1 + |v|)). The GPU and the
    host evaluate the covariances with different exp implementations, whose results may differ in the last bit,
    and each side's solve is backward stable to about that size. For entrywise relative perturbations of at
    most eps of a covariance matrix C with nonnegative entries, |dC|_2 <= eps |C|_2, so the weights move by at
    most eps cond(C) |w|_2 to first order and the estimate v = w'z by eps cond |w|_2 |z|_2. Two c5 systems
    checked in extended precision: condition 6.1e5, the oracle 6.2e-10 from the exact solve and the GPU 1e-11
    (bound 4.3e-9); condition 3.2e5 with v = -0.05, the GPU 1.6e-9 and the oracle 1e-10 from it (bound
    5.9e-8; one-ulp random perturbations of its entries moved v by up to 1.0e-9)."""
    nb = [i for i in ref["neighbors"][t] if i >= 0]
    d = np.sqrt(((w.coords[nb][:, None] - w.coords[nb][None]) ** 2).sum(-1))
    cov = np.where(d > 0, np.exp(-3 * (d / 200.0) ** 2), 1.0 + 1e-4)
    _, _, wt = oracle.krige("ordinary", targets[t], w.coords[nb], w.values[nb], w.variogram)
    size = np.linalg.norm(wt) * np.linalg.norm(w.values[nb])
    return max(floor, np.finfo(float).eps * np.linalg.cond(cov) * size / (1.0 + abs(ref["value"][t])))


@pytest.mark.parametrize("holes,blocks", [(160, 2000), (1600, 20000)])
def test_ill_conditioned_systems(oracle, holes, blocks):
    # c5: clustered holes, 10 % of samples copied 0.01 m away, Gaussian model with a 1e-4 nugget, 64
    # neighbours; at 160 holes (20,000 samples) and at its full 1,600 holes (220,000 samples), with 20,000
    # blocks of the 10.24M-block model. Condition numbers reach ~5e5: each FP64 estimate is held to 1e-10, or
    # where the last bits of its covariances could move it further, to cond_tolerance; variances to 1e-10.
    # The mixed form refines these systems iteratively from their FP32 factors: fewer than 5 % may fall back
    # to FP64, and every result is held to 1e-6 against the oracle.
    w = W.c5(holes=holes)
    rng = np.random.default_rng(0)
    cells = np.sort(rng.choice(w.geometry.cells(), blocks, replace=False))
    targets = oracle.centroids(w.geometry.origin, w.geometry.size, w.geometry.count, w.geometry.rotation)[cells]
    ref = oracle.estimate_many(targets, w.coords, w.values, w.search, w.variogram)
    fp64 = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    assert_same_neighbors(fp64, oracle, w.coords, w.search, w.variogram, targets[:300])
    got = fp64.predict_full(targets)
    fin = np.isfinite(ref["value"])
    assert np.array_equal(fin, np.isfinite(got["value"])) and np.array_equal(got["status"], ref["status"])
    for t in np.nonzero(fin & ~close(got["value"], ref["value"], 1e-10))[0]:
        assert close(got["value"][t], ref["value"][t], cond_tolerance(oracle, w, ref, targets, t, 1e-10)), t
    assert np.all(close(got["variance"][fin], ref["variance"][fin], 1e-10))
    mixed = OrdinaryKriging(w.variogram, w.search, precision="mixed").fit(w.coords, w.values).predict_full(targets)
    assert np.array_equal(fin, np.isfinite(mixed["value"]))
    assert np.array_equal(mixed["status"] & 0x0F, ref["status"].astype(np.int8))
    fallback = np.mean((mixed["status"][fin] & 0x10) != 0)
    assert fallback < 0.05, f"{fallback:.1%} of the systems fell back to FP64"
    for k in ("value", "variance", "lagrange"):
        assert np.all(close(mixed[k][fin], ref[k][fin], 1e-6)), k
    np.testing.assert_array_equal(mixed["n_used"][fin], ref["n_used"][fin])



def test_octants_of_samples_on_the_sector_planes(oracle):
    """Samples within a few ulps of the three octant planes through each target, under rotated searches at
    UTM-sized coordinates: the kernel's fast sector test (axes w - axes t against a rounding bound) must
    hand every such sample to the reference-order evaluation, so the lists equal the oracle's."""
    rng = np.random.default_rng(21)
    x0, y0, z0 = 512_345.25, 6_954_321.5, 1_150.0
    targets = np.column_stack([x0 + rng.uniform(0, 200, 40), y0 + rng.uniform(0, 200, 40),
                               z0 + rng.uniform(-50, 50, 40)])
    vg = Variogram([Structure("spherical", 1.0, 100.0)])
    for rot in [(30.0, 10.0, 0.0), (0.0, 0.0, 0.0), (-65.0, 45.0, 20.0)]:
        axes = oracle.block_frame(*rot)  # rows: the octant frame
        pts = []
        for t in targets:
            for r in range(3):
                u, v = axes[(r + 1) % 3], axes[(r + 2) % 3]
                for _ in range(12):
                    w = t + rng.uniform(-40, 40) * u + rng.uniform(-40, 40) * v
                    w = w + axes[r] * rng.choice([0.0, 1e-13, -1e-13, 1e-11, -1e-11, 1e-9])
                    for _ in range(int(rng.integers(0, 3))):
                        a = int(rng.integers(0, 3))
                        w[a] = np.nextafter(w[a], np.inf if rng.random() < 0.5 else -np.inf)
                    pts.append(w)
        coords = np.array(pts)
        s = Search(radius=60.0, max_samples=24, min_samples=1, octant=True, max_per_sector=3, rotation=rot,
                   ratios=(0.8, 0.5))
        ok = OrdinaryKriging(vg, s).fit(coords, np.zeros(len(coords)))
        assert_same_neighbors(ok, oracle, coords, s, vg, targets)
