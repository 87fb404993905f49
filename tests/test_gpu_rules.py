"""Searches with hole and sector rules (search.rs:476-577) on the GPU against the oracle's SearchTree:
neighbour lists identical index for index and in order, equal success flags, and the estimates and
leave-one-out estimates to 1e-10 (FP64 form)."""

import numpy as np
import pytest
from test_gpu_parity import assert_same_estimates

from boitata_b200 import OrdinaryKriging, Search
from boitata_b200 import workloads as W
from boitata_b200.estimation import hole_codes

pytestmark = pytest.mark.gpu


def drill_holes(holes=12):
    """c2's drill holes, cut to `holes` x `holes` collars; hole label per composite."""
    w = W.c2(holes=holes)
    labels = [f"DH{i // 125:03d}" for i in range(len(w.coords))]
    return w, labels


def assert_same_neighbors(est, oracle, coords, search, vg, targets, codes):
    idx, cnt, good = est.neighbors(targets)
    tree = oracle.Tree(coords, search, vg, codes)
    for t, target in enumerate(targets):
        want_ok, want = tree.neighbors(target)
        got = idx[t, : cnt[t]].tolist()
        assert got == want, f"target {t} at {target}: {got} != {want}"
        assert bool(good[t]) == want_ok, f"target {t}"


def targets_in(w, k, seed, lo=(0, 0, 0), hi=(300, 300, 250)):
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, (k, 3))


@pytest.mark.parametrize("search", [
    Search(radius=250.0, octant=True, max_per_sector=4, max_samples=32, max_per_hole=3),
    Search(radius=250.0, max_samples=24, max_per_hole=2),
    Search(radius=120.0, octant=True, max_per_sector=2, max_samples=24, min_sectors=6, max_empty_sectors=1,
           max_per_hole=2, min_holes=6),
    Search(radius=200.0, sectors=6, max_per_sector=3, max_samples=16, max_per_hole=4),
    Search(radius=90.0, sectors=12, max_per_sector=2, max_samples=20, min_sectors=9, max_empty_sectors=2,
           min_holes=4),
], ids=["octant+hole", "hole", "all-rules", "plane+hole", "plane-rules"])
def test_rule_searches_match_the_oracle(oracle, search):
    w, labels = drill_holes()
    codes = hole_codes(labels)
    t = targets_in(w, 400, 5)
    est = OrdinaryKriging(w.variogram, search).fit(w.coords, w.values, holes=labels)
    assert_same_neighbors(est, oracle, w.coords, search, w.variogram, t, codes)
    got = est.predict_full(t)
    ref = oracle.estimate_many(t, w.coords, w.values, search, w.variogram, holes=codes, neighbors=False)
    assert_same_estimates(got, ref, 1e-10)


def test_unlabelled_samples_count_as_their_own_holes(oracle):
    w, _ = drill_holes(8)
    s = Search(radius=150.0, octant=True, max_per_sector=3, max_samples=24, min_holes=20, max_per_hole=1)
    t = targets_in(w, 200, 6, hi=(200, 200, 250))
    est = OrdinaryKriging(w.variogram, s).fit(w.coords, w.values)
    assert_same_neighbors(est, oracle, w.coords, s, w.variogram, t, None)


def test_leave_one_out_with_hole_rules(oracle):
    w, labels = drill_holes(6)
    codes = hole_codes(labels)
    s = Search(radius=150.0, octant=True, max_per_sector=3, max_samples=16, max_per_hole=2, min_holes=3)
    est = OrdinaryKriging(w.variogram, s).fit(w.coords, w.values, holes=labels)
    cv = est.cross_validate()
    ref = oracle.estimate_many(None, w.coords, w.values, s, w.variogram, holes=codes, loo=True, neighbors=False)
    fin = np.isfinite(ref["value"])
    assert np.array_equal(fin, np.isfinite(np.asarray(cv.estimate)))
    a, b = np.asarray(cv.estimate)[fin], ref["value"][fin]
    assert np.all(np.abs(a - b) <= 1e-10 * (1 + np.maximum(np.abs(a), np.abs(b))))


def test_quadrants_with_a_hole_cap_on_planar_data(oracle):
    rng = np.random.default_rng(9)
    xyz = np.column_stack([rng.uniform(0, 500, 3000), rng.uniform(0, 500, 3000), np.full(3000, 10.0)])
    vals = rng.lognormal(size=3000)
    labels = [f"L{i % 400}" for i in range(3000)]
    w = W.c1()
    s = Search(radius=200.0, octant=True, max_per_sector=3, max_samples=12, max_per_hole=1, max_empty_sectors=1)
    est = OrdinaryKriging(w.variogram, s).fit(xyz, vals, holes=labels)
    t = np.column_stack([rng.uniform(0, 500, 300), rng.uniform(0, 500, 300), np.full(300, 10.0)])
    assert_same_neighbors(est, oracle, xyz, s, w.variogram, t, hole_codes(labels))


def boundary_clusters(P, axes, rng, targets=40):
    """Per target (1 km apart, so no search sees another's samples): for each boundary of P plane sectors, two
    samples within a few ulps of it in the search frame (near, 10-20 m), and one inside each sector (50-60 m).
    Samples whose offset's host-libm atan2 is not correctly rounded are left out: at those the reference's
    sector depends on its platform's libm (tests/test_sector_angles.py), and the oracle shares this host's."""
    from test_sector_angles import libm_misrounds

    M = np.asarray(axes)
    T = np.column_stack([1000.0 * np.arange(targets), np.zeros(targets), np.full(targets, 100.0)])
    pts = []
    for t in T:
        for k in range(P):
            for r, th in ((rng.uniform(10, 20), 2 * np.pi * k / P), (rng.uniform(10, 20), 2 * np.pi * k / P),
                          (rng.uniform(50, 60), 2 * np.pi * (k + 0.5) / P)):
                d = np.array([-r * np.sin(th), r * np.cos(th), rng.uniform(-3, 3)])
                d[0] = np.nextafter(d[0], np.inf if rng.random() < 0.5 else -np.inf)
                s = t + M.T @ d
                v = s - t
                # the search frame's offset as the reference computes it (nalgebra column order, no FMA)
                dd = [(M[r_, 0] * v[0] + M[r_, 1] * v[1]) + M[r_, 2] * v[2] for r_ in range(3)]
                if dd[0] != 0.0 and dd[1] != 0.0 and libm_misrounds(-dd[0], dd[1]):
                    continue
                pts.append(s)
    return T, np.array(pts)


@pytest.mark.parametrize("P", [4, 6, 12])
@pytest.mark.parametrize("rotation", [None, (30.0, 20.0, 10.0)])
def test_plane_sectors_at_their_boundaries(oracle, P, rotation):
    """Samples within a few ulps of every plane-sector boundary (search.rs:428-434), one per sector taken:
    the lists are the oracle's index for index."""
    from boitata_b200 import Structure, Variogram

    rng = np.random.default_rng(P)
    kw = {} if rotation is None else dict(rotation=rotation, ratios=(1.0, 1.0))
    s = Search(radius=100.0, sectors=P, max_per_sector=1, max_samples=P, min_samples=1, **kw)
    axes = oracle.block_frame(*(rotation or (0.0, 0.0, 0.0)))
    T, X = boundary_clusters(P, axes, rng)
    vg = Variogram([Structure("spherical", 1.0, 200.0)], nugget=0.1)
    est = OrdinaryKriging(vg, s).fit(X, rng.uniform(0, 1, len(X)))
    assert_same_neighbors(est, oracle, X, s, vg, T, None)


@pytest.mark.parametrize("per_octant,most", [(16, 32), (40, 64)])
def test_octant_caps_beyond_a_lanes_heap(oracle, per_octant, most):
    """Octant caps whose eight lists exceed a search lane's 64 heap slots (16 or 40 a sector) run in the
    rules kernel: lists equal the oracle's tree, estimates to 1e-10."""
    w, _ = drill_holes()
    s = Search(radius=250.0, octant=True, max_per_sector=per_octant, max_samples=most)
    est = OrdinaryKriging(w.variogram, s).fit(w.coords, w.values)
    targets = targets_in(w, 300, 7)
    assert_same_neighbors(est, oracle, w.coords, s, w.variogram, targets, None)
    ref = oracle.estimate_many(targets, w.coords, w.values, s, w.variogram, neighbors=False)
    assert_same_estimates(est.predict_full(targets), ref, 1e-10)
