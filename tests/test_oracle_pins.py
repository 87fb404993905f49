"""Pins of the oracle against the reference's own known-answer and property tests.

The reference (Rust) cannot be built here, and it has no numeric golden
vectors from outside software: every pin it holds for this path is a
property or a cross-method equality. These are those tests, ported to the
oracle (file:line of each original in its docstring).
"""

import math

import numpy as np
import pytest
from conftest import close

from boitata_b200 import Search, Structure, Variogram
from boitata_b200.workloads import Stream, lcg


def ns(**kw):
    class N:
        pass

    o = N()
    o.__dict__.update(kw)
    return o


def nested():
    """kernel.rs:139-159: nugget 0.1, spherical 0.6/80, exponential 0.3/200, az 30 dip 10, ratios 0.5/0.25."""
    return Variogram([Structure("spherical", 0.6, 80.0), Structure("exponential", 0.3, 200.0)], nugget=0.1,
                     rotation=(30.0, 10.0, 0.0), ratios=(0.5, 0.25))


def system(u, n):
    """kernel.rs:162-176: n samples scattered around a target at UTM-sized coordinates."""
    origin = np.array([650_000.0, 7_400_000.0, 1_200.0])
    d = u.uniform(4 * n).reshape(n, 4)
    xyz = origin + d[:, :3] * [200.0, 200.0, 50.0]
    return origin + [100.0, 100.0, 25.0], xyz, d[:, 3] * 3.0


def test_lcg_matches_the_reference_generator():
    s, out = 7, []
    for _ in range(100):
        s = (s * 6364136223846793005 + 1442695040888963407) % (1 << 64)
        out.append((s >> 11) / float(1 << 53))
    assert np.array_equal(lcg(7, 100), np.array(out))


def test_kernel_matches_lu(oracle):
    """kernel.rs:182-210."""
    vg, u = nested(), Stream(7)
    for trial in range(300):
        n = 1 + trial % 40
        t, xyz, v = system(u, n)
        for kind, kp in [("ordinary", 0.0), ("simple", 1.2), ("indicator", 1.5)]:
            s1, fast, wf = oracle.krige(kind, t, xyz, v, vg, kparam=kp, which="kernel")
            s2, slow, ws = oracle.krige(kind, t, xyz, v, vg, kparam=kp, which="lu")
            assert s1 == s2 == 0
            for k in ("value", "variance", "lagrange"):
                assert close(fast[k], slow[k], 1e-9), (trial, kind, k)
            assert np.all(close(wf, ws, 1e-9))


def test_ordinary_weights_sum_to_one(oracle):
    """kernel.rs:212-223."""
    vg, u = nested(), Stream(11)
    for n in [1, 5, 32, 64]:
        t, xyz, v = system(u, n)
        st, e, w = oracle.krige("ordinary", t, xyz, v, vg, which="kernel")
        assert st == 0 and abs(w.sum() - 1.0) < 1e-10


def test_exact_at_a_datum_without_nugget(oracle):
    """kernel.rs:225-238."""
    vg = nested()
    vg = Variogram(vg.structures, nugget=0.0, rotation=vg.rotation, ratios=vg.ratios)
    _, xyz, v = system(Stream(3), 20)
    st, e, _ = oracle.krige("ordinary", xyz[4], xyz, v, vg, which="kernel")
    assert abs(e["value"] - v[4]) < 1e-9 and e["variance"] < 1e-9


def test_duplicates_are_singular_before_the_guard(oracle):
    """kernel.rs:240-255."""
    vg = nested()
    vg = Variogram(vg.structures, nugget=0.0, rotation=vg.rotation, ratios=vg.ratios)
    t, xyz, v = system(Stream(5), 6)
    xyz, v = np.vstack([xyz, xyz[:1]]), np.append(v, v[0])
    assert oracle.krige("ordinary", t, xyz, v, vg, which="kernel")[0] == oracle.SINGULAR
    st, e, w = oracle.krige("ordinary", t, xyz, v, vg)
    assert st == 0 and w[0] == w[6]


def test_falls_back_beyond_max_and_without_a_sill(oracle):
    """kernel.rs:257-265."""
    t, xyz, v = system(Stream(9), 65)
    assert oracle.krige("ordinary", t, xyz, v, nested(), which="kernel")[0] == oracle.NONE
    power = Variogram([Structure("power", 1.0, 100.0, exponent=1.5)])
    assert oracle.krige("ordinary", t, xyz[:8], v[:8], power, which="kernel")[0] == oracle.NONE
    assert oracle.krige("ordinary", t, xyz[:0], v[:0], nested(), which="kernel")[0] == oracle.NONE


def test_measurement_error_enters_the_diagonal(oracle):
    """kernel.rs:267-278."""
    t, xyz, v = system(Stream(13), 10)
    err = np.zeros(10)
    err[2] = 0.4
    _, fast, _ = oracle.krige("ordinary", t, xyz, v, nested(), err=err, which="kernel")
    _, slow, _ = oracle.krige("ordinary", t, xyz, v, nested(), err=err, which="lu")
    assert close(fast["value"], slow["value"], 1e-9) and close(fast["variance"], slow["variance"], 1e-9)


def sph(sill=1.0, rng=100.0, nugget=0.0):
    return Variogram([Structure("spherical", sill, rng)], nugget=nugget)


def test_krige_unit_cases(oracle):
    """krige.rs:218-260: weights sum to 1, exact interpolation, SK reverts to the mean far away."""
    pts = np.array([[0.0, 0.0], [50.0, 0.0], [0.0, 50.0]])
    st, e, w = oracle.krige("ordinary", (10.0, 10.0, 0.0), pts, [1.0, 2.0, 3.0], sph())
    assert abs(w.sum() - 1) < 1e-9 and e["variance"] >= 0
    st, e, _ = oracle.krige("ordinary", (0.0, 0.0, 0.0), pts, [5.0, 2.0, 3.0], sph())
    assert abs(e["value"] - 5.0) < 1e-6 and e["variance"] < 1e-6
    st, e, _ = oracle.krige("simple", (1e4, 1e4, 0.0), pts[:2], [5.0, 2.0], sph(), kparam=3.0)
    assert abs(e["value"] - 3.0) < 1e-6 and abs(e["variance"] - 1.0) < 1e-6


def test_efficiency_and_slope(oracle):
    """krige.rs:262-291."""
    pts = np.array([[0.0, 0, 0], [50.0, 0, 0], [0.0, 50, 0], [60.0, 70, 0]])
    vals = [5.0, 2.0, 3.0, 1.0]
    vg = sph()
    _, at, _ = oracle.krige("ordinary", (0.0, 0.0, 0.0), pts, vals, vg)
    eff = (at["support"] - at["variance"]) / at["support"]
    cov = at["support"] - at["variance"] - at["lagrange"]
    assert abs(eff - 1) < 1e-9 and abs(cov / (cov - at["lagrange"]) - 1) < 1e-9
    t = (90.0, 20.0, 0.0)
    _, ok, w = oracle.krige("ordinary", t, pts, vals, vg)
    c = sum(w[i] * oracle.cov_points(vg, pts[i], t) for i in range(4))
    var = sum(w[i] * w[j] * oracle.cov_points(vg, pts[i], pts[j]) for i in range(4) for j in range(4))
    covz = ok["support"] - ok["variance"] - ok["lagrange"]
    assert abs(covz / (covz - ok["lagrange"]) - c / var) < 1e-9
    assert abs((covz - ok["lagrange"]) - var) < 1e-9


def test_measurement_error_blends_the_datum_with_its_neighbors(oracle):
    """krige.rs:293-321."""
    others = np.array([[50.0, 0, 0], [0.0, 50, 0], [60.0, 70, 0]])
    ov = [2.0, 3.0, 1.0]
    t = (0.0, 0.0, 0.0)
    for kind, kp in [("ordinary", 0.0), ("simple", 2.0)]:
        _, loo, _ = oracle.krige(kind, t, others, ov, sph(), kparam=kp)
        allp = np.vstack([[0.0, 0, 0], others])
        _, e0, _ = oracle.krige(kind, t, allp, [5.0] + ov, sph(), kparam=kp, err=[0.0, 0, 0, 0])
        assert abs(e0["value"] - 5.0) < 1e-9
        for ev in [0.1, 0.5, 2.0]:
            _, e, _ = oracle.krige(kind, t, allp, [5.0] + ov, sph(), kparam=kp, err=[ev, 0, 0, 0])
            k = loo["variance"] / (loo["variance"] + ev)
            assert abs(e["value"] - (loo["value"] + k * (5.0 - loo["value"]))) < 1e-9
            assert abs(e["variance"] - loo["variance"] * (1 - k)) < 1e-9


def test_negative_weights_and_indicator_bounds(oracle):
    """krige.rs:350-388."""
    pts = np.array([[10.0, 0, 0], [20.0, 0, 0], [0.0, 15, 0], [-30.0, -5, 0]])
    g = Variogram([Structure("gaussian", 1.0, 60.0)])
    _, e, w = oracle.krige("ordinary", (0.0, 0.0, 0.0), pts, [1.0, 2, 3, 4], g)
    assert w[w < 0].sum() < 0
    _, e, _ = oracle.krige("indicator", (10.0, 10.0, 0.0), pts[:3] * [5, 2.5, 1], [1.0, 4.0, 2.0], sph(),
                           kparam=2.5)
    assert -1e-6 <= e["value"] <= 1 + 1e-6


def pair_and_lattice(n, gap):
    s = [(10.0, 10.0, 1.0), (10.0 + gap, 10.0, 5.0)]
    k = 0
    while len(s) < n:
        x, y = (k % 9) * 7.0 - 20.0, (k // 9) * 7.0 - 20.0
        if abs(x - 10.0) + abs(y - 10.0) > 1.0:
            s.append((x, y, 3.0 + math.sin(k * 0.3)))
        k += 1
    a = np.array(s)
    return np.column_stack([a[:, :2], np.zeros(n)]), a[:, 2]


def test_twins_krige_as_one_sample(oracle):
    """lib.rs:111-137."""
    locs = np.array([[0.0, 0, 0], [10.0, 0, 0], [0.0, 0, 0], [5.0, 5, -0.0], [5.0, 5, 0]])
    vg = Variogram([Structure("spherical", 1.0, 50.0)])
    t = (2.0, 2.0, 0.0)
    _, est, w = oracle.krige("ordinary", t, locs, [1.0, 2, 3, 4, 6], vg)
    _, one, _ = oracle.krige("ordinary", t, locs[[0, 1, 3]], [2.0, 2.0, 5.0], vg)
    assert abs(est["value"] - one["value"]) < 1e-12 and abs(est["variance"] - one["variance"]) < 1e-12
    assert w[0] == w[2] and w[3] == w[4]


def test_near_coincident_pair_outcome_independent_of_n(oracle):
    """coincident.rs:147-169."""
    vg = Variogram([Structure("spherical", 1.0, 50.0)])
    t = (12.0, 11.0, 0.0)
    for gap in [0.0, 1e-12, 1e-7, 1e-6]:
        for kind, kp in [("ordinary", 0.0), ("simple", 3.0), ("indicator", 2.0)]:
            a = oracle.krige(kind, t, *pair_and_lattice(64, gap), vg, kparam=kp)
            b = oracle.krige(kind, t, *pair_and_lattice(65, gap), vg, kparam=kp)
            for st, e, w in (a, b):
                assert st == 0 and w[0] == w[1] and np.isfinite(e["value"]) and np.isfinite(e["variance"])
            if kind != "simple":
                assert abs(a[2].sum() - 1) < 1e-12
            assert (a[1]["n_used"], b[1]["n_used"]) == (64, 65)


def test_a_datum_repeated_krige_as_its_mean(oracle):
    """coincident.rs:224-246."""
    vg = Variogram([Structure("exponential", 0.8, 40.0)], nugget=0.2)
    xyz, v = pair_and_lattice(20, 0.0)
    others, ov = xyz[2:], v[2:]
    t = (12.0, 11.0, 0.0)
    at = np.array([[10.0, 10.0, 0.0]])
    three = oracle.krige("ordinary", t, np.vstack([at, at, at, others]), np.concatenate([[1.0, 2.0, 6.0], ov]), vg,
                         err=np.concatenate([[0.3] * 3, np.zeros(len(ov))]))
    one = oracle.krige("ordinary", t, np.vstack([at, others]), np.concatenate([[3.0], ov]), vg,
                       err=np.concatenate([[0.1], np.zeros(len(ov))]))
    assert close(three[1]["value"], one[1]["value"], 1e-9) and close(three[1]["variance"], one[1]["variance"], 1e-9)
    assert close(3 * three[2][0], one[2][0], 1e-9) and close(three[1]["lagrange"], one[1]["lagrange"], 1e-9)


def test_indicator_twins_average_their_indicators(oracle):
    """coincident.rs:248-256."""
    xyz, v = pair_and_lattice(10, 0.0)
    _, e, _ = oracle.krige("indicator", xyz[0], xyz, v, Variogram([Structure("spherical", 1.0, 50.0)]), kparam=2.0)
    assert close(e["value"], 0.5, 1e-9) and e["variance"] < 1e-9


def cloud(n, seed, scale):
    return lcg(seed, 3 * n).reshape(n, 3) * np.asarray(scale)


def brute(points, q, radius2):
    d = ((points[:, 0] - q[0]) ** 2 + (points[:, 1] - q[1]) ** 2) + (points[:, 2] - q[2]) ** 2
    keep = np.nonzero(d <= radius2)[0]
    bits = d[keep].view(np.uint64)
    order = np.lexsort((keep, bits))
    return list(zip(bits[order].tolist(), keep[order].tolist()))


def test_grid_visits_every_point_within_the_radius_nearest_first(oracle):
    """grid.rs:421-444."""
    for scale, n in [([1000.0, 1000, 100], 3000), ([1000.0, 1000, 0], 2000), ([0.0, 0, 500], 500),
                     ([3000.0, 20, 5], 1500)]:
        pts = cloud(n, 7, scale)
        targets = cloud(60, 11, np.asarray(scale) * 1.6 + 1.0)
        for t in targets:
            q = t - 0.3 * np.asarray(scale) - 0.5
            for r2 in [0.0, 2500.0, 40_000.0, math.inf]:
                assert oracle.grid_visit(pts, q, r2) == brute(pts, q, r2)


def test_grid_duplicates_come_in_index_order_and_nan_never(oracle):
    """grid.rs:446-460."""
    pts = np.vstack([np.tile([5.0, 5.0, 5.0], (100, 1)), [[math.nan, 0.0, 0.0]], cloud(50, 3, [10.0, 10, 10])])
    got = oracle.grid_visit(pts, np.array([5.0, 5.0, 5.0]), math.inf)
    assert got == brute(pts, [5.0, 5, 5], math.inf)
    assert all(i != 100 for _, i in got) and [i for _, i in got[:100]] == list(range(100))


def test_grid_stops_when_told(oracle):
    """grid.rs:462-472."""
    assert len(oracle.grid_visit(cloud(1000, 5, [100.0, 100, 100]), np.array([50.0, 50, 50]), math.inf, 5)) == 5


def params(min_samples, max_samples, radius, **kw):
    return ns(min_samples=min_samples, max_samples=max_samples, radius=radius, octant=kw.get("octant", False),
              max_per_hole=kw.get("max_per_hole"), max_per_octant=kw.get("max_per_octant"),
              min_sectors=kw.get("min_sectors"), max_empty_sectors=kw.get("max_empty_sectors"),
              min_holes=kw.get("min_holes"), sectors=None, max_per_sector=None,
              anisotropy=kw.get("anisotropy"))


def test_search_unit_cases(oracle):
    """search.rs:1121-1181."""
    two = np.array([[0.0, 0, 0], [1.0, 0, 0]])
    for m in [2 ** 61, 1 << 40]:
        s = params(1, m, 100.0, octant=True)
        assert len(oracle.Tree(two, s).neighbors((0.5, 0.0, 0.0))[1]) == 2
    three = np.array([[1.0, 0, 0], [2.0, 0, 0], [100.0, 0, 0]])
    p = params(1, 2, 10.0)
    assert oracle.scan_neighbors((0.0, 0.0, 0.0), three, p) == (True, [0, 1])
    assert oracle.Tree(three, p).neighbors((0.0, 0.0, 0.0)) == (True, [0, 1])
    four = np.array([[1.0, 0, 0], [2.0, 0, 0], [3.0, 0, 0], [4.0, 0, 0]])
    hp = params(1, 10, 100.0, max_per_hole=2)
    assert oracle.scan_neighbors((0.0, 0.0, 0.0), four, hp, holes=[1, 1, 1, 2]) == (True, [0, 1, 3])
    assert not oracle.scan_neighbors((0.0, 0.0, 0.0), four[:1], params(5, 10, 100.0))[0]
    assert not oracle.Tree(four[:1], params(5, 10, 100.0)).neighbors((0.0, 0.0, 0.0))[0]


def test_tree_matches_the_scan(oracle):
    """search.rs:1183-1270 (the cases without high-grade or soft domain rules)."""
    u = Stream(12345)
    pts = u.uniform(3 * 3000).reshape(3000, 3) * [1000.0, 1000, 100]
    holes = np.arange(3000) // 20
    an = (35.0, 10.0, 0.0, 1.0, 0.4, 0.2)
    cases = [params(1, 16, 120.0), params(1, 24, 200.0, octant=True),
             params(1, 12, 150.0, max_per_hole=3, anisotropy=an), params(1, 16, 150.0, octant=True),
             params(1, 16, 150.0, anisotropy=an),
             params(1, 24, 60.0, octant=True, max_per_octant=2, min_sectors=6, max_empty_sectors=1, max_per_hole=2,
                    min_holes=6)]
    for p in cases:
        tree = oracle.Tree(pts, p, holes=holes)
        for t in u.uniform(3 * 60).reshape(60, 3) * [1000.0, 1000, 100]:
            assert tree.neighbors(t) == oracle.scan_neighbors(t, pts, p, holes=holes)


def test_octants_follow_the_ellipse(oracle):
    """search.rs:1405-1438."""
    sa, ca = math.sin(math.radians(30)), math.cos(math.radians(30))
    at = lambda along, across, z: (along * sa + across * ca, along * ca - across * sa, z)  # noqa: E731
    pts = np.array([at(a, c, 0.0) for c, a in zip([-0.5, 0.5, -0.4, 0.4], [4.0, 5.0, 6.0, 7.0])] + [(-20.0, -20, 0)])
    p = params(1, 4, 100.0, octant=True, anisotropy=(30.0, 0.0, 0.0, 1.0, 0.5, 0.5))
    ok, got = oracle.scan_neighbors((0.0, 0.0, 0.0), pts, p)
    assert sorted(got) == [0, 1, 4]


def test_search_check_rules(oracle):
    """search.rs:214-264."""
    assert oracle.check_search(params(1, 16, 100.0))
    assert not oracle.check_search(params(1, 16, 0.0))
    assert not oracle.check_search(params(5, 4, 100.0))
    assert not oracle.check_search(params(1, 16, 100.0, max_per_octant=2))
    assert not oracle.check_search(params(1, 16, 100.0, octant=True, max_empty_sectors=4))


def test_rotation_conventions(oracle):
    """rotation.rs:54-70: azimuth clockwise from north, dip positive down."""
    assert np.allclose(oracle.rotation_matrix(0, 0, 0)[0], [0, 1, 0], atol=1e-12)
    assert np.allclose(oracle.rotation_matrix(90, 0, 0)[0], [1, 0, 0], atol=1e-12)
    assert np.allclose(oracle.rotation_matrix(0, 30, 0)[0], [0, math.cos(math.radians(30)), -0.5], atol=1e-12)
    assert np.array_equal(oracle.block_frame(0, 0, 0) + 0.0, np.eye(3))


def test_model_shapes(oracle):
    """model.rs:335-397."""
    assert oracle.shape("spherical", 0.0, 100.0) == 0.0
    assert abs(oracle.shape("spherical", 100.0, 100.0) - 1) < 1e-12
    assert oracle.shape("spherical", 200.0, 100.0) == 1.0
    assert abs(oracle.shape("cubic", 100.0, 100.0) - 1) < 1e-9 and oracle.shape("cubic", 150.0, 100.0) == 1.0
    assert oracle.shape("pentaspherical", 25.0, 100.0) < oracle.shape("pentaspherical", 75.0, 100.0) < 1
    assert abs(oracle.shape("circular", 100.0, 100.0) - 1) < 1e-9
    for h in [10.0, 55.0, 130.0]:
        assert abs(oracle.shape("matern", h, 100.0, 0.5) - oracle.shape("exponential", h, 100.0)) < 1e-12
    assert oracle.shape("matern", 20.0, 100.0, 2.5) < oracle.shape("matern", 20.0, 100.0, 0.5)
    assert abs(oracle.shape("power", 100.0, 100.0, 1.5) - 1) < 1e-12
    assert max(oracle.shape("sinehole", i * 10.0, 100.0) for i in range(1, 40)) > 1


@pytest.mark.parametrize("model,param", [("spherical", 0), ("exponential", 0), ("gaussian", 0), ("cubic", 0),
                                         ("pentaspherical", 0), ("circular", 0), ("sinehole", 0), ("matern", 0.5),
                                         ("matern", 1.5), ("matern", 2.5), ("power", 1.5)])
def test_shape_derivative_matches_finite_differences(oracle, model, param):
    """model.rs:399-430."""
    eps = 1e-4
    for h in [7.0, 23.0, 61.0, 140.0]:
        fd = (oracle.shape(model, h + eps, 100.0, param) - oracle.shape(model, h - eps, 100.0, param)) / (2 * eps)
        assert abs(fd - oracle.shape_d1(model, h, 100.0, param)) < 1e-6


def test_leave_one_out_equals_refit_without_the_sample(oracle):
    """batch.rs:375-460 / python test_estimation.py:186-204: LOO searches as if the sample were absent."""
    rng = np.random.default_rng(3)
    coords = np.column_stack([rng.uniform(0, 100, (150, 2)), np.zeros(150)])
    values = np.sin(coords[:, 0] / 15) + coords[:, 1] / 50
    vg = Variogram([Structure("spherical", 1.0, 40.0)])
    s = Search(radius=50, max_samples=4, octant=True, max_per_sector=1)
    loo = oracle.estimate_many(None, coords, values, s, vg, loo=True)
    for i in range(0, 150, 7):
        rest = np.arange(150) != i
        one = oracle.estimate_many(coords[i:i + 1], coords[rest], values[rest], s, vg)
        assert close(loo["value"][i], one["value"][0], 1e-9) or (np.isnan(loo["value"][i]) and np.isnan(one["value"][0]))


def test_results_do_not_depend_on_thread_count(oracle):
    """batch.rs:256-305."""
    i = np.arange(200)
    x, y = (i * 37 % 101).astype(float), (i * 53 % 97).astype(float)
    coords = np.column_stack([x, y, np.zeros(200)])
    values = np.sin(x / 10) + y / 50
    targets = np.column_stack([(np.arange(400) % 20) * 5.0, (np.arange(400) // 20) * 5.0, np.zeros(400)])
    vg = Variogram([Structure("spherical", 1.0, 40.0)])
    s = Search(radius=30.0, min_samples=4, max_samples=12)
    a = oracle.estimate_many(targets, coords, values, s, vg, threads=1)
    b = oracle.estimate_many(targets, coords, values, s, vg, threads=8)
    for k in ("value", "variance"):
        assert np.array_equal(a[k].view(np.uint64), b[k].view(np.uint64))


# ---- block kriging (crates/estimation/src/block.rs:200-371) ----

def test_block_discretization_centres_on_the_block(oracle):
    """block.rs:205-212."""
    off = oracle.block_offsets((10.0, 10.0, 10.0), (3, 3, 3))
    assert len(off) == 27
    pts = off + np.array([100.0, 200.0, 300.0])
    assert abs(pts[:, 0].mean() - 100.0) < 1e-9


def test_block_variance_below_point_variance(oracle):
    """block.rs:214-248."""
    vg = sph()
    xyz = np.array([[0.0, 0, 0], [60.0, 0, 0], [0.0, 60, 0]])
    vals = [1.0, 2.0, 3.0]
    c = (30.0, 30.0, 0.0)
    st, block, w = oracle.block_krige(c, oracle.block_offsets((20.0, 20.0, 20.0), (3, 3, 3)), xyz, vals, vg)
    _, point, _ = oracle.krige("ordinary", c, xyz, vals, vg)
    assert st == 0 and block["variance"] <= point["variance"] + 1e-9
    assert abs(w.sum() - 1.0) < 1e-9


def test_block_nugget_averages_out(oracle):
    """block.rs:267-296: C(B,B) = C - gamma_bar over a segment; a pure nugget leaves 0 and variance 1/2."""
    c0, c, a, l = 0.4, 1.0, 100.0, 60.0
    xyz = np.array([[-50.0, 0, 0], [70.0, 0, 0]])
    off = oracle.block_offsets((l, 0.0, 0.0), (400, 1, 1))
    _, e, _ = oracle.block_krige((0.0, 0.0, 0.0), off, xyz, [1.0, 2.0], sph(c, a, c0))
    gamma_bar = c * (l / (2 * a) - l ** 3 / (20 * a ** 3))
    assert abs(e["support"] - (c - gamma_bar)) < 1e-4
    pure = Variogram([], nugget=1.0)
    off = oracle.block_offsets((l, 1.0, 1.0), (400, 1, 1))
    _, e, _ = oracle.block_krige((0.0, 0.0, 0.0), off, xyz, [1.0, 2.0], pure)
    assert e["support"] == 0.0 and abs(e["variance"] - 0.5) < 1e-12


def test_block_sample_on_a_node_sees_no_nugget(oracle):
    """block.rs:298-310."""
    off = oracle.block_offsets((30.0, 30.0, 30.0), (3, 3, 3))

    def block(x):
        return oracle.block_krige((0.0, 0.0, 0.0), off, np.array([[x, 0.0, 0.0], [40.0, 25.0, 0.0]]), [1.0, 3.0],
                                  sph(nugget=0.5))

    (_, on, won), (_, off_, woff) = block(0.0), block(1e-9)
    assert abs(won[0] - woff[0]) < 1e-9 and abs(on["variance"] - off_["variance"]) < 1e-9


def test_one_point_block_is_point_kriging(oracle):
    """block.rs:312-340."""
    vg = Variogram([Structure("spherical", 0.7, 100.0)], nugget=0.3)
    one = oracle.block_offsets((10.0, 10.0, 10.0), (1, 1, 1))
    c = (0.0, 0.0, 0.0)
    xyz = np.array([[50.0, 0.0, 0.0]])
    _, point, _ = oracle.krige("ordinary", c, xyz, [1.0], vg)
    _, block, _ = oracle.block_krige(c, one, xyz, [1.0], vg)
    gamma50 = 0.3 + 0.7 * (1.5 * 0.5 - 0.5 * 0.5 ** 3)
    assert abs(point["variance"] - 2 * gamma50) < 1e-9 and abs(block["variance"] - point["variance"]) < 1e-9
    assert block["support"] == 1.0
    xyz = np.array([[0.0, 0.0, 0.0], [40.0, 25.0, 0.0]])
    _, point, wp = oracle.krige("ordinary", c, xyz, [1.0, 3.0], vg)
    _, block, wb = oracle.block_krige(c, one, xyz, [1.0, 3.0], vg)
    assert abs(wb[0] - wp[0]) < 1e-9 and abs(block["variance"] - point["variance"]) < 1e-9


def test_block_with_no_nugget_uses_point_covariances(oracle):
    """With no nugget, block_cov_points equals cov_points (block.rs:355-370). Checked here on the results:
    the oracle's block kriging equals a dense numpy solve of the same bordered system."""
    off = oracle.block_offsets((30.0, 30.0, 30.0), (3, 3, 3))
    xyz = np.array([[0.0, 0.0, 0.0], [40.0, 25.0, 0.0], [-20.0, 10.0, 5.0]])
    _, e, w = oracle.block_krige((0.0, 0.0, 0.0), off, xyz, [1.0, 3.0, 2.0], sph())
    pts = off
    cov = lambda h: 1.0 - (1.5 * (h / 100) - 0.5 * (h / 100) ** 3 if h < 100 else 1.0)
    rhs = np.array([np.mean([cov(np.linalg.norm(x - p)) for p in pts]) for x in xyz])
    C = np.array([[cov(np.linalg.norm(a - b)) for b in xyz] for a in xyz])
    K = np.block([[C, np.ones((3, 1))], [np.ones((1, 3)), np.zeros((1, 1))]])
    sol = np.linalg.solve(K, np.r_[rhs, 1.0])
    assert np.allclose(w, sol[:3], atol=1e-12) and abs(e["lagrange"] - sol[3]) < 1e-12


def scattered_nearest(seed, n, t):
    """n samples in a 40 m box around t, nearest first (a search's selection order)."""
    rng = np.random.default_rng(seed)
    xyz = np.asarray(t) + rng.uniform(-20.0, 20.0, (n, 3)) * [1.0, 1.0, 0.5]
    return xyz[np.argsort(((xyz - t) ** 2).sum(1), kind="stable")]


def test_prefix_quality_matches_direct_solves(oracle):
    """kriging_algebra.rs:1115-1157: each leading part's slope and efficiency equal those of kriging it."""
    vg = nested()
    t = np.array([1.0, 2.0, 5.0])
    xyz = scattered_nearest(17, 24, t)
    sill = vg.total_sill()
    osl, oef, ook = oracle.prefix_quality(t, xyz, vg)
    ssl, sef, sok = oracle.prefix_quality(t, xyz, vg, ordinary=False)
    assert ook.all() and sok.all()
    for n in range(1, 25):
        _, ok, _ = oracle.krige("ordinary", t, xyz[:n], np.zeros(n), vg)
        cov = sill - ok["variance"] - ok["lagrange"]
        assert close(osl[n - 1], cov / (cov - ok["lagrange"]), 1e-9)
        assert close(oef[n - 1], (sill - ok["variance"]) / sill, 1e-9)
        _, sk, _ = oracle.krige("simple", t, xyz[:n], np.zeros(n), vg, kparam=1.0)
        assert close(ssl[n - 1], 1.0, 1e-9) and close(sef[n - 1], (sill - sk["variance"]) / sill, 1e-9)


@pytest.mark.parametrize("calibration", [("target_slope", 0.8), ("target_slope", 0.95),
                                         ("target_efficiency", 0.3), ("target_efficiency", 0.99)])
def test_calibrated_count_takes_the_fewest_that_meet_the_target(oracle, calibration):
    """kriging_algebra.rs:1159-1189 through estimate_many: n >= min_samples; where met, the n-sample part
    meets the target and no shorter part from min_samples does; else every sample is used."""
    vg = nested()
    key, target = calibration
    rng = np.random.default_rng(5)
    xyz = rng.uniform(0.0, 60.0, (300, 3)) * [1.0, 1.0, 0.3]
    values = rng.normal(size=300)
    targets = rng.uniform(5.0, 55.0, (40, 3)) * [1.0, 1.0, 0.3]
    for trial, t in enumerate(targets):
        mn = 1 + trial % 4
        s = Search(radius=1e9, max_samples=20, min_samples=mn, **{key: target})
        plain = Search(radius=1e9, max_samples=20, min_samples=mn)
        r = oracle.estimate_many(t[None], xyz, values, s, vg, neighbors=False, diagnostics=True)
        full = oracle.estimate_many(t[None], xyz, values, plain, vg)
        chosen = full["neighbors"][0]
        sl, ef, ok = oracle.prefix_quality(t, xyz[chosen], vg)
        q = sl if key == "target_slope" else ef
        n, met = int(r["n_used"][0]), r["target_met"][0]
        assert mn <= n <= 20
        if met == 1:
            assert ok[n - 1] and q[n - 1] >= target
            assert not any(ok[k - 1] and q[k - 1] >= target for k in range(mn, n))
        else:
            assert met == 0 and n == 20
            assert not any(ok[k - 1] and q[k - 1] >= target for k in range(mn, 21))
        _, one, w = oracle.krige("ordinary", t, xyz[chosen[:n]], values[chosen[:n]], vg)
        assert r["value"][0] == one["value"] and abs(w[:n].sum() - 1.0) < 1e-10


def test_calibration_balances_octants_round_robin(oracle):
    """search.rs:913-936: a calibrated octant search krigs its samples taken from the octants in turn."""
    vg = Variogram([Structure("spherical", 1.0, 50.0)], nugget=0.05)
    rng = np.random.default_rng(9)
    xyz = rng.uniform(0.0, 100.0, (400, 3)) * [1.0, 1.0, 0.2]
    values = rng.normal(size=400)
    t = np.array([50.0, 50.0, 10.0])
    plain = Search(radius=60.0, max_samples=24, octant=True, max_per_sector=3)
    cal = Search(radius=60.0, max_samples=24, octant=True, max_per_sector=3, target_efficiency=-1e9)
    chosen = oracle.estimate_many(t[None], xyz, values, plain, vg)["neighbors"][0]
    chosen = chosen[chosen >= 0]
    d = xyz[chosen] - t
    octant = (d[:, 0] >= 0) * 4 + (d[:, 1] >= 0) * 2 + (d[:, 2] >= 0)
    rank = np.array([np.sum(octant[: i + 1] == octant[i]) for i in range(len(chosen))])
    order = chosen[np.argsort(rank, kind="stable")]
    r = oracle.estimate_many(t[None], xyz, values, cal, vg, neighbors=False, diagnostics=True)
    assert r["n_used"][0] == 1 and r["target_met"][0] == 1  # any efficiency meets: the first of the turn
    _, one, _ = oracle.krige("ordinary", t, xyz[order[:1]], values[order[:1]], vg)
    assert r["value"][0] == one["value"]
    cal = Search(radius=60.0, max_samples=24, octant=True, max_per_sector=3, target_efficiency=0.999)
    r = oracle.estimate_many(t[None], xyz, values, cal, vg, neighbors=False)
    _, all_, _ = oracle.krige("ordinary", t, xyz[order], values[order], vg)
    assert r["n_used"][0] == len(order) and close(r["value"][0], all_["value"], 1e-12)


def test_calibration_arguments_are_checked_as_the_reference_does():
    """crates/py/src/estimation.rs:458-473, 819-827."""
    from boitata_b200 import InvalidInput, OrdinaryKriging, SimpleKriging

    s = Search(radius=60, max_samples=24, min_samples=2, target_slope=0.9)
    assert (s.target_slope, s.target_efficiency) == (0.9, None)
    with pytest.raises(InvalidInput, match="at most one"):
        Search(radius=60, target_slope=0.9, target_efficiency=0.5)
    with pytest.raises(InvalidInput, match="target_slope"):
        Search(radius=60, target_slope=0.0)
    with pytest.raises(InvalidInput, match="target_efficiency"):
        Search(radius=60, target_efficiency=1.5)
    with pytest.raises(InvalidInput, match="simple kriging"):
        SimpleKriging(nested(), s, mean=1.0)
    OrdinaryKriging(nested(), s)
    SimpleKriging(nested(), Search(radius=60, target_efficiency=0.5), mean=1.0)


# ---- k-fold and hard domains (crates/estimation/src/batch.rs tests) ----------
def batch_samples():
    """batch.rs:256-263: 200 samples at (37 i mod 101, 53 i mod 97, 0), value sin(x / 10) + y / 50."""
    i = np.arange(200)
    x, y = (i * 37 % 101).astype(float), (i * 53 % 97).astype(float)
    return np.column_stack([x, y, np.zeros(200)]), np.sin(x / 10.0) + y / 50.0


def batch_grid():
    """batch.rs:582-586: a 30 x 30 grid of targets 5 apart."""
    i = np.arange(900)
    return np.column_stack([(i % 30) * 5.0, (i // 30) * 5.0, np.zeros(900)])


def domain_of(p):
    """batch.rs:991-997."""
    v = p[0] + 0.3 * p[1]
    return 0 if v < 45.0 else (1 if v < 80.0 else 2)


def batch_search(min_samples, radius):
    from boitata_b200 import Search

    return Search(radius=radius, max_samples=12, min_samples=min_samples)


def spherical_40():
    from boitata_b200 import Structure, Variogram

    return Variogram([Structure("spherical", 1.0, 40.0)])


def same_bits(a, b):
    return all(np.array_equal(a[k].view(np.int64), b[k].view(np.int64)) for k in ("value", "variance")) and \
        np.array_equal(a["status"], b["status"])


def test_k_fold_with_one_sample_per_fold_is_leave_one_out(oracle):
    # batch.rs:349-372
    xyz, v = batch_samples()
    s, vg = batch_search(4, 30.0), spherical_40()
    loo = oracle.estimate_many(None, xyz, v, s, vg, loo=True, neighbors=False)
    folds = oracle.k_fold(len(xyz), xyz, v, s, vg)
    assert np.sum(loo["status"] == 0) > 150
    assert same_bits(loo, folds)
    with pytest.raises(ValueError):
        oracle.k_fold(1, xyz, v, s, vg)


def test_k_fold_never_splits_a_hole(oracle):
    # batch.rs:463-489: every seventh sample untagged, the others in holes of five; every sample is estimated
    # for k = 2, 5 and n.
    xyz, v = batch_samples()
    i = np.arange(len(xyz))
    holes = np.where(i % 7 == 0, -1, 1000 - i // 5)
    s, vg = batch_search(2, 60.0), spherical_40()
    for k in (2, 5, len(xyz)):
        out = oracle.k_fold(k, xyz, v, s, vg, holes=holes)
        assert np.all(out["status"] == 0), k


def test_hard_domains_are_separate_estimations(oracle):
    # batch.rs:1047-1075: with hard boundaries a domain's targets (and its samples' leave-one-out) are
    # estimated as if the other domains' samples did not exist.
    xyz, v = batch_samples()
    targets = batch_grid()
    dom = np.array([domain_of(p) for p in xyz])
    tdom = np.array([domain_of(p) for p in targets])
    s, vg = batch_search(2, 30.0), spherical_40()
    hard = oracle.estimate_many(targets, xyz, v, s, vg, domains=dom, target_domains=tdom, neighbors=False)
    hard_cv = oracle.estimate_many(None, xyz, v, s, vg, loo=True, domains=dom, neighbors=False)
    for d in range(3):
        own = dom == d
        at = tdom == d
        alone = oracle.estimate_many(targets[at], xyz[own], v[own], s, vg, neighbors=False)
        assert same_bits(alone, {k: x[at] for k, x in hard.items()})
        cv = oracle.estimate_many(None, xyz[own], v[own], s, vg, loo=True, neighbors=False)
        assert same_bits(cv, {k: x[own] for k, x in hard_cv.items()})
    assert np.sum(hard["status"] == 0) > 300
    # A target of a domain without samples is not estimated.
    none = oracle.estimate_many(targets[:5], xyz, v, s, vg, domains=dom, target_domains=np.full(5, -1),
                                neighbors=False)
    assert np.all(none["status"] == 1) and np.all(np.isnan(none["value"]))


@pytest.mark.parametrize("rules", [{}, {"max_per_hole": 4}, {"max_per_hole": 4, "octant": True}],
                         ids=["plain", "per_hole", "per_hole_octant"])
def test_search_scale_tree_matches_brute_force(oracle, rules):
    """tests/search_scale.rs:73-127 on a subset: the oracle's tree equals the test's brute force among
    504,100 drill-hole composites at lattice targets (exact ties), including the three targets that once
    lost a neighbour."""
    from search_scale_case import brute, composites, targets

    locs, vals, holes = composites()
    t = targets()
    sub = np.r_[np.arange(0, len(t) - 3, 311), len(t) - 3, len(t) - 2, len(t) - 1]
    s = Search(radius=200.0, min_samples=4, max_samples=32, **rules)
    ref = oracle.estimate_many(t[sub], locs, vals, s, Variogram([("spherical", 1.0, 100.0)]), holes=holes)
    for j, k in enumerate(sub):
        b = brute(t[k], locs, holes, 200.0, 32, 4, **rules)
        assert (b is None) == (ref["status"][j] == 1), k
        if b is not None:
            got = ref["neighbors"][j]
            assert got[got >= 0].tolist() == b, k
