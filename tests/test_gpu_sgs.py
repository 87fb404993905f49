"""Sequential Gaussian simulation on the GPU against the oracle's one-node-at-a-time restatement of
crates/simulation/src/sgs.rs:586-760 (same data scores, node order and normal draws): node scores to 1e-9 in
|a-b| <= tol (1 + max(|a|, |b|)) and the same kriged / marginal split; any batch gives the same bits (the
realization is the sequential one); and the properties of the reference's SGS tests (sgs.rs:933-1195)."""

import numpy as np
import pytest
from conftest import close

import boitata_b200 as bt
from boitata_b200 import workloads as W
from boitata_b200.simulation import sgs_scores, unit_sill
from boitata_b200.transforms import normal_score

pytestmark = pytest.mark.gpu


def case(n_nodes, seed=5, holes=False):
    w = W.c1()
    scores, _ = normal_score(w.values)
    rng = np.random.default_rng(seed)
    nodes = rng.uniform(0, 1000, (n_nodes, 3)) * [1.0, 1.0, 0.2]
    z = rng.standard_normal(n_nodes)
    codes = (np.arange(len(w.coords)) // 5) if holes else None
    return w, scores, nodes, z, codes


@pytest.mark.parametrize("search", [
    dict(ranges=(300.0, 300.0, 100.0), max_samples=16, min_samples=4),
    dict(radius=120.0, octant=True, max_per_sector=3, max_samples=24, min_samples=1, rotation=(30.0, 0.0, 0.0),
         ratios=(0.5, 0.3)),
    dict(ranges=(250.0, 250.0, 80.0), max_samples=20, max_per_hole=2, min_samples=2),
    dict(ranges=(300.0, 300.0, 100.0), max_samples=72, min_samples=8),
])
def test_sgs_matches_the_sequential_oracle(oracle, search):
    holes = "max_per_hole" in search
    w, scores, nodes, z, codes = case(3000, holes=holes)
    s = bt.Search(**search)
    vg = unit_sill(w.variogram)
    got, how, rounds = sgs_scores(w.coords, scores, codes, nodes, z, s, vg)
    want, whow = oracle.sgs(w.coords, scores, nodes, z, s, vg, holes=codes)
    np.testing.assert_array_equal(how, whow)
    assert np.all(close(got, want, 1e-9)), np.max(np.abs(got - want))
    assert rounds >= 1 and np.any(how == 1)


def test_any_batch_gives_the_sequential_realization():
    w, scores, nodes, z, _ = case(2000, seed=6)
    s = bt.Search(ranges=(300.0, 300.0, 100.0), max_samples=16, min_samples=4)
    vg = unit_sill(w.variogram)
    one, _, r1 = sgs_scores(w.coords, scores, None, nodes, z, s, vg, batch=1)
    assert r1 == len(nodes)  # one node per round: the plain sequential loop
    for batch in (16, 512, None, 100000):
        other, _, _ = sgs_scores(w.coords, scores, None, nodes, z, s, vg, batch=batch)
        np.testing.assert_array_equal(one, other)


def test_nodes_on_data_take_the_data_value_and_data_are_honoured():
    # sgs.rs:1114-1140 and :933-972.
    vg = bt.Variogram([bt.Structure("spherical", 1.0, 30.0)])
    sim = bt.SGS(vg, bt.Search(50.0, max_samples=8, min_samples=1))
    sim.fit([[0.0, 0.0, 0.0], [10.0, 0.0, 0.0], [20.0, 0.0, 0.0]], [1.0, 5.0, 3.0])
    r = sim.simulate([[10.0, 0.0, 0.0], [5.0, 0.0, 0.0], [15.0, 0.0, 0.0]], n=5, seed=4).realizations
    assert np.all(r[:, 0] == 5.0) and np.all((r[:, 1:] >= 1.0) & (r[:, 1:] <= 5.0))
    vg = bt.Variogram([bt.Structure("spherical", 1.0, 200.0)])
    sim = bt.SGS(vg, bt.Search(float("inf"), max_samples=8, min_samples=1))
    sim.fit([[0.0, 0.0, 0.0], [100.0, 0.0, 0.0], [0.0, 100.0, 0.0], [100.0, 100.0, 0.0]], [1.0, 5.0, 3.0, 8.0])
    r = sim.simulate([[0.0, 0.0, 0.0], [50.0, 50.0, 0.0]], n=3, seed=42).realizations
    assert np.all(r[:, 0] == 1.0)


def test_seeds_reproduce_and_differ():
    # sgs.rs:974-1032.
    vg = bt.Variogram([bt.Structure("exponential", 1.0, 150.0)])
    data = [[0.0, 0.0, 0.0], [100.0, 0.0, 0.0], [0.0, 100.0, 0.0]]
    grid = [[i * 5.0, 25.0, 0.0] for i in range(20)]
    sim = bt.SGS(vg, bt.Search(float("inf"), max_samples=12, min_samples=1)).fit(data, [1.0, 5.0, 3.0])
    a, b = sim.simulate(grid, seed=7).realizations, sim.simulate(grid, seed=7).realizations
    np.testing.assert_array_equal(a, b)
    assert not np.array_equal(a, sim.simulate(grid, seed=8).realizations)


def test_ensemble_statistics():
    # sgs.rs:1166-1195: the ensemble mean approaches kriging between equal data, and far from the data
    # the ensemble reproduces the data histogram.
    vg = bt.Variogram([bt.Structure("spherical", 1.0, 200.0)])
    s = bt.Search(float("inf"), max_samples=8, min_samples=1)
    sim = bt.SGS(vg, s).fit([[0.0, 0.0, 0.0], [100.0, 0.0, 0.0], [0.0, 100.0, 0.0], [100.0, 100.0, 0.0]],
                            [2.0, 2.0, 2.0, 2.0])
    assert abs(sim.simulate([[50.0, 50.0, 0.0]], n=50, seed=100).mean[0] - 2.0) < 0.2
    locs = [[float(i * 7 % 20), float(i * 3 % 20), 0.0] for i in range(20)]
    vals = np.arange(1.0, 21.0)
    far = bt.SGS(bt.Variogram([bt.Structure("spherical", 1.0, 10.0)]), s).fit(locs, vals)
    e = far.simulate([[1e4, 1e4, 0.0]], n=400, seed=100)
    assert abs(e.mean[0] - 10.5) < 0.8 and abs(e.variance[0] / 33.25 - 1.0) < 0.25


def test_simulated_scores_keep_the_variogram_sill_c1():
    w = W.c1()
    sim = bt.SGS(w.variogram, w.search).fit(w.coords, w.values)
    g = bt.Geometry((0.0, 0.0, 0.0), (40.0, 40.0, 20.0), (25, 25, 10))
    r = sim.simulate(g, n=2, seed=1)
    assert r.realizations.shape == (2, 6250) and np.all(np.isfinite(r.realizations))
    assert w.values.min() <= r.realizations.min() and r.realizations.max() <= w.values.max()
    assert abs(np.median(r.realizations) / np.median(w.values) - 1.0) < 0.3
