"""The reference's search scale test on the GPU (crates/estimation/tests/search_scale.rs:73-127): 504,100
composites of 5,041 drill holes, every 53rd target of a 200 x 200 x 25 lattice of 5 m blocks (where exact
distance ties are common) plus three targets where a tree search once lost a neighbour, and three searches:
plain, four per hole, four per hole with octants. The engine's neighbour lists must be, index for index, the
test's brute force (restated in search_scale_case.py) on a subset and the oracle's tree on every target."""

import numpy as np
import pytest
from search_scale_case import brute, composites, targets

import boitata_b200 as bt

pytestmark = pytest.mark.gpu

CASES = [{}, {"max_per_hole": 4}, {"max_per_hole": 4, "octant": True}]
VG = bt.Variogram([("spherical", 1.0, 100.0)])


@pytest.fixture(scope="module")
def case():
    locs, vals, holes = composites()
    return locs, vals, holes, targets()


@pytest.mark.parametrize("rules", CASES, ids=["plain", "per_hole", "per_hole_octant"])
def test_lattice_targets_among_drill_holes_match_brute_force(oracle, case, rules):
    locs, vals, holes, t = case
    s = bt.Search(radius=200.0, min_samples=4, max_samples=32, **rules)
    ok = bt.OrdinaryKriging(VG, s).fit(locs, vals, holes=holes)
    idx, cnt, good = ok.neighbors(t)
    ref = oracle.estimate_many(t, locs, vals, s, VG, holes=holes)
    found = ref["status"] != 1  # the oracle's search succeeded (status 1: SearchFailed)
    np.testing.assert_array_equal(good, found)
    for j in range(len(t)):
        if found[j]:
            want = ref["neighbors"][j]
            assert idx[j, : cnt[j]].tolist() == want[want >= 0].tolist(), j
    sub = np.r_[np.arange(0, len(t) - 3, 19), len(t) - 3, len(t) - 2, len(t) - 1]
    for j in sub:
        b = brute(t[j], locs, holes, 200.0, 32, 4, **rules)
        assert (b is None) == (not good[j]), j
        if b is not None:
            assert idx[j, : cnt[j]].tolist() == b, j
