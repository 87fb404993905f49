"""The normal-score transform the simulation takes (crates/transforms/src/normal_score.rs, normal.rs), pinned
by the reference's own tests of it (normal.rs:72-103, normal_score.rs:265-340), and the simulation's host-side
argument checks (crates/py/src/estimation.rs:319-331, sgs.rs:857-862)."""

import math

import numpy as np
import pytest

import boitata_b200 as bt
from boitata_b200.simulation import _back, unit_sill
from boitata_b200.transforms import normal_score, phi, probit


def test_phi_is_accurate_in_the_tails_and_known_values():
    assert abs(phi(-3.0) / 1.349_898_031_630_096e-3 - 1.0) < 1e-12
    assert abs(phi(-6.0) / 9.865_876_450_377_016e-10 - 1.0) < 1e-12
    assert abs(phi(0.0) - 0.5) < 1e-6 and abs(phi(1.0) - 0.8413447) < 1e-5 and abs(phi(-1.96) - 0.025) < 1e-3


def test_probit_inverts_phi_and_quantiles():
    for z in (-2.0, -0.5, 0.0, 0.7, 1.5, 2.3):
        assert abs(z - probit(phi(z))) < 1e-4
    assert abs(probit(0.5)) < 1e-6 and abs(probit(0.975) - 1.959964) < 1e-4
    assert probit(0.0) == probit(1e-15) and probit(1.0) == probit(1.0 - 1e-15)


def test_scores_are_standard_normal_ish():
    scores, _ = normal_score(np.arange(1.0, 101.0))
    assert abs(scores.mean()) < 1e-6 and abs(scores.min() + scores.max()) < 1e-6


def test_forward_inverts_back_and_averages_ties():
    scores, table = normal_score([0.0, 0.0, 1.0, 3.0, 7.0])
    for y in (-0.3, 0.1, 0.6):
        assert abs(table.forward(table.back(y)) - y) < 1e-12
    assert abs(table.forward(0.0) - (scores[0] + scores[1]) / 2.0) < 1e-12


def test_back_transform_round_trips_and_is_monotone():
    vals = [2.0, 5.0, 1.0, 9.0, 4.0, 7.0]
    scores, table = normal_score(vals)
    for v, s in zip(vals, scores):
        assert abs(table.back(s) - v) < 1e-6
    _, t5 = normal_score([1.0, 2.0, 3.0, 4.0, 5.0])
    assert t5.back(-3.0) < t5.back(0.0) < t5.back(3.0)


def test_tails_stay_within_bounds():
    _, table = normal_score([1.0, 2.0, 3.0, 4.0, 5.0])
    assert table.back(-8.0) == 1.0 and table.back(8.0) == 5.0
    wide = table.with_tails(0.0, 10.0)
    low, high = wide.back(-2.0), wide.back(2.5)
    assert 0.0 < low < 1.0 and abs(wide.forward(low) + 2.0) < 1e-6
    assert 5.0 < high < 10.0 and abs(wide.forward(high) - 2.5) < 1e-6


def test_weighted_and_zero_weight_samples():
    scores, table = normal_score([1.0, 2.0, 3.0, 4.0], [0.4, 0.3, 0.2, 0.1])
    assert len(scores) == 4 and np.all(np.diff(scores) > 0)
    assert abs(scores[0] - probit(0.2)) < 1e-15
    s2, t2 = normal_score([1.0, 2.0, 3.0, 4.0], [1.0, 0.0, 1.0, 1.0])
    assert len(t2.values) == 3 and s2[1] == t2.forward(2.0)
    with pytest.raises(bt.InvalidInput):
        normal_score([1.0, 2.0], [1.0, -1.0])


def test_vectorised_back_transform_equals_the_scalar_one():
    rng = np.random.default_rng(3)
    scores, table = normal_score(rng.lognormal(size=200))
    s = np.concatenate([rng.normal(size=500) * 1.5, [-9.0, 9.0, scores[0], scores[-1]]])
    got = _back(table, s)
    want = np.array([table.back(x) for x in s])
    assert np.all(np.abs(got - want) <= 1e-13 * (1 + np.abs(want)))


def test_unit_sill_scales_nugget_and_sills():
    vg = bt.Variogram([bt.Structure("spherical", 2.0, 30.0), bt.Structure("exponential", 1.0, 90.0)], nugget=1.0)
    u = unit_sill(vg)
    assert math.isclose(u.total_sill(), 1.0) and u.nugget == 0.25 and u.structures[0].sill == 0.5
    power = bt.Variogram([bt.Structure("power", 1.0, 10.0, exponent=1.5)])
    assert unit_sill(power) is power


def test_sgs_arguments_are_checked():
    vg = bt.Variogram([bt.Structure("spherical", 1.0, 30.0)])
    with pytest.raises(bt.InvalidInput, match="target_slope"):
        bt.SGS(vg, bt.Search(30.0, target_slope=0.9))
    with pytest.raises(bt.InvalidInput, match="sill"):
        bt.SGS(bt.Variogram([bt.Structure("power", 1.0, 10.0)]), bt.Search(30.0))
    with pytest.raises(bt.Unsupported):
        bt.SGS(vg, [bt.Search(10.0), bt.Search(30.0)])
    sgs = bt.SGS(vg, bt.Search(30.0))
    assert sgs.n_samples is None
    with pytest.raises(bt.InvalidInput, match="not fitted"):
        sgs.simulate(np.zeros((2, 3)))
    assert sgs.fit(np.eye(3), [1.0, 2.0, 3.0]).n_samples == 3
