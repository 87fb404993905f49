"""Host logic of calibrate_search (no GPU): the cells a suggestion grid spans, the searches they vary, the
global bias, and the argument checks made before any estimate (python/boitata/estimation.py:569-799)."""

import numpy as np
import pytest

import boitata_b200 as bt
from boitata_b200.calibrate import _cells, _cv_scores


def test_cells_run_cheapest_first_and_vary_every_pass():
    base = bt.Search(radius=30, max_samples=8)
    cells = _cells(base, {"max_samples": [16, 4, 8], "factors": [2, 1], "min_holes": [None, 3]})
    assert [c[:3] for c in cells] == [(m, f, h) for m in (4, 8, 16) for f in (1, 2) for h in (None, 3)]
    for m, f, h, s in cells:
        assert (s.max_samples, s.radius, s.min_holes) == (m, 30 * f, h)
    passes = _cells([base, bt.Search(radius=1e4, min_holes=2)], {"factors": [1, 3]})
    assert [[p.max_samples for p in c[3]] for c in passes] == [[8, 8], [8, 8]]
    assert [[p.min_holes for p in c[3]] for c in passes] == [[None, None], [None, None]]
    assert [c[3][1].radius for c in passes] == [1e4, 3e4]
    with pytest.raises(bt.InvalidInput, match="suggest takes max_samples, factors and min_holes, not radius"):
        _cells(base, {"radius": [1]})


def test_vary_checks_the_search_it_makes():
    s = bt.Search(radius=10, max_samples=8, min_holes=6)
    assert s._vary(2.0, 4, None).min_holes is None  # min_holes replaced before the check
    with pytest.raises(bt.InvalidInput, match="min_holes"):
        s._vary(1.0, 4, 5)
    with pytest.raises(bt.InvalidInput, match="factors"):
        s._vary(0.0, 4, None)
    sectors = bt.Search(radius=10, max_samples=12, sectors=4)
    assert sectors._vary(1.0, 20, None).max_per_sector == 5  # the default cap follows max_samples


def test_global_bias_is_the_relative_difference_of_weighted_means():
    est, data = np.array([1.0, 2.0, np.nan, 3.0]), np.array([1.0, 3.0, np.nan])
    g = bt.global_bias(est, data, weights=[1.0, 1.0, 5.0, 2.0], data_weights=[3.0, 1.0, 1.0])
    assert g["estimate_mean"] == pytest.approx((1 + 2 + 6) / 4)
    assert g["data_mean"] == pytest.approx((3 + 3) / 4)
    assert g["relative"] == pytest.approx(g["estimate_mean"] / g["data_mean"] - 1)


def test_cross_validation_scores_weight_the_estimated_samples():
    a = np.array([1.0, 2.0, 3.0, 4.0])
    e = np.array([1.5, np.nan, 2.5, 4.5])
    w = np.array([1.0, 9.0, 2.0, 1.0])
    got = _cv_scores(a, e, w)
    ok = np.isfinite(e)
    err = e[ok] - a[ok]
    assert got["cv_mean_error"] == pytest.approx(np.average(err, weights=w[ok]))
    assert got["cv_rmse"] == pytest.approx(np.sqrt(np.average(err ** 2, weights=w[ok])))
    assert np.isnan(_cv_scores(a, np.full(4, np.nan), None)["cv_slope"])


class _Fitted:
    """Stands in for a fitted estimator: the argument checks read only its sample values."""

    values = np.arange(5.0)


def test_arguments_are_checked_before_estimating():
    s = bt.Search(radius=10)
    with pytest.raises(bt.InvalidInput, match="sequence of scenarios"):
        bt.calibrate_search(_Fitted(), s, [[0.0, 0.0]])
    with pytest.raises(bt.InvalidInput, match="sequence of scenarios"):
        bt.calibrate_search(_Fitted(), [], [[0.0, 0.0]])
    with pytest.raises(bt.InvalidInput, match="one scenario"):
        bt.calibrate_search(_Fitted(), [s, s], [[0.0, 0.0]], suggest={})
    with pytest.raises(bt.InvalidInput, match="HermiteAnamorphosis"):
        bt.calibrate_search(_Fitted(), [s], [[0.0, 0.0]], cutoffs=[1.0])
    with pytest.raises(bt.Unsupported, match="anamorphosis"):
        bt.calibrate_search(_Fitted(), [s], [[0.0, 0.0]], cutoffs=[1.0], anamorphosis=object())
    with pytest.raises(bt.InvalidInput, match="one of domains or domain_column"):
        bt.calibrate_search(_Fitted(), [s], [[0.0, 0.0]], domains="a", domain_column="d")
    with pytest.raises(bt.InvalidInput, match="pass the fitted samples as data="):
        bt.calibrate_search(_Fitted(), [s], [[0.0, 0.0]], weights="w")
    with pytest.raises(bt.InvalidInput, match="3 weights for 5 fitted samples"):
        bt.calibrate_search(_Fitted(), [s], [[0.0, 0.0]], weights=np.ones(3))


def test_defaulted_arguments_are_keyword_only():
    """python/tests/test_estimation.py:1291-1306: arguments with defaults are keyword-only."""
    vg, s = bt.Variogram([("spherical", 1.0, 40.0)]), bt.Search(radius=50)
    xy, z = np.zeros((3, 2)), np.zeros(3)
    ok = bt.OrdinaryKriging(vg, s)
    for call in (lambda: ok.fit(xy, z, None), lambda: ok.predict(xy, True), lambda: bt.global_bias(z, z, None),
                 lambda: bt.calibrate_search(ok, [s], xy, 5), lambda: ok.cross_validate(5)):
        with pytest.raises(TypeError):
            call()


@pytest.mark.parametrize(("options", "match"), [({"discretization": (0, 4, 1)}, "discretization"),
                                                 ({"size": (10, float("nan"))}, "size"),
                                                 ({"size": (10, 0)}, "size"), ({"size": (10, -1, 5)}, "size")])
def test_block_kriging_rejects_bad_support(options, match):
    """python/tests/test_estimation.py:1040-1052."""
    vg, s = bt.Variogram([("spherical", 1.0, 40.0)]), bt.Search(radius=50)
    with pytest.raises(bt.InvalidInput, match=match):
        bt.BlockKriging(vg, s, **{"size": (10, 10), **options})


def test_weight_declustering_needs_a_kriging_estimator():
    with pytest.raises(bt.InvalidInput, match="linear in the data"):
        bt.weight_declustering(np.zeros((3, 2)), np.zeros(3), np.zeros((2, 2)), estimator=object())
    d = bt.Declustering(weights=np.ones(2), mean=1.0, cell_size=float("nan"))
    assert d.mean == 1.0 and np.isnan(d.cell_size)
