"""Estimator persistence in the reference's Parquet format (crates/py/src/persist.rs, crates/io/src/parquet.rs):
the JSON envelope under the "boitata" key with serde's names and tags, unfitted round trips, and the errors
the reference's tests expect (python/tests/test_persist.py:209-247). Fitted round trips run on the GPU."""

import json
import math

import numpy as np
import pyarrow.parquet as pq
import pytest

import boitata_b200 as bt
from boitata_b200 import persist


def model():
    return bt.Variogram([bt.Structure("spherical", 0.7, 40.0), bt.Structure("matern", 0.2, 90.0, order=2.5)],
                        nugget=0.1, rotation=(30.0, 10.0, 0.0), ratios=(0.5, 0.25))


def test_envelope_follows_serde_names_order_and_tags():
    s = bt.Search(float("inf"), max_samples=12, min_samples=2, octant=True, max_per_sector=3, target_slope=0.9)
    est = bt.OrdinaryKriging(model(), [s, bt.Search(60.0, sectors=6, min_holes=2)])
    d = json.loads(persist.envelope(est))
    assert list(d)[:3] == ["type", "format", "fitted"] and d["type"] == "OrdinaryKriging" and d["format"] == 1
    assert d["fitted"] is False and d["method"] == {"Kriging": "Ordinary"}
    assert d["variogram"] == {
        "nugget": 0.1,
        "structures": [{"model": "Spherical", "sill": 0.7, "range": 40.0},
                       {"model": {"Matern": {"order": 2.5}}, "sill": 0.2, "range": 90.0}],
        "anisotropy": {"azimuth": 30.0, "dip": 10.0, "rake": 0.0, "major": 1.0, "semi": 0.5, "minor": 0.25},
    }
    first, second = d["search"]
    assert list(first) == ["min_samples", "max_samples", "radius", "max_per_hole", "octant", "anisotropy",
                           "high_grade", "calibration", "max_per_octant"]
    assert first["radius"] == "inf" and first["calibration"] == {"slope": 0.9} and first["max_per_octant"] == 3
    assert second["sectors"] == {"count": 6, "max_per_sector": 3} and second["min_holes"] == 2
    assert d["drift_data"] == [] and d["units"] == [None, None, None]
    sk = json.loads(persist.envelope(bt.SimpleKriging(model(), bt.Search(30.0), mean=2.5)))
    assert sk["method"] == {"Kriging": {"Simple": {"mean": 2.5}}}
    ik = json.loads(persist.envelope(bt.IndicatorKriging(model(), s, 1.2)))
    assert ik["method"] == {"Kriging": {"Indicator": {"threshold": 1.2}}}
    bk = json.loads(persist.envelope(bt.BlockKriging(model(), s, (10.0, 10.0, 5.0), discretization=(3, 3, 2))))
    assert bk["method"] == {"Block": {"size": [10.0, 10.0, 5.0], "disc": {"nx": 3, "ny": 3, "nz": 2},
                                      "rotation": [0.0, 0.0, 0.0]}}
    power = bt.Variogram([bt.Structure("power", 0.5, 10.0, exponent=1.5)])
    assert json.loads(persist.envelope(bt.OrdinaryKriging(power, s)))["variogram"]["structures"][0]["model"] == {
        "Power": {"exponent": 1.5}}


@pytest.mark.parametrize("make", [
    lambda s: bt.OrdinaryKriging(model(), [s, s.scaled(2.0, min_samples=1)]),
    lambda s: bt.SimpleKriging(model(), s, mean=-1.5),
    lambda s: bt.IndicatorKriging(model(), s, 0.75),
    lambda s: bt.BlockKriging(model(), s, (20.0, 10.0, 5.0), discretization=(2, 3, 1)),
])
def test_unfitted_round_trip_keeps_every_parameter(tmp_path, make):
    s = bt.Search(ranges=(80.0, 40.0, 20.0), rotation=(15.0, 0.0, 5.0), max_samples=24, min_samples=3,
                  octant=True, max_per_sector=4, min_sectors=3, max_empty_sectors=2, target_efficiency=0.4)
    est = make(s)
    path = tmp_path / "model.parquet"
    est.to_parquet(path)
    back = type(est).from_parquet(path)
    assert type(back) is type(est)
    assert json.loads(persist.envelope(back)) == json.loads(persist.envelope(est))
    assert pq.read_table(path).num_rows == 0


def test_wrong_class_missing_file_and_newer_format(tmp_path):
    path = tmp_path / "ok.parquet"
    bt.OrdinaryKriging(model(), bt.Search(30.0)).to_parquet(path)
    with pytest.raises(bt.InvalidInput, match="expected a SimpleKriging"):
        bt.SimpleKriging.from_parquet(path)
    with pytest.raises(bt.FileError):
        bt.OrdinaryKriging.from_parquet(tmp_path / "missing.parquet")
    table = pq.read_table(path)
    meta = json.loads(table.schema.metadata[b"boitata"])
    meta["format"] = 2
    pq.write_table(table.replace_schema_metadata({b"boitata": json.dumps(meta).encode()}), tmp_path / "new.parquet")
    with pytest.raises(bt.InvalidInput, match="newer"):
        bt.OrdinaryKriging.from_parquet(tmp_path / "new.parquet")


def test_options_this_engine_does_not_run_are_refused(tmp_path):
    path = tmp_path / "ok.parquet"
    bt.OrdinaryKriging(model(), bt.Search(30.0)).to_parquet(path)
    table = pq.read_table(path)
    meta = json.loads(table.schema.metadata[b"boitata"])
    meta["search"][0]["high_grade"] = {"threshold": 5.0, "radius": 10.0}
    pq.write_table(table.replace_schema_metadata({b"boitata": json.dumps(meta).encode()}), tmp_path / "hg.parquet")
    with pytest.raises(bt.Unsupported, match="high-grade"):
        bt.OrdinaryKriging.from_parquet(tmp_path / "hg.parquet")


def test_nonfinite_floats_are_strings():
    assert persist._num(math.inf) == "inf" and persist._num(-math.inf) == "-inf" and persist._num(math.nan) == "NaN"
    assert persist._unnum("inf", "r") == math.inf and math.isnan(persist._unnum("NaN", "r"))
    assert persist._unnum(3, "r") == 3.0 and isinstance(persist._unnum(3, "r"), float)
    with pytest.raises(bt.InvalidInput):
        persist._unnum("x", "r")
    assert np.isnan(persist._unnum("NaN", "r"))


def test_parameters_round_trip_through_json_and_pickle():
    """Variogram, Structure and Search to_json / from_json (crates/py/src/variogram.rs:196-208, 569-579,
    estimation.rs:401-412) and pickle give the same JSON back; an infinite radius survives; the envelope's
    type and format are checked (python/tests/test_persist.py:121-135 of the reference)."""
    import pickle

    objs = [bt.Variogram([("spherical", 0.7, 50.0), bt.Structure("matern", 0.2, 30.0, order=2.5)], nugget=0.1,
                         rotation=(30.0, 10.0, 0.0), ratios=(0.5, 0.2)),
            bt.Structure("exponential", 1.0, 30.0), bt.Structure("power", 1.0, 1.0, exponent=1.5),
            bt.Search(np.inf, rotation=(10.0, 0.0, 0.0), ratios=(0.5, 0.5)),
            bt.Search(30.0, sectors=6, max_per_sector=2, min_holes=2, target_efficiency=0.5)]
    for obj in objs:
        for back in (type(obj).from_json(obj.to_json()), pickle.loads(pickle.dumps(obj))):
            assert type(back) is type(obj) and back.to_json() == obj.to_json()
    assert bt.Search.from_json(bt.Search(np.inf).to_json()).radius == np.inf
    text = objs[0].to_json()
    assert text.startswith('{"type":"Variogram","format":1,"nugget":0.1,"structures":[{"model":"Spherical"')
    with pytest.raises(bt.InvalidInput, match="expected a Search"):
        bt.Search.from_json(text)
    with pytest.raises(bt.InvalidInput, match=r"^format 2 is newer"):
        bt.Variogram.from_json(text.replace('"format":1', '"format":2'))
