"""CPU-side checks: the C ABI library loads and exports every declared entry
point, and the host layer validates parameters as the reference does."""

import ctypes
import os
import re
import warnings

import numpy as np
import pytest

import boitata_b200 as bt
from boitata_b200 import _native
from boitata_b200.estimation import distinct, points

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"\b(btk_[a-z_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_entry_point():
    from boitata_b200 import build

    if not os.path.exists(_native.LIB_PATH):
        build.build()
    lib = ctypes.CDLL(_native.LIB_PATH)
    names = declared()
    assert "btk_predict_geometry_device" in names and len(names) >= 12
    for name in names:
        assert hasattr(lib, name), name
    assert set(_native.SIGNATURES) <= set(names)
    assert lib.btk_version  # loads without a GPU


def test_engine_refuses_to_run_without_a_cuda_device():
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    with pytest.raises(_native.EngineError, match="CUDA"):
        bt.OrdinaryKriging(bt.Variogram([("spherical", 1.0, 10.0)]), bt.Search(radius=5)).fit(
            [[0.0, 0.0], [1.0, 1.0]], [1.0, 2.0])


def test_search_constructor_rules():
    """crates/py/src/estimation.rs:414-510 and search.rs:214-264."""
    with pytest.raises(bt.InvalidInput, match="radius or ranges, not both"):
        bt.Search(radius=10, ranges=(10, 10, 10))
    with pytest.raises(bt.InvalidInput, match="give radius or ranges"):
        bt.Search()
    with pytest.raises(bt.InvalidInput, match="ratios with radius"):
        bt.Search(ranges=(10, 5, 2), ratios=(0.5, 0.5))
    with pytest.raises(bt.InvalidInput, match="max_per_sector needs octant"):
        bt.Search(radius=10, max_per_sector=2)
    with pytest.raises(bt.InvalidInput, match="min_samples <= max_samples"):
        bt.Search(radius=10, min_samples=20, max_samples=16)
    with pytest.raises(bt.InvalidInput, match="min_sectors and max_empty_sectors need"):
        bt.Search(radius=10, min_sectors=2)
    s = bt.Search(ranges=(300, 300, 100), max_samples=16)
    assert s.radius == 300 and s.anisotropy == (0.0, 0.0, 0.0, 1.0, 1.0, 1.0 / 3.0)
    o = bt.Search(radius=250, octant=True, max_per_sector=4, max_samples=32)
    assert o.max_per_octant == 4 and o.anisotropy is None
    c = o.to_c()
    assert c.octant == 1 and c.max_per_octant == 4 and c.max_per_hole == -1


def test_variogram_constructor_rules():
    """crates/py/src/variogram.rs:164-177, 328-361 and model.rs:47-59."""
    with pytest.raises(bt.InvalidInput, match="nugget"):
        bt.Variogram([("spherical", 1.0, 10.0)], nugget=-1)
    with pytest.raises(bt.InvalidInput, match="unknown model"):
        bt.Variogram([("sphere", 1.0, 10.0)])
    with pytest.raises(bt.InvalidInput, match="range finite and > 0"):
        bt.Structure("spherical", 1.0, 0.0)
    vg = bt.Variogram([("Spherical", 0.5, 80.0), bt.Structure("matern", 0.45, 250.0)], nugget=0.05)
    assert vg.anisotropy is None and vg.total_sill() == pytest.approx(1.0)
    assert vg.structures[1].order == 1.5
    assert bt.Variogram([("hole", 1, 10)]).structures[0].model == "sinehole"
    assert bt.Variogram([("spherical", 1, 10)], rotation=(30, 10, 0), ratios=(0.75, 0.25)).anisotropy == (
        30.0, 10.0, 0.0, 1.0, 0.75, 0.25)


def test_simple_kriging_rejects_a_variogram_without_a_sill():
    """python/tests/test_estimation.py:38-44."""
    power = bt.Variogram([("power", 1.0, 1.5)])
    with pytest.raises(bt.InvalidInput, match="simple kriging needs a variogram with a sill"):
        bt.SimpleKriging(power, bt.Search(radius=1000), mean=1.0)


def test_fit_drops_samples_sharing_a_location_with_a_warning():
    """crates/py/src/args.rs:318-376: the first of each group is kept; -0 equals 0."""
    locs = points([[0.0, 0.0], [1.0, 1.0], [-0.0, 0.0], [2.0, 2.0], [1.0, 1.0]])
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        keep = distinct(locs, ["a", "b", "c", "d", "e"])
    assert keep.tolist() == [0, 1, 3]
    assert "2 locations hold several samples" in str(w[0].message) and "holes a, c" in str(w[0].message)
    assert distinct(points([[0.0, 0.0], [1.0, 0.0]])).tolist() == [0, 1]


def test_coordinates_and_values_must_be_finite():
    with pytest.raises(bt.InvalidInput, match="finite"):
        points([[0.0, np.nan]])
    with pytest.raises(bt.InvalidInput, match="shape"):
        points([[0.0, 1.0, 2.0, 3.0]])
    assert points([[1.0, 2.0]]).tolist() == [[1.0, 2.0, 0.0]]


def test_block_kriging_arguments_are_checked_as_the_reference_does():
    """crates/py/src/estimation.rs:1414-1439: size finite and > 0, discretization at least 1 per axis."""
    import pytest

    from boitata_b200 import BlockKriging, InvalidInput, Search, Structure, Variogram

    vg = Variogram([Structure("spherical", 1.0, 100.0)])
    s = Search(radius=100.0, max_samples=8)
    for size, disc in [((10.0, 0.0, 10.0), (4, 4, 1)), ((10.0, float("nan"), 1.0), (4, 4, 1)),
                       ((10.0, 10.0, -1.0), (4, 4, 1)), ((10.0, 10.0, 10.0), (0, 4, 1)),
                       ((10.0, 10.0, 10.0), (4, 4)), ((10.0,), (4, 4, 1))]:
        with pytest.raises(InvalidInput):
            BlockKriging(vg, s, size, discretization=disc)
    b = BlockKriging(vg, s, (10.0, 20.0))
    assert b.size == (10.0, 20.0, 1.0) and b.discretization == (4, 4, 1)


def test_table_columns_rows_and_exchange():
    from boitata_b200 import Table

    t = Table({"value": np.array([1.0, np.nan, 3.0]), "pass": np.array([1.0, np.nan, 2.0])})
    assert t.column_names == ["value", "pass"] and t.num_rows == 3 and len(t) == 3
    np.testing.assert_array_equal(t["pass"], [1.0, np.nan, 2.0])
    f = t.filter(np.isfinite(t["value"]))
    assert f.num_rows == 2 and f["value"].tolist() == [1.0, 3.0]
    assert t.with_column("slope", np.ones(3)).column_names == ["value", "pass", "slope"]
    assert t.to_pyarrow().column_names == ["value", "pass"]
    assert list(t.to_pandas().columns) == ["value", "pass"]
    with pytest.raises(KeyError):
        t["missing"]
    with pytest.raises(bt.InvalidInput):
        Table({"a": np.ones(2), "b": np.ones(3)})


def test_oracle_diagnostics_columns(oracle):
    """The oracle's neighborhood_stats restatement on a hand-made case: distances 1, 2 (sorted), two holes."""
    xyz = np.array([[2.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.5, 0.0]])
    s = bt.Search(radius=10.0, max_samples=2, min_samples=1)
    vg = bt.Variogram([bt.Structure("spherical", 1.0, 10.0)])
    r = oracle.estimate_many(np.zeros((1, 3)), xyz, [1.0, 2.0, 3.0], s, vg, holes=np.array([5, 5, 6]),
                             neighbors=False, diagnostics=True)
    assert r["n_used"][0] == 2 and r["n_within"][0] == 2
    assert r["mean_distance"][0] == pytest.approx((1.0 + 1.5) / 2)
    assert r["n_holes"][0] == 2
    r = oracle.estimate_many(np.zeros((1, 3)), xyz, [1.0, 2.0, 3.0], bt.Search(radius=10.0, max_samples=3), vg,
                             holes=np.array([5, 5, 6]), neighbors=False, diagnostics=True)
    assert r["n_holes"][0] == 2 and r["mean_distance"][0] == pytest.approx(4.5 / 3)
    assert r["negative_weight_sum"][0] <= 0.0


def test_ctypes_mirrors_match_the_c_header_layouts(tmp_path):
    """Every struct the Python layer passes through the C ABI has the size and field offsets of its
    declaration in include/boitata_b200.h (a C probe compiled with gcc prints them)."""
    import subprocess

    pairs = {"btk_aniso": _native.Aniso, "btk_structure": _native.StructureC, "btk_variogram": _native.VariogramC,
             "btk_search": _native.SearchC, "btk_geometry": _native.GeometryC, "btk_tuning": _native.TuningC,
             "btk_outputs": _native.OutputsC, "btk_diagnostics": _native.DiagnosticsC}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "boitata_b200.h"', "int main(void) {"]
    for cname, py in pairs.items():
        lines.append(f'  printf("{cname} :sizeof %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src, exe = tmp_path / "probe.c", tmp_path / "probe"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        cname, key, value = line.split()
        got[(cname, key)] = int(value)
    for cname, py in pairs.items():
        assert got[(cname, ":sizeof")] == ctypes.sizeof(py), cname
        for field, _ in py._fields_:
            assert got[(cname, field)] == getattr(py, field).offset, (cname, field)


def test_block_model_takes_the_reference_constructor():
    from boitata_b200.errors import InvalidInput, Unsupported

    m = bt.BlockModel((1.0, 2.0, 3.0), (2.5, 2.5, 1.0), (4, 3, 2), rotation=(30.0, 0.0, 0.0))
    assert (m.origin, m.size, m.count, m.rotation) == ((1.0, 2.0, 3.0), (2.5, 2.5, 1.0), (4, 3, 2), (30.0, 0.0, 0.0))
    assert len(m) == 24 and isinstance(m.geometry, bt.Geometry)
    g = bt.Geometry((0, 0, 0), (1, 1, 1), (2, 2, 2))
    assert bt.BlockModel(g).geometry is g
    with pytest.raises(InvalidInput):
        bt.BlockModel((0, 0, 0), (1, 1, 1))
    with pytest.raises(InvalidInput):
        bt.BlockModel(g, (1, 1, 1), (2, 2, 2))
    with pytest.raises(Unsupported):
        bt.BlockModel((0, 0, 0), (1, 1, 1), (2, 2, 2), index=[0, 3])
    flat = bt.BlockModel(origin=(5.0, 5.0), size=(10, 10), count=(20, 20))
    assert (flat.origin, flat.size, flat.count, len(flat)) == ((5.0, 5.0, 0.0), (10.0, 10.0, 1.0), (20, 20, 1), 400)


def test_search_passes_scale_the_ellipsoid():
    """Search.passes / scaled (crates/py/src/estimation.rs:276-307, 511-557): the ellipsoid widened by each
    factor, rotation and rules kept, plane sectors at their default cap follow a new max_samples."""
    base = bt.Search(ranges=(40, 20, 10), rotation=(45, 0, 0), max_samples=12, sectors=4, min_holes=2)
    passes = bt.Search.passes(base)
    assert [p.ranges for p in passes] == [(40, 20, 10), (80, 40, 20), (120, 60, 30)]
    assert all((p.rotation, p.sectors, p.min_holes, p.max_samples) == ((45, 0, 0), 4, 2, 12) for p in passes)
    custom = bt.Search.passes(base, (1, 1.5), min_samples=(4, 2), max_samples=(12, 24))
    assert [(p.radius, p.min_samples, p.max_samples, p.max_per_sector) for p in custom] == [
        (40, 4, 12, 3), (60, 2, 24, 6)]
    kept = bt.Search.passes(bt.Search(radius=40, sectors=4, max_per_sector=2), (1, 2), max_samples=(16, 32))
    assert [p.max_per_sector for p in kept] == [2, 2]
    for bad in ({"factors": ()}, {"factors": (1, -2)}, {"factors": (1, float("inf"))}, {"max_samples": (8,)},
                {"min_samples": (20, 20, 20)}):
        with pytest.raises(bt.InvalidInput):
            bt.Search.passes(base, **bad)
    s = bt.Search(radius=50, octant=True, max_per_hole=3, rotation=(30, 10, 5), ratios=(0.5, 0.2))
    assert (s.octant, s.max_per_hole, s.rotation, s.ratios) == (True, 3, (30, 10, 5), (0.5, 0.2))
    plain = bt.Search(radius=50)
    assert not plain.octant
    assert plain.max_per_hole is plain.rotation is plain.ratios is plain.ranges is None


def test_sector_and_hole_rules_are_checked_and_kept():
    """The rules round-trip through Search.to_json / from_json (crates/py/src/estimation.rs:401-412) and
    the constructor rejects what search.rs:214-264 rejects."""
    s = bt.Search(radius=50, octant=True, max_per_sector=2, min_sectors=3, max_empty_sectors=1, min_holes=2)
    assert (s.max_per_sector, s.min_sectors, s.max_empty_sectors, s.min_holes) == (2, 3, 1, 2)
    back = bt.Search.from_json(s.to_json())
    assert (back.max_per_sector, back.min_sectors, back.max_empty_sectors, back.min_holes) == (2, 3, 1, 2)
    assert s.to_json().startswith('{"type":"Search","format":1,"min_samples":1,"max_samples":16,"radius":50.0')
    plain = bt.Search.from_json(bt.Search(radius=50, octant=True).to_json())
    assert plain.max_per_sector is plain.min_sectors is plain.max_empty_sectors is plain.min_holes is None
    aniso = bt.Search(ranges=(40, 20, 10), rotation=(45, 10, 5), sectors=4, max_samples=12, target_slope=0.9)
    again = bt.Search.from_json(aniso.to_json())
    assert (again.ranges, again.rotation, again.sectors, again.max_per_sector, again.target_slope) == (
        (40, 20, 10), (45, 10, 5), 4, 3, 0.9)
    with pytest.raises(bt.InvalidInput, match="expected a Search"):
        bt.Search.from_json('{"type":"Variogram","format":1}')
    with pytest.raises(bt.InvalidInput, match="newer"):
        bt.Search.from_json(s.to_json().replace('"format":1', '"format":2'))
    for bad in ({"min_sectors": 2}, {"max_empty_sectors": 1}, {"octant": True, "min_sectors": 9},
                {"octant": True, "min_sectors": 0}, {"octant": True, "max_empty_sectors": 4},
                {"sectors": 6, "min_sectors": 7}, {"sectors": 6, "max_empty_sectors": 6},
                {"octant": True, "max_per_sector": 0}, {"min_holes": 0}, {"min_holes": 17}):
        with pytest.raises(bt.InvalidInput):
            bt.Search(radius=50, **bad)


def test_cross_validation_summary_statistics():
    """CrossValidation's rmse, slope and standardized error (python/boitata/estimation.py:110-145) over the
    estimated samples only."""
    from boitata_b200.estimation import CrossValidation

    r = np.random.default_rng(0)
    actual = r.normal(size=50)
    est = 0.7 * actual + 0.3 * r.normal(size=50)
    est[3] = np.nan
    cv = CrossValidation(actual, est, np.full(50, 0.25))
    ok = ~np.isnan(est)
    assert cv.rmse == pytest.approx(np.sqrt(np.mean((est[ok] - actual[ok]) ** 2)), rel=1e-14)
    assert cv.slope == pytest.approx(np.polyfit(est[ok], actual[ok], 1)[0], rel=1e-12)
    assert cv.standardized_squared_error == pytest.approx(np.mean((est[ok] - actual[ok]) ** 2) / 0.25, rel=1e-14)


def test_point_sets_and_named_columns():
    """PointSet / BlockModel attribute columns (crates/py/src/containers.rs:75-210) and the estimators'
    column arguments (python/boitata/estimation.py:226-330, _columns.py:13-27), checked before any device
    work."""
    r = np.random.default_rng(3)
    xy = r.uniform(0, 100, (150, 2))
    zone = np.where(xy[:, 0] < 50, "W", "E")
    samples = bt.PointSet(xy, {"grade": np.sin(xy[:, 0] / 15), "zone": zone})
    assert len(samples) == 150 and samples.coords.shape == (150, 3) and not samples.coords[:, 2].any()
    assert samples.column_names == ["grade", "zone"] and "zone" in samples
    np.testing.assert_array_equal(samples["zone"], zone)
    w = samples.with_column("w", np.linspace(1, 2, 150))
    assert w.column_names == ["grade", "zone", "w"] and samples.column_names == ["grade", "zone"]
    with pytest.raises(bt.MissingColumn, match='did you mean "grade"'):
        samples["grades"]
    with pytest.raises(KeyError):
        samples["rock"]
    with pytest.raises(bt.InvalidInput, match="expected 150"):
        samples.with_column("short", np.zeros(3))
    with pytest.raises(bt.InvalidInput, match="expected 150"):
        bt.PointSet(xy, {"bad": np.zeros(4)})
    blocks = bt.BlockModel(origin=(0, 0), size=(10, 10), count=(10, 10), attributes={"zone": np.arange(100) % 2})
    assert blocks.column_names == ["zone"] and blocks.with_column("ok", np.ones(100))["ok"].shape == (100,)
    ok = bt.OrdinaryKriging(bt.Variogram([("spherical", 1.0, 40.0)]), bt.Search(radius=50))
    with pytest.raises(bt.InvalidInput, match="one of domains or domain_column"):
        ok.fit(samples, "grade", domains=zone, domain_column="zone")
    with pytest.raises(bt.InvalidInput, match="needs a container"):
        ok.fit(xy, "grade")
    with pytest.raises(bt.MissingColumn):
        ok.fit(samples, "gold")
    with pytest.raises(bt.InvalidInput, match="one of domains or domain_column"):
        ok.predict(samples, domains=zone, domain_column="zone")
    with pytest.raises(bt.MissingColumn):
        ok.predict(samples, domain_column="rock")
    assert issubclass(bt.InvalidInput, bt.BoitataError) and issubclass(bt.MissingColumn, bt.BoitataError)


def test_hole_labels_are_keyed_as_the_reference_keys_them():
    """crates/py/src/args.rs:14-45, 257-292: labels keyed by their text (1, 1.0 and "1" are one hole; True and
    "true" too), None and NaN each a hole of their own, infinite labels rejected before any device work."""
    from boitata_b200.estimation import hole_codes

    np.testing.assert_array_equal(hole_codes([1, 1.0, "1", True, "true", None, np.nan, 2.5, "a"]),
                                  [0, 0, 0, 1, 1, 2, 3, 4, 5])
    np.testing.assert_array_equal(hole_codes(np.array([None] * 4, dtype=object)), [0, 1, 2, 3])
    np.testing.assert_array_equal(hole_codes(np.full(3, np.nan)), [0, 1, 2])
    for bad in ([np.inf, 1.0], [[1, 2], [3, 4]], "DH1"):
        with pytest.raises(bt.InvalidInput, match="sequence of labels"):
            hole_codes(bad)
    xy = np.random.default_rng(3).uniform(0, 100, (150, 2))
    ok = bt.OrdinaryKriging(bt.Variogram([("spherical", 1.0, 40.0)]), bt.Search(radius=50))
    with pytest.raises(bt.InvalidInput, match="holes must be a 1-D sequence of labels"):
        ok.fit(xy, xy[:, 0], holes=np.full(150, np.inf))
