"""Estimator persistence in the reference's Parquet format.

crates/py/src/persist.rs:1-203 with crates/io/src/parquet.rs:31, 146-160,
487-496 and the estimator's Tabular impl (crates/py/src/estimation.rs:
1110-1170): the fitted samples as nullable float64 columns x, y, z, value,
hole, error_variance and domain (null where a sample has none), and the
parameters as one JSON object under the schema metadata key "boitata":

    {"type": <class name>, "format": 1, "fitted": <bool>, "method": ...,
     "variogram": ..., "search": [...], "drift_data": [], "units": [...]}

with serde's field names, field order and enum tags for the estimator's
`method` (Kind / Block), the variogram (crates/variogram/src/{composite,
model,aniso}.rs) and each search pass (crates/estimation/src/search.rs:31-
100, flattened into the Python Search with its length_unit). Floats that
may be infinite or NaN are written as "inf", "-inf", "NaN"
(crates/core/src/nonfinite.rs). A file the reference wrote loads here and
predicts as the saved estimator did; options this engine does not run
(high-grade, soft boundaries, external drift) raise Unsupported.
"""

import json
import math
import os

import numpy as np

from .errors import InvalidInput, Unsupported

FORMAT = 1
KEY = b"boitata"
ROW_GROUP = 1 << 20
COLUMNS = ("x", "y", "z", "value", "hole", "error_variance", "domain")

_MODEL_NAMES = {"spherical": "Spherical", "exponential": "Exponential", "gaussian": "Gaussian", "cubic": "Cubic",
                "pentaspherical": "PentaSpherical", "circular": "Circular", "sinehole": "SineHole"}
_MODEL_KEYS = {v: k for k, v in _MODEL_NAMES.items()}


class FileError(InvalidInput, OSError):
    """A file that cannot be read or written (the reference's boitata.errors.FileError)."""


def _num(v):
    """nonfinite.rs: finite floats as numbers, the others as "NaN", "inf", "-inf"."""
    v = float(v)
    if math.isfinite(v):
        return v
    return "NaN" if math.isnan(v) else ("inf" if v > 0 else "-inf")


def _unnum(v, what):
    if isinstance(v, bool) or v is None:
        raise InvalidInput(f"{what}: expected a number")
    if isinstance(v, (int, float)):
        return float(v)
    table = {"NaN": math.nan, "inf": math.inf, "-inf": -math.inf}
    if v not in table:
        raise InvalidInput(f"{what}: {v!r} is not a number")
    return table[v]


def _angles(a):
    """aniso.rs:17-25 (Angles): azimuth, dip, rake, major, semi, minor."""
    if a is None:
        return None
    return dict(zip(("azimuth", "dip", "rake", "major", "semi", "minor"), (float(x) for x in a)))


def _unangles(d, what):
    """(rotation, ratios) of serialized Angles; this engine's ellipsoids have a major range of 1."""
    if d is None:
        return (0.0, 0.0, 0.0), (1.0, 1.0)
    rake = d["rake"] if "rake" in d else d.get("pitch")
    major = float(d["major"])
    if major != 1.0:
        raise Unsupported(f"{what}: anisotropy with a major range of {major} (this engine takes ratios, major 1)")
    return (float(d["azimuth"]), float(d["dip"]), float(rake)), (float(d["semi"]), float(d["minor"]))


def variogram_json(vg):
    """composite.rs:12-18, model.rs:10-40."""
    structures = []
    for s in vg.structures:
        if s.model == "matern":
            model = {"Matern": {"order": float(s.order)}}
        elif s.model == "power":
            model = {"Power": {"exponent": float(s.exponent)}}
        else:
            model = _MODEL_NAMES[s.model]
        structures.append({"model": model, "sill": float(s.sill), "range": float(s.range)})
    return {"nugget": float(vg.nugget), "structures": structures, "anisotropy": _angles(vg.anisotropy)}


def variogram_from(d):
    from .variogram import Structure, Variogram

    if d is None:
        raise Unsupported("an estimator without a variogram is not run by this engine")
    out = []
    for s in d["structures"]:
        m = s["model"]
        if isinstance(m, str):
            if m not in _MODEL_KEYS:
                raise InvalidInput(f"unknown variogram model {m!r}")
            out.append(Structure(_MODEL_KEYS[m], s["sill"], s["range"]))
        elif "Matern" in m:
            out.append(Structure("matern", s["sill"], s["range"], order=m["Matern"]["order"]))
        elif "Power" in m:
            out.append(Structure("power", s["sill"], s["range"], exponent=m["Power"]["exponent"]))
        else:
            raise InvalidInput(f"unknown variogram model {m!r}")
    rotation, ratios = _unangles(d.get("anisotropy"), "variogram")
    return Variogram(out, nugget=d["nugget"], rotation=rotation, ratios=ratios)


def search_json(s):
    """search.rs:31-81 in field order, optional fields skipped when None as serde skips them; the Python
    Search's own soft and length_unit (crates/py/src/estimation.rs:211-221) are None here."""
    out = {"min_samples": int(s.min_samples), "max_samples": int(s.max_samples), "radius": _num(s.radius),
           "max_per_hole": None if s.max_per_hole is None else int(s.max_per_hole), "octant": bool(s.octant)}
    if s.sectors is not None:
        out["sectors"] = {"count": int(s.sectors), "max_per_sector": int(s.max_per_sector)}
    out["anisotropy"] = _angles(s.anisotropy)
    out["high_grade"] = None
    if s.target_slope is not None:
        out["calibration"] = {"slope": _num(s.target_slope)}
    elif s.target_efficiency is not None:
        out["calibration"] = {"efficiency": _num(s.target_efficiency)}
    for key in ("max_per_octant", "min_sectors", "max_empty_sectors", "min_holes"):
        v = getattr(s, key)
        if v is not None:
            out[key] = int(v)
    return out


def search_from(d):
    from .search import Search

    if d.get("high_grade") is not None:
        raise Unsupported("high-grade restrictions are not run by this engine")
    if d.get("soft") is not None:
        raise Unsupported("soft domain boundaries are not run by this engine")
    rotation, ratios = _unangles(d.get("anisotropy"), "search")
    cal = d.get("calibration") or {}
    sectors = d.get("sectors")
    kw = dict(max_samples=int(d["max_samples"]), min_samples=int(d["min_samples"]), octant=bool(d["octant"]),
              max_per_hole=d.get("max_per_hole"), min_sectors=d.get("min_sectors"),
              max_empty_sectors=d.get("max_empty_sectors"), min_holes=d.get("min_holes"))
    if sectors is not None:
        kw.update(sectors=int(sectors["count"]), max_per_sector=int(sectors["max_per_sector"]))
    elif d.get("max_per_octant") is not None:
        kw.update(max_per_sector=int(d["max_per_octant"]))
    if "slope" in cal:
        kw["target_slope"] = _unnum(cal["slope"], "target_slope")
    if "efficiency" in cal:
        kw["target_efficiency"] = _unnum(cal["efficiency"], "target_efficiency")
    if d.get("anisotropy") is not None:
        kw.update(rotation=rotation, ratios=ratios)
    return Search(_unnum(d["radius"], "radius"), **kw)


def method_json(est):
    """The estimator's Method (crates/py/src/estimation.rs:696-725) with its Kind (krige.rs:19-27)."""
    from .estimation import BlockKriging, IndicatorKriging, SimpleKriging

    if isinstance(est, BlockKriging):
        nx, ny, nz = est.discretization
        return {"Block": {"size": [float(v) for v in est.size], "disc": {"nx": nx, "ny": ny, "nz": nz},
                          "rotation": [0.0, 0.0, 0.0]}}
    if isinstance(est, SimpleKriging):
        return {"Kriging": {"Simple": {"mean": float(est.mean)}}}
    if isinstance(est, IndicatorKriging):
        return {"Kriging": {"Indicator": {"threshold": float(est.threshold)}}}
    return {"Kriging": "Ordinary"}


def envelope_of(name, fields):
    """persist.rs:20-33: {"type": name, "format": 1, <fields>...}, compact, non-finite floats as strings."""
    return json.dumps({"type": name, "format": FORMAT, **fields}, separators=(",", ":"), allow_nan=False)


def envelope(est):
    """persist.rs:20-33 and :85-92: type and format first, then fitted, then the estimator's fields."""
    fields = {"type": type(est).__name__, "format": FORMAT, "fitted": est._samples is not None,
              "method": method_json(est), "variogram": variogram_json(est.variogram),
              "search": [search_json(s) for s in est.searches], "drift_data": [], "units": [None, None, None],
              "precision": est.precision}  # this engine's own field; serde ignores unknown fields
    labels = getattr(est, "_domain_labels", None)
    if labels is not None:  # the fitted domain labels, indexed by the domain column's codes
        fields["domains"] = [_label_json(v) for v in labels]
    return json.dumps(fields, separators=(",", ":"), allow_nan=False)


def _label_json(v):
    """A domain label as JSON: string, boolean, or number (integral numbers as integers)."""
    if isinstance(v, (bool, np.bool_)):
        return bool(v)
    if isinstance(v, str):
        return v
    f = float(v)
    return int(f) if f == int(f) and abs(f) < 9e15 else f


def columns(est):
    """sample_columns (crates/py/src/estimation.rs:1110-1122) of the fitted samples, or None."""
    if est._samples is None:
        return None
    locs, vals, err = est._samples
    n = len(vals)
    holes = getattr(est, "_holes", None)
    return {"x": locs[:, 0].astype(np.float64), "y": locs[:, 1].astype(np.float64),
            "z": locs[:, 2].astype(np.float64), "value": np.asarray(vals, dtype=np.float64),
            "hole": None if holes is None else np.asarray(holes, dtype=np.float64),
            "error_variance": np.zeros(n) if err is None else np.asarray(err, dtype=np.float64),
            "domain": None if getattr(est, "_domains", None) is None else np.asarray(est._domains, dtype=np.float64),
            "_rows": n}


def to_parquet(est, path):
    import pyarrow as pa
    import pyarrow.parquet as pq

    meta = envelope(est)
    cols = columns(est) or {"_rows": 0}
    n = cols.pop("_rows")
    arrays = []
    for name in (COLUMNS if est._samples is not None else ()):
        v = cols.get(name)
        arrays.append(pa.nulls(n, pa.float64()) if v is None else pa.array(v, type=pa.float64()))
    fields = [pa.field(name, pa.float64(), nullable=True) for name in (COLUMNS if arrays else ())]
    schema = pa.schema(fields, metadata={KEY: meta.encode()})
    table = pa.Table.from_arrays(arrays, schema=schema) if arrays else pa.Table.from_pylist([], schema=schema)
    try:
        pq.write_table(table, os.fspath(path), compression="zstd", row_group_size=ROW_GROUP,
                       data_page_version="2.0")
    except OSError as e:
        raise FileError(f"cannot write {os.fspath(path)}: {e}") from e


def _open(name, text):
    """persist.rs:35-51: the envelope's fields once its type and format are checked."""
    try:
        d = json.loads(text)
    except ValueError as e:
        raise InvalidInput(f"boitata metadata is not JSON: {e}") from None
    if not isinstance(d, dict):
        raise InvalidInput("expected a JSON object")
    found = d.pop("type", None)
    if found != name:
        raise InvalidInput(f"expected a {name}, found {json.dumps(found)}")
    fmt = d.pop("format", None)
    if isinstance(fmt, bool) or not isinstance(fmt, int) or fmt < 0:
        raise InvalidInput("missing or invalid format number")
    if fmt > FORMAT:
        raise InvalidInput(f"format {fmt} is newer than this boitata reads (up to {FORMAT}); upgrade boitata")
    return d


def from_parquet(cls, path):
    import pyarrow.parquet as pq

    path = os.fspath(path)
    if not os.path.exists(path):
        raise FileError(f"no such file: {path}")
    try:
        table = pq.read_table(path)
    except OSError as e:
        raise FileError(f"cannot read {path}: {e}") from e
    meta = (table.schema.metadata or {}).get(KEY)
    if meta is None:
        raise InvalidInput("no boitata metadata")
    d = _open(cls.__name__, meta.decode())
    fitted = d.pop("fitted", None) is True
    labels = d.get("domains")
    if d.get("drift_data"):
        raise Unsupported("external-drift estimators are not run by this engine")
    est = _build(cls, d)
    if d.get("precision") in ("fp64", "mixed"):
        est.precision = d["precision"]
    if fitted:
        got = {}
        for name in table.column_names:
            col = table.column(name)
            if str(col.type) != "double":
                raise InvalidInput(f"column {name} is not float64")
            got[name] = col.to_numpy(zero_copy_only=False)
        for name in ("x", "y", "z", "value", "hole", "error_variance", "domain"):
            if name not in got:
                raise InvalidInput(f"missing column {name}")
        for name in ("x", "y", "z", "value", "error_variance"):
            if np.isnan(got[name]).any() and table.column(name).null_count:
                raise InvalidInput(f"null in column {name}")
        doms = None
        if labels:
            codes = got["domain"]
            if np.isnan(codes).any() or np.any((codes < 0) | (codes >= len(labels)) | (codes != np.floor(codes))):
                raise InvalidInput("domain codes must index the fitted domains")
            doms = [labels[int(c)] for c in codes]
        elif (~np.isnan(got["domain"])).any():
            raise InvalidInput("domain codes without fitted domains")
        holes = got["hole"]
        has = ~np.isnan(holes)
        if has.any():
            h = holes[has]
            if np.any((h < 0) | (h != np.floor(h)) | (h >= 2.0 ** 32 - 1)):
                raise InvalidInput("hole codes must be indices")
        hole_labels = None if not has.any() else [int(v) if ok else None for v, ok in zip(holes, has)]
        err = got["error_variance"]
        est.fit(np.column_stack([got["x"], got["y"], got["z"]]), got["value"], holes=hole_labels,
                error_variance=None if not err.any() else err, domains=doms)
    return est


def _build(cls, d):
    """An unfitted estimator of class `cls` from the envelope's fields."""
    from .estimation import BlockKriging, IndicatorKriging, OrdinaryKriging, SimpleKriging

    method = d.get("method")
    vg = variogram_from(d.get("variogram"))
    searches = [search_from(s) for s in d.get("search", [])]
    search = searches if len(searches) != 1 else searches[0]
    if isinstance(method, dict) and "Block" in method:
        b = method["Block"]
        if any(float(v) != 0.0 for v in b.get("rotation", [0.0, 0.0, 0.0])):
            raise Unsupported("a block method fixed to a rotated model is not run by this engine")
        disc = b["disc"]
        if not issubclass(cls, BlockKriging):
            raise InvalidInput(f"{cls.__name__} cannot hold a block-kriging method")
        return cls(vg, search, tuple(b["size"]), discretization=(disc["nx"], disc["ny"], disc["nz"]))
    kind = method.get("Kriging") if isinstance(method, dict) else None
    if kind == "Ordinary" and issubclass(cls, OrdinaryKriging):
        return cls(vg, search)
    if isinstance(kind, dict) and "Simple" in kind and issubclass(cls, SimpleKriging):
        return cls(vg, search, mean=kind["Simple"]["mean"])
    if isinstance(kind, dict) and "Indicator" in kind and issubclass(cls, IndicatorKriging):
        return cls(vg, search, kind["Indicator"]["threshold"])
    raise Unsupported(f"method {json.dumps(method)} is not run by this engine as {cls.__name__}")
