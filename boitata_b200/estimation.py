"""Estimators with the reference's call surface: fit on samples, predict at targets.

Mirrors python/boitata/estimation.py:209-423 (`_Base.fit/predict/
cross_validate`, `OrdinaryKriging`, `SimpleKriging`, `IndicatorKriging`) and
the pyo3 engine behind it (crates/py/src/estimation.rs:1213-1868): samples
sharing a location keep the first one with a warning (args.rs:318-376),
targets a search cannot fill are NaN, several searches run as passes on the
targets earlier passes left (batch.rs:132-147). The kriging itself runs in
the CUDA engine through its C ABI; `precision` selects the FP64 form
(default, the reference's arithmetic) or the mixed form (FP32 factorisation
refined in FP64; a system whose refinement does not converge is re-solved in
FP64). Hard domains (`fit(domains=)`, `predict(domains=)`) restrict each
target to its own domain's samples; `cross_validate(folds=k)` runs the
reference's k-fold scheme (batch.rs:197-243).
"""

import contextlib
import ctypes
import math
import warnings
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .errors import InvalidInput, Unsupported
from .geometry import BlockModel, Geometry, PointSet
from .search import Search
from .table import Table
from .variogram import Variogram

DIAGNOSTICS = ("negative_weight_sum", "mean_distance", "n_holes", "target_met")

PRECISIONS = {"fp64": N.FP64, "mixed": N.MIXED}


def points(coords):
    """(n, 2) or (n, 3) finite coordinates as an (n, 3) float64 array (containers.rs:15-54)."""
    a = np.asarray(coords, dtype=np.float64)
    if a.ndim != 2 or a.shape[1] not in (2, 3):
        raise InvalidInput("coordinates must be a 2-D array of shape (n, 2) or (n, 3)")
    if not np.all(np.isfinite(a)):
        raise InvalidInput("coordinates must be finite")
    if a.shape[1] == 2:
        a = np.column_stack([a, np.zeros(len(a))])
    return np.ascontiguousarray(a)


def column(data, arg, what):
    """`arg`, or the column of the container `data` it names (python/boitata/_columns.py:13-27)."""
    if not isinstance(arg, str):
        return arg
    if not isinstance(data, (PointSet, BlockModel)):
        raise InvalidInput(f'{what} names column "{arg}"; that needs a container')
    return data[arg]


def domains_of(data, domains, domain_column):
    """The domains given, or the container's column `domain_column` (estimation.py:675-678)."""
    if domain_column is None:
        return domains
    if domains is not None:
        raise InvalidInput("give one of domains or domain_column")
    return column(data, str(domain_column), "domain_column")


def held_samples(search, n):
    """The samples a system can hold, the width of the engine's neighbour rows: max_samples, or the n fitted
    samples when there are fewer (never below min_samples or min_holes). btk_api.cu's held_samples."""
    floor = max(n, search.min_samples, search.min_holes if search.min_holes is not None else -1)
    return min(search.max_samples, floor)


def finite(values, what, n=None):
    v = np.ascontiguousarray(np.asarray(values, dtype=np.float64))
    if v.ndim != 1:
        raise InvalidInput(f"{what} must be a 1-D numeric array")
    if not np.all(np.isfinite(v)):
        raise InvalidInput(f"{what} must be finite; drop missing values first")
    if n is not None and len(v) != n:
        raise InvalidInput(f"{what}: expected {n} values, got {len(v)}")
    return v


def _hole_text(v):
    """A hole label as the reference keys it (crates/py/src/args.rs:14-45): the text of a string, boolean
    ("true" / "false") or finite number (integral values without a decimal point, so 1, 1.0 and "1" are one
    hole); None for None and NaN."""
    if v is None:
        return None
    if isinstance(v, str):
        return v
    if isinstance(v, (bool, np.bool_)):
        return "true" if v else "false"
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    try:
        f = float(v)
    except (TypeError, ValueError):
        f = math.inf
    if math.isnan(f):
        return None
    if not math.isfinite(f):
        raise InvalidInput("holes must be a 1-D sequence of labels: strings, finite numbers or booleans, None or "
                           "NaN for none")
    return str(int(f)) if f == math.floor(f) and abs(f) < 9e15 else repr(f)


def hole_codes(labels):
    """Integer codes of hole labels (crates/py/src/args.rs:257-292): one per distinct label text, in order of
    first appearance, and a fresh one for each row without a label (None or NaN), which then counts as a
    hole of its own."""
    if isinstance(labels, str):
        raise InvalidInput("holes must be a sequence of labels")
    items = labels.to_pylist() if hasattr(labels, "to_pylist") else np.asarray(labels).tolist()
    if not isinstance(items, list) or any(isinstance(v, list) for v in items):
        raise InvalidInput("holes must be a 1-D sequence of labels: strings, finite numbers or booleans, None or "
                           "NaN for none")
    codes, out = {}, np.empty(len(items), dtype=np.int64)
    nxt = 0
    for i, v in enumerate(items):
        key = _hole_text(v)
        if key is None:
            out[i] = nxt
            nxt += 1
            continue
        if key not in codes:
            codes[key] = nxt
            nxt += 1
        out[i] = codes[key]
    return out


def _label_key(v):
    """A domain label as the reference keys it (crates/py/src/args.rs:16-37): strings, booleans, integral
    numbers as integers, other finite numbers; None for a missing label (None or NaN)."""
    if v is None:
        return None
    if isinstance(v, (bool, np.bool_)):
        return ("bool", bool(v))
    if isinstance(v, str):
        return ("str", v)
    if isinstance(v, (int, np.integer)):
        return ("num", int(v))
    try:
        f = float(v)
    except (TypeError, ValueError):
        f = None
    if f is None or math.isinf(f):
        raise InvalidInput(f"domain labels must be strings, finite numbers or booleans, not {v!r}")
    if math.isnan(f):
        return None
    return ("num", int(f)) if f == int(f) and abs(f) < 9e15 else ("num", f)


def _labels(obj, n):
    """A sequence of n labels, or one label for all (crates/py/src/estimation.rs:250-265)."""
    if isinstance(obj, (str, bool, int, float, np.generic)) or not hasattr(obj, "__len__"):
        return [obj] * n
    labels = list(obj)
    if len(labels) != n:
        raise InvalidInput(f"domains: expected {n} values, got {len(labels)}")
    return labels


def domain_codes(obj, n):
    """(fitted labels by code, int32 codes of the n samples): one code per distinct label in order of first
    appearance (crates/py/src/estimation.rs:1321-1333); every sample needs a label."""
    fitted, code, out = [], {}, np.empty(n, dtype=np.int32)
    for i, v in enumerate(_labels(obj, n)):
        k = _label_key(v)
        if k is None:
            raise InvalidInput(f"domain labels must be strings, finite numbers or booleans, not {v!r}")
        if k not in code:
            code[k] = len(fitted)
            fitted.append(v)
        out[i] = code[k]
    return fitted, out


def target_codes(fitted, obj, n, method="predict"):
    """Codes of n target labels among the fitted ones, -1 for a domain without samples
    (crates/py/src/estimation.rs:1337-1360)."""
    if fitted is None and obj is None:
        return None
    if fitted is not None and obj is None:
        raise InvalidInput(f"fitted with domains; {method} needs domains too")
    if fitted is None:
        raise InvalidInput(f"fitted without domains; {method} takes none")
    code = {_label_key(v): c for c, v in enumerate(fitted)}
    out = np.empty(n, dtype=np.int32)
    for i, v in enumerate(_labels(obj, n)):
        k = _label_key(v)
        if k is None:
            raise InvalidInput(f"domain labels must be strings, finite numbers or booleans, not {v!r}")
        out[i] = code.get(k, -1)
    return out


def distinct(locs, holes=None, domains=None):
    """Rows to keep so no two samples share a location (within a domain, with domains): the first of each
    group, with a UserWarning naming the dropped groups (args.rs:318-376 over eda::duplicates with
    tolerance 0, which treats -0 as 0)."""
    key = np.ascontiguousarray(locs + 0.0)
    if domains is not None:
        key = np.column_stack([key, np.asarray(domains, dtype=np.float64)])
    _, first, inverse, counts = np.unique(key, axis=0, return_index=True, return_inverse=True, return_counts=True)
    inverse = inverse.ravel()
    if np.all(counts == 1):
        return np.arange(len(locs))
    keep = np.sort(first)
    groups = []
    for g in np.nonzero(counts > 1)[0]:
        rows = np.nonzero(inverse == g)[0]
        groups.append(rows)
    groups.sort(key=lambda r: r[0])
    lines = []
    for rows in groups[:20]:
        who = (f"holes {', '.join(str(holes[i]) for i in rows)}" if holes is not None
               else f"rows {', '.join(str(i) for i in rows)}")
        x, y, z = locs[rows[0]]
        lines.append(f"{who} at ({x}, {y}, {z})")
    if len(groups) > 20:
        lines.append(f"and {len(groups) - 20} more")
    warnings.warn(f"{len(groups)} locations hold several samples; kept the first of each: {'; '.join(lines)}",
                  UserWarning, stacklevel=3)
    return keep


@dataclass(frozen=True)
class CrossValidation:
    """Cross-validation results; NaN where a sample had too few neighbours (estimation.py:112-170)."""

    actual: np.ndarray
    estimate: np.ndarray
    variance: np.ndarray

    @property
    def error(self):
        return self.estimate - self.actual

    @property
    def mean_error(self):
        return float(np.nanmean(self.error))

    @property
    def mean_squared_error(self):
        return float(np.nanmean(self.error ** 2))

    @property
    def rmse(self):
        return float(np.sqrt(self.mean_squared_error))

    @property
    def standardized_squared_error(self):
        """Mean of error^2 / variance over the estimated samples (near 1 for a calibrated variance)."""
        return float(np.nanmean(self.error ** 2 / self.variance))

    @property
    def correlation(self):
        ok = np.isfinite(self.estimate)
        return float(np.corrcoef(self.actual[ok], self.estimate[ok])[0, 1])

    @property
    def slope(self):
        """Least-squares slope of the actual values on the estimates; below 1 shows conditional bias."""
        ok = np.isfinite(self.estimate)
        e, a = self.estimate[ok], self.actual[ok]
        de = e - e.mean()
        return float(np.dot(de, a - a.mean()) / np.dot(de, de))


class _Base:
    _kind = N.ORDINARY

    def __init__(self, variogram, search, *, kparam=0.0, precision="fp64", device=0):
        if variogram is None:
            raise InvalidInput("kriging needs a variogram")
        if not isinstance(variogram, Variogram):
            raise InvalidInput("variogram must be a Variogram")
        searches = self._searches(search)
        if self._kind == N.SIMPLE and not variogram.is_stationary():
            raise InvalidInput("simple kriging needs a variogram with a sill: every structure must be stationary "
                               "(not power); use ordinary kriging")
        if precision not in PRECISIONS:
            raise InvalidInput(f"precision must be one of {sorted(PRECISIONS)}")
        self.variogram = variogram
        self.searches = searches
        self._kparam = float(kparam)
        self.precision = precision
        self._device = device
        self._ctx = None
        self._pass = None
        self._samples = None

    def _searches(self, search):
        """`search` (a Search or passes) as the list of passes, checked for this estimator."""
        searches = list(search) if isinstance(search, (list, tuple)) else [search]
        if not searches or not all(isinstance(s, Search) for s in searches):
            raise InvalidInput("search must be a Search or a sequence of Search (passes)")
        if self._kind == N.SIMPLE and any(s.target_slope is not None for s in searches):
            raise InvalidInput("simple kriging has a slope of regression of 1; calibrate it with target_efficiency")
        return searches

    def with_search(self, search):
        """A copy with `search` (a Search or passes) in place of the searches, keeping the variogram, the
        precision and the fitted samples, holes, error variances and domains
        (crates/py/src/estimation.rs:1742-1756). The copy indexes the samples for its searches on a context
        of its own."""
        import copy

        searches = self._searches(search)
        out = copy.copy(self)
        out.searches = searches
        out._ctx, out._pass = None, None
        if out._samples is not None:
            out._ctx = N.Context(out._device)
            out._use_pass(0)
        return out

    # -- fit --------------------------------------------------------------
    def fit(self, coords, values, *, holes=None, error_variance=None, domains=None, domain_column=None):
        """Stores the samples; samples sharing a location keep the first one, with a warning. With
        `domains` (one label per sample: strings, finite numbers or booleans) a target is estimated from
        the samples of its own domain only (hard boundaries), shared locations are dropped within a domain
        only, and predict needs the targets' domains too (python/boitata/estimation.py:226-250).
        `coords` may be a PointSet or BlockModel whose columns `values`, `holes`, `error_variance` and
        `domain_column` name."""
        values = column(coords, values, "values")
        holes = column(coords, holes, "holes")
        error_variance = column(coords, error_variance, "error_variance")
        domains = domains_of(coords, domains, domain_column)
        if isinstance(coords, Geometry):
            coords = BlockModel(coords)
        if isinstance(coords, BlockModel):
            coords = coords.centroids(self._ctx)
        elif isinstance(coords, PointSet):
            coords = coords.coords
        locs = points(coords)
        n = len(locs)
        vals = finite(values, "values", n)
        err = None
        if error_variance is not None:
            err = finite(error_variance, "error_variance", n)
            if np.any(err < 0):
                raise InvalidInput("error_variance must be >= 0")
        if holes is not None:
            holes = list(holes)
            if len(holes) != n:
                raise InvalidInput(f"holes: expected {n} values, got {len(holes)}")
        fitted, codes = (None, None) if domains is None else domain_codes(domains, n)
        keep = distinct(locs, holes, codes)
        locs, vals = np.ascontiguousarray(locs[keep]), np.ascontiguousarray(vals[keep])
        err = None if err is None else np.ascontiguousarray(err[keep])
        self._holes = None if holes is None else np.ascontiguousarray(hole_codes(holes)[keep])
        self._domain_labels = fitted
        self._domains = None if codes is None else np.ascontiguousarray(codes[keep])
        self._samples = (locs, vals, err)
        if self._ctx is None:
            self._ctx = N.Context(self._device)
        self._pass = None
        self._use_pass(0)
        return self

    # -- persistence (crates/py/src/persist.rs) ---------------------------------
    def to_parquet(self, path):
        """Writes the samples as Parquet columns and the parameters as JSON in the file metadata, in the
        reference's format (python/boitata/estimation.py:377-383)."""
        from . import persist

        persist.to_parquet(self, path)

    @classmethod
    def from_parquet(cls, path):
        """Reads `to_parquet` output, or a file the reference wrote; predictions match the saved
        estimator's bit for bit (python/boitata/estimation.py:385-402)."""
        from . import persist

        return persist.from_parquet(cls, path)

    def __getstate__(self):
        from . import persist

        cols = persist.columns(self)
        doms = getattr(self, "_domains", None)
        labels = getattr(self, "_domain_labels", None)
        return {"meta": persist.envelope(self), "columns": cols, "holes": getattr(self, "_holes", None),
                "domains": None if doms is None else [labels[c] for c in doms]}

    def __setstate__(self, state):
        from . import persist

        d = persist._open(type(self).__name__, state["meta"])
        fitted = d.pop("fitted", None) is True
        other = persist._build(type(self), d)
        self.__dict__.update(other.__dict__)
        self.precision = d.get("precision", self.precision)
        cols = state["columns"]
        if fitted and cols is not None:
            holes = state["holes"]
            err = cols["error_variance"]
            self.fit(np.column_stack([cols["x"], cols["y"], cols["z"]]), cols["value"],
                     holes=None if holes is None else [int(h) for h in holes],
                     error_variance=None if not err.any() else err, domains=state.get("domains"))

    def _use_pass(self, p):
        if self._pass == p:
            return
        ctx = self._ctx
        s = self.searches[p].to_c()
        if self._pass is None:
            locs, vals, err = self._samples
            vg = self.variogram.to_c()
            holes = getattr(self, "_holes", None)
            rc = ctx._lib.btk_fit(ctx.handle, len(locs), locs.ctypes.data, vals.ctypes.data,
                                  None if err is None else err.ctypes.data,
                                  None if holes is None else holes.ctypes.data, ctypes.byref(s), ctypes.byref(vg))
            ctx.check(rc, "fit")
            doms = getattr(self, "_domains", None)
            if doms is not None:
                ctx.check(ctx._lib.btk_set_domains(ctx.handle, doms.ctypes.data), "domains")
        else:
            ctx.check(ctx._lib.btk_set_search(ctx.handle, ctypes.byref(s)), "search")
        self._pass = p

    def _fitted(self):
        if self._samples is None:
            raise InvalidInput("estimator is not fitted; call fit first")

    @property
    def values(self):
        self._fitted()
        return self._samples[1].copy()

    # -- predict ------------------------------------------------------------
    def _run(self, xyz, precision, diagnostics=False, domains=None):
        m = len(xyz)
        out = {k: np.full(m, np.nan) for k in ("value", "variance", "lagrange")}
        out["n_used"] = np.zeros(m, dtype=np.int32)
        out["status"] = np.zeros(m, dtype=np.int8)
        if diagnostics:
            out["negative_weight_sum"] = np.full(m, np.nan)
            out["mean_distance"] = np.full(m, np.nan)
            out["n_holes"] = np.zeros(m, dtype=np.int32)
            out["target_met"] = np.full(m, -1, dtype=np.int8)
        if m == 0:
            return out
        o = N.OutputsC(out["value"].ctypes.data, out["variance"].ctypes.data, out["lagrange"].ctypes.data,
                       out["n_used"].ctypes.data, out["status"].ctypes.data)
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        ctx = self._ctx
        d = N.DiagnosticsC(*(out[k].ctypes.data for k in DIAGNOSTICS)) if diagnostics else None
        dom = None if domains is None else np.ascontiguousarray(domains, dtype=np.int32)
        rc = ctx._lib.btk_predict_ex(ctx.handle, m, xyz.ctypes.data, None, None if dom is None else dom.ctypes.data,
                                     self._kind, self._kparam, PRECISIONS[precision], ctypes.byref(o),
                                     None if d is None else ctypes.byref(d))
        ctx.check(rc, "predict")
        return out

    def _level(self, targets):
        """Centroids of a single-layer model turned only in azimuth take the
        elevation of 2-D data (crates/py/src/estimation.rs:960-992)."""
        g = targets.geometry
        locs = self._samples[0]
        if g.count[2] != 1 or g.rotation[1] != 0.0 or g.rotation[2] != 0.0:
            return None
        z = locs[0, 2]
        return z if math.isfinite(z) and np.all(locs[:, 2] == z) else None

    def predict_full(self, targets, *, precision=None, diagnostics=False, domains=None, domain_column=None):
        """Every output of the engine: value, variance, lagrange, n_used, status and pass (1-based, 0 unfilled);
        with `diagnostics`, also negative_weight_sum, mean_distance and n_holes of the samples used.
        `domains`: the targets' domain labels (one per target, or one for all) when fitted with domains."""
        self._fitted()
        precision = precision or self.precision
        if precision not in PRECISIONS:
            raise InvalidInput(f"precision must be one of {sorted(PRECISIONS)}")
        domains = domains_of(targets, domains, domain_column)
        if isinstance(targets, Geometry):
            targets = BlockModel(targets)
        xyz = self._locate(targets)
        codes = target_codes(getattr(self, "_domain_labels", None), domains, len(xyz))
        with self._support(targets):
            return self._passes(xyz, precision, diagnostics, codes)

    def _locate(self, targets):
        """(m, 3) target points: a BlockModel's centroids (made on the device; a single layer turned only in
        azimuth at the elevation of 2-D data), a PointSet's coordinates, or an array's."""
        if isinstance(targets, Geometry):
            targets = BlockModel(targets)
        if isinstance(targets, BlockModel):
            xyz = targets.centroids(self._ctx)
            z = self._level(targets)
            if z is not None:
                xyz[:, 2] = z
            return xyz
        if isinstance(targets, PointSet):
            return targets.coords
        return points(targets)

    def _support(self, targets):
        """Context manager setting the engine's target support for one prediction (point support here)."""
        return contextlib.nullcontext()

    def _passes(self, xyz, precision, diagnostics=False, codes=None):
        m = len(xyz)
        if m == 0:  # no targets: empty columns of every output
            res = self._run(xyz, precision, diagnostics)
            res["pass"] = np.zeros(0, dtype=np.int32)
            return res
        res = None
        remaining = np.arange(m)
        for p in range(len(self.searches)):
            if len(remaining) == 0:
                break
            self._use_pass(p)
            out = self._run(xyz[remaining], precision, diagnostics, None if codes is None else codes[remaining])
            if res is None:
                res = {k: v.copy() for k, v in out.items()}
                res["pass"] = np.where(np.isfinite(out["value"]), 1, 0).astype(np.int32)
            else:
                got = np.isfinite(out["value"])
                for k in out:
                    res[k][remaining[got]] = out[k][got]
                res["pass"][remaining[got]] = p + 1
                st = out["status"]
                res["status"][remaining[~got]] = st[~got]
            remaining = np.nonzero(~np.isfinite(res["value"]))[0]
        return res

    def predict(self, targets, *, return_variance=False, diagnostics=False, precision=None, domains=None,
                domain_column=None):
        """Estimates at targets; NaN where the search found too few samples (estimation.py:273-335).

        targets : (n, 2|3) array, PointSet, Geometry or BlockModel (centroids made on the device).
        domains : the targets' domain labels (one per target, or one for all), when fitted with domains; a
            target of a domain without samples is NaN.
        domain_column : the column of `targets` (a PointSet or BlockModel) holding their domains.
        """
        domains = domains_of(targets, domains, domain_column)
        if diagnostics:
            return self._diagnostics(targets, precision, domains)
        res = self.predict_full(targets, precision=precision, domains=domains)
        if return_variance:
            return res["value"], res["variance"]
        return res["value"]

    def _support_variance(self, targets):
        """C(v, v) of the targets' support: the sill for points (krige.rs:40-42)."""
        return self.variogram.total_sill()

    def _diagnostics(self, targets, precision, domains=None):
        """The diagnostics table (crates/py/src/estimation.rs:1046-1105): NaN where unestimated. With hard
        domains every sample used is of the target's domain, so n_other_domain is 0."""
        res = self.predict_full(targets, precision=precision, diagnostics=True, domains=domains)
        est = np.isfinite(res["value"])
        nan = lambda v: np.where(est, v, np.nan)  # noqa: E731
        sv = nan(np.full(len(est), self._support_variance(targets)))
        var, mu = res["variance"], res["lagrange"]
        cov = sv - var - mu  # Cov(Z, Z*) (krige.rs:58-61)
        est_var = cov - mu  # Var(Z*) (krige.rs:63-68)
        passes = np.maximum(res["pass"], 1) - 1
        full = res["n_used"] >= np.array([s.max_samples for s in self.searches])[passes]
        with np.errstate(divide="ignore", invalid="ignore"):
            columns = {
                "value": res["value"],
                "variance": var,
                "efficiency": (sv - var) / sv,
                "slope": cov / est_var,
                "n_samples": nan(res["n_used"].astype(np.float64)),
                "pass": nan(res["pass"].astype(np.float64)),
                "n_holes": nan(res["n_holes"].astype(np.float64)),
                "n_other_domain": nan(np.zeros(len(est))),
                "mean_distance": res["mean_distance"],
                "negative_weight_sum": res["negative_weight_sum"],
                "lagrange": mu,
                "support_variance": sv,
                "estimate_variance": est_var,
                "max_samples_reached": nan(full.astype(np.float64)),
                "target_met": np.where(est & (res["target_met"] >= 0), res["target_met"], np.nan),
            }
        return Table(columns)

    def predict_kinds(self, targets, kinds, *, mean=0.0, precision=None):
        """Every output at `targets` with a kriging kind per target ("ordinary" / "simple" / "indicator", or
        0 / 1 / 2) in one launch, sharing `mean` (simple) or threshold (indicator); first pass only."""
        self._fitted()
        precision = precision or self.precision
        codes = {"ordinary": N.ORDINARY, "simple": N.SIMPLE, "indicator": N.INDICATOR}
        k = np.array([codes.get(x, x) if isinstance(x, str) else x for x in kinds], dtype=np.int8)
        xyz = points(targets)
        m = len(xyz)
        if len(k) != m:
            raise InvalidInput(f"kinds: expected {m} values, got {len(k)}")
        out = {key: np.full(m, np.nan) for key in ("value", "variance", "lagrange")}
        out["n_used"] = np.zeros(m, dtype=np.int32)
        out["status"] = np.zeros(m, dtype=np.int8)
        self._use_pass(0)
        o = N.OutputsC(out["value"].ctypes.data, out["variance"].ctypes.data, out["lagrange"].ctypes.data,
                       out["n_used"].ctypes.data, out["status"].ctypes.data)
        ctx = self._ctx
        rc = ctx._lib.btk_predict_kinds(ctx.handle, m, xyz.ctypes.data, k.ctypes.data, float(mean),
                                        PRECISIONS[precision], ctypes.byref(o))
        ctx.check(rc, "predict")
        return out

    def cross_validate(self, *, folds=None, precision=None):
        """Re-estimates every sample from the others, through the same passes (estimation.py:337-355):
        leave-one-out when `folds` is None, else k-fold (batch.rs:197-243): each sample estimated without the
        samples of its fold, where the j-th of the sorted hole ids goes to fold j % k (holes stay whole) and
        an untagged sample i to fold i % k; each held-out sample in its own domain."""
        self._fitted()
        precision = precision or self.precision
        n = len(self._samples[0])
        est = np.full(n, np.nan)
        var = np.full(n, np.nan)
        if folds is not None:
            k = int(folds)
            if k != folds or k < 2:
                raise InvalidInput("k must be ≥ 2")
            fold = self._folds(k)
        for p in range(len(self.searches)):
            remaining = np.nonzero(~np.isfinite(est))[0]
            if len(remaining) == 0:
                break
            if folds is None:
                self._use_pass(p)
                value, variance = np.full(n, np.nan), np.full(n, np.nan)
                o = N.OutputsC(value.ctypes.data, variance.ctypes.data, None, None, None)
                ctx = self._ctx
                ctx.check(ctx._lib.btk_cross_validate(ctx.handle, self._kind, self._kparam, PRECISIONS[precision],
                                                      ctypes.byref(o)), "cross_validate")
            else:
                value, variance = self._k_fold(fold, k, remaining, p, precision)
            fill = ~np.isfinite(est) & np.isfinite(value)
            est[fill], var[fill] = value[fill], variance[fill]
        return CrossValidation(self._samples[1].copy(), est, var)

    def _folds(self, k):
        """Fold of each fitted sample (batch.rs:210-220): rank of its hole id among the sorted ids, or its
        index when untagged, modulo k."""
        n = len(self._samples[0])
        holes = getattr(self, "_holes", None)
        if holes is None:
            return np.arange(n) % k
        ids = np.unique(holes)
        return np.searchsorted(ids, holes) % k

    def _k_fold(self, fold, k, which, p, precision):
        """Estimates at samples `which` with search pass p, each from a fit of the samples outside its fold
        (a new index per fold, as the reference builds a new tree over the training samples)."""
        n = len(self._samples[0])
        value, variance = np.full(n, np.nan), np.full(n, np.nan)
        locs, vals, err = self._samples
        holes, doms = getattr(self, "_holes", None), getattr(self, "_domains", None)
        s = self.searches[p].to_c()
        vg = self.variogram.to_c()
        for f in range(k):
            test = which[fold[which] == f]
            if len(test) == 0:
                continue
            train = np.nonzero(fold != f)[0]
            ctx = N.Context(self._device)
            sub = lambda a: None if a is None else np.ascontiguousarray(a[train])  # noqa: E731
            tl, tv, te, th, td = sub(locs), sub(vals), sub(err), sub(holes), sub(doms)
            rc = ctx._lib.btk_fit(ctx.handle, len(train), tl.ctypes.data, tv.ctypes.data,
                                  None if te is None else te.ctypes.data, None if th is None else th.ctypes.data,
                                  ctypes.byref(s), ctypes.byref(vg))
            ctx.check(rc, "fit")
            if td is not None:
                ctx.check(ctx._lib.btk_set_domains(ctx.handle, td.ctypes.data), "domains")
            m = len(test)
            xyz = np.ascontiguousarray(locs[test])
            v, sv = np.full(m, np.nan), np.full(m, np.nan)
            o = N.OutputsC(v.ctypes.data, sv.ctypes.data, None, None, None)
            dom = None if doms is None else np.ascontiguousarray(doms[test])
            ctx.check(ctx._lib.btk_predict_ex(ctx.handle, m, xyz.ctypes.data, None,
                                              None if dom is None else dom.ctypes.data, self._kind, self._kparam,
                                              PRECISIONS[precision], ctypes.byref(o), None), "k-fold predict")
            value[test], variance[test] = v, sv
            del ctx
        return value, variance

    def neighbors(self, targets, *, loo=False, search_pass=0, domains=None):
        """Neighbour lists (selection order, -1 padded), counts and success flags of the search; `domains`
        as for predict when fitted with domains."""
        self._fitted()
        self._use_pass(search_pass)
        k = held_samples(self.searches[search_pass], len(self._samples[0]))
        if loo:
            m = len(self._samples[0])
            xyz = None
        else:
            xyz = points(targets)
            m = len(xyz)
        idx = np.empty((m, k), dtype=np.int64)
        cnt = np.empty(m, dtype=np.int32)
        ok = np.empty(m, dtype=np.int8)
        ctx = self._ctx
        codes = None if loo else target_codes(getattr(self, "_domain_labels", None), domains, m, "neighbors")
        rc = ctx._lib.btk_neighbors(ctx.handle, m, None if xyz is None else xyz.ctypes.data, 1 if loo else 0,
                                    None if codes is None else codes.ctypes.data, idx.ctypes.data, cnt.ctypes.data,
                                    ok.ctypes.data)
        ctx.check(rc, "neighbors")
        return idx, cnt, ok.astype(bool)


class OrdinaryKriging(_Base):
    """Kriging with an unknown, locally constant mean (weights sum to 1)."""

    _kind = N.ORDINARY

    def __init__(self, variogram, search, *, precision="fp64", device=0):
        super().__init__(variogram, search, precision=precision, device=device)


class SimpleKriging(_Base):
    """Kriging with a known global `mean`."""

    _kind = N.SIMPLE

    def __init__(self, variogram, search, *, mean=0.0, precision="fp64", device=0):
        mean = float(mean)
        if not math.isfinite(mean):
            raise InvalidInput("mean must be finite")
        super().__init__(variogram, search, kparam=mean, precision=precision, device=device)
        self.mean = mean


class IndicatorKriging(_Base):
    """Ordinary kriging of the indicator `value <= threshold`; estimates are probabilities."""

    _kind = N.INDICATOR

    def __init__(self, variogram, search, threshold, *, precision="fp64", device=0):
        super().__init__(variogram, search, kparam=float(threshold), precision=precision, device=device)
        self.threshold = float(threshold)


class BlockKriging(_Base):
    """Ordinary kriging of block averages; targets are block centres of `size`
    (python/boitata/estimation.py:475-485, crates/estimation/src/block.rs).

    `size` runs along the axes of a rotated BlockModel given as targets, and
    along the world axes for coordinates. Each size must be finite and > 0,
    and `discretization` at least 1 per axis, or InvalidInput is raised; a
    ``(1, 1, 1)`` discretization is point support, nugget included.
    Cross-validation runs at point support, as in the reference.
    """

    _kind = N.ORDINARY

    def __init__(self, variogram, search, size, *, discretization=(4, 4, 1), precision="fp64", device=0):
        size = [float(v) for v in size]
        if len(size) == 2:
            size.append(1.0)
        if len(size) != 3:
            raise InvalidInput(f"size needs 2 or 3 values, got {len(size)}")
        disc = tuple(int(v) for v in discretization)
        if len(disc) != 3 or any(v < 1 for v in disc):
            raise InvalidInput(f"discretization must be at least 1 per axis, got {disc}")
        if not all(math.isfinite(v) and v > 0.0 for v in size):
            raise InvalidInput(f"size must be finite and > 0, got {tuple(size)}")
        if disc[0] * disc[1] * disc[2] > 4096:
            raise Unsupported("block discretizations of more than 4096 points are not run by this engine")
        super().__init__(variogram, search, precision=precision, device=device)
        self.size = tuple(size)
        self.discretization = disc

    @contextlib.contextmanager
    def _support(self, targets):
        rot = targets.geometry.rotation if isinstance(targets, BlockModel) else (0.0, 0.0, 0.0)
        ctx = self._ctx
        size = (ctypes.c_double * 3)(*self.size)
        disc = (ctypes.c_int32 * 3)(*self.discretization)
        r = (ctypes.c_double * 3)(*rot)
        ctx.check(ctx._lib.btk_set_support(ctx.handle, size, disc, r), "block support")
        try:
            yield
        finally:
            ctx._lib.btk_set_support(ctx.handle, None, None, None)

    def _support_variance(self, targets):
        return self.support_variance(targets if isinstance(targets, (BlockModel, Geometry)) else None)

    def support_variance(self, targets=None):
        """C(B,B), the mean covariance within a block (the reference's support_variance), for blocks turned
        as `targets` (a BlockModel or Geometry) or along the world axes."""
        self._fitted()
        if isinstance(targets, Geometry):
            targets = BlockModel(targets)
        out = ctypes.c_double(0.0)
        with self._support(targets):
            self._ctx.check(self._ctx._lib.btk_support_variance(self._ctx.handle, ctypes.byref(out)), "support")
        return out.value
