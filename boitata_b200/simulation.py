"""Sequential Gaussian simulation, the caller of the kriging path that the
reference's simulations are built on (crates/simulation/src/sgs.rs).

Per realization (sgs.rs:281-760): the data are normal-score transformed
(declustering weights optional), the nodes are visited along a random path,
each node on a datum takes the datum's value, and every other node is
simple-kriged (mean 0, the variogram scaled to a unit sill, sgs.rs:857-862)
from the data and the nodes simulated before it, draws a score from that
Gaussian (or from the standard normal where its search finds too few
samples) and joins the conditioning set; scores are back-transformed through
the data's table. The sequential loop runs on the GPU (btk_sgs_simulate):
windows of the path in parallel, nodes that an earlier unsimulated node
could reach searched again, so each realization is the sequential one.

The random path and the normal draws come from numpy's generator seeded with
(seed, realization): a realization follows its seed reproducibly, but it is
not the reference's realization for that seed, whose generator (rand 0.8
StdRng and rand_distr's ziggurat normal) is not restated here.
"""

import ctypes
import math

import numpy as np

from . import _native as N
from .errors import InvalidInput, Unsupported
from .estimation import distinct, finite, hole_codes, points
from .geometry import BlockModel, Geometry
from .search import Search
from .transforms import normal_score
from .variogram import Structure, Variogram


def unit_sill(vg):
    """sgs.rs:857-862 with composite.rs:55-61: a stationary variogram scaled to a total sill of 1."""
    c0 = vg.total_sill()
    if not (vg.is_stationary() and c0 > 0.0):
        return vg
    k = 1.0 / c0
    st = [Structure(s.model, s.sill * k, s.range, order=s.order, exponent=s.exponent) for s in vg.structures]
    return Variogram(st, nugget=vg.nugget * k, rotation=vg.rotation, ratios=vg.ratios)


def _key(p):
    """sgs.rs:864-867: a location key equal for 0.0 and -0.0."""
    return tuple(float(v) + 0.0 for v in p)


class Simulation:
    """Realizations (n, nodes) in data units, with their ensemble mean and variance."""

    def __init__(self, realizations, rounds):
        self.realizations = realizations
        self.rounds = rounds

    @property
    def mean(self):
        return self.realizations.mean(axis=0)

    @property
    def variance(self):
        return self.realizations.var(axis=0)


class SGS:
    """Sequential Gaussian simulation with `variogram` (of the normal scores) and `search`."""

    def __init__(self, variogram, search, *, device=0):
        if not isinstance(variogram, Variogram):
            raise InvalidInput("variogram must be a Variogram")
        searches = list(search) if isinstance(search, (list, tuple)) else [search]
        if not searches or not all(isinstance(s, Search) for s in searches):
            raise InvalidInput("search must be a Search or a sequence of Search (passes)")
        if len(searches) > 1:
            raise Unsupported("SGS with several search passes is not run by this engine")
        if searches[0].calibrated():
            raise InvalidInput("SGS does not take target_slope or target_efficiency; they calibrate the ordinary, "
                               "simple, indicator, universal, external-drift and block kriging estimators")
        if not variogram.is_stationary():
            raise InvalidInput("simple kriging needs a variogram with a sill: every structure must be stationary "
                               "(not power); use ordinary kriging")
        self.variogram = variogram
        self.search = searches[0]
        self._device = device
        self._data = None
        self._ctx = None

    @property
    def n_samples(self):
        return None if self._data is None else len(self._data[1])

    def fit(self, coords, values, *, weights=None, holes=None):
        """Stores the conditioning data and their declustered normal scores (sgs.rs:97-168)."""
        locs = points(coords)
        n = len(locs)
        vals = finite(values, "values", n)
        if n == 0:
            raise InvalidInput("no conditioning data")
        w = None if weights is None else finite(weights, "weights", n)
        if holes is not None and len(holes) != n:
            raise InvalidInput(f"holes: expected {n} values, got {len(holes)}")
        # Samples sharing a location keep the first, with a warning naming them (crates/py/src/simulation.rs
        # `located`, args.rs:318-376), before the normal-score transform.
        keep = distinct(locs, None if holes is None else list(holes))
        if len(keep) < n:
            locs, vals = locs[keep], vals[keep]
            w = None if w is None else w[keep]
            holes = None if holes is None else [list(holes)[i] for i in keep]
        scores, table = normal_score(vals, w)
        codes = None if holes is None else hole_codes(list(holes))
        self._data = (np.ascontiguousarray(locs), np.ascontiguousarray(vals), scores, table, codes)
        return self

    def _targets(self, targets):
        if isinstance(targets, Geometry):
            targets = BlockModel(targets)
        if isinstance(targets, BlockModel):
            if self._ctx is None:
                self._ctx = N.Context(self._device)
            return targets.centroids(self._ctx)
        return points(targets)

    def simulate(self, targets, *, n=1, seed=0, batch=None):
        """`n` realizations at the nodes `targets` (points, Geometry or BlockModel); realization r follows
        (seed, r)."""
        if self._data is None:
            raise InvalidInput("SGS is not fitted; call fit first")
        n = int(n)
        if n < 1:
            raise InvalidInput("n must be at least 1")
        if batch is not None and int(batch) < 1:
            raise InvalidInput("batch must be at least 1")
        locs, vals, scores, table, codes = self._data
        nodes = np.ascontiguousarray(self._targets(targets), dtype=np.float64)
        m = len(nodes)
        first = {}
        for i, p in enumerate(locs):
            first.setdefault(_key(p), i)
        on_datum = np.array([first.get(_key(p), -1) for p in nodes], dtype=np.int64)
        out = np.empty((n, m))
        rounds = []
        if self._ctx is None:
            self._ctx = N.Context(self._device)
        nd = len(locs)
        data_holes = codes if codes is not None else np.arange(nd, dtype=np.int64)
        for r in range(n):
            rng = np.random.default_rng((int(seed), r))
            path = rng.permutation(m)
            order = path[on_datum[path] < 0]  # nodes that draw, in path order
            z = rng.standard_normal(len(order))
            sc, _, nr = sgs_scores(locs, scores, data_holes, nodes[order], z, self.search, unit_sill(self.variogram),
                                   batch=batch, context=self._ctx)
            row = np.empty(m)
            row[on_datum >= 0] = vals[on_datum[on_datum >= 0]]
            row[order] = _back(table, sc)
            out[r] = row
            rounds.append(nr)
        return Simulation(out, rounds)


def sgs_scores(locs, scores, holes, nodes, z, search, variogram, *, batch=None, context=None, device=0):
    """The sequential loop on the GPU (btk_sgs_simulate): scores of `nodes`, given in simulation order, from
    data `locs` with normal `scores` and hole codes `holes` (None: each datum its own hole), drawing z[j] for
    node j; `variogram` as kriged (scaled to a unit sill by the caller). Returns (scores, how: 1 kriged,
    2 marginal, parallel rounds)."""
    ctx = context or N.Context(device)
    locs, nodes = points(locs), points(nodes)
    nd, m = len(locs), len(nodes)
    data_holes = np.arange(nd, dtype=np.int64) if holes is None else np.asarray(holes, dtype=np.int64)
    xyz = np.ascontiguousarray(np.vstack([locs, nodes]))
    v = np.ascontiguousarray(np.concatenate([np.asarray(scores, dtype=np.float64), np.zeros(m)]))
    h = np.ascontiguousarray(np.concatenate([data_holes, data_holes.max(initial=-1) + 1 + np.arange(m)]),
                             dtype=np.int64)
    s, vg = search.to_c(), variogram.to_c()
    ctx.check(ctx._lib.btk_fit(ctx.handle, len(xyz), xyz.ctypes.data, v.ctypes.data, None, h.ctypes.data,
                               ctypes.byref(s), ctypes.byref(vg)), "fit")
    sc = np.empty(m)
    how = np.empty(m, dtype=np.int8)
    nr = ctypes.c_int64(0)
    zc = np.ascontiguousarray(z, dtype=np.float64)
    if len(zc) != m:
        raise InvalidInput(f"z: expected {m} values, got {len(zc)}")
    ctx.check(ctx._lib.btk_sgs_simulate(ctx.handle, nd, zc.ctypes.data, int(batch or 0), sc.ctypes.data,
                                        how.ctypes.data, ctypes.byref(nr)), "simulate")
    return sc, how, nr.value


def _back(table, scores):
    """NormalScoreTable::back (normal_score.rs:209-222) over an array of scores."""
    from scipy.special import erfc

    phi = lambda x: 0.5 * erfc(-np.asarray(x, dtype=np.float64) / math.sqrt(2.0))  # noqa: E731
    xs, ys = table.scores, table.values
    nt = len(xs)
    s = np.asarray(scores, dtype=np.float64)
    if nt == 1:
        return np.full(len(s), ys[0])
    hi = np.clip(np.searchsorted(xs, s, side="right"), 1, nt - 1)
    x0, x1, y0, y1 = xs[hi - 1], xs[hi], ys[hi - 1], ys[hi]
    with np.errstate(divide="ignore", invalid="ignore"):
        mid = np.where(np.abs(x1 - x0) < 2.2250738585072014e-308, y0, y0 + (y1 - y0) * (s - x0) / (x1 - x0))
    lo, top = table.tails
    low = lo + (ys[0] - lo) * (phi(s) / phi(xs[0]))
    edge = phi(xs[nt - 1])
    high = ys[nt - 1] + (top - ys[nt - 1]) * ((phi(s) - edge) / (1.0 - edge))
    return np.where(s < xs[0], low, np.where(s > xs[nt - 1], high, mid))
