"""Declustering weights from kriging weights.

The call surface is the reference's `weight_declustering`
(python/boitata/estimation.py:540-566): each sample's weight is the sum of
the kriging weights it receives when the estimator estimates a dense set of
targets, scaled to sum to the number of samples
(crates/estimation/src/batch.rs:76-125, crates/py/src/estimation.rs:
1509-1585). The weights of every target come from the engine
(`btk_predict_weights`: search, solve and the FP64 weights pass on the
GPU); this module adds them up, in target order, the order the reference
sums them in, so a call is reproducible to the bit.
"""

import copy
import ctypes
import threading
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .errors import InvalidInput
from .estimation import PRECISIONS, _Base, column, points
from .geometry import BlockModel, Geometry, PointSet


@dataclass(frozen=True)
class Declustering:
    """Declustering weights, one per sample (samples sharing a location share one weight), and the declustered
    mean; `cell_size` is NaN for weights from an estimator (crates/py/src/transforms.rs:2215-2264)."""

    weights: np.ndarray
    mean: float
    cell_size: float


_LOCAL = threading.local()


def _context(device):
    """A context of this thread for declustering calls on `device`, kept between calls: each call fits its
    samples on it again, and its device buffers, grown by earlier calls, are reused instead of allocated."""
    cache = getattr(_LOCAL, "contexts", None)
    if cache is None:
        cache = _LOCAL.contexts = {}
    if device not in cache:
        cache[device] = N.Context(device)
    return cache[device]


def _seq_sum(x):
    """Left-to-right sum, as an iterator's sum."""
    return float(np.cumsum(x)[-1]) if len(x) else 0.0


def _sample_points(coords, ctx):
    if isinstance(coords, Geometry):
        coords = BlockModel(coords)
    if isinstance(coords, BlockModel):
        return coords.centroids(ctx)
    if isinstance(coords, PointSet):
        return points(coords.coords)
    return points(coords)


def _pass_weights(est, p, xyz, codes):
    """(estimated, per-target lists, per-target weights) of search pass p at targets xyz."""
    m = len(xyz)
    est._use_pass(p)
    value, status = np.full(m, np.nan), np.zeros(m, dtype=np.int8)
    k = int(est.searches[p].max_samples)
    idx = np.full((m, k), -1, dtype=np.int64)
    w = np.zeros((m, k))
    o = N.OutputsC(value.ctypes.data, None, None, None, status.ctypes.data)
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    ctx = est._ctx
    rc = ctx._lib.btk_predict_weights(ctx.handle, m, xyz.ctypes.data, est._kind, est._kparam, PRECISIONS["fp64"],
                                      None if codes is None else codes.ctypes.data, ctypes.byref(o),
                                      idx.ctypes.data, w.ctypes.data)
    ctx.check(rc, "weights")
    return np.isfinite(value), idx, w


def weight_declustering(coords, values, targets, *, estimator):
    """Declustering weights from estimation weights: each sample's weight is the sum of the kriging weights it
    receives when `estimator` estimates `targets`, scaled to sum to the number of samples
    (python/boitata/estimation.py:540-566).

    coords : sample locations ((n, 2) or (n, 3)), or a PointSet / BlockModel whose column `values` may name.
    targets : a dense set of points, or a BlockModel (its centroids), covering the domain; targets the search
        leaves unestimated add nothing.
    estimator : an OrdinaryKriging, SimpleKriging, IndicatorKriging or BlockKriging whose search passes,
        variogram and kind give the weights; it is neither fitted nor changed.

    Returns a Declustering: `weights` per sample (samples sharing a location share the weight of the one
    kept, split evenly), the declustered `mean`, and `cell_size` NaN. Kriging can give negative weights, so a
    screened sample's weight can be below 0.
    """
    if not isinstance(estimator, _Base):
        raise InvalidInput("weight declustering needs an estimator linear in the data (a kriging estimator)")
    vals = np.asarray(column(coords, values, "values"), dtype=np.float64)
    locs = _sample_points(coords, None)
    est = copy.copy(estimator)
    est._pass = est._samples = None
    est._holes = est._domains = est._domain_labels = None
    est._ctx = _context(est._device)
    est.fit(locs, vals)  # samples sharing a location keep the first, with a warning
    kept = est._samples[0]
    n_all, n_kept = len(locs), len(kept)

    if isinstance(targets, Geometry):
        targets = BlockModel(targets)
    xyz = est._locate(targets)
    m = len(xyz)
    tidx, sidx, wts = [], [], []
    remaining = np.arange(m)
    with est._support(targets):
        for p in range(len(est.searches)):
            if len(remaining) == 0:
                break
            got, idx, w = _pass_weights(est, p, xyz[remaining], None)
            use = got[:, None] & (idx >= 0)
            t = np.broadcast_to(remaining[:, None], idx.shape)
            tidx.append(t[use]), sidx.append(idx[use]), wts.append(w[use])
            remaining = remaining[~got]
    t_all = np.concatenate(tidx) if tidx else np.zeros(0, dtype=np.int64)
    order = np.argsort(t_all, kind="stable")  # target order; each target's list stays in its order
    # bincount adds each bin's weights in input order, from 0.0: the reference's sum, term for term
    sums = (np.bincount(np.concatenate(sidx)[order], weights=np.concatenate(wts)[order], minlength=n_kept)
            if len(order) else np.zeros(n_kept))
    total = _seq_sum(sums)
    if not total > 0.0:
        raise InvalidInput("no target was estimated")
    sums = sums * (n_kept / total)

    # Samples sharing a location share the weight of the one kept.
    key = lambda a: [tuple(r) for r in (np.asarray(a, dtype=np.float64) + 0.0).view(np.uint64)]  # noqa: E731
    where = {kk: i for i, kk in enumerate(key(kept))}
    owner = np.array([where[kk] for kk in key(locs)], dtype=np.int64)
    shared = np.bincount(owner, minlength=n_kept)
    weights = sums[owner] / shared[owner] * (n_all / n_kept)
    mean = _seq_sum(weights * vals) / n_all
    return Declustering(weights=weights, mean=mean, cell_size=float("nan"))
