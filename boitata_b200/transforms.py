"""Normal-score transform of a variable and its back-transform, as the
reference's simulations take them (crates/transforms/src/normal_score.rs:
38-262, crates/transforms/src/normal.rs:7-70).

Scores match the (optionally declustered) empirical quantiles of the data to
standard-normal quantiles at the midpoint of each sorted sample's weight;
the table of (value, score) pairs back-transforms by linear interpolation,
and beyond its ends linearly in probability toward the tails (the data range
by default). The quantile function is Acklam's rational approximation
(P. J. Acklam, "An algorithm for computing the inverse normal cumulative
distribution function", 2003: its published coefficients, absolute error
about 1e-9); the CDF is 0.5 erfc(-x / sqrt 2).
"""

import math

import numpy as np

from .errors import InvalidInput

# Acklam's published coefficients: central region (a, b), tails (c, d).
_A = (-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02, 1.383577518672690e+02,
      -3.066479806614716e+01, 2.506628277459239e+00)
_B = (-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02, 6.680131188771972e+01,
      -1.328068155288572e+01)
_C = (-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00, -2.549732539343734e+00,
      4.374664141464968e+00, 2.938163982698783e+00)
_D = (7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00, 3.754408661907416e+00)
_PLOW = 0.02425


def probit(p):
    """Standard-normal quantile of p, clamped to [1e-15, 1 - 1e-15] (normal.rs:17-70)."""
    p = min(max(float(p), 1e-15), 1.0 - 1e-15)
    if p < _PLOW:
        q = math.sqrt(-2.0 * math.log(p))
        return ((((((_C[0] * q + _C[1]) * q + _C[2]) * q + _C[3]) * q + _C[4]) * q + _C[5])
                / ((((_D[0] * q + _D[1]) * q + _D[2]) * q + _D[3]) * q + 1.0))
    if p <= 1.0 - _PLOW:
        q = p - 0.5
        r = q * q
        return ((((((_A[0] * r + _A[1]) * r + _A[2]) * r + _A[3]) * r + _A[4]) * r + _A[5]) * q
                / (((((_B[0] * r + _B[1]) * r + _B[2]) * r + _B[3]) * r + _B[4]) * r + 1.0))
    q = math.sqrt(-2.0 * math.log(1.0 - p))
    return -((((((_C[0] * q + _C[1]) * q + _C[2]) * q + _C[3]) * q + _C[4]) * q + _C[5])
             / ((((_D[0] * q + _D[1]) * q + _D[2]) * q + _D[3]) * q + 1.0))


def phi(x):
    """Standard-normal CDF (normal.rs:7-10)."""
    return 0.5 * math.erfc(-float(x) / math.sqrt(2.0))


class NormalScoreTable:
    """Monotone value <-> score table with linear tails in probability (normal_score.rs:15-28, 190-262)."""

    def __init__(self, values, scores, tails):
        self.values = np.asarray(values, dtype=np.float64)
        self.scores = np.asarray(scores, dtype=np.float64)
        self.tails = (float(tails[0]), float(tails[1]))

    def with_tails(self, lower, upper):
        n = len(self.values)
        return NormalScoreTable(self.values, self.scores,
                                (min(lower, self.values[0]), max(upper, self.values[n - 1])))

    def back(self, score):
        """normal_score.rs:209-222."""
        n, (lo, hi) = len(self.values), self.tails
        score = float(score)
        if n > 1 and score < self.scores[0]:
            fraction = phi(score) / phi(self.scores[0])
            return lo + (self.values[0] - lo) * fraction
        if n > 1 and score > self.scores[n - 1]:
            edge = phi(self.scores[n - 1])
            fraction = (phi(score) - edge) / (1.0 - edge)
            return self.values[n - 1] + (hi - self.values[n - 1]) * fraction
        return _lookup(self.scores, self.values, score)

    def forward(self, value):
        """normal_score.rs:225-245: a value tied in the table gets the mean score of its ties."""
        value = float(value)
        first = int(np.searchsorted(self.values, value, side="left"))
        last = int(np.searchsorted(self.values, value, side="right"))
        if last > first:
            return float(sum(self.scores[first:last])) / (last - first)
        n, (lo, hi) = len(self.values), self.tails
        if n > 1 and value < self.values[0]:
            fraction = min(max((value - lo) / (self.values[0] - lo), 0.0), 1.0)
            return probit(fraction * phi(self.scores[0]))
        if n > 1 and value > self.values[n - 1]:
            edge = phi(self.scores[n - 1])
            fraction = min(max((value - self.values[n - 1]) / (hi - self.values[n - 1]), 0.0), 1.0)
            return probit(edge + fraction * (1.0 - edge))
        return _lookup(self.values, self.scores, value)


def _lookup(xs, ys, x):
    """normal_score.rs:247-262: linear interpolation on the bracketing pair."""
    n = len(xs)
    if n == 0:
        return math.nan
    if n == 1:
        return float(ys[0])
    hi = min(max(int(np.searchsorted(xs, x, side="right")), 1), n - 1)
    x0, x1, y0, y1 = float(xs[hi - 1]), float(xs[hi]), float(ys[hi - 1]), float(ys[hi])
    if abs(x1 - x0) < 2.2250738585072014e-308:
        return y0
    return y0 + (y1 - y0) * (x - x0) / (x1 - x0)


def normalized_weights(weights, n):
    """normal_score.rs:136-150."""
    if weights is None:
        return np.full(n, 1.0 / n)
    w = np.asarray(weights, dtype=np.float64)
    s = float(sum(w.tolist()))
    if not math.isfinite(s) or s <= 0.0 or np.any(~np.isfinite(w)) or np.any(w < 0.0):
        raise InvalidInput("weights must be finite and >= 0, with a finite sum > 0")
    return w / s


def normal_score(values, weights=None):
    """(scores aligned with `values`, table) of the forward transform (normal_score.rs:38-134, uncensored):
    samples sorted stably by value, each scored at the midpoint of its cumulative weight; zero-weight
    samples are left out of the CDF and scored from the table."""
    v = np.asarray(values, dtype=np.float64)
    n = len(v)
    if n == 0:
        raise InvalidInput("no values")
    if weights is not None and len(weights) != n:
        raise InvalidInput("weights length mismatch")
    order = np.argsort(v, kind="stable")
    w = normalized_weights(weights, n)
    floor = 1e-10 * max(0.0, float(np.max(w)))
    kept = [int(i) for i in order if w[i] > floor]
    if len(kept) < n:
        total = 0.0
        for i in kept:
            total += w[i]
        w = w / total
    scores = np.zeros(n)
    cum = 0.0
    tv, ts = [], []
    for i in kept:
        wi = w[i]
        p = cum + wi / 2.0
        cum += wi
        z = probit(p)
        scores[i] = z
        tv.append(v[i])
        ts.append(z)
    table = NormalScoreTable(tv, ts, (tv[0], tv[-1]))
    if len(kept) < n:
        lo, hi = tv[0], tv[-1]
        for i in order:
            if w[i] <= floor:
                scores[i] = table.forward(min(max(v[i], lo), hi))
    return scores, table
