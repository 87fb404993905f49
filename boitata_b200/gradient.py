"""Gradients of kriging objectives with respect to the variogram.

The reference cross-validates (python/boitata/estimation.py:337-355 ->
crates/estimation/src/batch.rs:165-190) and predicts block models, but has
no gradient of either. Here two objectives, each over neighbourhoods frozen
at the fitted variogram, come with their gradients from a hand-written
adjoint kernel (btk_loo_gradient, btk_mean_gradient) that reuses each
system's forward factorisation and recomputes covariance derivatives
instead of storing matrices:
- LeaveOneOut: the mean squared leave-one-out error of ordinary kriging;
- BlockMean: the mean ordinary-kriging estimate over a block model.
Both take precision="fp64" or "mixed" (FP32 factorisation with FP64
refinement and FP64 gradient sums). `objective` (and `loo_loss`,
`block_mean`) puts them behind torch.autograd.

Parameter vector theta (float64): nugget, the sill of each structure, the
major range of each structure, the semi/major and minor/major ratios, and
the azimuth, dip and rake in degrees of the one anisotropy the structures
share (crates/variogram/src/composite.rs:13-18, aniso.rs:18-26).
"""

import ctypes

import numpy as np

from . import _native as N
from .errors import InvalidInput
from .variogram import Structure, Variogram


def theta_of(vg):
    """theta of a variogram (no anisotropy = ratios 1, 1 and angles 0)."""
    a = vg.anisotropy or (0.0, 0.0, 0.0, 1.0, 1.0, 1.0)
    return np.array([vg.nugget, *(s.sill for s in vg.structures), *(s.range for s in vg.structures), a[4], a[5],
                     a[0], a[1], a[2]], dtype=np.float64)


def variogram_of(template, theta):
    """The variogram with `template`'s models and the parameters `theta`."""
    theta = np.asarray(theta, dtype=np.float64)
    ns = len(template.structures)
    if theta.shape != (1 + 2 * ns + 5,):
        raise InvalidInput(f"theta needs {1 + 2 * ns + 5} values for {ns} structures")
    st = [Structure(s.model, theta[1 + k], theta[1 + ns + k], order=s.order, exponent=s.exponent)
          for k, s in enumerate(template.structures)]
    semi, minor, az, dip, rake = theta[1 + 2 * ns:]
    return Variogram(st, nugget=theta[0], rotation=(az, dip, rake), ratios=(semi, minor))


def _variogram_c(vg):
    c = vg.to_c()
    if not c.aniso.on:  # a point of theta: ratios 1, angles 0
        c.aniso.on, c.aniso.major, c.aniso.semi, c.aniso.minor = 1, 1.0, 1.0, 1.0
    return c


PRECISIONS = {"fp64": N.FP64, "mixed": N.MIXED}


class _Frozen:
    """A kriging objective over neighbourhoods frozen at construction, with its gradient from the adjoint
    kernel. `precision`: "fp64", or "mixed" (FP32 factorisation refined in FP64, FP64 gradient sums)."""

    _entry, _range_entry, _what = None, None, None

    def __init__(self, estimator, precision, sharded, group):
        estimator._fitted()
        if estimator._kind != N.ORDINARY:
            raise InvalidInput(f"the {self._what} gradient is for ordinary kriging")
        if precision not in PRECISIONS:
            raise InvalidInput(f"precision must be one of {sorted(PRECISIONS)}")
        self.estimator = estimator
        self.template = estimator.variogram
        self.precision = precision
        self.sharded, self.group = sharded, group

    @property
    def theta0(self):
        return theta_of(self.template)

    def range_sums(self, theta, first, count, grad=True):
        """Partial sums over systems first .. first + count - 1: [objective sum, systems counted,
        gradient sums...]."""
        vg = variogram_of(self.template, theta)
        c = _variogram_c(vg)
        out = np.zeros(2 + 1 + 2 * len(vg.structures) + 5)
        ctx = self.estimator._ctx
        rc = getattr(ctx._lib, self._range_entry)(ctx.handle, ctypes.byref(c), int(first), int(count),
                                                  1 if grad else 0, PRECISIONS[self.precision], out.ctypes.data)
        ctx.check(rc, f"{self._what} range")
        return out

    def evaluate(self, theta, grad=True, values=False):
        """(objective, gradient or None, number of systems in it[, estimates])."""
        if self.sharded:
            if values:
                raise InvalidInput("the estimates are per rank; evaluate(values=True) needs sharded=False")
            from .shard import objective_sharded

            return objective_sharded(self, theta, group=self.group, grad=grad)
        vg = variogram_of(self.template, theta)
        c = _variogram_c(vg)
        ns = len(vg.structures)
        g = np.zeros(1 + 2 * ns + 5)
        obj = ctypes.c_double(0.0)
        nv = ctypes.c_int64(0)
        est = np.empty(self.n) if values else None
        ctx = self.estimator._ctx
        rc = getattr(ctx._lib, self._entry)(ctx.handle, ctypes.byref(c), 1 if grad else 0,
                                            PRECISIONS[self.precision], ctypes.byref(obj),
                                            g.ctypes.data if grad else None, ctypes.byref(nv),
                                            None if est is None else est.ctypes.data)
        ctx.check(rc, f"{self._what} gradient")
        out = (obj.value, g if grad else None, nv.value)
        return out + (est,) if values else out


class LeaveOneOut(_Frozen):
    """Leave-one-out loss and gradient of a fitted ordinary-kriging estimator,
    neighbourhoods frozen at the time of construction. With sharded=True
    (one process per GPU under torch.distributed, the estimator fitted on
    every rank) each rank takes a contiguous share of the left-out samples and
    one all-reduce over `group` combines the partial sums (boitata_b200.shard),
    so every rank gets the whole loss and gradient."""

    _entry, _range_entry, _what = "btk_loo_gradient", "btk_loo_gradient_range", "leave-one-out"

    def __init__(self, estimator, *, precision="fp64", sharded=False, group=None):
        super().__init__(estimator, precision, sharded, group)
        estimator._use_pass(0)
        ctx = estimator._ctx
        ctx.check(ctx._lib.btk_loo_freeze(ctx.handle), "freeze")
        self.n = len(estimator._samples[0])


class BlockMean(_Frozen):
    """The mean ordinary-kriging estimate over the centroids of a block model (a Geometry) and its
    gradient with respect to the variogram, each centroid's neighbourhood frozen at construction by one
    search with the fitted variogram. The reference has no gradient of any kind; its forward here is
    predict over the centroids (crates/estimation/src/batch.rs:15-38 with kernel.rs:24-123). With
    sharded=True each rank takes a contiguous range of cells and one all-reduce combines the sums."""

    _entry, _range_entry, _what = "btk_mean_gradient", "btk_mean_gradient_range", "block-mean"

    def __init__(self, estimator, geometry, *, precision="fp64", sharded=False, group=None):
        super().__init__(estimator, precision, sharded, group)
        estimator._use_pass(0)
        ctx = estimator._ctx
        g = geometry.to_c()
        ctx.check(ctx._lib.btk_mean_freeze(ctx.handle, ctypes.byref(g)), "freeze")
        self.geometry = geometry
        self.n = geometry.cells()


def _function():
    import torch

    class FrozenObjective(torch.autograd.Function):
        """value = FrozenObjective.apply(theta, obj): FP64 scalar of a LeaveOneOut or BlockMean; backward
        gives dvalue/dtheta from the adjoint kernel."""

        @staticmethod
        def forward(ctx, theta, obj):
            value, g, _ = obj.evaluate(theta.detach().cpu().numpy().astype(np.float64), grad=True)
            ctx.save_for_backward(torch.from_numpy(g).to(theta.device, theta.dtype))
            return torch.tensor(value, dtype=theta.dtype, device=theta.device)

        @staticmethod
        def backward(ctx, grad_out):
            (g,) = ctx.saved_tensors
            return grad_out * g, None

    return FrozenObjective


_cls = None


def objective(theta, obj):
    """Differentiable value of `obj` (a LeaveOneOut or a BlockMean) at torch tensor `theta`."""
    global _cls
    if _cls is None:
        _cls = _function()
    return _cls.apply(theta, obj)


def loo_loss(theta, loo):
    """Differentiable leave-one-out loss of `loo` (a LeaveOneOut) at torch tensor `theta`."""
    return objective(theta, loo)


def block_mean(theta, bm):
    """Differentiable mean estimate of `bm` (a BlockMean) at torch tensor `theta`."""
    return objective(theta, bm)
