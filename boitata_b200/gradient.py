"""Gradient of the leave-one-out cross-validation loss with respect to the variogram.

The reference cross-validates (python/boitata/estimation.py:337-355 ->
crates/estimation/src/batch.rs:165-190) but has no gradient of it. Here the
mean squared leave-one-out error of ordinary kriging, with every sample's
neighbourhood frozen at the fitted variogram, and its gradient come from a
hand-written adjoint kernel (btk_loo_gradient) that reuses each system's
forward factorisation and recomputes covariance derivatives instead of
storing matrices. `LeaveOneOutLoss` puts it behind torch.autograd.

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


class LeaveOneOut:
    """Leave-one-out loss and gradient of a fitted ordinary-kriging estimator,
    neighbourhoods frozen at the time of construction. With sharded=True
    (one process per GPU under torch.distributed, the estimator fitted on
    every rank) each rank takes a contiguous share of the left-out samples and
    one all-reduce over `group` combines the partial sums (boitata_b200.shard),
    so every rank gets the whole loss and gradient."""

    def __init__(self, estimator, *, sharded=False, group=None):
        estimator._fitted()
        if estimator._kind != N.ORDINARY:
            raise InvalidInput("the leave-one-out gradient is for ordinary kriging")
        self.estimator = estimator
        self.template = estimator.variogram
        estimator._use_pass(0)
        ctx = estimator._ctx
        ctx.check(ctx._lib.btk_loo_freeze(ctx.handle), "freeze")
        self.n = len(estimator._samples[0])
        self.sharded, self.group = sharded, group

    @property
    def theta0(self):
        return theta_of(self.template)

    def evaluate(self, theta, grad=True, values=False):
        """(loss, gradient or None, number of samples in the loss[, estimates])."""
        if self.sharded:
            if values:
                raise InvalidInput("leave-one-out estimates are per rank; evaluate(values=True) needs sharded=False")
            from .shard import loo_loss_sharded

            return loo_loss_sharded(self, theta, group=self.group, grad=grad)
        vg = variogram_of(self.template, theta)
        c = _variogram_c(vg)
        ns = len(vg.structures)
        g = np.zeros(1 + 2 * ns + 5)
        loss = ctypes.c_double(0.0)
        nv = ctypes.c_int64(0)
        est = np.empty(self.n) if values else None
        ctx = self.estimator._ctx
        rc = ctx._lib.btk_loo_gradient(ctx.handle, ctypes.byref(c), 1 if grad else 0, ctypes.byref(loss),
                                       g.ctypes.data if grad else None, ctypes.byref(nv),
                                       None if est is None else est.ctypes.data)
        ctx.check(rc, "leave-one-out gradient")
        out = (loss.value, g if grad else None, nv.value)
        return out + (est,) if values else out


def _function():
    import torch

    class LeaveOneOutLoss(torch.autograd.Function):
        """loss = LeaveOneOutLoss.apply(theta, loo): FP64 scalar; backward gives dloss/dtheta."""

        @staticmethod
        def forward(ctx, theta, loo):
            loss, g, _ = loo.evaluate(theta.detach().cpu().numpy().astype(np.float64), grad=True)
            ctx.save_for_backward(torch.from_numpy(g).to(theta.device, theta.dtype))
            return torch.tensor(loss, dtype=theta.dtype, device=theta.device)

        @staticmethod
        def backward(ctx, grad_out):
            (g,) = ctx.saved_tensors
            return grad_out * g, None

    return LeaveOneOutLoss


_cls = None


def loo_loss(theta, loo):
    """Differentiable leave-one-out loss of `loo` (a LeaveOneOut) at torch tensor `theta`."""
    global _cls
    if _cls is None:
        _cls = _function()
    return _cls.apply(theta, loo)
