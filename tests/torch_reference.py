"""FP64 dense references of the leave-one-out loss and of the mean estimate
of a set of targets (test infrastructure).

Each system's bordered ordinary-kriging matrix [C 1; 1' 0] is built from
the variogram parameters theta in torch and solved densely; torch autograd
then gives the gradient the engine's adjoint kernel must match. Tensors may
live on any device. The covariance follows crates/variogram/src/{model,composite}.rs and
the frame crates/core/src/rotation.rs:8-16 with aniso.rs:88-94.
"""

import math

import torch


def shape(model, t):
    if model == "spherical":
        return torch.where(t >= 1, torch.ones_like(t), 1.5 * t - 0.5 * t ** 3)
    if model == "exponential":
        return 1 - torch.exp(-3 * t)
    if model == "gaussian":
        return 1 - torch.exp(-3 * t * t)
    raise NotImplementedError(model)


def frame(semi, minor, az, dip, rake):
    k = math.pi / 180
    sa, ca = torch.sin(az * k), torch.cos(az * k)
    sd, cd = torch.sin(dip * k), torch.cos(dip * k)
    sr, cr = torch.sin(rake * k), torch.cos(rake * k)
    z, o = torch.zeros_like(sa), torch.ones_like(sa)
    r1 = torch.stack([torch.stack([sa, ca, z]), torch.stack([-ca, sa, z]), torch.stack([z, z, o])])
    r2 = torch.stack([torch.stack([cd, z, -sd]), torch.stack([z, o, z]), torch.stack([sd, z, cd])])
    r3 = torch.stack([torch.stack([o, z, z]), torch.stack([z, cr, sr]), torch.stack([z, -sr, cr])])
    d = torch.diag(torch.stack([o, 1 / semi, 1 / minor]))
    return d @ (r3 @ r2 @ r1)


def loo_loss(theta, models, coords, values, nbr, rows=None):
    """Mean squared leave-one-out error; nbr (n x k) frozen neighbour indices (all systems full). With
    `rows` (indices of left-out samples) the mean over those samples only."""
    ns = len(models)
    nugget, sills, ranges = theta[0], theta[1:1 + ns], theta[1 + ns:1 + 2 * ns]
    M = frame(*theta[1 + 2 * ns:])
    if rows is None:
        rows = torch.arange(len(coords), device=coords.device)
    nbr = nbr[rows]
    X = coords[nbr]                             # n, k, 3
    P = (X - coords[rows][:, None, :]) @ M.T    # n, k, 3
    n, k, _ = P.shape
    eye = torch.eye(k, dtype=P.dtype, device=P.device)
    D = P[:, :, None, :] - P[:, None, :, :]
    H = torch.sqrt((D * D).sum(-1) + eye)  # the diagonal is replaced below
    h0 = torch.sqrt((P * P).sum(-1))

    def cov(h):
        return sum(sills[s] * (1 - shape(models[s], h / ranges[s])) for s in range(ns))

    C = cov(H) * (1 - eye) + eye * (nugget + sills.sum())
    K = torch.ones((n, k + 1, k + 1), dtype=P.dtype, device=P.device)
    K[:, :k, :k] = C
    K[:, k, k] = 0
    b = torch.ones((n, k + 1), dtype=P.dtype, device=P.device)
    b[:, :k] = cov(h0)
    x = torch.linalg.solve(K, b)
    est = (x[:, :k] * values[nbr]).sum(-1)
    return ((est - values[rows]) ** 2).mean()


def mean_estimate(theta, models, coords, values, targets, nbr):
    """Mean ordinary-kriging estimate over `targets` (m x 3), each kriged from its frozen neighbour list
    (nbr, m x k, -1 padded; every target with at least one sample). Padded slots are decoupled rows of the
    bordered system (unit diagonal, no covariance, no unbiasedness term), so their weights are zero."""
    ns = len(models)
    nugget, sills, ranges = theta[0], theta[1:1 + ns], theta[1 + ns:1 + 2 * ns]
    M = frame(*theta[1 + 2 * ns:])
    live = nbr >= 0
    idx = torch.where(live, nbr, torch.zeros_like(nbr))
    X = coords[idx]                               # m, k, 3
    P = (X - targets[:, None, :]) @ M.T           # m, k, 3
    m, k, _ = P.shape
    eye = torch.eye(k, dtype=P.dtype, device=P.device)
    D = P[:, :, None, :] - P[:, None, :, :]
    pair = live[:, :, None] & live[:, None, :]
    # Lags of live pairs only: padded slots share one point, and sqrt at 0 would poison the gradient.
    d2 = torch.where(pair & (eye == 0), (D * D).sum(-1), torch.ones_like(eye))
    H = torch.sqrt(d2)
    h0 = torch.sqrt(torch.where(live, (P * P).sum(-1), torch.ones_like(live, dtype=P.dtype)))

    def cov(h):
        return sum(sills[s] * (1 - shape(models[s], h / ranges[s])) for s in range(ns))

    C = torch.where(pair, cov(H) * (1 - eye) + eye * (nugget + sills.sum()), eye.expand(m, k, k))
    K = torch.zeros((m, k + 1, k + 1), dtype=P.dtype, device=P.device)
    K[:, :k, :k] = C
    lv = live.to(P.dtype)
    K[:, :k, k] = lv
    K[:, k, :k] = lv
    b = torch.zeros((m, k + 1), dtype=P.dtype, device=P.device)
    b[:, :k] = torch.where(live, cov(h0), torch.zeros_like(h0))
    b[:, k] = 1
    x = torch.linalg.solve(K, b)
    est = (x[:, :k] * values[idx] * lv).sum(-1)
    return est.mean(), est
