"""Leave-one-out loss and its variogram gradient (the adjoint kernel).

References, both FP64 over the same frozen neighbourhoods: central finite
differences (h = 1e-6) of the oracle's leave-one-out loss, and torch
autograd through dense bordered solves (tests/torch_reference.py). The
reference implementation has no gradient, so neither is pinned to it; the
loss itself is the oracle's kriging at 1e-10.
"""

import numpy as np
import pytest
import torch
import torch_reference as TR
from conftest import close

from boitata_b200 import OrdinaryKriging
from boitata_b200 import workloads as W
from boitata_b200.gradient import LeaveOneOut, loo_loss, theta_of, variogram_of


def frozen(oracle, w):
    tree = oracle.Tree(w.coords, w.search, w.variogram)
    return np.array([tree.neighbors(w.coords[i], left_out=i)[1] for i in range(len(w.coords))])


def oracle_loss(oracle, w, nbr, theta):
    r = oracle.krige_lists(w.coords, w.coords, w.values, nbr, variogram_of(w.variogram, theta))
    ok = r["status"] == 0
    return float(np.mean((r["value"][ok] - w.values[ok]) ** 2)), r["value"]


def oracle_fd(oracle, w, nbr, theta, h=1e-6):
    e = np.eye(len(theta))
    return np.array([(oracle_loss(oracle, w, nbr, theta + h * e[p])[0] -
                      oracle_loss(oracle, w, nbr, theta - h * e[p])[0]) / (2 * h) for p in range(len(theta))])


def torch_grad(w, nbr, theta):
    t = torch.tensor(theta, requires_grad=True)
    loss = TR.loo_loss(t, [s.model for s in w.variogram.structures], torch.tensor(w.coords),
                       torch.tensor(w.values), torch.tensor(nbr))
    loss.backward()
    return loss.item(), t.grad.numpy()


def test_torch_reference_matches_the_oracle(oracle):
    w = W.c4(n=300)
    nbr = frozen(oracle, w)
    th = theta_of(w.variogram)
    lt, gt = torch_grad(w, nbr, th)
    assert close(lt, oracle_loss(oracle, w, nbr, th)[0], 1e-12)
    assert np.allclose(gt, oracle_fd(oracle, w, nbr, th), rtol=1e-5, atol=1e-9)


@pytest.mark.gpu
def test_loo_loss_and_gradient_match_the_references(oracle):
    w = W.c4(n=1500)
    est = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    loo = LeaveOneOut(est)
    idx, cnt, _ = est.neighbors(None, loo=True)
    nbr = frozen(oracle, w)
    assert np.array_equal(idx, nbr), "frozen neighbourhoods differ from the oracle's"
    th = theta_of(w.variogram)
    rng = np.random.default_rng(0)
    for trial in range(3):
        theta = th if trial == 0 else th * (1 + 0.1 * rng.uniform(-1, 1, len(th)))
        loss, g, nv, values = loo.evaluate(theta, values=True)
        ref_loss, ref_values = oracle_loss(oracle, w, nbr, theta)
        assert nv == len(w.coords)
        assert np.all(close(values, ref_values, 1e-10))
        assert close(loss, ref_loss, 1e-10)
        lt, gt = torch_grad(w, nbr, theta)
        assert np.allclose(g, gt, rtol=1e-8, atol=1e-12), (g, gt)
        assert np.allclose(g, oracle_fd(oracle, w, nbr, theta), rtol=1e-5, atol=1e-9)


@pytest.mark.gpu
def test_autograd_function_gives_the_adjoint_gradient():
    w = W.c4(n=800)
    loo = LeaveOneOut(OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values))
    theta = torch.tensor(theta_of(w.variogram), requires_grad=True)
    loss = loo_loss(theta, loo)
    (2.0 * loss).backward()
    _, g, _ = loo.evaluate(theta.detach().numpy())
    np.testing.assert_allclose(theta.grad.numpy(), 2.0 * g, rtol=1e-14)
    with torch.no_grad():
        step = theta - 0.01 * theta.grad / theta.grad.abs().max()
    assert loo.evaluate(step.numpy(), grad=False)[0] < loss.item()
