"""Kriging objectives and their variogram gradients (the adjoint kernel):
the leave-one-out loss and the mean estimate of a block model.

References, both FP64 over the same frozen neighbourhoods: central finite
differences (h = 1e-6) of the oracle's objective, and torch autograd
through dense bordered solves (tests/torch_reference.py). The reference
implementation has no gradient, so neither is pinned to it; the objectives
themselves are the oracle's kriging at 1e-10 (FP64 form) or 1e-8 (mixed
form: FP32 factorisation, FP64 refinement and gradient sums).
"""

import numpy as np
import pytest
import torch
import torch_reference as TR
from conftest import close

from boitata_b200 import Geometry, OrdinaryKriging, Search
from boitata_b200 import workloads as W
from boitata_b200.gradient import BlockMean, LeaveOneOut, block_mean, loo_loss, theta_of, variogram_of


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


# (value tolerance, gradient rtol against the torch reference) per form
FORMS = {"fp64": (1e-10, 1e-8), "mixed": (1e-8, 1e-6)}


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_loo_loss_and_gradient_match_the_references(oracle, precision):
    vtol, gtol = FORMS[precision]
    w = W.c4(n=1500)
    est = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    loo = LeaveOneOut(est, precision=precision)
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
        assert np.all(close(values, ref_values, vtol))
        assert close(loss, ref_loss, vtol)
        lt, gt = torch_grad(w, nbr, theta)
        assert np.allclose(g, gt, rtol=gtol, atol=1e-12), (g, gt)
        assert np.allclose(g, oracle_fd(oracle, w, nbr, theta), rtol=1e-5, atol=1e-9)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_loo_gradient_at_full_c4_size(oracle, precision):
    """c4 at its full 20,000 samples (32 neighbours each): loss and gradient against the torch FP64 dense
    reference over every system."""
    vtol, gtol = FORMS[precision]
    w = W.c4(device=torch.device("cuda", 0))
    est = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    loo = LeaveOneOut(est, precision=precision)
    idx, _, _ = est.neighbors(None, loo=True)
    th = theta_of(w.variogram)
    loss, g, nv = loo.evaluate(th)
    assert nv == len(w.coords)
    dev = torch.device("cuda", 0)
    t = torch.tensor(th, requires_grad=True, device=dev)
    ref = TR.loo_loss(t, [s.model for s in w.variogram.structures], torch.tensor(w.coords, device=dev),
                      torch.tensor(w.values, device=dev), torch.tensor(idx, device=dev))
    ref.backward()
    assert close(loss, ref.item(), vtol)
    np.testing.assert_allclose(g, t.grad.cpu().numpy(), rtol=gtol, atol=1e-12)


@pytest.mark.gpu
def test_loo_gradient_with_64_samples(oracle):
    """Systems of up to 64 samples take the two-warp form of the kernel."""
    w = W.c4(n=1200)
    s = Search(radius=float("inf"), max_samples=48, min_samples=1)
    est = OrdinaryKriging(w.variogram, s).fit(w.coords, w.values)
    th = theta_of(w.variogram)
    idx, _, _ = est.neighbors(None, loo=True)
    t = torch.tensor(th, requires_grad=True)
    ref = TR.loo_loss(t, [x.model for x in w.variogram.structures], torch.tensor(w.coords), torch.tensor(w.values),
                      torch.tensor(idx))
    ref.backward()
    for precision in ("fp64", "mixed"):
        vtol, gtol = FORMS[precision]
        loss, g, nv = LeaveOneOut(est, precision=precision).evaluate(th)
        assert nv == len(w.coords) and close(loss, ref.item(), vtol)
        np.testing.assert_allclose(g, t.grad.numpy(), rtol=gtol, atol=1e-12)


def small_c5():
    """c5's model on a tenth of its holes, and a 40 x 40 x 8 block model over one corner of its box."""
    w = W.c5(holes=160)
    return w, Geometry((100.0, 100.0, 50.0), (5.0, 5.0, 12.5), (40, 40, 8))


@pytest.mark.gpu
def test_block_mean_matches_predict_and_the_references(oracle):
    w, geo = small_c5()
    est = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    th = theta_of(w.variogram)
    fp64 = BlockMean(est, geo)
    mean, g, nv, values = fp64.evaluate(th, values=True)
    pred = est.predict_full(geo)
    # The FP64 objective is the prediction path's estimate, bit for bit.
    np.testing.assert_array_equal(values, pred["value"])
    fin = np.isfinite(values)
    assert nv == fin.sum() and close(mean, values[fin].mean(), 1e-12)
    cent = oracle.centroids(geo.origin, geo.size, geo.count, geo.rotation)
    idx, cnt, good = est.neighbors(cent)
    nbr = np.where(good[:, None], idx, -1)[fin]
    dev = torch.device("cuda", 0)
    t = torch.tensor(th, requires_grad=True, device=dev)
    ref, _ = TR.mean_estimate(t, [s.model for s in w.variogram.structures], torch.tensor(w.coords, device=dev),
                              torch.tensor(w.values, device=dev), torch.tensor(cent[fin], device=dev),
                              torch.tensor(nbr, device=dev))
    ref.backward()
    assert close(mean, ref.item(), 1e-10)
    # Condition numbers reach ~5e5 here: two FP64 solves differ by ~1e-10 relative.
    np.testing.assert_allclose(g, t.grad.cpu().numpy(), rtol=1e-6, atol=1e-10)

    def oracle_mean(theta):
        r = oracle.krige_lists(cent[fin], w.coords, w.values, nbr, variogram_of(w.variogram, theta))
        return r["value"].mean()

    h, e = 1e-6, np.eye(len(th))
    fd = np.array([(oracle_mean(th + h * e[p]) - oracle_mean(th - h * e[p])) / (2 * h) for p in range(len(th))])
    np.testing.assert_allclose(g, fd, rtol=1e-3, atol=1e-4)
    mixed = BlockMean(est, geo, precision="mixed")
    m2, g2, nv2, v2 = mixed.evaluate(th, values=True)
    assert nv2 == nv and np.all(close(v2[fin], values[fin], 1e-8)) and close(m2, mean, 1e-8)
    np.testing.assert_allclose(g2, g, rtol=1e-5, atol=1e-9)
    # tuning.mixed_large: the mixed form's systems above 32 samples by the FP64 kernel, as in prediction.
    from boitata_b200.autotune import get_tuning, set_tuning

    set_tuning(est._ctx, dict(get_tuning(est._ctx), mixed_large=1))
    m3, g3, nv3, v3 = mixed.evaluate(th, values=True)
    assert m3 == mean and nv3 == nv
    np.testing.assert_array_equal(g3, g)
    np.testing.assert_array_equal(v3, values)
    set_tuning(est._ctx, dict(get_tuning(est._ctx), mixed_large=0))


@pytest.mark.gpu
def test_block_mean_autograd_and_sharded_sums():
    from boitata_b200 import shard

    w, geo = small_c5()
    est = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    bm = BlockMean(est, geo)
    theta = torch.tensor(theta_of(w.variogram), requires_grad=True)
    value = block_mean(theta, bm)
    value.backward()
    mean, g, nv = bm.evaluate(theta.detach().numpy())
    assert value.item() == mean
    np.testing.assert_allclose(theta.grad.numpy(), g, rtol=1e-14)
    parts = [shard.loo_sums(bm, theta.detach().numpy(), f, c) for f, c in shard.split(bm.n, 3)]
    m3, g3, n3 = shard.finish(np.sum(parts, axis=0))
    assert n3 == nv and close(m3, mean, 1e-13)
    np.testing.assert_allclose(g3, g, rtol=1e-11, atol=1e-14)


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
