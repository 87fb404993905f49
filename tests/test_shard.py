"""The path over several ranks (boitata_b200.shard): slabs of a block model and leave-one-out sums reduced
across ranks. The host logic runs as gloo ranks on CPU with world size 2, against single-process results
of the oracle and of the FP64 torch reference; the engine's range sums run on one GPU."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import _shard_workers as SW
from boitata_b200 import BlockModel, Geometry, shard
from boitata_b200 import workloads as W


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(fn, world, data, tmp_path):
    mp.spawn(fn, args=(world, free_port(), str(tmp_path), data), nprocs=world, join=True)
    return [np.load(os.path.join(tmp_path, f"rank{r}.npz")) for r in range(world)]


def test_split_is_a_balanced_partition():
    for n in (0, 1, 7, 80, 1001):
        for world in (1, 2, 3, 8):
            parts = shard.split(n, world)
            assert sum(c for _, c in parts) == n
            assert all(parts[i][0] + parts[i][1] == parts[i + 1][0] for i in range(world - 1))
            assert max(c for _, c in parts) - min(c for _, c in parts) <= 1


def test_slabs_are_whole_k_layers_covering_the_model():
    g = Geometry((0.0, 0.0, 0.0), (2.5, 2.5, 3.125), (20, 30, 13))
    for world in (1, 2, 4, 13):
        cells = [shard.slab(g, r, world) for r in range(world)]
        assert cells[0][0] == 0 and sum(c for _, c in cells) == g.cells()
        for f, c in cells:
            assert f % (20 * 30) == 0 and c % (20 * 30) == 0


def test_leave_one_out_sums_reduce_over_two_gloo_ranks(oracle, tmp_path):
    import torch
    import torch_reference as TR

    from boitata_b200.gradient import theta_of

    w = W.c4(n=240)
    tree = oracle.Tree(w.coords, w.search, w.variogram)
    nbr = np.array([tree.neighbors(w.coords[i], left_out=i)[1] for i in range(len(w.coords))])
    theta = theta_of(w.variogram)
    models = [s.model for s in w.variogram.structures]
    t = torch.tensor(theta, requires_grad=True)
    full = TR.loo_loss(t, models, torch.tensor(w.coords), torch.tensor(w.values), torch.tensor(nbr))
    full.backward()
    data = {"coords": w.coords, "values": w.values, "nbr": nbr, "theta": theta, "models": models}
    for r in run_ranks(SW.loo_rank, 2, data, tmp_path):
        assert int(r["cnt"]) == len(w.coords)
        assert abs(float(r["loss"]) - full.item()) <= 1e-13 * (1 + abs(full.item()))
        np.testing.assert_allclose(r["grad"], t.grad.numpy(), rtol=1e-11, atol=1e-15)


def test_block_model_slabs_gather_over_two_gloo_ranks(oracle, tmp_path):
    w = W.c1()
    g = Geometry((0.0, 0.0, 0.0), (20.0, 20.0, 10.0), (12, 10, 7))
    data = {"geometry": g, "coords": w.coords, "values": w.values, "search": w.search, "variogram": w.variogram}
    ranks = run_ranks(SW.slab_rank, 2, data, tmp_path)
    xyz = oracle.centroids(g.origin, g.size, g.count, g.rotation)
    want = oracle.estimate_many(xyz, w.coords, w.values, w.search, w.variogram, threads=1, neighbors=False)
    for r in ranks:
        np.testing.assert_array_equal(r["full"][:, 0], want["value"])
        np.testing.assert_array_equal(r["full"][:, 1], want["variance"])
    assert int(ranks[0]["count"]) + int(ranks[1]["count"]) == g.cells()


@pytest.mark.gpu
def test_engine_range_sums_add_up_to_the_whole():
    from boitata_b200 import OrdinaryKriging
    from boitata_b200.gradient import LeaveOneOut, theta_of

    w = W.c4(n=3000)
    est = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    loo = LeaveOneOut(est)
    th = theta_of(w.variogram)
    loss, grad, n = loo.evaluate(th)
    parts = [shard.loo_sums(loo, th, f, c) for f, c in shard.split(loo.n, 3)]
    got = shard.finish(np.sum(parts, axis=0))
    assert got[2] == n
    assert abs(got[0] - loss) <= 1e-12 * (1 + abs(loss))
    np.testing.assert_allclose(got[1], grad, rtol=1e-10, atol=1e-14)
    single = LeaveOneOut(est, sharded=True).evaluate(th)  # one rank: the whole range
    assert single[2] == n and abs(single[0] - loss) <= 1e-12 * (1 + abs(loss))


@pytest.mark.gpu
def test_slabs_of_a_block_model_give_the_whole_models_bits():
    from boitata_b200 import OrdinaryKriging

    w = W.c2()
    g = Geometry((100.0, 100.0, 60.0), (2.5, 2.5, 3.125), (40, 40, 24))
    est = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    whole = est.predict_full(g)
    for world in (2, 3):
        vals = []
        for r in range(world):
            first, count = shard.slab(g, r, world)
            vals.append(est.predict_full(BlockModel(g).centroids(est._ctx, first, count))["value"])
        np.testing.assert_array_equal(np.concatenate(vals), whole["value"])
