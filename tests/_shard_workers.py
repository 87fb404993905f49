"""Rank bodies for the multi-process shard tests (gloo on CPU). Module level so that spawned processes can
import them; each writes its result to out_dir/rank<r>.npz."""

import os
import sys

import numpy as np


def _init(rank, world, port):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    return dist


def loo_rank(rank, world, port, out_dir, data):
    """Partial leave-one-out sums of this rank's samples from the FP64 torch reference, reduced with
    shard.all_reduce_sum and finished with shard.finish."""
    sys.path.insert(0, os.path.dirname(__file__))
    import torch
    import torch_reference as TR

    from boitata_b200 import shard

    dist = _init(rank, world, port)
    try:
        coords, values, nbr, theta, models = (data[k] for k in ("coords", "values", "nbr", "theta", "models"))
        first, count = shard.split(len(coords), world)[rank]
        rows = torch.arange(first, first + count)
        t = torch.tensor(theta, requires_grad=True)
        mean = TR.loo_loss(t, models, torch.tensor(coords), torch.tensor(values), torch.tensor(nbr), rows=rows)
        part = mean * count
        part.backward()
        sums = np.concatenate([[part.item(), float(count)], t.grad.numpy()])
        loss, grad, cnt = shard.finish(shard.all_reduce_sum(sums))
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), loss=loss, grad=grad, cnt=cnt)
    finally:
        dist.destroy_process_group()


def slab_rank(rank, world, port, out_dir, data):
    """The oracle's kriging of this rank's slab of a block model, gathered with shard.all_gather_rows."""
    sys.path.insert(0, os.path.dirname(os.path.dirname(__file__)))
    from boitata_b200 import shard
    from oracle import oracle as O

    dist = _init(rank, world, port)
    try:
        g = data["geometry"]
        first, count = shard.slab(g, rank, world)
        xyz = O.centroids(g.origin, g.size, g.count, g.rotation, first, count)
        r = O.estimate_many(xyz, data["coords"], data["values"], data["search"], data["variogram"], threads=1,
                            neighbors=False)
        full = shard.all_gather_rows(np.column_stack([r["value"], r["variance"]]))
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), full=full, first=first, count=count)
    finally:
        dist.destroy_process_group()
