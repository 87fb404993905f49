"""The kriging path over several ranks, one process per GPU.

Targets are independent (crates/estimation/src/batch.rs:15-38 krigs each on
its own), so a block model splits into contiguous slabs of k-layers, one per
rank, with the samples (a few MB) replicated on every rank and nothing
exchanged on the data path. A slab is a range of cell indices of the whole
model (row index i + nx (j + ny k), block_model.rs:62-86), so each rank's
centroids, and its FP64 results, are bit for bit those of the unsharded run.

The leave-one-out loss and gradient split over the left-out samples, and the
block-model mean over the cells: each rank sums its range's objective
terms, count and gradient terms (btk_loo_gradient_range,
btk_mean_gradient_range) and one all-reduce of those 2 + p FP64 values
gives every rank the same value and gradient.

`group` is a torch.distributed process group (None: the default group when
torch.distributed is initialised, else a single rank).
"""

import ctypes

import numpy as np

from .errors import InvalidInput
from .geometry import BlockModel, Geometry


def rank_world(group=None):
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def split(n, world):
    """Contiguous, balanced (first, count) ranges of range(n) for ranks 0 .. world - 1."""
    if world < 1 or n < 0:
        raise InvalidInput("split needs n >= 0 and at least one rank")
    return [(n * r // world, n * (r + 1) // world - n * r // world) for r in range(world)]


def slab(geometry, rank, world):
    """(first cell, cell count) of `rank`'s k-layers of `geometry`."""
    nx, ny, nz = geometry.count
    k0, nk = split(nz, world)[rank]
    return k0 * nx * ny, nk * nx * ny


def _device(group):
    import torch
    import torch.distributed as dist

    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"


def all_reduce_sum(values, group=None):
    """Sum of a float64 vector over the ranks, on every rank."""
    values = np.asarray(values, dtype=np.float64)
    if rank_world(group)[1] == 1:
        return values.copy()
    import torch
    import torch.distributed as dist

    t = torch.as_tensor(values).to(_device(group))
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def all_gather_rows(local, group=None):
    """Every rank's `local` array (same trailing shape and dtype, any length) concatenated in rank order,
    on every rank."""
    local = np.ascontiguousarray(local)
    _, world = rank_world(group)
    if world == 1:
        return local.copy()
    import torch
    import torch.distributed as dist

    dev = _device(group)
    n = torch.tensor([local.shape[0]], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    sizes = [int(s.item()) for s in sizes]
    buf = np.zeros((max(sizes),) + local.shape[1:], dtype=local.dtype)
    buf[: local.shape[0]] = local
    t = torch.from_numpy(buf).to(dev)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    return np.concatenate([p.cpu().numpy()[:s] for p, s in zip(parts, sizes)])


def predict_slab(estimator, geometry, *, group=None, precision=None):
    """This rank's slab of `geometry` kriged by `estimator` (fitted on every rank): (first cell, outputs of
    predict_full for cells first .. first + count - 1)."""
    if not isinstance(geometry, Geometry):
        raise InvalidInput("predict_slab needs a Geometry")
    rank, world = rank_world(group)
    first, count = slab(geometry, rank, world)
    xyz = BlockModel(geometry).centroids(estimator._ctx, first, count)
    return first, estimator.predict_full(xyz, precision=precision)


def predict_sharded(estimator, geometry, *, group=None, precision=None, keys=("value", "variance")):
    """Kriging of the whole block model with each rank taking its slab, gathered on every rank in cell
    order: {key: array over all cells}."""
    _, out = predict_slab(estimator, geometry, group=group, precision=precision)
    return {k: all_gather_rows(np.asarray(out[k]), group) for k in keys}


def loo_sums(loo, theta, first, count, grad=True):
    """Partial sums of a LeaveOneOut (or BlockMean) over systems first .. first + count - 1: [objective sum,
    systems counted, gradient sums...]."""
    return loo.range_sums(theta, first, count, grad)


def finish(sums):
    """(loss, gradient, systems) from summed partial sums."""
    sums = np.asarray(sums, dtype=np.float64)
    cnt = sums[1]
    if cnt <= 0:
        return float("nan"), np.full(len(sums) - 2, np.nan), 0
    return float(sums[0] / cnt), sums[2:] / cnt, int(round(cnt))


def objective_sharded(obj, theta, *, group=None, grad=True):
    """A LeaveOneOut's loss or a BlockMean's mean, and its gradient, with the systems split over the ranks:
    (value, gradient or None, systems), the same on every rank."""
    rank, world = rank_world(group)
    first, count = split(obj.n, world)[rank]
    value, g, cnt = finish(all_reduce_sum(loo_sums(obj, theta, first, count, grad), group))
    return value, (g if grad else None), cnt


loo_loss_sharded = objective_sharded


__all__ = ["rank_world", "split", "slab", "all_reduce_sum", "all_gather_rows", "predict_slab", "predict_sharded",
           "loo_sums", "finish", "objective_sharded", "loo_loss_sharded"]
