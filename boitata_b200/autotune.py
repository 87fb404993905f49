"""Autotuner for the engine's launch configuration.

The tunables (btk_tuning in include/boitata_b200.h):
- samples per grid cell (the cell size of the search grid);
- the block-model tile one search warp serves (32 cells);
- warps per search CTA (shared-memory granularity);
- resident solve CTAs per SM;
- the table size of the tile-shared solve (0: per-system assembly);
- for the mixed form, the tile solve's factorisation with its trailing updates on the tensor pipe or not;
- for the mixed form, the kernel of the systems above 32 samples: FP32 with FP64 refinement, or FP64.

They are picked by timing the real workload. The time is the sum of the search and solve kernels, taken
with CUDA events on the launch stream. Three stages run, each at the best of the one before: cell size x
tile, then search CTA warps, then table size x solve CTAs per SM, then (mixed form) the tensor pipe and the
large systems' kernel. Block models (autotune_geometry) and
device target arrays (autotune_device, e.g. uneven neighbour counts with per-target kinds in one launch)
are tuned alike. The choice is cached per workload signature in a JSON file (BTK_TUNING_CACHE, or
~/.cache/boitata_b200/tuning.json) and applied to the context.
"""

import ctypes
import json
import os

import numpy as np

from . import _native as N

TILES = [(4, 4, 2), (8, 4, 1), (2, 4, 4), (4, 8, 1), (8, 2, 2), (4, 2, 4), (2, 2, 8)]
SAMPLES_PER_CELL = [1.0, 2.0, 4.0]
SEARCH_WARPS = [0, 2, 8]
SOLVE_BLOCKS = [0, 2, 3]
TILE_UNION = [0, 64, 72, 96]


def cache_path():
    return os.environ.get("BTK_TUNING_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "boitata_b200",
                                                           "tuning.json"))


def get_tuning(ctx):
    t = N.TuningC()
    ctx.check(ctx._lib.btk_get_tuning(ctx.handle, ctypes.byref(t)), "tuning")
    return {"samples_per_cell": t.samples_per_cell, "tile": tuple(t.tile), "search_warps": t.search_warps,
            "solve_blocks_per_sm": t.solve_blocks_per_sm, "tile_union": t.tile_union, "host_chunk": t.host_chunk,
            "tile_tensor": t.tile_tensor, "mixed_large": t.mixed_large}


def set_tuning(ctx, cfg):
    t = N.TuningC()
    t.samples_per_cell = float(cfg["samples_per_cell"])
    for a in range(3):
        t.tile[a] = int(cfg["tile"][a])
    t.search_warps = int(cfg["search_warps"])
    t.solve_blocks_per_sm = int(cfg["solve_blocks_per_sm"])
    t.tile_union = int(cfg.get("tile_union", 64))
    t.host_chunk = int(cfg.get("host_chunk", 0))
    t.tile_tensor = int(cfg.get("tile_tensor", 0))
    t.mixed_large = int(cfg.get("mixed_large", 0))
    ctx.check(ctx._lib.btk_set_tuning(ctx.handle, ctypes.byref(t)), "tuning")


def signature(estimator, geometry, precision):
    s = estimator.searches[0]
    return json.dumps({"n": int(len(estimator._samples[0])), "max": s.max_samples, "octant": s.octant,
                       "radius": s.radius, "anisotropy": s.anisotropy or estimator.variogram.anisotropy,
                       "models": [x.model for x in estimator.variogram.structures],
                       "count": None if geometry is None else geometry.count,
                       "precision": precision}, sort_keys=True, default=str)


def time_geometry(estimator, geometry, precision, steps=2):
    """Median search + solve kernel time (ms) of one prediction over `geometry`."""
    import torch

    ctx = estimator._ctx
    m = geometry.cells()
    dev = torch.device("cuda", estimator._device)
    outs = [torch.empty(m, dtype=torch.float64, device=dev) for _ in range(3)]
    outs += [torch.empty(m, dtype=torch.int32, device=dev), torch.empty(m, dtype=torch.int8, device=dev)]
    oc = N.OutputsC(*(t.data_ptr() for t in outs))
    g = geometry.to_c()
    prec = {"fp64": N.FP64, "mixed": N.MIXED}[precision]
    ctx.check(ctx._lib.btk_set_timing(ctx.handle, 1), "timing")
    times = []
    try:
        for i in range(steps + 1):
            ctx.check(ctx._lib.btk_predict_geometry_device(ctx.handle, ctypes.byref(g), estimator._kind,
                                                           estimator._kparam, prec, ctypes.byref(oc), None),
                      "predict")
            p = (ctypes.c_float * 3)()
            ctx.check(ctx._lib.btk_phase_ms(ctx.handle, p), "timing")
            if i > 0:
                times.append(sum(p))
    finally:
        ctx._lib.btk_set_timing(ctx.handle, 0)
    return float(np.median(times))


def time_device(estimator, m, d_xyz, d_kinds=None, *, kparam=0.0, precision="mixed", steps=2):
    """Median search + solve kernel time (ms) of one prediction at m device targets (d_xyz: x, y, z arrays of
    m doubles back to back; d_kinds: one int8 kind per target, or None for the estimator's kind)."""
    import torch

    ctx = estimator._ctx
    dev = torch.device("cuda", estimator._device)
    outs = [torch.empty(m, dtype=torch.float64, device=dev) for _ in range(3)]
    outs += [torch.empty(m, dtype=torch.int32, device=dev), torch.empty(m, dtype=torch.int8, device=dev)]
    oc = N.OutputsC(*(t.data_ptr() for t in outs))
    prec = {"fp64": N.FP64, "mixed": N.MIXED}[precision]
    ctx.check(ctx._lib.btk_set_timing(ctx.handle, 1), "timing")
    times = []
    try:
        for i in range(steps + 1):
            if d_kinds is None:
                rc = ctx._lib.btk_predict_device(ctx.handle, m, d_xyz, estimator._kind, estimator._kparam, prec,
                                                 ctypes.byref(oc), None)
            else:
                rc = ctx._lib.btk_predict_kinds_device(ctx.handle, m, d_xyz, d_kinds, kparam, prec, ctypes.byref(oc),
                                                       None)
            ctx.check(rc, "predict")
            p = (ctypes.c_float * 3)()
            ctx.check(ctx._lib.btk_phase_ms(ctx.handle, p), "timing")
            if i > 0:
                times.append(sum(p))
    finally:
        ctx._lib.btk_set_timing(ctx.handle, 0)
    return float(np.median(times))


def _search(ctx, base, timer, table, mixed=False, large=False):
    """The stages over the tunables, each at the best of the one before; returns (best, ms). The mixed form
    adds the tile solve's factorisation with and without the tensor pipe and, when systems can hold more
    than 32 samples (`large`), their per-system kernel in FP32 with refinement or in FP64."""
    best, best_ms = dict(base), float("inf")
    for ppc in SAMPLES_PER_CELL:
        for tile in TILES:
            cfg = dict(base, samples_per_cell=ppc, tile=tile)
            set_tuning(ctx, cfg)
            ms = timer()
            table.append((dict(cfg), ms))
            if ms < best_ms:
                best, best_ms = dict(cfg), ms
    stage1 = dict(best)
    for sw in SEARCH_WARPS:
        cfg = dict(stage1, search_warps=sw)
        if cfg == stage1:
            continue
        set_tuning(ctx, cfg)
        ms = timer()
        table.append((dict(cfg), ms))
        if ms < best_ms:
            best, best_ms = dict(cfg), ms
    stage2 = dict(best)
    for tu in TILE_UNION:
        for sb in SOLVE_BLOCKS:
            cfg = dict(stage2, tile_union=tu, solve_blocks_per_sm=sb)
            if cfg == stage2:
                continue
            set_tuning(ctx, cfg)
            ms = timer()
            table.append((dict(cfg), ms))
            if ms < best_ms:
                best, best_ms = dict(cfg), ms
    stage3 = dict(best)
    if mixed and stage3["tile_union"] > 0:
        cfg = dict(stage3, tile_tensor=1 - int(stage3.get("tile_tensor", 0)))
        set_tuning(ctx, cfg)
        ms = timer()
        table.append((dict(cfg), ms))
        if ms < best_ms:
            best, best_ms = dict(cfg), ms
    stage4 = dict(best)
    if mixed and large:
        cfg = dict(stage4, mixed_large=1 - int(stage4.get("mixed_large", 0)))
        set_tuning(ctx, cfg)
        ms = timer()
        table.append((dict(cfg), ms))
        if ms < best_ms:
            best, best_ms = dict(cfg), ms
    return best, best_ms


def _tune(estimator, key, timer, use_cache, mixed=False):
    estimator._fitted()
    estimator._use_pass(0)
    ctx = estimator._ctx
    path = cache_path()
    cache = {}
    if use_cache and os.path.exists(path):
        try:
            with open(path) as f:
                cache = json.load(f)
        except (OSError, ValueError):
            cache = {}
    if use_cache and key in cache:
        cfg = cache[key]["best"]
        cfg["tile"] = tuple(cfg["tile"])
        set_tuning(ctx, cfg)
        return {"best": cfg, "ms": cache[key]["ms"], "table": [], "cached": True}
    table = []
    from .estimation import held_samples

    large = any(held_samples(s, len(estimator._samples[0])) > 32 for s in estimator.searches)
    best, best_ms = _search(ctx, get_tuning(ctx), timer, table, mixed, large)
    set_tuning(ctx, best)
    if use_cache:
        cache[key] = {"best": {**best, "tile": list(best["tile"])}, "ms": best_ms}
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            with open(path, "w") as f:
                json.dump(cache, f, indent=1)
        except OSError:
            pass
    return {"best": best, "ms": best_ms, "table": table, "cached": False}


def autotune_geometry(estimator, geometry, *, precision="mixed", steps=2, use_cache=True):
    """Picks and applies the fastest tuning for kriging `geometry` with `estimator` (fitted, first pass).
    Returns {"best": config, "ms": time, "table": [(config, ms), ...], "cached": bool}."""
    key = signature(estimator, geometry, precision)
    return _tune(estimator, key, lambda: time_geometry(estimator, geometry, precision, steps), use_cache,
                 precision == "mixed")


def autotune_device(estimator, m, d_xyz, d_kinds=None, *, kparam=0.0, precision="mixed", steps=2, use_cache=True,
                    tag=""):
    """As autotune_geometry for m device targets (btk_predict_device, or btk_predict_kinds_device with
    d_kinds); `tag` names the target set in the cache key (the targets themselves are not hashed)."""
    key = signature(estimator, None, precision)[:-1] + f', "targets": {m}, "kinds": {d_kinds is not None}, ' \
        f'"tag": {json.dumps(tag)}}}'
    return _tune(estimator, key,
                 lambda: time_device(estimator, m, d_xyz, d_kinds, kparam=kparam, precision=precision, steps=steps),
                 use_cache, precision == "mixed")
