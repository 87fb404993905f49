"""Launch configuration: results do not depend on the tuning, and a captured graph replays the call."""

import ctypes

import numpy as np
import pytest

from boitata_b200 import Geometry, OrdinaryKriging
from boitata_b200 import _native as N
from boitata_b200 import workloads as W
from boitata_b200.autotune import autotune_geometry, get_tuning, set_tuning

pytestmark = pytest.mark.gpu


def device_outputs(m):
    import torch

    outs = [torch.empty(m, dtype=torch.float64, device="cuda") for _ in range(3)]
    outs += [torch.empty(m, dtype=torch.int32, device="cuda"), torch.empty(m, dtype=torch.int8, device="cuda")]
    return outs, N.OutputsC(*(t.data_ptr() for t in outs))


def predict(est, geo, prec, outs, oc):
    ctx = est._ctx
    g = geo.to_c()
    ctx.check(ctx._lib.btk_predict_geometry_device(ctx.handle, ctypes.byref(g), 0, 0.0, prec, ctypes.byref(oc),
                                                   None), "predict")
    import torch

    torch.cuda.synchronize()
    return [t.clone().cpu().numpy() for t in outs]


def test_results_do_not_depend_on_the_tuning():
    w = W.c2()
    geo = Geometry((0.0, 0.0, 0.0), (2.5, 2.5, 3.125), (40, 40, 40))
    est = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    outs, oc = device_outputs(geo.cells())
    base = predict(est, geo, N.FP64, outs, oc)
    cfg = get_tuning(est._ctx)
    assert cfg["tile_union"] > 0  # the tile-shared solve is the default
    # Tables of 32 and 40 samples: tiles overflow and are retried as halves, some of which overflow too.
    for ppc, tile, sw, sb, tu in [(1.0, (8, 4, 1), 2, 2, 0), (4.0, (2, 2, 8), 8, 3, 64), (2.0, (4, 4, 2), 0, 0, 96),
                                  (2.0, (4, 4, 2), 0, 0, 32), (2.0, (4, 4, 2), 0, 0, 40)]:
        set_tuning(est._ctx, dict(cfg, samples_per_cell=ppc, tile=tile, search_warps=sw, solve_blocks_per_sm=sb,
                                  tile_union=tu))
        got = predict(est, geo, N.FP64, outs, oc)
        for a, b in zip(got, base):
            np.testing.assert_array_equal(a, b)


def test_tile_and_per_system_mixed_forms_agree():
    """The mixed form through the tile-shared kernel and through the per-system kernel: both refine to the
    FP64 solution, so they agree far inside the mixed form's 1e-6 tolerance."""
    w = W.c2()
    geo = Geometry((100.0, 100.0, 50.0), (2.5, 2.5, 3.125), (40, 40, 40))
    est = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    outs, oc = device_outputs(geo.cells())
    cfg = get_tuning(est._ctx)
    tiled = predict(est, geo, N.MIXED, outs, oc)
    exact = predict(est, geo, N.FP64, outs, oc)
    set_tuning(est._ctx, dict(cfg, tile_union=0))
    per_system = predict(est, geo, N.MIXED, outs, oc)
    # A 40-sample table: most tiles overflow it and are retried as two halves of 8 targets, and halves
    # that still do not fit go to the per-system kernel.
    set_tuning(est._ctx, dict(cfg, tile_union=40))
    halves = predict(est, geo, N.MIXED, outs, oc)
    for k in (0, 1):
        scale = 1.0 + np.maximum(np.abs(exact[k]), np.abs(tiled[k]))
        assert np.nanmax(np.abs(tiled[k] - exact[k]) / scale) < 1e-9
        assert np.nanmax(np.abs(tiled[k] - per_system[k]) / scale) < 1e-9
        assert np.nanmax(np.abs(halves[k] - exact[k]) / scale) < 1e-9
    for got in (per_system, halves):
        np.testing.assert_array_equal(tiled[3], got[3])
        np.testing.assert_array_equal(tiled[4] & 0x0F, got[4] & 0x0F)


def test_graph_replay_matches_the_call_and_autotune_keeps_results():
    import torch

    w = W.c2()
    geo = Geometry((0.0, 0.0, 0.0), (2.5, 2.5, 3.125), (40, 40, 40))
    est = OrdinaryKriging(w.variogram, w.search, precision="mixed").fit(w.coords, w.values)
    ctx = est._ctx
    outs, oc = device_outputs(geo.cells())
    for prec in (N.MIXED, N.FP64):
        want = predict(est, geo, prec, outs, oc)
        for t in outs:
            t.fill_(0)
        g = geo.to_c()
        ctx.check(ctx._lib.btk_graph_capture_geometry(ctx.handle, ctypes.byref(g), 0, 0.0, prec, ctypes.byref(oc)),
                  "capture")
        for t in outs:
            t.fill_(0)
        stream = torch.cuda.Stream()
        for _ in range(2):
            ctx.check(ctx._lib.btk_graph_launch(ctx.handle, ctypes.c_void_p(stream.cuda_stream)), "replay")
        stream.synchronize()
        for a, b in zip([t.cpu().numpy() for t in outs], want):
            np.testing.assert_array_equal(a, b)
    tuned = autotune_geometry(est, geo, precision="mixed", steps=1, use_cache=False)
    assert tuned["ms"] > 0 and len(tuned["table"]) >= 21 + 2 + 11
    got = predict(est, geo, N.MIXED, outs, oc)
    for a, b in zip(got, predict(est, geo, N.MIXED, outs, oc)):
        np.testing.assert_array_equal(a, b)


def test_caller_order_does_not_change_results():
    """btk_predict sorts caller-supplied targets into Morton order; the FP64 form gives the same bits for any
    input order, and a result lands at its own target's index."""
    w = W.c2()
    rng = np.random.default_rng(7)
    t = np.column_stack([rng.uniform(50, 450, 20000), rng.uniform(50, 450, 20000), rng.uniform(10, 240, 20000)])
    est = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    a = est.predict_full(t)
    perm = rng.permutation(len(t))
    b = est.predict_full(t[perm])
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm))
    for k in a:
        np.testing.assert_array_equal(np.asarray(b[k])[inv], np.asarray(a[k]))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_host_chunks_give_the_unchunked_results(precision):
    """A host call in chunks of tuning.host_chunk targets (the copies of chunks c - 1 out and c + 1 in overlap
    chunk c's kernels; each chunk is ordered and solved on its own) gives the one-chunk results: FP64 bit for
    bit, with the diagnostics; the mixed form far inside its 1e-6 tolerance."""
    w = W.c2()
    t = np.random.default_rng(8).uniform(0.0, 1.0, (150_000, 3)) * [500.0, 500.0, 250.0]
    kinds = np.where(np.arange(len(t)) % 7 == 0, "simple", "ordinary")
    est = OrdinaryKriging(w.variogram, w.search, precision=precision).fit(w.coords, w.values)
    whole = est.predict_full(t, diagnostics=True)
    whole_kinds = est.predict_kinds(t, kinds, mean=1.0)
    set_tuning(est._ctx, dict(get_tuning(est._ctx), host_chunk=40_000))  # four chunks
    parts = est.predict_full(t, diagnostics=True)
    parts_kinds = est.predict_kinds(t, kinds, mean=1.0)
    if precision == "fp64":
        for k in ("value", "variance", "lagrange", "n_used", "status"):
            np.testing.assert_array_equal(parts_kinds[k], whole_kinds[k])
    for k in ("n_used", "n_holes", "negative_weight_sum", "mean_distance"):
        np.testing.assert_array_equal(parts[k], whole[k])
    np.testing.assert_array_equal(parts["status"] & 0x0F, whole["status"] & 0x0F)
    assert np.isfinite(whole["value"]).mean() > 0.5
    for k in ("value", "variance", "lagrange"):
        if precision == "fp64":
            np.testing.assert_array_equal(parts[k], whole[k])
        else:
            fin = np.isfinite(whole[k])
            np.testing.assert_array_equal(fin, np.isfinite(parts[k]))
            scale = 1.0 + np.maximum(np.abs(whole[k][fin]), np.abs(parts[k][fin]))
            assert np.max(np.abs(parts[k][fin] - whole[k][fin]) / scale) < 1e-9, k


def test_device_calls_match_the_host_calls():
    """btk_predict_device and btk_predict_kinds_device (device x, y, z arrays and outputs, queued on a torch
    stream) give the host calls' results bit for bit: the same targets take the same order and tiles."""
    import torch

    w = W.c2()
    t = np.random.default_rng(10).uniform(0.0, 1.0, (60_000, 3)) * [500.0, 500.0, 250.0]
    kinds = np.where(np.arange(len(t)) % 5 == 0, N.SIMPLE, N.ORDINARY).astype(np.int8)
    keys = ("value", "variance", "lagrange", "n_used", "status")
    dxyz = torch.from_numpy(np.ascontiguousarray(t.T)).cuda()
    dkinds = torch.from_numpy(kinds).cuda()
    stream = torch.cuda.Stream()
    for precision, code in (("fp64", N.FP64), ("mixed", N.MIXED)):
        est = OrdinaryKriging(w.variogram, w.search, precision=precision).fit(w.coords, w.values)
        ctx = est._ctx
        host, host_kinds = est.predict_full(t), est.predict_kinds(t, kinds, mean=1.0)
        assert np.isfinite(host["value"]).mean() > 0.5
        outs, oc = device_outputs(len(t))
        ctx.check(ctx._lib.btk_predict_device(ctx.handle, len(t), ctypes.c_void_p(dxyz.data_ptr()), N.ORDINARY, 0.0,
                                              code, ctypes.byref(oc), ctypes.c_void_p(stream.cuda_stream)), "device")
        stream.synchronize()
        for got, k in zip(outs, keys):
            np.testing.assert_array_equal(got.cpu().numpy(), host[k])
        ctx.check(ctx._lib.btk_predict_kinds_device(ctx.handle, len(t), ctypes.c_void_p(dxyz.data_ptr()),
                                                    ctypes.c_void_p(dkinds.data_ptr()), 1.0, code, ctypes.byref(oc),
                                                    ctypes.c_void_p(stream.cuda_stream)), "kinds")
        stream.synchronize()
        for got, k in zip(outs, keys):
            np.testing.assert_array_equal(got.cpu().numpy(), host_kinds[k])


def test_lattice_targets_in_any_order_match_the_block_model():
    """Block centroids passed as coordinates, in the model's order and shuffled, are found to be a lattice and
    take the block-model path's tile order; either way the FP64 results are the block-model call's, bit for
    bit."""
    from boitata_b200 import BlockModel

    w = W.c2()
    geo = Geometry((0.0, 0.0, 0.0), (2.5, 2.5, 3.125), (60, 60, 30))
    est = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    want = est.predict_full(geo)
    cent = BlockModel(geo).centroids(est._ctx)
    perm = np.random.default_rng(3).permutation(len(cent))
    for t, back in ((cent, np.arange(len(cent))), (cent[perm], np.argsort(perm))):
        got = est.predict_full(t)
        for k in ("value", "variance", "lagrange", "n_used", "status"):
            np.testing.assert_array_equal(got[k][back], want[k])


def test_target_order_never_changes_results():
    """The order the engine gives caller targets (the lattice tile order, or Hilbert when they are not a
    lattice) is invisible: FP64 results are the same bits for every permutation of the targets. Cases: a
    flat lattice (one z), a lattice with blocks missing, a lattice too long for the tile keys (Hilbert) and a
    rotated lattice (Hilbert). A NaN target, which only the C ABI takes, turns the lattice order off and
    gets NaN; the other targets keep their results."""
    w = W.c2()
    est = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    rng = np.random.default_rng(21)
    g = np.stack(np.meshgrid(np.arange(40), np.arange(30), np.arange(6), indexing="ij"), -1).reshape(-1, 3)
    lattice = g * [5.0, 5.0, 6.25] + [100.0, 120.0, 10.0]
    a = np.deg2rad(30.0)
    rot = np.array([[np.cos(a), -np.sin(a), 0.0], [np.sin(a), np.cos(a), 0.0], [0.0, 0.0, 1.0]])
    g2 = np.stack(np.meshgrid(np.arange(60), np.arange(50), indexing="ij"), -1).reshape(-1, 2)
    flat = np.column_stack([g2 * 5.0 + [100.0, 120.0], np.full(len(g2), 10.0)])  # 3,000: ordered (2,048 up)
    holed = lattice[rng.random(len(lattice)) > 0.3]
    long = np.vstack([lattice, [[100.0 + 5.0 * 600_000, 120.0, 10.0]]])
    rotated = (lattice - 250.0) @ rot.T + 250.0
    keys = ("value", "variance", "lagrange", "n_used", "status")
    for t in (flat, holed, long, rotated):
        want = est.predict_full(t)
        perm = rng.permutation(len(t))
        got = est.predict_full(t[perm])
        back = np.argsort(perm)
        for k in keys:
            np.testing.assert_array_equal(got[k][back], want[k])
        assert np.isfinite(want["value"]).sum() >= len(t) - 1
    want = est.predict_full(lattice)
    nan = np.ascontiguousarray(lattice.copy())
    nan[17, 1] = np.nan
    out = {k: np.full(len(nan), np.nan) for k in ("value", "variance", "lagrange")}
    out["n_used"] = np.zeros(len(nan), dtype=np.int32)
    out["status"] = np.zeros(len(nan), dtype=np.int8)
    oc = N.OutputsC(*(out[k].ctypes.data for k in keys))
    ctx = est._ctx
    ctx.check(ctx._lib.btk_predict(ctx.handle, len(nan), nan.ctypes.data, N.ORDINARY, 0.0, N.FP64,
                                   ctypes.byref(oc)), "predict")
    assert np.isnan(out["value"][17])
    keep = np.arange(len(nan)) != 17
    for k in keys:
        np.testing.assert_array_equal(out[k][keep], want[k][keep])
