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
    for ppc, tile, sw, sb in [(1.0, (8, 4, 1), 2, 2), (4.0, (2, 2, 8), 8, 3), (2.0, (4, 4, 2), 0, 0)]:
        set_tuning(est._ctx, dict(cfg, samples_per_cell=ppc, tile=tile, search_warps=sw, solve_blocks_per_sm=sb))
        got = predict(est, geo, N.FP64, outs, oc)
        for a, b in zip(got, base):
            np.testing.assert_array_equal(a, b)


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
    assert tuned["ms"] > 0 and len(tuned["table"]) >= 21
    got = predict(est, geo, N.MIXED, outs, oc)
    for a, b in zip(got, predict(est, geo, N.MIXED, outs, oc)):
        np.testing.assert_array_equal(a, b)
