"""btk_solve_noalloc: kriging for callers that cannot allocate device memory.

Some callers cannot call cudaMalloc: a host that owns every device
allocation through its own arena or pool, or a plugin running inside
another program's CUDA context with a fixed memory budget. They own every
buffer and hand the engine device pointers; the entry point's only scratch
is a static device array inside the library. This test gives it buffers
allocated by torch (standing in for such a host), fed with the neighbour
lists of the engine's own search, and checks that two calls in a row give
the results of the ordinary predict path.

This file sorts last so that a run stopping at the first failure has
already run every other test.
"""

import ctypes

import numpy as np
import pytest
from conftest import close

from boitata_b200 import OrdinaryKriging
from boitata_b200 import _native as N
from boitata_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_no_alloc_entry_point_matches_predict():
    import torch

    from oracle import oracle

    w = W.c1()
    g = w.geometry
    targets = oracle.centroids(g.origin, g.size, g.count, g.rotation)[::5]
    ok = OrdinaryKriging(w.variogram, w.search, precision="mixed").fit(w.coords, w.values)
    want = ok.predict_full(targets)
    idx, cnt, good = ok.neighbors(targets)
    locs, vals, _ = ok._samples
    m, k = idx.shape
    dev = torch.device("cuda", 0)

    def d(a, dtype):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dtype=dtype, device=dev)

    sx, sy, sz = (d(locs[:, a], torch.float64) for a in range(3))
    sv = d(vals, torch.float64)
    tx, ty, tz = (d(targets[:, a], torch.float64) for a in range(3))
    nbr = d(np.where(idx < 0, 0, idx).astype(np.int64), torch.int64).to(torch.int32)
    count = d(cnt, torch.int32)
    status = d(np.where(good, N.ST_OK, N.ST_SEARCH_FAILED).astype(np.int8), torch.int8)
    lib = N.library()
    stream = torch.cuda.Stream(dev)
    vg = w.variogram.to_c()
    err = ctypes.create_string_buffer(256)
    for call in range(2):
        out = {key: torch.full((m,), float("nan"), dtype=torch.float64, device=dev)
               for key in ("value", "variance", "lagrange")}
        out["n_used"] = torch.zeros(m, dtype=torch.int32, device=dev)
        out["status"] = torch.full((m,), -1, dtype=torch.int8, device=dev)
        oc = N.OutputsC(*(out[key].data_ptr() for key in ("value", "variance", "lagrange", "n_used", "status")))
        rc = lib.btk_solve_noalloc(0, ctypes.byref(vg), N.ORDINARY, 0.0, sx.data_ptr(), sy.data_ptr(),
                                   sz.data_ptr(), sv.data_ptr(), None, m, tx.data_ptr(), ty.data_ptr(),
                                   tz.data_ptr(), nbr.data_ptr(), k, count.data_ptr(), status.data_ptr(),
                                   ctypes.byref(oc), ctypes.c_void_p(stream.cuda_stream), err, len(err))
        assert rc == N.OK, err.value.decode()
        stream.synchronize()
        got = {key: v.cpu().numpy() for key, v in out.items()}
        fin = np.isfinite(want["value"])
        assert np.array_equal(fin, np.isfinite(got["value"])), f"call {call}: NaN pattern"
        assert np.array_equal(got["status"] & 0x0F, want["status"] & 0x0F), f"call {call}: status"
        assert np.array_equal(got["n_used"][fin], want["n_used"][fin])
        for key in ("value", "variance", "lagrange"):
            assert np.all(close(got[key][fin], want[key][fin], 1e-6)), f"call {call}: {key}"


def test_no_alloc_entry_point_rejects_calls_beyond_its_limit():
    lib = N.library()
    err = ctypes.create_string_buffer(256)
    vg = N.VariogramC()
    vg.nstruct = 1
    vg.s[0].model, vg.s[0].sill, vg.s[0].range = N.MODELS["spherical"], 1.0, 10.0
    oc = N.OutputsC(None, None, None, None, None)  # the size check comes before any other
    rc = lib.btk_solve_noalloc(0, ctypes.byref(vg), N.ORDINARY, 0.0, None, None, None, None, None, 262144 + 1,
                               None, None, None, None, 16, None, None, ctypes.byref(oc), None, err, len(err))
    assert rc == N.EINVAL and "at most 262144 systems" in err.value.decode()
