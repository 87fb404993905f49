"""btk_solve_noalloc: kriging for callers that cannot allocate device memory.

Some callers cannot call cudaMalloc: a host that owns every device
allocation through its own arena or pool, or a plugin running inside
another program's CUDA context with a fixed memory budget. They own every
buffer and hand the engine device pointers; the entry point's only scratch
is a static device array inside the library. These tests give it buffers
allocated by torch (standing in for such a host), fed with the neighbour
lists of the engine's own search, and check its results against the oracle
(the reference's kriging restated on the CPU) on the same lists, call after
call: the scratch array keeps the last call's contents, so each call must
start its re-solve list from zero.

This file sorts last so that a run stopping at the first failure has
already run every other test.
"""

import ctypes

import numpy as np
import pytest
from conftest import close

from boitata_b200 import OrdinaryKriging, Structure, Variogram
from boitata_b200 import _native as N
from boitata_b200 import workloads as W

pytestmark = pytest.mark.gpu

ST = {0: 0, 1: 1, 2: 2}  # oracle status -> engine status (ok, search failed, singular)


class Case:
    """Device buffers of one call: samples, targets and the engine's neighbour lists."""

    def __init__(self, coords, values, err, targets, variogram, search):
        import torch

        ok = OrdinaryKriging(variogram, search).fit(coords, values, error_variance=err)
        idx, cnt, good = ok.neighbors(targets)
        self.coords, self.values, self.err, self.targets, self.variogram = coords, values, err, targets, variogram
        self.idx, self.cnt, self.good = idx, cnt, good
        self.m, self.k = idx.shape
        dev = torch.device("cuda", 0)

        def d(a, dtype):
            return torch.from_numpy(np.ascontiguousarray(a)).to(dtype=dtype, device=dev)

        self.sx, self.sy, self.sz = (d(coords[:, a], torch.float64) for a in range(3))
        self.sv = d(values, torch.float64)
        self.se = None if err is None else d(err, torch.float64)
        self.tx, self.ty, self.tz = (d(targets[:, a], torch.float64) for a in range(3))
        self.nbr = d(np.where(idx < 0, 0, idx).astype(np.int64), torch.int64).to(torch.int32)
        self.count = d(cnt, torch.int32)
        self.status = d(np.where(good, N.ST_OK, N.ST_SEARCH_FAILED).astype(np.int8), torch.int8)

    def oracle(self, oracle):
        return oracle.krige_lists(self.targets, self.coords, self.values, self.idx, self.variogram, err=self.err,
                                  skip_coincident=False)

    def call(self, stream, n_samples=None, count=None, nbr=None):
        import torch

        dev = self.sx.device
        out = {key: torch.full((self.m,), float("nan"), dtype=torch.float64, device=dev)
               for key in ("value", "variance", "lagrange")}
        out["n_used"] = torch.zeros(self.m, dtype=torch.int32, device=dev)
        out["status"] = torch.full((self.m,), -1, dtype=torch.int8, device=dev)
        oc = N.OutputsC(*(out[key].data_ptr() for key in ("value", "variance", "lagrange", "n_used", "status")))
        vg = self.variogram.to_c()
        err = ctypes.create_string_buffer(256)
        ns = len(self.coords) if n_samples is None else n_samples
        rc = N.library().btk_solve_noalloc(
            0, ctypes.byref(vg), N.ORDINARY, 0.0, self.sx.data_ptr(), self.sy.data_ptr(), self.sz.data_ptr(),
            self.sv.data_ptr(), None if self.se is None else self.se.data_ptr(), ns, self.m, self.tx.data_ptr(),
            self.ty.data_ptr(), self.tz.data_ptr(), (self.nbr if nbr is None else nbr).data_ptr(), self.k,
            (self.count if count is None else count).data_ptr(), self.status.data_ptr(), ctypes.byref(oc),
            ctypes.c_void_p(stream.cuda_stream), err, len(err))
        assert rc == N.OK, err.value.decode()
        stream.synchronize()
        return {key: v.cpu().numpy() for key, v in out.items()}


def assert_matches_oracle(got, ref, tol, what):
    fin = np.isfinite(ref["value"])
    assert np.array_equal(fin, np.isfinite(got["value"])), f"{what}: NaN pattern"
    want_st = np.vectorize(ST.get)(ref["status"]).astype(np.int8)
    assert np.array_equal(got["status"] & 0x0F, want_st), f"{what}: status"
    assert np.array_equal(got["n_used"][fin], ref["n_used"][fin]), f"{what}: n_used"
    for key in ("value", "variance", "lagrange"):
        assert np.all(close(got[key][fin], ref[key][fin], tol)), f"{what}: {key}"


def c1_case(step, err=False):
    from oracle import oracle

    w = W.c1()
    g = w.geometry
    targets = oracle.centroids(g.origin, g.size, g.count, g.rotation)[::step]
    e = np.random.default_rng(3).uniform(0.0, 0.05, len(w.coords)) if err else None
    return Case(w.coords, w.values, e, targets, w.variogram, w.search)


def twin_case():
    """c1's samples plus 300 twins 1.5e-6 m away (outside the 1e-6 m coincident rule) under a
    variogram without nugget: C between twins is 1 - 1.5e-8, which FP32 rounds to 1, so the FP32
    factorisation of every system holding a pair fails and the FP64 re-solve list fills."""
    from oracle import oracle

    w = W.c1()
    rng = np.random.default_rng(8)
    pick = rng.choice(len(w.coords), 300, replace=False)
    coords = np.vstack([w.coords, w.coords[pick] + [1.5e-6, 0.0, 0.0]])
    values = np.concatenate([w.values, w.values[pick] * 1.01])
    vg = Variogram([Structure("spherical", 1.0, 150.0)], nugget=0.0, ratios=(1.0, 1.0 / 3.0))
    g = w.geometry
    targets = oracle.centroids(g.origin, g.size, g.count, g.rotation)[::7]
    return Case(coords, values, None, targets, vg, w.search)


def test_no_alloc_matches_the_oracle_call_after_call(oracle):
    import torch

    stream = torch.cuda.Stream(torch.device("cuda", 0))
    twins = twin_case()  # 7,143 targets
    plain = c1_case(5)   # 10,000 targets: the twins' stale list would stay in bounds, were it not cleared
    with_err = c1_case(9, err=True)
    ref_twins, ref_plain, ref_err = twins.oracle(oracle), plain.oracle(oracle), with_err.oracle(oracle)
    first = twins.call(stream)
    assert_matches_oracle(first, ref_twins, 1e-6, "twins, call 1")
    flagged = (first["status"] & N.ST_FP64_FALLBACK) != 0
    assert flagged.sum() > 100, "the twin systems should have gone to the FP64 re-solve"
    second = plain.call(stream)
    assert_matches_oracle(second, ref_plain, 1e-6, "plain, after the twins")
    # Nothing of the previous call's re-solve list may reach this call.
    assert ((second["status"] & N.ST_FP64_FALLBACK) != 0).sum() <= (ref_plain["status"] == 0).sum() // 1000
    third = with_err.call(stream)
    assert_matches_oracle(third, ref_err, 1e-6, "measurement errors")
    again = twins.call(stream)
    assert_matches_oracle(again, ref_twins, 1e-6, "twins, call 4")
    assert np.array_equal(again["status"], first["status"]), "re-solve flags differ between two equal calls"
    for key in ("value", "variance", "lagrange"):
        np.testing.assert_array_equal(again[key], first[key])


def test_no_alloc_checks_the_callers_lists():
    import torch

    stream = torch.cuda.Stream(torch.device("cuda", 0))
    case = c1_case(50)
    base = case.call(stream)
    # A count above max_samples, and an index past the samples, fail their target alone (BTK_ST_INVALID);
    # the kernel reads nothing outside the caller's buffers.
    a, b = np.flatnonzero(case.good & (case.cnt > 0))[[3, 7]]
    count = case.count.clone()
    count[int(a)] = case.k + 1
    nbr = case.nbr.clone()
    nbr[int(b), 0] = len(case.coords)
    got = case.call(stream, count=count, nbr=nbr)
    assert got["status"][a] == N.ST_INVALID and got["status"][b] == N.ST_INVALID
    assert np.isnan(got["value"][a]) and np.isnan(got["value"][b])
    keep = np.ones(case.m, dtype=bool)
    keep[[a, b]] = False
    np.testing.assert_array_equal(got["value"][keep], base["value"][keep])
    # The same lists against a smaller sample count: every target holding a higher index fails.
    limit = len(case.coords) // 2
    got = case.call(stream, n_samples=limit)
    uses_high = np.array([np.any(case.idx[t, : case.cnt[t]] >= limit) for t in range(case.m)])
    run = case.good & (case.cnt > 0)
    assert np.all(got["status"][uses_high & run] == N.ST_INVALID)
    np.testing.assert_array_equal(got["value"][~uses_high], base["value"][~uses_high])


def test_no_alloc_entry_point_rejects_calls_beyond_its_limit():
    lib = N.library()
    err = ctypes.create_string_buffer(256)
    vg = N.VariogramC()
    vg.nstruct = 1
    vg.s[0].model, vg.s[0].sill, vg.s[0].range = N.MODELS["spherical"], 1.0, 10.0
    oc = N.OutputsC(None, None, None, None, None)  # the size check comes before any other
    rc = lib.btk_solve_noalloc(0, ctypes.byref(vg), N.ORDINARY, 0.0, None, None, None, None, None, 10, 262144 + 1,
                               None, None, None, None, 16, None, None, ctypes.byref(oc), None, err, len(err))
    assert rc == N.EINVAL and "at most 262144 systems" in err.value.decode()
