"""The mixed form's tile solve with its trailing updates on the tensor pipe (tuning.tile_tensor = 1).

The factorisation is blocked: 8-column panels on the CUDA cores, the
trailing lower triangle updated by split-TF32 mma (btk_tile.cu factor_tc).
Its results are held to the mixed form's bar against the oracle (1e-6 per
result in |a - b| <= tol (1 + max(|a|, |b|)), NaN pattern, status and
n_used equal), and they differ in the last bits from the unblocked FP32
elimination's, which shows the other factorisation ran.
"""

import numpy as np
import pytest
from conftest import close
from test_gpu_parity import assert_same_estimates, centroids

from boitata_b200 import OrdinaryKriging
from boitata_b200 import workloads as W
from boitata_b200.autotune import get_tuning, set_tuning
from boitata_b200.errors import InvalidInput

pytestmark = pytest.mark.gpu


def tensor(est, on=1):
    set_tuning(est._ctx, dict(get_tuning(est._ctx), tile_tensor=on))
    return est


def test_tensor_form_c1_block_model(oracle):
    w = W.c1()
    targets = centroids(oracle, w)
    est = tensor(OrdinaryKriging(w.variogram, w.search, precision="mixed").fit(w.coords, w.values))
    got = est.predict_full(targets)
    ref = oracle.estimate_many(targets, w.coords, w.values, w.search, w.variogram, neighbors=False)
    assert_same_estimates(got, ref, 1e-6)
    on_device = est.predict_full(w.geometry)
    for k in ("value", "variance", "lagrange"):
        np.testing.assert_array_equal(on_device[k], got[k])


def test_tensor_form_c2_model_200k_blocks(oracle):
    """200,000 blocks of the 3.2M-block c2 model (every 16th cell), whole geometry on the device."""
    w = W.c2()
    cells = np.arange(0, w.geometry.cells(), 16)
    targets = centroids(oracle, w)[cells]
    ref = oracle.estimate_many(targets, w.coords, w.values, w.search, w.variogram, neighbors=False)
    est = OrdinaryKriging(w.variogram, w.search, precision="mixed").fit(w.coords, w.values)
    plain = est.predict_full(w.geometry)
    got = tensor(est).predict_full(w.geometry)
    sel = {k: v[cells] for k, v in got.items()}
    assert_same_estimates(sel, ref, 1e-6)
    fin = np.isfinite(got["value"])
    assert not np.array_equal(got["value"][fin], plain["value"][fin])
    assert np.all(close(got["value"][fin], plain["value"][fin], 1e-6))
    # Refinement and re-solve flags stay rare (bit 0x10: the FP64 re-solve took the system).
    assert np.mean((got["status"][fin] & 0x10) != 0) < 0.01


def test_tensor_form_uneven_counts_and_kinds(oracle):
    # c3: 4-64 samples (the tile takes n <= 32), simple kriging on every 10th target in the same launch.
    w = W.c3()
    targets = centroids(oracle, w, 3)
    kinds = np.where(np.arange(len(targets)) % 10 == 0, "simple", "ordinary")
    est = tensor(OrdinaryKriging(w.variogram, w.search, precision="mixed").fit(w.coords, w.values))
    got = est.predict_kinds(targets, kinds, mean=1.0)
    for kind in ("ordinary", "simple"):
        sel = kinds == kind
        ref = oracle.estimate_many(targets[sel], w.coords, w.values, w.search, w.variogram, kind=kind, kparam=1.0,
                                   neighbors=False)
        assert_same_estimates({k: v[sel] for k, v in got.items()}, ref, 1e-6)


def test_tensor_form_ill_conditioned_systems(oracle):
    # Gaussian model with a 1e-4 nugget and near-duplicate samples: condition numbers reach ~5e5, the
    # systems go through the refinement; every result at 1e-6 against the oracle.
    w = W.c5(holes=160)
    rng = np.random.default_rng(0)
    cent = centroids(oracle, w)
    targets = cent[rng.choice(len(cent), 2000, replace=False)]
    ref = oracle.estimate_many(targets, w.coords, w.values, w.search, w.variogram, neighbors=False)
    est = tensor(OrdinaryKriging(w.variogram, w.search, precision="mixed").fit(w.coords, w.values))
    got = est.predict_full(targets)
    fin = np.isfinite(ref["value"])
    assert np.array_equal(fin, np.isfinite(got["value"]))
    assert np.array_equal(got["status"] & 0x0F, ref["status"].astype(np.int8))
    assert np.mean((got["status"][fin] & 0x10) != 0) < 0.05
    for k in ("value", "variance", "lagrange"):
        assert np.all(close(got[k][fin], ref[k][fin], 1e-6)), k


def test_tensor_switch_is_checked():
    w = W.c1()
    est = OrdinaryKriging(w.variogram, w.search, precision="mixed").fit(w.coords[:500], w.values[:500])
    with pytest.raises(InvalidInput, match="tile_tensor"):
        tensor(est, 2)
    assert get_tuning(est._ctx)["tile_tensor"] == 0


def test_mixed_large_systems_by_the_fp64_kernel(oracle):
    """tuning.mixed_large = 1: the mixed form's systems above 32 samples are the FP64 form's, bit for bit;
    the rest keep the mixed tile solve; everything at 1e-6 against the oracle (c3: 4-64 samples)."""
    w = W.c3()
    targets = centroids(oracle, w, 3)
    est = OrdinaryKriging(w.variogram, w.search, precision="mixed").fit(w.coords, w.values)
    set_tuning(est._ctx, dict(get_tuning(est._ctx), mixed_large=1))
    got = est.predict_full(targets)
    fp64 = est.predict_full(targets, precision="fp64")
    ref = oracle.estimate_many(targets, w.coords, w.values, w.search, w.variogram, neighbors=False)
    assert_same_estimates(got, ref, 1e-6)
    large = (got["n_used"] > 32) & np.isfinite(got["value"])
    assert large.sum() > 1000
    for k in ("value", "variance", "lagrange"):
        np.testing.assert_array_equal(got[k][large], fp64[k][large])
    assert not np.any(got["status"][large] & 0x10)
    small = (got["n_used"] <= 32) & np.isfinite(got["value"])
    assert not np.array_equal(got["value"][small], fp64["value"][small])
    with pytest.raises(InvalidInput, match="mixed_large"):
        set_tuning(est._ctx, dict(get_tuning(est._ctx), mixed_large=3))


def test_mixed_tile_solve_with_a_large_sill(oracle):
    """Grades in units whose variance is about 1e6 (c2's samples, values x 1e3, sills and nugget x 1e6):
    the mixed tile solve tests its FP32 pivots against n ulp of C0 over each system's own pivots (not the
    padded rows' unit pivots), so its systems are not sent to the FP64 re-solve wholesale, and every result
    is held to 1e-6 against the oracle."""
    from boitata_b200 import Structure, Variogram

    w = W.c2()
    vg = w.variogram
    big = Variogram([Structure(s.model, s.sill * 1e6, s.range) for s in vg.structures], nugget=vg.nugget * 1e6,
                    rotation=vg.rotation, ratios=vg.ratios)
    values = w.values * 1e3
    rng = np.random.default_rng(9)
    targets = centroids(oracle, w)[rng.choice(w.geometry.cells(), 20000, replace=False)]
    ref = oracle.estimate_many(targets, w.coords, values, w.search, big, neighbors=False)
    for tensor_form in (0, 1):
        est = tensor(OrdinaryKriging(big, w.search, precision="mixed").fit(w.coords, values), tensor_form)
        got = est.predict_full(targets)
        assert_same_estimates(got, ref, 1e-6)
        fin = np.isfinite(got["value"])
        assert np.mean((got["status"][fin] & 0x10) != 0) < 0.01, tensor_form
