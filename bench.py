"""Headline benchmark: ordinary-kriging blocks/s on 3.2M blocks with at most 32 samples each.

Workload (c2 of boitata_b200.workloads): 50,000 drill-hole composites, a
200 x 200 x 80 block model (3.2M blocks), octant search (4 per octant, 32 at
most) in a rotated ellipsoid, nested spherical + exponential variogram. One
step = the whole kriging path over the block model (centroids, neighbour
search, assembly, solve, estimate and variance) with the samples resident
on the device. `value` is the mixed FP32/FP64 form; the FP64 form is
timed beside it, with the error of mixed against FP64 over every block and
of both forms against the FP64 oracle over the CPU baseline's sample of
blocks. The line also measures the other configurations: c3 (uneven
neighbour counts with simple kriging in the same launch) and c5 (10.24M
ill-conditioned blocks), each against the oracle, the c4 leave-one-out
gradient and the paths around the headline one.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun each rank krigs its own block model of the same size (the
grid shifted by half a block per rank) over the same samples: weak scaling,
no collective on the data path; rank 0 prints the JSON line. `--impl
reference` times the CPU restatement of the reference path (the reference
itself is Rust and is not buildable here) on a bounded sample of the same
blocks, with every host thread.
"""

import argparse
import ctypes
import hashlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# DRAM bytes per system of k_tile<mixed> from one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum over
# the systems of the launch), valid for the tile kernel's sources whose hash is TILE_TRAFFIC_SOURCE: when they
# change, the line reports no traffic until a new capture is made.
TILE_DRAM_BYTES_PER_SYSTEM = (132878336 + 12759808) / 800000
TILE_WARP_INSTRUCTIONS_PER_SYSTEM = 2754602618 / 800000  # sm__inst_executed.sum of the same capture
TILE_TRAFFIC_SOURCE = "c862de9d82734b4b"
TILE_SOURCES = ("boitata_b200/csrc/btk_tile.cu", "boitata_b200/csrc/btk_device.cuh", "boitata_b200/csrc/btk_internal.h")


def tile_source_hash():
    h = hashlib.sha256()
    for f in TILE_SOURCES:
        with open(os.path.join(ROOT, f), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:16]


def hbm_peak():
    """Measured HBM copy bandwidth of this pool's B200s (GB/s) and where it came from."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, a STREAM-style copy)"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback (an earlier copy measurement on this pool)"


METRIC = "OK blocks/s @3.2M blocks n≤32: mixed vs FP64 GPU at ≤1e-6 rel; LOO-grad ms"
UNIT = "blocks/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--cpu-sample", type=int, default=400_000, help="blocks in the CPU baseline sample")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-grad", action="store_true")
    p.add_argument("--no-tune", action="store_true")
    p.add_argument("--no-callers", action="store_true", help="skip the dense-LU, calibration and SGS lines")
    p.add_argument("--no-configs", action="store_true", help="skip the c3 and c5 configurations")
    p.add_argument("--grid", default=None, help="block counts NXxNYxNZ in place of 200x200x80 (profiling cases)")
    p.add_argument("--profile", action="store_true",
                   help="profiling case: warm-up and two steps of each form, no timing, no JSON line")
    p.add_argument("--tuning", default=None,
                   help="launch configuration per form as JSON, the bench line's config.tuning "
                        "({\"fp64\": {...}, \"mixed\": {...}}); skips the autotuner")
    return p.parse_args()


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=None)
    return ws, rank, local


def workload_config(w, blocks):
    return {
        "workload": "c2: 50,000 drill-hole composites (400 vertical holes, 125 x 2 m), 200x200x80 blocks of "
                    "2.5x2.5x3.125 m, octant search 4 per octant / 32 max, radius 250 m in a (30,10,0) "
                    "0.75/0.25 ellipsoid, nugget 0.05 + sph 0.5 (80 m) + exp 0.45 (250 m)",
        "blocks": blocks,
        "samples": int(len(w.coords)),
        "max_samples": 32,
        "kind": "ordinary",
    }


def cpu_baseline(w, sample_blocks, threads=0):
    """The oracle (CPU restatement of the reference path) on every host thread over a fixed sample of blocks:
    (the baseline record, the oracle's per-block results, the sampled cell indices)."""
    from oracle import oracle

    g = w.geometry
    cent = oracle.centroids(g.origin, g.size, g.count, g.rotation)
    step = max(1, len(cent) // sample_blocks)
    cells = np.arange(0, len(cent), step)[:sample_blocks]
    targets = np.ascontiguousarray(cent[cells])
    cores = threads or oracle.num_threads()
    t0 = time.perf_counter()
    ref = oracle.estimate_many(targets, w.coords, w.values, w.search, w.variogram, threads=cores, neighbors=False)
    dt = time.perf_counter() - t0
    return ({"value": len(targets) / dt, "unit": UNIT, "cores": cores, "kind": "port",
             "sample": f"every {step}th block of the {len(cent)}-block model ({len(targets)} blocks), "
                       f"{dt:.2f} s on {cores} threads"}, ref, cells)


ORACLE_STATUS = {0: 0, 1: 1, 2: 2, 3: 3, 4: 4}  # oracle status -> engine status


def oracle_error(got, ref, cells=None):
    """Error of one GPU form against the FP64 oracle, per result, in the reference tests' convention
    |a - b| / (1 + max(|a|, |b|)) (crates/estimation/src/kernel.rs:178-180), over value, variance and
    lagrange; with the NaN pattern and the status (fallback flag masked) compared block for block."""
    pick = (lambda a: a) if cells is None else (lambda a: a[cells])
    errs = []
    fin = np.isfinite(ref["value"])
    for key in ("value", "variance", "lagrange"):
        a, b = pick(got[key])[fin], ref[key][fin]
        errs.append(np.abs(a - b) / (1.0 + np.maximum(np.abs(a), np.abs(b))))
    e = np.concatenate(errs)
    st = pick(got["status"]) & 0x0F
    want = np.vectorize(ORACLE_STATUS.get)(ref["status"]).astype(np.int8)
    nan_same = np.isfinite(pick(got["value"])) == fin
    return {"max": float(e.max()) if len(e) else None, "p99": float(np.percentile(e, 99)) if len(e) else None,
            "nan_pattern_equal": bool(nan_same.all()), "nan_pattern_differs": int((~nan_same).sum()),
            "status_equal": bool(np.array_equal(st, want)), "status_differs": int((st != want).sum()),
            "n_used_equal": bool(np.array_equal(pick(got["n_used"])[fin], ref["n_used"][fin])),
            "blocks": int(len(fin))}


class Clocks:
    """nvidia-smi samples during the timed region (median SM clock, throttle reasons seen)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, mx, reasons = [], None, set()
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for k, name in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def flops_per_system(n, structures):
    """Algorithmic FLOPs of one system of n samples: n(n+1)/2 (9 + sum f_s) lags and models, n^3/3
    Cholesky, n^2/2 pivots, 4n^2 solves, 8n epilogue, 15n projection (f_sph 8, f_exp 6, f_gauss 7)."""
    f = {"spherical": 8, "exponential": 6, "gaussian": 7}
    fs = sum(f.get(s, 8) for s in structures)
    n = np.asarray(n, dtype=np.float64)
    return n * (n + 1) / 2 * (9 + fs) + n ** 3 / 3 + n ** 2 / 2 + 4 * n ** 2 + 8 * n + 15 * n


def rel_err(a, b):
    ok = np.isfinite(a) & np.isfinite(b)
    e = np.abs(a[ok] - b[ok]) / (1 + np.maximum(np.abs(a[ok]), np.abs(b[ok])))
    return e


def objective_times(obj, theta, first, count, warmup, steps, dev, ws=1):
    """Kernel times (ms, CUDA events on the launch stream, median over steps, max over ranks) of the objective
    alone and with its gradient, over systems first .. first + count - 1; and the summed partial sums."""
    import torch

    from boitata_b200 import shard

    ctx = obj.estimator._ctx
    ctx._lib.btk_set_timing(ctx.handle, 1)
    times, sums = {}, None
    for grad in (False, True):
        ms = []
        for i in range(warmup + max(steps, 3)):
            sums = shard.loo_sums(obj, theta, first, count, grad)
            p3 = (ctypes.c_float * 3)()
            ctx.check(ctx._lib.btk_phase_ms(ctx.handle, p3), "phase timing")
            if i >= warmup:
                ms.append(p3[0])
        t = np.array([float(np.median(ms))])
        if ws > 1:
            import torch.distributed as dist

            tt = torch.tensor(t, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = tt.cpu().numpy()
        times[grad] = float(t[0])
    ctx._lib.btk_set_timing(ctx.handle, 0)
    return times, sums


def loo_gradient(args, dev, ws=1, rank=0):
    """c4: leave-one-out loss of 20,000 samples (32 neighbours, frozen) and its 10-parameter gradient, in the
    FP64 form and the mixed form (FP32 factorisation, FP64 refinement and gradient sums); kernel times from
    CUDA events on the launch stream, forward alone and forward with the adjoint. With several ranks the
    samples are split over them (boitata_b200.shard) and the partial sums are all-reduced; the time is the
    slowest rank's kernel time. loo_grad_ms is the faster form's forward with the adjoint."""
    import torch

    from boitata_b200 import OrdinaryKriging, shard, workloads
    from boitata_b200.gradient import LeaveOneOut, theta_of

    w = workloads.c4(device=dev)
    torch.cuda.empty_cache()
    est = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    theta = theta_of(w.variogram)
    forms = {}
    for precision in ("fp64", "mixed"):
        loo = LeaveOneOut(est, precision=precision)
        first, count = shard.split(loo.n, ws)[rank]
        times, sums = objective_times(loo, theta, first, count, args.warmup, args.steps, dev, ws)
        loss, g, cnt = shard.finish(shard.all_reduce_sum(sums))
        forms[precision] = {"forward_ms": times[False], "forward_and_adjoint_ms": times[True],
                            "adjoint_over_forward": (times[True] - times[False]) / times[False],
                            "loss": loss, "grad": [float(x) for x in g], "systems": cnt}
    gd = np.array(forms["mixed"]["grad"]) - np.array(forms["fp64"]["grad"])
    best = min(forms, key=lambda k: forms[k]["forward_and_adjoint_ms"])
    return {"loo_grad_ms": forms[best]["forward_and_adjoint_ms"],
            "loo_grad": {"samples": int(len(w.coords)), "parameters": int(len(theta)), "form": best,
                         "forms": forms, "ranks": ws,
                         "mixed_vs_fp64": {"loss": abs(forms["mixed"]["loss"] - forms["fp64"]["loss"]) /
                                           abs(forms["fp64"]["loss"]),
                                           "grad_max_rel": float(np.max(np.abs(gd) / np.maximum(
                                               np.abs(forms["fp64"]["grad"]), 1e-12)))},
                         "what": "c4: mean squared leave-one-out error of ordinary kriging, 32 nearest samples "
                                 "frozen at theta0, gradient w.r.t. nugget, 2 sills, 2 ranges, 2 ratios, "
                                 "3 angles (adjoint in the same kernel as the forward); samples split over the "
                                 "ranks, partial sums all-reduced"}}


def callers(dev):
    """The paths around the headline one, each timed once warm (wall clock around the host call, inputs on
    the host): the dense LU of 128-sample and power-model systems, a calibrated search and weight declustering
    over c1's 50,000 blocks, and one sequential Gaussian simulation of 400,000 nodes conditioned on c2's 50,000
    composites."""
    import torch

    import boitata_b200 as bt
    from boitata_b200 import workloads
    from boitata_b200.simulation import sgs_scores, unit_sill
    from boitata_b200.transforms import normal_score

    out = {}
    w = workloads.c1()
    g = w.geometry
    cases = {
        "dense_lu_128": (w.variogram, bt.Search(ranges=(300.0, 300.0, 100.0), max_samples=128, min_samples=1)),
        "power_model_32": (bt.Variogram([bt.Structure("power", 0.02, 100.0, exponent=1.5)], nugget=0.1,
                                        ratios=(1.0, 1.0 / 3.0)),
                           bt.Search(ranges=(300.0, 300.0, 100.0), max_samples=32, min_samples=1)),
        "calibrated_slope_0.9": (w.variogram, bt.Search(ranges=(300.0, 300.0, 100.0), max_samples=48, min_samples=4,
                                                         target_slope=0.9)),
    }
    for name, (vg, s) in cases.items():
        ok = bt.OrdinaryKriging(vg, s).fit(w.coords, w.values)
        ok.predict_full(g)
        torch.cuda.synchronize()
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            ok.predict_full(g)
            ts.append(time.perf_counter() - t0)
        out[name] = {"blocks_per_s": g.cells() / float(np.median(ts)), "blocks": g.cells(),
                     "workload": "c1 samples and block model, " + name.replace("_", " ")}
    # Weight declustering: the kriging weights each c1 sample receives over the 50,000 blocks (search,
    # solve and the FP64 weights pass on the device, the target-order sum on the host).
    est = bt.OrdinaryKriging(w.variogram, w.search)
    bt.weight_declustering(w.coords, w.values, g, estimator=est)
    ts = []
    for _ in range(3):
        t0 = time.perf_counter()
        bt.weight_declustering(w.coords, w.values, g, estimator=est)
        ts.append(time.perf_counter() - t0)
    out["weight_declustering"] = {"blocks_per_s": g.cells() / float(np.median(ts)), "blocks": g.cells(),
                                  "workload": "c1 samples and block model, OK weights summed per sample"}
    w2 = workloads.c2()
    scores, _ = normal_score(w2.values)
    sim_grid = bt.Geometry((0.0, 0.0, 0.0), (5.0, 5.0, 6.25), (100, 100, 40))
    ctx = bt._native.Context(0)
    nodes = bt.BlockModel(sim_grid).centroids(ctx)
    rng = np.random.default_rng(1)
    order, z = rng.permutation(len(nodes)), rng.standard_normal(len(nodes))
    vg = unit_sill(w2.variogram)
    # Warm at full size: the first run grows the context's buffers to 400k nodes (device allocations).
    sgs_scores(w2.coords, scores, None, nodes[order], z, w2.search, vg, context=ctx)
    t0 = time.perf_counter()
    _, how, rounds = sgs_scores(w2.coords, scores, None, nodes[order], z, w2.search, vg, context=ctx)
    dt = time.perf_counter() - t0
    out["sgs"] = {"nodes_per_s": len(nodes) / dt, "nodes": len(nodes), "seconds": dt, "rounds": rounds,
                  "kriged": int((how == 1).sum()),
                  "workload": "c2 composites (normal scores) conditioning a 100x100x40 grid of 5x5x6.25 m nodes, "
                              "one realization, c2's octant search, FP64"}
    return out


class Replay:
    """One captured CUDA graph of a prediction on a context, replayed on `stream` with CUDA events around
    each replay and L2 flushed between replays (outside the events)."""

    def __init__(self, ctx, stream, flush):
        self.ctx, self.stream, self.flush = ctx, stream, flush

    def time(self, warmup, steps):
        import torch

        lib, h = self.ctx._lib, self.ctx.handle
        for _ in range(warmup):
            self.ctx.check(lib.btk_graph_launch(h, ctypes.c_void_p(self.stream.cuda_stream)), "replay")
        torch.cuda.synchronize()
        before = self.ctx.launches()
        ms = []
        for _ in range(steps):
            self.flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(self.stream)
            self.ctx.check(lib.btk_graph_launch(h, ctypes.c_void_p(self.stream.cuda_stream)), "replay")
            e1.record(self.stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return float(np.mean(ms)), self.ctx.launches() - before


def device_outputs(m, dev):
    import torch

    from boitata_b200 import _native as N

    outs = {k: torch.empty(m, dtype=torch.float64, device=dev) for k in ("value", "variance", "lagrange")}
    outs["n_used"] = torch.empty(m, dtype=torch.int32, device=dev)
    outs["status"] = torch.empty(m, dtype=torch.int8, device=dev)
    oc = N.OutputsC(*(outs[k].data_ptr() for k in ("value", "variance", "lagrange", "n_used", "status")))
    return outs, oc


def host_copy(outs):
    return {k: v.cpu().numpy() for k, v in outs.items()}


def config_c3(args, dev, stream, flush, tune=True):
    """c3: c1's box with a 10x sample-density gradient along x (2,000 samples), the 50,000 block centroids
    of c1's model as device targets, neighbour counts 4 to 64, simple kriging (mean 1.0) on every 10th target
    and ordinary kriging on the rest in the same call; each form autotuned, captured into one CUDA graph and
    replayed; every block checked against the FP64 oracle (ordinary and simple kriging per block)."""
    import torch

    from boitata_b200 import OrdinaryKriging, workloads
    from boitata_b200 import _native as N
    from boitata_b200.autotune import autotune_device
    from oracle import oracle

    w = workloads.c3()
    g = w.geometry
    targets = oracle.centroids(g.origin, g.size, g.count, g.rotation)
    m = len(targets)
    sk = np.arange(m) % 10 == 0
    kinds = np.where(sk, N.SIMPLE, N.ORDINARY).astype(np.int8)
    est = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    ctx = est._ctx
    lib, h = ctx._lib, ctx.handle
    d_xyz = torch.from_numpy(np.ascontiguousarray(targets.T).ravel()).to(dev)
    d_kinds = torch.from_numpy(kinds).to(dev)
    outs, oc = device_outputs(m, dev)
    out = {"workload": "c3: 2,000 samples with density rising 10x along x in 1000x1000x200 m, 50x50x20 block "
                       "centroids (50,000 device targets), Search(radius=150, min_samples=4, max_samples=64), "
                       "simple kriging (mean 1.0) on every 10th target in the same launch",
           "blocks": m}
    got = {}
    for prec, name in ((N.FP64, "fp64"), (N.MIXED, "mixed")):
        if tune:
            t = autotune_device(est, m, d_xyz.data_ptr(), d_kinds.data_ptr(), kparam=1.0, precision=name, steps=2,
                                tag="c3 block centroids, every 10th simple")
            out.setdefault("tuning", {})[name] = {**t["best"], "tile": list(t["best"]["tile"])}
        ctx.check(lib.btk_graph_capture_device(h, m, d_xyz.data_ptr(), d_kinds.data_ptr(), N.ORDINARY, 1.0, prec,
                                               ctypes.byref(oc)), "capture")
        ms, launches = Replay(ctx, stream, flush).time(args.warmup, max(args.steps, 5))
        got[name] = host_copy(outs)
        out[name] = {"blocks_per_s": m / (ms * 1e-3), "ms_per_step": ms, "gpu_launches_per_step":
                     launches / max(args.steps, 5)}
    # The mixed form's other kernel for its systems above 32 samples, timed the same way.
    from boitata_b200.autotune import get_tuning, set_tuning

    tuned = get_tuning(ctx)
    set_tuning(ctx, dict(tuned, mixed_large=1 - int(tuned["mixed_large"])))
    ctx.check(lib.btk_graph_capture_device(h, m, d_xyz.data_ptr(), d_kinds.data_ptr(), N.ORDINARY, 1.0, N.MIXED,
                                           ctypes.byref(oc)), "capture")
    ms, _ = Replay(ctx, stream, flush).time(args.warmup, max(args.steps, 5))
    got["mixed_alt"] = host_copy(outs)
    out["mixed_alt"] = {"blocks_per_s": m / (ms * 1e-3), "ms_per_step": ms,
                        "large_systems": "fp64 kernel" if not tuned["mixed_large"] else
                        "fp32 factorisation, fp64 refinement"}
    out["mixed"]["large_systems"] = "fp64 kernel" if tuned["mixed_large"] else "fp32 factorisation, fp64 refinement"
    set_tuning(ctx, tuned)
    n_used = got["fp64"]["n_used"]
    ok = (got["fp64"]["status"] & 0x0F) == 0
    out["n_used"] = {"min": int(n_used[ok].min()), "max": int(n_used[ok].max()), "mean": float(n_used[ok].mean())}
    out["mixed_over_fp64"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    out["fp64_fallback_systems"] = int(np.sum((got["mixed"]["status"] & 0x10) != 0))
    ref = {}
    for kind, sel in (("ordinary", ~sk), ("simple", sk)):
        r = oracle.estimate_many(targets[sel], w.coords, w.values, w.search, w.variogram, kind=kind, kparam=1.0,
                                 neighbors=False)
        for k, v in r.items():
            ref.setdefault(k, np.empty(m, dtype=v.dtype))[sel] = v
    out["oracle_error"] = {name: oracle_error(got[name], ref) for name in ("fp64", "mixed", "mixed_alt")}
    out["launch"] = "btk_graph_capture_device (btk_predict_kinds_device: Hilbert order, search, tile solve, " \
                    "per-system kernels, FP64 re-solve) replayed per step; L2 flushed between steps"
    del est
    return out


def config_c5(args, dev, stream, flush, sample=20_000):
    """c5: 220,000 clustered composites (10 % copied 0.01 m away), Gaussian variogram with a 1e-4 nugget,
    octant search of up to 64 samples, 10.24M blocks; each form captured into one CUDA graph (centroids,
    search, solves, FP64 re-solves) and replayed; the mixed form's fallback fraction; a sample of blocks
    checked against the FP64 oracle."""
    from boitata_b200 import OrdinaryKriging, workloads
    from boitata_b200 import _native as N
    from oracle import oracle

    w = workloads.c5()
    est = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    ctx = est._ctx
    lib, h = ctx._lib, ctx.handle
    m = w.geometry.cells()
    gc = w.geometry.to_c()
    outs, oc = device_outputs(m, dev)
    out = {"workload": "c5: 220,000 composites (1,600 holes in 40 clusters, 125 x 2 m, plus 10% copied 0.01 m away), "
                       "Gaussian variogram (nugget 1e-4, range 200 m), 400x400x64 blocks (10.24M), octant search "
                       "8 per octant / 64 max, radius 300 m", "blocks": m, "samples": int(len(w.coords))}
    got = {}
    steps = max(2, min(args.steps, 3))
    from boitata_b200.autotune import get_tuning, set_tuning

    base = get_tuning(ctx)
    # The mixed form's systems above 32 samples (nearly all here) in FP32 with FP64 refinement, or by the FP64
    # kernel (btk_tuning.mixed_large); the mixed form is the faster of the two, as the autotuner picks.
    variants = ((N.FP64, "fp64", base), (N.MIXED, "mixed_fp32_large", dict(base, mixed_large=0)),
                (N.MIXED, "mixed_fp64_large", dict(base, mixed_large=1)))
    for prec, name, tun in variants:
        set_tuning(ctx, tun)
        ctx.check(lib.btk_graph_capture_geometry(h, ctypes.byref(gc), N.ORDINARY, 0.0, prec, ctypes.byref(oc)),
                  "capture")
        ms, _ = Replay(ctx, stream, flush).time(1, steps)
        st = outs["status"].cpu().numpy()
        got[name] = {k: v.cpu().numpy() for k, v in outs.items()}
        out[name] = {"blocks_per_s": m / (ms * 1e-3), "ms_per_step": ms}
        if prec == N.MIXED:
            fin = (st & 0x0F) == 0
            out[name]["fp64_fallback_fraction"] = float(np.mean((st[fin] & 0x10) != 0))
    pick = min(("mixed_fp32_large", "mixed_fp64_large"), key=lambda k: out[k]["ms_per_step"])
    out["mixed"] = dict(out[pick], large_systems="fp64 kernel" if pick == "mixed_fp64_large" else
                        "fp32 factorisation, fp64 refinement")
    got["mixed"] = got[pick]
    out["mixed_over_fp64"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    # The gradient of the global mean estimate with respect to the variogram (nugget, sill, range, 2 ratios,
    # 3 angles), neighbourhoods frozen at theta0, covariances recomputed in the adjoint; against one forward
    # step of the same form (the captured prediction above).
    from boitata_b200.gradient import BlockMean, theta_of

    del outs, oc
    theta = theta_of(w.variogram)
    grad = {}
    # The mixed form's gradient with either kernel for systems above 32 samples; "mixed" is the one the
    # forward picked.
    for name, large in (("fp64", 0), ("mixed_fp32_large", 0), ("mixed_fp64_large", 1)):
        set_tuning(ctx, dict(base, mixed_large=large))
        bm = BlockMean(est, w.geometry, precision="fp64" if name == "fp64" else "mixed")
        times, sums = objective_times(bm, theta, 0, bm.n, 1, 3, dev)
        grad[name] = {"objective_ms": times[False], "objective_and_gradient_ms": times[True],
                      "over_forward_step": times[True] / out[name]["ms_per_step"],
                      "mean": float(sums[0] / sums[1]), "systems": int(sums[1]),
                      "grad": [float(x) for x in sums[2:] / sums[1]]}
    set_tuning(ctx, base)
    grad["mixed"] = dict(grad[pick], over_forward_step=grad[pick]["objective_and_gradient_ms"] /
                         out["mixed"]["ms_per_step"])
    out["mean_gradient"] = grad
    out["c5_grad_ms"] = min(v["objective_and_gradient_ms"] for v in grad.values())
    out["c5_forward_ms"] = min(out["fp64"]["ms_per_step"], out["mixed"]["ms_per_step"])
    g = w.geometry
    cells = np.arange(0, m, m // sample)[:sample]
    cent = oracle.centroids(g.origin, g.size, g.count, g.rotation)[cells]
    ref = oracle.estimate_many(cent, w.coords, w.values, w.search, w.variogram, neighbors=False)
    out["oracle_error"] = {name: oracle_error(got[name], ref, cells)
                           for name in ("fp64", "mixed_fp32_large", "mixed_fp64_large")}
    out["oracle_error"]["sample"] = f"every {m // sample}th block ({len(cells)} blocks)"
    out["oracle_error"]["note"] = ("condition numbers reach ~5e5 here, so two FP64 evaluation orders differ by up "
                                   "to ~1e-15 x cond (about 1e-10) on their own")
    del est
    return out


def run_reference(args, ws, rank):
    if rank != 0:
        return
    from boitata_b200 import workloads

    w = workloads.c2()
    vals = []
    sample = min(args.cpu_sample, 60_000)
    for i in range(args.warmup + args.steps):
        r, _, _ = cpu_baseline(w, sample)
        if i >= args.warmup:
            vals.append(r["value"])
    v = float(statistics.mean(vals))
    cfg = workload_config(w, 3_200_000)
    cfg["sample_blocks_per_step"] = sample
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": sample / v * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded LCG, reference test generator)", "config": cfg,
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": r["cores"], "kind": "port", "sample": r["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference is Rust; no cargo/rustc here or on the GPU box, so this arm times the C++ "
                    "restatement of its CPU path (oracle/), every host thread"}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_init()
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return
    import torch

    from boitata_b200 import Geometry, OrdinaryKriging, workloads
    from boitata_b200 import _native as N

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = workloads.c2()
    g0 = w.geometry
    count = tuple(int(c) for c in args.grid.split("x")) if args.grid else g0.count
    geo = Geometry((g0.origin[0] + 0.5 * g0.size[0] * rank, g0.origin[1], g0.origin[2]), g0.size, count,
                   g0.rotation)
    m = geo.cells()
    est = OrdinaryKriging(w.variogram, w.search, precision="mixed", device=local).fit(w.coords, w.values)
    ctx = est._ctx
    lib, h = ctx._lib, ctx.handle
    outs = {k: torch.empty(m, dtype=torch.float64, device=dev) for k in ("value", "variance", "lagrange")}
    outs["n_used"] = torch.empty(m, dtype=torch.int32, device=dev)
    outs["status"] = torch.empty(m, dtype=torch.int8, device=dev)
    oc = N.OutputsC(*(outs[k].data_ptr() for k in ("value", "variance", "lagrange", "n_used", "status")))
    gc = geo.to_c()
    # A stream of our own: torch's legacy default stream has handle 0, which
    # the C ABI reads as "the context's stream".
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    tunings = {}
    override = {}

    def use(prec):
        """Each form runs at its own tuned launch configuration (set outside the timed region)."""
        from boitata_b200.autotune import set_tuning

        if prec in override:
            set_tuning(ctx, override[prec])
        elif tunings:
            set_tuning(ctx, tunings[prec])

    def step(prec):
        use(prec)
        rc = lib.btk_predict_geometry_device(h, ctypes.byref(gc), N.ORDINARY, 0.0, prec, ctypes.byref(oc),
                                             ctypes.c_void_p(stream.cuda_stream))
        ctx.check(rc, "predict")

    def capture(prec):
        use(prec)
        ctx.check(lib.btk_graph_capture_geometry(h, ctypes.byref(gc), N.ORDINARY, 0.0, prec, ctypes.byref(oc)),
                  "capture")

    def replay():
        ctx.check(lib.btk_graph_launch(h, ctypes.c_void_p(stream.cuda_stream)), "replay")

    def barrier():
        if ws > 1:
            import torch.distributed as dist

            dist.barrier()

    tuning = {}
    if args.tuning:
        from boitata_b200.autotune import get_tuning

        given = json.loads(args.tuning)
        for prec, name in ((N.FP64, "fp64"), (N.MIXED, "mixed")):
            tunings[prec] = {**get_tuning(ctx), **{k: v for k, v in given[name].items() if k not in ("ms", "cached")}}
            tuning[name] = {**tunings[prec], "tile": list(tunings[prec]["tile"]), "given": True}
    if not args.profile and not args.no_tune and not args.tuning:
        from boitata_b200.autotune import autotune_geometry

        for prec, name in ((N.FP64, "fp64"), (N.MIXED, "mixed")):
            tuned = autotune_geometry(est, geo, precision=name, steps=2)
            tunings[prec] = dict(tuned["best"])
            tuning[name] = {**tuned["best"], "tile": list(tuned["best"]["tile"]), "ms": tuned["ms"],
                            "cached": tuned["cached"]}
    for _ in range(args.warmup):
        step(N.MIXED)
        step(N.FP64)
    torch.cuda.synchronize()
    if args.profile:
        for prec in (N.MIXED, N.FP64, N.MIXED, N.FP64):
            step(prec)
        torch.cuda.synchronize()
        print(f"profile case done: {m} blocks, {ctx.launches()} launches", flush=True)
        return
    results = {}
    for prec in (N.FP64, N.MIXED):
        step(prec)
        torch.cuda.synchronize()
        results[prec] = host_copy(outs)

    def time_graph(prec):
        """Mean ms of args.steps replays of the step's CUDA graph (max over ranks), and the launches."""
        capture(prec)  # the whole step as one CUDA graph
        for _ in range(2):
            replay()
        barrier()
        torch.cuda.synchronize()
        before = ctx.launches()
        ms = []
        for _ in range(args.steps):
            flush.zero_()  # L2 (126 MB) flushed between steps, outside the timed events
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            replay()
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        n = ctx.launches() - before
        torch.cuda.synchronize()
        barrier()
        total = torch.tensor([sum(ms)], dtype=torch.float64, device=dev)
        if ws > 1:
            import torch.distributed as dist

            dist.all_reduce(total, op=dist.ReduceOp.MAX)
        return total.item() / args.steps, ms, n

    def solve_phase(prec, reps=3):
        """Mean per-phase kernel ms (search, solve, FP64 re-solve) of untimed steps."""
        lib.btk_set_timing(h, 1)
        acc = np.zeros(3)
        for _ in range(reps):
            flush.zero_()
            step(prec)
            p3 = (ctypes.c_float * 3)()
            ctx.check(lib.btk_phase_ms(h, p3), "phase timing")
            acc += np.array(p3[:])
        lib.btk_set_timing(h, 0)
        return acc / reps

    timed = {}
    launches = {}
    with Clocks(local) as clk:
        for prec in (N.MIXED, N.FP64):
            ms_avg, ms, launches[prec] = time_graph(prec)
            timed[prec] = (ms_avg, ms)
    clocks = clk.summary()

    # The mixed tile solve's two factorisations (btk_tuning.tile_tensor): the tuned one is the line's
    # value; the other is timed the same way here.
    from boitata_b200.autotune import get_tuning

    use(N.MIXED)
    tuned_tensor = int(get_tuning(ctx).get("tile_tensor", 0))
    override[N.MIXED] = dict(get_tuning(ctx), tile_tensor=1 - tuned_tensor)
    step(N.MIXED)
    torch.cuda.synchronize()
    alt_result = host_copy(outs)
    with Clocks(local) as clk_alt:
        alt_ms = time_graph(N.MIXED)[0]
    alt_phase = solve_phase(N.MIXED)
    del override[N.MIXED]

    # Per-phase kernel times (CUDA events on the launch stream), untimed pass.
    phases = {prec: solve_phase(prec) for prec in (N.MIXED, N.FP64)}
    peak64 = lib.btk_peak_flops(h, 1)
    peak32 = lib.btk_peak_flops(h, 0)

    mixed, fp64 = results[N.MIXED], results[N.FP64]
    v64, vmx = fp64["value"], mixed["value"]
    s64, smx = fp64["variance"], mixed["variance"]
    n_used = fp64["n_used"]
    st64 = fp64["status"]
    err = np.concatenate([rel_err(vmx, v64), rel_err(smx, s64)])
    nan_same = int(np.sum(np.isfinite(vmx) == np.isfinite(v64)))
    fallback = int(np.sum((mixed["status"] & 0x10) != 0))
    flops = float(np.sum(flops_per_system(n_used[st64 == 0], [s.model for s in w.variogram.structures])))

    ms_mixed, ms_fp64 = timed[N.MIXED][0], timed[N.FP64][0]
    solve_ms = phases[N.MIXED][1]
    if TILE_TRAFFIC_SOURCE == tile_source_hash():
        traffic = TILE_DRAM_BYTES_PER_SYSTEM * m
        traffic_source = ("dram__bytes_read.sum + dram__bytes_write.sum of k_tile<mixed> per system from one ncu "
                          "capture of these kernel sources (hash " + TILE_TRAFFIC_SOURCE + "), times the systems "
                          "of one launch (the per-target streams grow in proportion)")
    else:
        traffic, traffic_source = None, "no ncu capture of the current tile kernel sources"
    issue_view = None
    if traffic is not None and clocks.get("sm_mhz"):
        # The tile solve is issue-bound: its warp instructions (same capture) against one instruction a
        # clock per scheduler, four per SM, at the SM clock sampled during the timed region.
        inst = TILE_WARP_INSTRUCTIONS_PER_SYSTEM * m
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        peak_issue = sms * 4 * clocks["sm_mhz"] * 1e6
        issue_view = {"warp_instructions_per_step": inst, "achieved_per_s": inst / (solve_ms * 1e-3),
                      "peak_per_s": peak_issue, "frac": inst / (solve_ms * 1e-3) / peak_issue,
                      "source": "sm__inst_executed.sum of k_tile<mixed> per system from the capture named in "
                                "traffic_source; peak: 4 warp instructions a clock per SM at the median sampled "
                                "SM clock"}
    value = ws * m / (ms_mixed * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_mixed, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64 (mixed); f64 form beside it", "data": "synthetic (seeded LCG, reference test generator)",
        "config": {**workload_config(w, m), "precision": "mixed", "parallelism": f"replicas x{ws} (weak)",
                   "l2": "flushed between timed steps (256 MB write, outside the events)",
                   "launch": "one CUDA graph per step (centroids, search, solve, FP64 re-solve)",
                   "tuning": tuning},
        "fp64": {"value": ws * m / (ms_fp64 * 1e-3), "ms_per_step": ms_fp64},
        "mixed_over_fp64": ms_fp64 / ms_mixed,
        "mixed_vs_fp64_error": {"max": float(err.max()) if len(err) else None,
                                "p99": float(np.percentile(err, 99)) if len(err) else None,
                                "nan_pattern_equal": nan_same, "blocks": m, "fp64_fallback_systems": fallback,
                                "metric": "|a-b| / (1 + max(|a|, |b|)) over value and variance"},
        "phases_ms": {"mixed": {"search": phases[N.MIXED][0], "solve": phases[N.MIXED][1],
                                "fp64_resolve": phases[N.MIXED][2]},
                      "fp64": {"search": phases[N.FP64][0], "solve": phases[N.FP64][1]}},
        "roofline": {"bound": "fp64", "kernel": "k_tile<mixed> (tile-shared FP64 covariance table, FP32 factor, "
                                               "FP64 refinement) and the per-system kernels for its leftovers",
                     "achieved": flops / (solve_ms * 1e-3) / 1e12, "peak": peak64 / 1e12, "unit": "TFLOP/s",
                     "frac": (flops / (solve_ms * 1e-3)) / peak64,
                     "traffic": traffic,
                     "traffic_source": traffic_source,
                     "peak_source": "measured in this run: CUDA-core FP64 FMA loop (btk_peak_flops)",
                     "fp32_peak": peak32 / 1e12,
                     "algorithmic_flops_per_step": flops,
                     # The same launches against HBM: the tile solve reads the neighbour table and targets
                     # and writes the outputs; its tables live in shared memory, so HBM is far from bound.
                     "hbm_view": None if traffic is None else {
                         "achieved_gbs": traffic / (solve_ms * 1e-3) / 1e9, "peak_gbs": hbm_peak()[0],
                         "frac": traffic / (solve_ms * 1e-3) / 1e9 / hbm_peak()[0], "peak_source": hbm_peak()[1]},
                     "issue_view": issue_view},
        "gpu_launches": int(launches[N.MIXED]),
        "clocks": clocks,
    }
    forms = {tuned_tensor: (ms_mixed, phases[N.MIXED][1], mixed), 1 - tuned_tensor: (alt_ms, alt_phase[1], alt_result)}
    line["tile_factorisation"] = {
        "tuned": "tensor" if tuned_tensor else "unblocked",
        "forms": {name: {"ms_per_step": forms[v][0], "blocks_per_s": ws * m / (forms[v][0] * 1e-3),
                         "solve_ms": forms[v][1], "mixed_over_fp64": ms_fp64 / forms[v][0],
                         "vs_fp64_max_error": float(np.nanmax(np.concatenate([
                             rel_err(forms[v][2]["value"], v64), rel_err(forms[v][2]["variance"], s64)]))),
                         "fp64_fallback_systems": int(np.sum((forms[v][2]["status"] & 0x10) != 0))}
                  for v, name in ((0, "unblocked"), (1, "tensor"))},
        "about": "mixed tile solve: 'unblocked' = FP32 right-looking LDL^T, packed FMA, two systems a warp; "
                 "'tensor' = 8-column panels on the CUDA cores, trailing updates as split-TF32 mma.sync "
                 "(m16n8k8, three per tile); both with the same FP64 residual test and refinement",
        "clocks_alt": clk_alt.summary(),
    }

    if not args.no_e2e:
        cent = np.empty((m, 3))
        ctx.check(lib.btk_centroids(h, ctypes.byref(gc), 0, m, cent.ctypes.data), "centroids")
        tgt = torch.from_numpy(cent).pin_memory()
        hv = torch.empty(m, dtype=torch.float64).pin_memory()
        hs = torch.empty(m, dtype=torch.float64).pin_memory()
        ho = N.OutputsC(hv.data_ptr(), hs.data_ptr(), None, None, None)

        def e2e_time(hc, steps):
            """Mean wall seconds of btk_predict with pipeline chunks of hc targets (0: one chunk)."""
            use(N.MIXED)
            from boitata_b200.autotune import set_tuning

            set_tuning(ctx, dict(get_tuning(ctx), host_chunk=hc))
            e2e = []
            for i in range(args.warmup + steps):
                flush.zero_()
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                ctx.check(lib.btk_predict(h, m, ctypes.c_void_p(tgt.data_ptr()), N.ORDINARY, 0.0, N.MIXED,
                                          ctypes.byref(ho)), "predict")
                dt = time.perf_counter() - t0
                if i >= args.warmup:
                    e2e.append(dt)
            t = torch.tensor([sum(e2e) / len(e2e)], dtype=torch.float64, device=dev)
            if ws > 1:
                import torch.distributed as dist

                dist.all_reduce(t, op=dist.ReduceOp.MAX)  # every rank takes the same choice
            return t.item()

        # The host call's copy/compute pipeline (btk_tuning.host_chunk): the chunk is picked by timing, as the
        # autotuner picks the kernels' launch shapes, then timed over the full step count.
        trial = {hc: e2e_time(hc, 2) for hc in (0, -(-m // 2), -(-m // 4), -(-m // 8))}
        best_chunk = min(trial, key=trial.get)
        t_best = e2e_time(best_chunk, args.steps)
        line["e2e"] = {"value": ws * m / t_best, "unit": UNIT, "h2d_bytes_per_step": m * 24,
                       "d2h_bytes_per_step": m * 16, "host_chunk": best_chunk,
                       "host_chunk_trials_ms": {str(k): v * 1e3 for k, v in trial.items()},
                       "path": "btk_predict (C ABI, host buffers): H2D of pinned targets, search, solve, D2H of "
                               "value and variance, in pipelined chunks of host_chunk targets (0: one); wall clock "
                               "around the synchronous call"}

    if not args.no_grad:
        line.update(loo_gradient(args, dev, ws, rank))

    if rank == 0 and ws == 1 and not args.no_callers:
        line["callers"] = callers(dev)
    if rank == 0 and ws == 1 and not args.no_configs:
        line["configs"] = {"c3": config_c3(args, dev, stream, flush, tune=not args.no_tune),
                           "c5": config_c5(args, dev, stream, flush)}
    if rank == 0 and ws == 1 and not args.no_cpu:
        base, ref, cells = cpu_baseline(w, args.cpu_sample)
        line["cpu_baseline"] = base
        line["oracle_error"] = {"fp64": oracle_error(fp64, ref, cells), "mixed": oracle_error(mixed, ref, cells),
                                "mixed_" + ("unblocked" if tuned_tensor else "tensor"): oracle_error(alt_result, ref,
                                                                                                   cells),
                                "sample": base["sample"],
                                "metric": "|a-b| / (1 + max(|a|, |b|)) over value, variance and lagrange against "
                                          "the FP64 oracle (crates/estimation/src/kernel.rs:178-180)",
                                "tolerance": {"fp64": 1e-10, "mixed": 1e-6}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
