"""Headline benchmark: ordinary-kriging blocks/s on 3.2M blocks with at most 32 samples each.

Workload (c2 of boitata_b200.workloads): 50,000 drill-hole composites, a
200 x 200 x 80 block model (3.2M blocks), octant search (4 per octant, 32 at
most) in a rotated ellipsoid, nested spherical + exponential variogram. One
step = the whole kriging path over the block model (centroids, neighbour
search, assembly, solve, estimate and variance) with the samples resident
on the device. `value` is the mixed FP32/FP64 form; the FP64 form is
timed beside it, with the error of mixed against FP64 over every block.

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

# DRAM bytes per system of k_tile<mixed>: (132,827,648 read + 16,656,896 written) / 800,000 systems in the
# ncu capture of profiles/k_tile_c2_800k_blocks.md.
TILE_DRAM_BYTES_PER_SYSTEM = (132827648 + 16656896) / 800000

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
    """The oracle (CPU restatement of the reference path) on every host thread over a fixed sample of blocks."""
    from oracle import oracle

    g = w.geometry
    cent = oracle.centroids(g.origin, g.size, g.count, g.rotation)
    step = max(1, len(cent) // sample_blocks)
    targets = np.ascontiguousarray(cent[::step][:sample_blocks])
    cores = threads or oracle.num_threads()
    t0 = time.perf_counter()
    oracle.estimate_many(targets, w.coords, w.values, w.search, w.variogram, threads=cores, neighbors=False)
    dt = time.perf_counter() - t0
    return {"value": len(targets) / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"every {step}th block of the 3.2M-block model ({len(targets)} blocks), "
                      f"{dt:.2f} s on {cores} threads"}


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


def loo_gradient(args, dev, ws=1, rank=0):
    """c4: leave-one-out loss of 20,000 samples (32 neighbours, frozen) and its 10-parameter gradient;
    kernel times from CUDA events on the launch stream, forward alone and forward with the adjoint. With
    several ranks the samples are split over them (boitata_b200.shard) and the partial sums are
    all-reduced; the time is the slowest rank's kernel time."""
    import torch

    from boitata_b200 import OrdinaryKriging, shard, workloads
    from boitata_b200.gradient import LeaveOneOut, theta_of

    w = workloads.c4(device=dev)
    torch.cuda.empty_cache()
    est = OrdinaryKriging(w.variogram, w.search).fit(w.coords, w.values)
    loo = LeaveOneOut(est)
    theta = theta_of(w.variogram)
    first, count = shard.split(loo.n, ws)[rank]
    ctx = est._ctx
    ctx._lib.btk_set_timing(ctx.handle, 1)
    times = {}
    for grad in (False, True):
        ms = []
        for i in range(args.warmup + max(args.steps, 3)):
            sums = shard.loo_sums(loo, theta, first, count, grad)
            p3 = (ctypes.c_float * 3)()
            ctx.check(ctx._lib.btk_phase_ms(ctx.handle, p3), "phase timing")
            if i >= args.warmup:
                ms.append(p3[0])
        t = np.array([float(np.median(ms))])
        if ws > 1:
            import torch.distributed as dist

            tt = torch.tensor(t, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = tt.cpu().numpy()
        times[grad] = float(t[0])
    loss, g, _ = shard.finish(shard.all_reduce_sum(sums))
    ctx._lib.btk_set_timing(ctx.handle, 0)
    return {"loo_grad_ms": times[True],
            "loo_grad": {"samples": int(len(w.coords)), "parameters": int(len(theta)), "loss": loss,
                         "forward_ms": times[False], "forward_and_adjoint_ms": times[True],
                         "adjoint_over_forward": (times[True] - times[False]) / times[False],
                         "grad_norm": float(np.linalg.norm(g)), "ranks": ws,
                         "what": "c4: mean squared leave-one-out error of ordinary kriging, 32 nearest samples "
                                 "frozen at theta0, gradient w.r.t. nugget, 2 sills, 2 ranges, 2 ratios, "
                                 "3 angles (FP64 adjoint, one kernel with the forward); samples split over the "
                                 "ranks, partial sums all-reduced"}}


def callers(dev):
    """The paths around the headline one, each timed once warm (wall clock around the host call, inputs on
    the host): the dense LU of 128-sample and power-model systems and a calibrated search over c1's 50,000
    blocks, and one sequential Gaussian simulation of 400,000 nodes conditioned on c2's 50,000 composites."""
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
    # C5: 220k clustered composites (10% near-twins 0.01 m away), Gaussian model with a 1e-4 nugget, octant
    # search with up to 64 samples, 10.24M blocks; FP64 (every system is ill-conditioned, so the mixed form
    # re-solves all of them in FP64), device outputs, one timed step after a warm one.
    w5 = workloads.c5()
    est = bt.OrdinaryKriging(w5.variogram, w5.search).fit(w5.coords, w5.values)
    c5ctx = est._ctx
    m5 = w5.geometry.cells()
    g5 = w5.geometry.to_c()
    v5 = torch.empty(m5, dtype=torch.float64, device=dev)
    s5 = torch.empty(m5, dtype=torch.float64, device=dev)
    o5 = bt._native.OutputsC(v5.data_ptr(), s5.data_ptr(), None, None, None)
    ts = []
    for _ in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        c5ctx.check(c5ctx._lib.btk_predict_geometry_device(c5ctx.handle, ctypes.byref(g5), bt._native.ORDINARY, 0.0,
                                                           bt._native.FP64, ctypes.byref(o5), None), "c5")
        torch.cuda.synchronize()
        ts.append(time.perf_counter() - t0)
    out["c5_fp64"] = {"blocks_per_s": m5 / ts[-1], "blocks": m5, "samples": int(len(w5.coords)),
                      "seconds": ts[-1], "finite": int(torch.isfinite(v5).sum().item()),
                      "workload": "C5: 10.24M blocks, octant search up to 64 samples, FP64, device outputs"}
    del est, v5, s5
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


def run_reference(args, ws, rank):
    if rank != 0:
        return
    from boitata_b200 import workloads

    w = workloads.c2()
    vals = []
    sample = min(args.cpu_sample, 60_000)
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(w, sample)
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

    def use(prec):
        """Each form runs at its own tuned launch configuration (set outside the timed region)."""
        if tunings:
            from boitata_b200.autotune import set_tuning

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
        results[prec] = {k: v.clone() for k, v in outs.items()}

    timed = {}
    launches = {}
    with Clocks(local) as clk:
        for prec in (N.MIXED, N.FP64):
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
            launches[prec] = ctx.launches() - before
            torch.cuda.synchronize()
            barrier()
            total = torch.tensor([sum(ms)], dtype=torch.float64, device=dev)
            if ws > 1:
                import torch.distributed as dist

                dist.all_reduce(total, op=dist.ReduceOp.MAX)
            timed[prec] = (total.item() / args.steps, ms)
    clocks = clk.summary()

    # Per-phase kernel times (CUDA events on the launch stream), untimed pass.
    lib.btk_set_timing(h, 1)
    phases = {}
    for prec in (N.MIXED, N.FP64):
        acc = np.zeros(3)
        for _ in range(3):
            flush.zero_()
            step(prec)
            p3 = (ctypes.c_float * 3)()
            ctx.check(lib.btk_phase_ms(h, p3), "phase timing")
            acc += np.array(p3[:])
        phases[prec] = acc / 3
    lib.btk_set_timing(h, 0)
    peak64 = lib.btk_peak_flops(h, 1)
    peak32 = lib.btk_peak_flops(h, 0)

    mixed, fp64 = results[N.MIXED], results[N.FP64]
    v64, vmx = fp64["value"].cpu().numpy(), mixed["value"].cpu().numpy()
    s64, smx = fp64["variance"].cpu().numpy(), mixed["variance"].cpu().numpy()
    n_used = fp64["n_used"].cpu().numpy()
    st64 = fp64["status"].cpu().numpy()
    err = np.concatenate([rel_err(vmx, v64), rel_err(smx, s64)])
    nan_same = int(np.sum(np.isfinite(vmx) == np.isfinite(v64)))
    fallback = int(np.sum((mixed["status"].cpu().numpy() & 0x10) != 0))
    flops = float(np.sum(flops_per_system(n_used[st64 == 0], [s.model for s in w.variogram.structures])))

    ms_mixed, ms_fp64 = timed[N.MIXED][0], timed[N.FP64][0]
    value = ws * m / (ms_mixed * 1e-3)
    solve_ms = phases[N.MIXED][1]
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
                     "traffic": TILE_DRAM_BYTES_PER_SYSTEM * m,
                     "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of k_tile<mixed> from one ncu "
                                       "capture at 800,000 blocks (profiles/k_tile_c2_800k_blocks.md), scaled by "
                                       "the systems per launch (the per-target streams grow in proportion)",
                     "peak_source": "measured in this run: CUDA-core FP64 FMA loop (btk_peak_flops)",
                     "fp32_peak": peak32 / 1e12,
                     "algorithmic_flops_per_step": flops,
                     # The same launches against HBM: the tile solve reads the neighbour table and targets
                     # and writes the outputs; its tables live in shared memory, so HBM is far from bound.
                     "hbm_view": {"achieved_gbs": TILE_DRAM_BYTES_PER_SYSTEM * m / (solve_ms * 1e-3) / 1e9,
                                  "peak_gbs": hbm_peak()[0],
                                  "frac": TILE_DRAM_BYTES_PER_SYSTEM * m / (solve_ms * 1e-3) / 1e9 / hbm_peak()[0],
                                  "peak_source": hbm_peak()[1]}},
        "gpu_launches": int(launches[N.MIXED]),
        "clocks": clocks,
    }

    if not args.no_e2e:
        cent = np.empty((m, 3))
        ctx.check(lib.btk_centroids(h, ctypes.byref(gc), 0, m, cent.ctypes.data), "centroids")
        tgt = torch.from_numpy(cent).pin_memory()
        hv = torch.empty(m, dtype=torch.float64).pin_memory()
        hs = torch.empty(m, dtype=torch.float64).pin_memory()
        ho = N.OutputsC(hv.data_ptr(), hs.data_ptr(), None, None, None)
        use(N.MIXED)
        e2e = []
        for i in range(args.warmup + args.steps):
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

            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        line["e2e"] = {"value": ws * m / t.item(), "unit": UNIT, "h2d_bytes_per_step": m * 24,
                       "d2h_bytes_per_step": m * 16,
                       "path": "btk_predict (C ABI, host buffers): H2D of pinned targets, search, solve, D2H of "
                               "value and variance; wall clock around the synchronous call"}

    if not args.no_grad:
        line.update(loo_gradient(args, dev, ws, rank))

    if rank == 0 and ws == 1 and not args.no_callers:
        line["callers"] = callers(dev)
    if rank == 0 and ws == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(w, args.cpu_sample)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
