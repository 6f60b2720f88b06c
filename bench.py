"""Benchmark of the ray vs displaced-surface query (Mrays/s).

Default workload (N=1): the GPU-scale plain-method scene, a radius-1 cube
sphere of 96 displaced patches (6 faces x 4 x 4, two base triangles each),
each patch its own 2048 x 2048 FP32 height map (seeded sines + value noise,
amplitude 0.08); one step intersects 1920 x 1080 jittered primary rays and
one cosine-weighted bounce ray per primary hit (closest hit, t/u/v/normal).
Inputs are seeded synthetic data of the reference benchmark's shape.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl dmap|reference]
                  [--config sphere|quad] [--precision f32|f64]

--impl reference times the reference's own CPU implementation of the query
(oracle/_ref: the reference sources compiled here; else the C oracle port)
on every host core over a bounded sample of the same workload.
Under torchrun (N > 1) each rank intersects a full batch of its own (the
camera jitter seeded by the rank) with a replicated scene, no collective on
the data path: weak scaling, value = all ranks' rays / max rank time.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from dmap_b200 import scenes  # noqa: E402

METRIC = "Mrays/s displaced-surface hits"
FLOP = {"node": 450, "leaf": 290, "sub": 285, "newton": 215}   # per-unit FLOPs of the reference algorithm
BYTES = {"ray": 32, "hit": 48, "node": 32, "leaf": 16}          # per-unit algorithmic bytes (FP32 records)


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def build_scene(config: str, small: bool, seed: int = scenes.SEED):
    """The scene and its primary rays; `seed` jitters the sphere's camera
    rays (each rank of a multi-GPU run takes its own batch)."""
    if config == "quad":
        return scenes.quad_scene(128 if small else 512), scenes.quad_camera_rays(*(64, 64) if small else (256, 256))
    texel = np.float16 if config == "sphere16" else np.float32
    sc = scenes.sphere_benchmark_scene(256 if small else 2048, texel, min(16, os.cpu_count() or 4))
    w, h = (480, 270) if small else (1920, 1080)
    return sc, scenes.sphere_camera_rays(w, h, seed=seed)


def extra_rays(config: str, sc, small: bool):
    """The precision variant's grazing rays: aimed at random base-surface
    points from 0.1-5 deg above the tangent plane, origins backed off."""
    if config != "sphere16":
        return np.zeros((0, 8), np.float32)
    p, m = scenes.base_points(sc, 100_000 if small else 1_000_000, seed=scenes.SEED + 7)
    return scenes.grazing_rays(p, m, seed=scenes.SEED + 8)


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def profiled_traffic_per_ray(args):
    """DRAM bytes per ray of one query, from the committed ncu summary of the
    same schedule (a line `traffic_bytes_per_ray <schedule> <value>`), or None."""
    p = ROOT / "profiles" / "traversal_sphere_dram.md"
    if not p.exists():
        return None
    for ln in p.read_text().splitlines():
        f = ln.strip().strip("`").split()
        if len(f) == 3 and f[0] == "traffic_bytes_per_ray" and f[1] == args.schedule:
            return float(f[2])
    return None


def work_per_ray(stats):
    s = stats.astype(np.float64).sum(axis=0)
    n = len(stats)
    flops = (FLOP["node"] * s[1] + FLOP["leaf"] * s[2] + FLOP["sub"] * s[3] + FLOP["newton"] * s[4]) / n
    byts = BYTES["ray"] + BYTES["hit"] + (BYTES["node"] * s[1] + BYTES["leaf"] * s[2]) / n
    return flops, byts, {k: float(s[i] / n) for i, k in enumerate(["triangle_tests", "node_tests", "leaf_tests",
                                                                      "sub_squares", "newton_iters"])}


CPU_STRIDE = 64   # the CPU legs answer every 64th ray of the step's ray list


def cpu_scene(sc, use_ref: bool):
    """The scene on the CPU checker: the reference's own sources compiled
    here (oracle/_ref) when present, else the C port; every patch."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import py_oracle
    lib = py_oracle.Reference() if use_ref and py_oracle.Reference.available() else py_oracle.Oracle()
    kind = "reference" if isinstance(lib, py_oracle.Reference) else "port"
    return py_oracle.CpuScene(lib, sc), kind


def stride_sample(rays_all, stride: int = CPU_STRIDE):
    """Every stride-th ray of the step's whole ray list (primaries then
    bounces, in order), so the sample keeps the workload's mix of misses,
    primary hits and bounce rays over all patches."""
    return np.ascontiguousarray(rays_all[::stride])


def sample_desc(n_sample, n_all, n_patches):
    return (f"{n_sample} rays: every {CPU_STRIDE}th of the step's {n_all} (primaries and bounces in proportion), "
            f"all {n_patches} patches, flat loop")


def time_cpu(cpu, sample, budget_s: float, threads: int):
    """Rays/s of the CPU flat loop on the sample, repeated to fill about
    budget_s seconds of CPU work."""
    t = time.perf_counter()
    cpu.intersect(sample, threads=threads, order="index")
    dt = time.perf_counter() - t
    reps = int(min(64, max(1, budget_s / max(dt, 1e-3))))
    t = time.perf_counter()
    for _ in range(reps):
        cpu.intersect(sample, threads=threads, order="index")
    return len(sample) * reps / (time.perf_counter() - t) / 1e6


def run_cpu(args, rank, world):
    """The reference arm: the reference's own C++ query (oracle/_ref, flat
    loop) on every host core. Its rays are the GPU arm's: the primaries, and
    one bounce per primary hit from the CPU's own FP64 hits (bit-identical
    to the device FP64 path's), then every CPU_STRIDE-th ray of that list
    per step."""
    sc, prim = build_scene(args.config, args.small)
    cpu, kind = cpu_scene(sc, True)
    threads = os.cpu_count() or 1
    h0, _ = cpu.intersect(prim, threads=threads, order="index")
    hit = h0[:, 10] >= 0
    bounce = scenes.bounce_rays(prim[hit], h0[hit, 0], h0[hit, 5:8])
    rays_all = np.concatenate([prim, bounce, extra_rays(args.config, sc, args.small)]).astype(np.float32)
    sample = stride_sample(rays_all)
    times = []
    for s in range(args.warmup + args.steps):
        t = time.perf_counter()
        cpu.intersect(sample, threads=threads, order="index")
        dt = time.perf_counter() - t
        if s >= args.warmup:
            times.append(dt)
    ms = 1e3 * float(np.mean(times))
    v = len(sample) / (ms * 1e-3) / 1e6
    desc = sample_desc(len(sample), len(rays_all), len(sc.assets))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name(args), "rays_per_step": len(rays_all), "sample_rays": len(sample),
                       "sample_objects": len(sc.assets), "order": "index (the reference's flat loop)"},
            "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": threads, "kind": kind, "sample": desc},
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def parity_fields(got, ref, extent, rays):
    """The timed step's FP32 hits against the FP64 device path's on the same
    rays and triangle order (the FP64 path equals the CPU oracle bit for
    bit): hit/miss set, false misses, and the t / uv / normal error. Hit/miss
    differences of rays within 1e-3 of tangent to the FP64 hit's surface
    (|cos| < 1e-3) are counted apart as the grazing band."""
    g_hit, r_hit = got["tri"] >= 0, ref["tri"] >= 0
    both = g_hit & r_hit
    d = rays[:, 3:6].astype(np.float64)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    grazing = r_hit & (np.abs(np.sum(d * ref["ng"], axis=1)) < 1e-3)
    diff = g_hit != r_hit
    out = {"rays": int(len(ref)), "hits": int(r_hit.sum()),
           "mismatched_hit_set": int((diff & ~grazing).sum()),
           "mismatched_in_grazing_band": int((diff & grazing).sum()),
           "false_misses": int((r_hit & ~g_hit).sum()),
           "extra_hits": int((g_hit & ~r_hit).sum()),
           "triangle_mismatch": int((both & (got["tri"] != ref["tri"])).sum())}
    if both.any():
        t_g = got["t"][both].astype(np.float64)
        t_r = ref["t"][both]
        dt = np.abs(t_g - t_r)
        out["max_abs_dt"] = float(dt.max())
        out["max_rel_dt"] = float(dt.max() / extent)
        out["t_equal_to_rounded_fp64"] = float(np.mean(t_g == t_r.astype(np.float32)))
        out["max_duv"] = float(np.abs(got["st"][both].astype(np.float64) - ref["st"][both]).max())
        out["max_dng"] = float(np.abs(got["ng"][both].astype(np.float64) - ref["ng"][both]).max())
    out["extent"] = extent
    out["bar"] = ("hit set identical outside the grazing band, zero false misses outside it, "
                  "max |dt| <= 1e-5 x extent")
    out["pass"] = bool(out["mismatched_hit_set"] == 0 and out.get("max_rel_dt", 0.0) <= 1e-5)
    return out


def scene_extent(dev, n_tri):
    """Diagonal of the union of the triangles' object boxes."""
    lo, hi = np.full(3, np.inf), np.full(3, -np.inf)
    for k in range(n_tri):
        info = dev.triangle_info(k)
        lo = np.minimum(lo, info[3:6])
        hi = np.maximum(hi, info[6:9])
    return float(np.linalg.norm(hi - lo))


def workload_name(args):
    if args.config == "quad":
        return "quad 512^2 FP32, 256x256 camera rays" if not args.small else "quad 128^2 (small)"
    if args.config == "sphere16":
        return ("cube sphere 96 patches x 2048^2 FP16 texels, 1920x1080 jittered primary + 1 diffuse bounce "
                "per hit + 1M grazing rays (0.1-5 deg)" if not args.small
                else "cube sphere 96 patches x 256^2 FP16 + 100k grazing (small)")
    return ("cube sphere 96 patches x 2048^2 FP32, 1920x1080 jittered primary + 1 diffuse bounce per hit"
            if not args.small else "cube sphere 96 patches x 256^2 (small)")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dmap", choices=["dmap", "reference"])
    ap.add_argument("--config", default="sphere",
                    choices=["sphere", "sphere16", "quad", "pathtrace", "serve", "pyramid", "tessellate", "emitter"])
    ap.add_argument("--requests", type=int, default=4096, help="serve: requests in the arrival trace")
    ap.add_argument("--interarrival-ms", type=float, default=15.0, help="serve: mean Poisson inter-arrival time")
    ap.add_argument("--no-plain", action="store_true", help="serve: skip the plain per-request comparison")
    ap.add_argument("--policy", default="oldest", choices=["oldest", "shortest"],
                    help="serve: the server's slot-filling policy")
    ap.add_argument("--build", default="fold", choices=["fold", "direct"], help="pyramid: the build to time")
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="keep --rounds / --blocks-per-sm instead of the autotuner's choice")
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"])
    ap.add_argument("--schedule", default="wavefront", choices=["wavefront", "simple"])
    ap.add_argument("--leaf", default="f32", choices=["f64", "f32"],
                    help="the FP32 path's certified leaf: the reference's FP64 leaf or the FP32 leaf")
    ap.add_argument("--order", default="nearest", choices=["nearest", "index"],
                    help="triangle order: nearest box entry first, or the reference's flat loop")
    ap.add_argument("--rounds", type=int, default=2)
    ap.add_argument("--blocks-per-sm", type=int, default=0,
                    help="walk CTAs per SM (0: the occupancy the scene's walk is compiled for)")
    ap.add_argument("--small", action="store_true", help="reduced sizes for quick checks (not a bench number)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            run_cpu(args, rank, world)
        return

    import torch
    import dmap_b200 as dm
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    if args.config == "pathtrace":
        run_pathtrace(args, rank, world, local, dist)
        return
    if args.config == "serve":
        run_serve(args, rank, world, local, dist)
        return
    if args.config == "pyramid":
        run_pyramid(args, rank, world, local, dist)
        return
    if args.config == "tessellate":
        run_tessellate(args, rank, world, local, dist)
        return
    if args.config == "emitter":
        run_emitter(args, rank, world, local, dist)
        return

    t_setup = time.perf_counter()
    # weak scaling: every rank answers a full batch of its own (the camera's
    # jitter seeded by the rank), so the work per GPU is fixed as N grows
    sc, prim = build_scene(args.config, args.small, scenes.SEED + rank)
    ctx = dm.Context(local)
    keep64 = args.precision == "f64" or True   # the FP64 path counts the reference algorithm's work
    dev = dm.Scene.from_synthetic(ctx, sc, keep_f64=keep64)
    opt = dm.TraversalOptions(precision=args.precision, schedule=args.schedule, rounds=args.rounds,
                              blocks_per_sm=args.blocks_per_sm, order=args.order, leaf_precision=args.leaf)
    ref_opt = dm.TraversalOptions(precision="f64", order=args.order)
    flat_opt = dm.TraversalOptions(precision="f64", order="index")
    # bounce rays from the FP64 hits of the reference's flat loop, frozen
    h0 = dev.intersect(prim, flat_opt, np.float64)
    hit = h0["tri"] >= 0
    bounce = scenes.bounce_rays(prim[hit], h0["t"][hit], h0["ng"][hit])
    rays_all = np.concatenate([prim, bounce, extra_rays(args.config, sc, args.small)]).astype(np.float32)
    # this rank's batch; all ranks together answer world x n_all rays a step
    n_all = len(rays_all)
    my = np.ascontiguousarray(rays_all)
    n = len(my)
    # algorithmic work of the query on these rays (FP64 path counters, same triangle order)
    h_ref, st = dev.intersect(my, ref_opt, np.float64, stats=True)
    flops_ray, bytes_ray, counts = work_per_ray(st)
    # and of the reference's flat loop (index order), for comparison
    counts_flat = work_per_ray(dev.intersect(my, flat_opt, np.float64, stats=True)[1])[2]
    # the measured path's own counters (its bounds are wider: more cells may pass)
    _, st_path = dev.intersect(my, opt, np.float64, stats=True)
    counts_path = work_per_ray(st_path)[2]
    rays_d = torch.from_numpy(my).cuda()
    hits_d = torch.empty((n, 12), dtype=torch.int32, device="cuda")   # 48 B hit32 records
    tuned = None
    if args.tune and args.precision == "f32" and args.schedule == "wavefront":
        # the launch shape the autotuner picks on these rays (setup, not timed)
        opt, tune_ms = dev.autotune(rays_d.data_ptr(), dm.F32, n, opt)
        tuned = {"rounds": opt.rounds, "blocks_per_sm": opt.blocks_per_sm, "sample_ms": tune_ms}
    setup_s = time.perf_counter() - t_setup
    # one explicit stream for the kernels, the L2 flush and the events
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step():
        dev.intersect_device(rays_d.data_ptr(), dm.F32, n, hits_d.data_ptr(), dm.F32, opt,
                             stream=stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    launches0 = ctx.kernel_launches
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with Clocks(local) as clk:
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        for e0, e1 in evs:
            flush.fill_(1.0)          # L2 flush between steps, outside the events
            e0.record(stream)
            step()
            e1.record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    launches = ctx.kernel_launches - launches0
    ms = float(np.sum([a.elapsed_time(b) for a, b in evs])) / args.steps
    ms_max = ms
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    value = world * n_all / (ms_max * 1e-3) / 1e6

    # end to end through the public host API: pinned host rays in, hits out, per step
    rays_h = torch.from_numpy(my).pin_memory()
    hits_h = torch.empty((n, 12), dtype=torch.int32).pin_memory()
    optc = opt.c()
    import ctypes
    L = dm.lib()

    def e2e_step():
        ctx.check(L.dmap_intersect_host(dev.h, rays_h.data_ptr(), dm.F32, n, ctypes.byref(optc),
                                        hits_h.data_ptr(), dm.F32, None), "dmap_intersect_host")

    for _ in range(max(1, args.warmup)):
        e2e_step()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = (time.perf_counter() - t0) / args.steps
    if dist:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = world * n_all / e2e_s / 1e6

    hbm, peak_src = peaks()
    # the unit is one query: its walk and leaf kernels run back to back on one
    # stream and the events bracket all of them
    achieved_gbs = bytes_ray * n / (ms * 1e-3) / 1e9
    traffic_ray = profiled_traffic_per_ray(args)
    traffic = traffic_ray * n if traffic_ray else None
    line = {"metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
            "config": {"workload": workload_name(args), "rays_per_step": n_all, "precision": args.precision,
                       "l2": "flushed between steps (256 MB write); pyramids 17 GB exceed L2",
                       "parallelism": f"replicated scene, one full ray batch per rank ({world} rank(s), camera "
                                      "jitter seeded by the rank)",
                       "rays_per_step_all_ranks": world * n_all,
                       "schedule": args.schedule, "order": args.order, "leaf": args.leaf, "autotuned": tuned,
                       "rounds": opt.rounds, "blocks_per_sm": opt.blocks_per_sm},
            "e2e": {"value": e2e, "unit": "Mrays/s", "h2d_bytes_per_step": int(my.nbytes),
                    "d2h_bytes_per_step": int(n * 48)},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": hbm, "unit": "GB/s",
                         "frac": achieved_gbs / hbm, "traffic": traffic, "peak_source": peak_src,
                         "kernel": f"one query: {launches // args.steps} launches of the walk and leaf kernels",
                         "bytes_per_ray": bytes_ray, "traffic_per_ray": traffic_ray},
            "roofline_fp32": {"achieved": flops_ray * n / (ms * 1e-3) / 1e12, "unit": "TFLOP/s",
                              "flops_per_ray": flops_ray, "nominal_peak": 74.4,
                              "note": "FP32 CUDA-core issue is the path's bound; no measured FP32 peak on file"},
            "work_per_ray": counts, "work_per_ray_path": counts_path, "work_per_ray_flat_loop": counts_flat,
            "setup_s": setup_s}
    clk_s = clk.summary()
    if clk_s:
        line["clocks"] = clk_s
    # parity of the last timed step's hits (outside the timed region)
    got = np.frombuffer(hits_d.cpu().numpy().tobytes(), dm.HIT32)
    line["parity"] = parity_fields(got, h_ref, scene_extent(dev, len(sc.tris)), my)
    line["parity"]["against"] = "FP64 device path, same rays and triangle order (equal to the CPU oracle)"
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cpu, kind = cpu_scene(sc, True)
            sample = stride_sample(rays_all)
            threads = os.cpu_count() or 1
            v = time_cpu(cpu, sample, 10.0, threads)
            line["cpu_baseline"] = {"value": v, "unit": "Mrays/s", "cores": threads, "kind": kind,
                                    "sample": sample_desc(len(sample), n_all, len(sc.assets))}
            del cpu
        except Exception as e:  # the baseline is reported, not required
            line["cpu_baseline"] = {"error": str(e)[:200]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def run_pathtrace(args, rank, world, local, dist):
    """The batched path tracer: cube sphere + ground plane + area emitter,
    1280x720 x 16 spp, depth <= 5, Russian roulette from depth 3; a step is
    one whole render (every extension and shadow query of its 14.7M paths),
    timed by the library's CUDA events on its stream."""
    import torch
    import dmap_b200 as dm
    t_setup = time.perf_counter()
    sc, _ = build_scene("sphere", args.small)
    sc = scenes.with_ground_and_emitter(sc, 512 if args.small else 4096)
    ctx = dm.Context(local)
    dev = dm.Scene.from_synthetic(ctx, sc)
    w, h, spp = (320, 180, 4) if args.small else (1280, 720, 16)
    view = scenes.path_tracer_view(w, h)
    opt = dm.TraversalOptions(schedule=args.schedule, rounds=args.rounds, blocks_per_sm=args.blocks_per_sm,
                              order=args.order, leaf_precision=args.leaf)

    def render(seed):
        return dev.render(view, sc.emitter, spp=spp, max_depth=5, rr_depth=3, seed=seed, options=opt, use_graph=True)

    setup_s = time.perf_counter() - t_setup
    for s in range(args.warmup):
        render(1000 + s)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms, rays, wall, launches, ext, shd = [], 0, 0.0, 0, 0, 0
    img = None
    with Clocks(local) as clk:
        for s in range(args.steps):
            t0 = time.perf_counter()
            img, st, _ = render(scenes.SEED + 7919 * rank + s)
            wall += time.perf_counter() - t0
            ms.append(st["device_ms"])
            ext += st["extension_rays"]
            shd += st["shadow_rays"]
            launches += st["kernel_launches"]
    if dist:
        dist.barrier()
    ms_step = float(np.mean(ms))
    rays_step = (ext + shd) / args.steps
    ms_max, wall_max, rays_all = ms_step, wall / args.steps, rays_step
    if dist:
        t = torch.tensor([ms_step, wall_max], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max, wall_max = float(t[0]), float(t[1])
        r = torch.tensor([rays_step], device="cuda", dtype=torch.float64)
        dist.all_reduce(r)
        rays_all = float(r.item())
    value = rays_all / (ms_max * 1e-3) / 1e6
    line = {"metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"path tracer: cube sphere 96 x {256 if args.small else 2048}^2 + ground "
                                   f"{512 if args.small else 4096}^2 + 0.5x0.5 emitter, {w}x{h} x {spp} spp, "
                                   "depth <= 5, RR from 3, one shadow ray per vertex",
                       "queries_per_step": rays_step, "extension_rays_per_step": ext / args.steps,
                       "shadow_rays_per_step": shd / args.steps, "paths_per_step": w * h * spp,
                       "l2": "pyramids 18 GB exceed L2", "graph": "one batch captured, replayed per batch",
                       "parallelism": f"replicated scene, {world} independent renders"},
            "e2e": {"value": rays_all / wall_max / 1e6, "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(img.nbytes)},
            "gpu_launches": int(launches), "setup_s": setup_s, "image_mean": float(img.mean())}
    clk_s = clk.summary()
    if clk_s:
        line["clocks"] = clk_s
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def run_pyramid(args, rank, world, local, dist):
    """The pyramid build (K1): the cube sphere's 96 maps of 2048^2 FP32
    texels, each built into its outward FP32 pyramid (the product path: the
    FP64 levels are scratch). A step builds all 96; its time is the sum of
    the build kernels' CUDA-event times. Algorithmic bytes per map: the node
    grid read once, the FP32 pyramid written once."""
    import torch
    import dmap_b200 as dm
    sc, _ = build_scene("sphere", args.small)
    ctx = dm.Context(local)
    per_map = []
    for s in range(args.warmup + args.steps):
        ms = 0.0
        with Clocks(local) as clk:
            for a in sc.assets:
                asset = dm.Asset(ctx, a.nodes, build=args.build)
                ms += asset.build_ms
                asset.close()
        if s >= args.warmup:
            per_map.append(ms)
    ms = float(np.mean(per_map))
    nodes = sc.assets[0].nodes.shape[0]
    n = nodes - 1
    cells = sum((n >> l) ** 2 for l in range(n.bit_length()))
    byts = len(sc.assets) * (nodes * nodes * 4 + 32 * cells)
    hbm, peak_src = peaks()
    gbs = byts / (ms * 1e-3) / 1e9
    line = {"metric": "pyramid build GB/s (algorithmic)", "value": gbs, "unit": "GB/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"pyramid build ({args.build}), 96 maps of {n}^2 FP32 texels, outward FP32 "
                                   "pyramid", "maps_per_step": len(sc.assets), "cells_per_map": cells},
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                         "traffic": None, "peak_source": peak_src,
                         "kernel": "pyramid_leaf_kernel + folds" if args.build == "fold"
                         else "direct_hull_* + direct_cells",
                         "bytes_per_map": byts / len(sc.assets)}}
    clk_s = clk.summary()
    if clk_s:
        line["clocks"] = clk_s
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_tessellate(args, rank, world, local, dist):
    """The oracle meshes: the texel-aligned tessellation (m = 1, the
    two-triangle leaf's surface) of 4 cube-sphere patches (8 base
    triangles over 2048^2 FP32 maps), through dmap_tessellate_texel on
    device buffers; a step is one whole call (count, scan, emit). The
    uniform tessellation of all 192 triangles at n = 256 is timed beside it.
    Algorithmic bytes: what the mesh holds, 152 B per face (9 + 6 + 9 floats
    and the 56-byte TexelFace record); the map reads are a few MB."""
    import ctypes as C
    import torch
    import dmap_b200 as dm
    sc_all, _ = build_scene("sphere", args.small)
    sub = scenes.Scene(sc_all.assets[:4], sc_all.tris[:8], sc_all.tri_asset[:8], name="4 patches")
    ctx = dm.Context(local)
    dev = dm.Scene.from_synthetic(ctx, sub)
    L = dm.lib()
    stream = torch.cuda.Stream()   # a stream of its own, so the events and the library's kernels share it
    sp = C.c_void_p(stream.cuda_stream)
    nf = C.c_int64()
    ctx.check(L.dmap_tessellate_texel(dev.h, 1, 0, None, None, None, None, C.byref(nf), sp), "count")
    F = nf.value
    pos = torch.empty(F * 9, dtype=torch.float32, device="cuda")
    uv = torch.empty(F * 6, dtype=torch.float32, device="cuda")
    nrm = torch.empty(F * 9, dtype=torch.float32, device="cuda")
    faces = torch.empty(F * dm.TEXEL_FACE.itemsize, dtype=torch.uint8, device="cuda")

    def texel():
        ctx.check(L.dmap_tessellate_texel(dev.h, 1, F, pos.data_ptr(), uv.data_ptr(), nrm.data_ptr(),
                                          faces.data_ptr(), C.byref(nf), sp), "dmap_tessellate_texel")

    dev_all = dm.Scene.from_synthetic(ctx, sc_all)
    n_u = 256
    Vt, Ft = (n_u + 1) * (n_u + 2) // 2 * dev_all.n_tri, n_u * n_u * dev_all.n_tri
    upos = torch.empty(Vt * 3, dtype=torch.float32, device="cuda")
    uuv = torch.empty(Vt * 2, dtype=torch.float32, device="cuda")
    unrm = torch.empty(Vt * 3, dtype=torch.float32, device="cuda")
    uidx = torch.empty(Ft * 3, dtype=torch.int32, device="cuda")

    def uniform():
        ctx.check(L.dmap_tessellate_uniform(dev_all.h, n_u, upos.data_ptr(), uuv.data_ptr(), unrm.data_ptr(),
                                            uidx.data_ptr(), sp), "dmap_tessellate_uniform")

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(args.steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        return float(np.mean(ms))

    l0 = ctx.kernel_launches
    with Clocks(local) as clk:
        ms = timed(texel)
    launches = (ctx.kernel_launches - l0) // (args.warmup + args.steps)
    ms_u = timed(uniform)
    face_bytes = 9 * 4 + 6 * 4 + 9 * 4 + dm.TEXEL_FACE.itemsize
    gbs = F * face_bytes / (ms * 1e-3) / 1e9
    u_bytes = Vt * 32 + Ft * 12
    hbm, peak_src = peaks()
    line = {"metric": "texel tessellation faces/s", "value": F / (ms * 1e-3), "unit": "faces/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "gpu_launches": launches,
            "config": {"workload": f"append_texel_tessellation m=1, 4 cube-sphere patches (8 triangles) of "
                                   f"{sub.assets[0].n_leaf}^2 FP32 maps", "faces": F,
                       "l2": "output larger than L2"},
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                         "traffic": None, "peak_source": peak_src, "kernel": "texel_kernel<count|emit> + scan",
                         "bytes_per_face": face_bytes},
            "uniform": {"workload": f"append_displaced_triangle n={n_u}, 192 triangles", "vertices": Vt,
                        "faces": Ft, "ms": ms_u, "GB/s": u_bytes / (ms_u * 1e-3) / 1e9}}
    if not args.no_cpu:
        sys.path.insert(0, str(ROOT / "oracle"))
        import py_oracle
        cpu = py_oracle.CpuScene(py_oracle.Oracle(), sub)
        t0 = time.perf_counter()
        got = cpu.tessellate_texel(0, 1)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": len(got["interior"]) / dt, "unit": "faces/s", "cores": 1, "kind": "port",
                                "sample": "triangle 0 of the workload through the oracle's restatement"}
    clk_s = clk.summary()
    if clk_s:
        line["clocks"] = clk_s
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_emitter(args, rank, world, local, dist):
    """Displaced-emitter sampling (DescentSampler, Product weights): 4
    cube-sphere patches (8 triangles) over 2048^2 FP32 maps with 2048^2
    emission tiles (seeded value noise, 30% dark texels); a step draws 4M
    samples spread over the triangles, 48 float uniforms each, through
    dmap_emitter_sample on device buffers, then re-walks their pdfs
    (dmap_emitter_pdf). Algorithmic bytes per sample: the uniforms read
    (192 B), the record written (96 B), and one 64 B FP64 pyramid node per
    weighed child (4 per descent level)."""
    import ctypes as C
    import torch
    import dmap_b200 as dm
    sc_all, _ = build_scene("sphere", args.small)
    sub = scenes.Scene(sc_all.assets[:4], sc_all.tris[:8], sc_all.tri_asset[:8], name="4 patches")
    ctx = dm.Context(local)
    dev = dm.Scene.from_synthetic(ctx, sub, keep_f64=True)
    rng = np.random.default_rng(scenes.SEED)
    tex = [(0.5 + 0.5 * scenes.value_noise(a.n_leaf, 32, rng)) * (rng.random((a.n_leaf, a.n_leaf)) > 0.3)
           for a in sub.assets]
    t0 = time.perf_counter()
    em = dm.Emitter(dev, tex, "product", beta=0.05)
    setup_s = time.perf_counter() - t0
    n, K = (1 << 20) if args.small else (4 << 20), 48
    tri = torch.from_numpy(np.arange(n, dtype=np.int32) % 8).cuda()
    uni = torch.rand((n, K), dtype=torch.float32, device="cuda", generator=torch.Generator("cuda").manual_seed(7))
    out = torch.empty(n * dm.EMITTER_POINT.itemsize, dtype=torch.uint8, device="cuda")
    uv = torch.empty((n, 2), dtype=torch.float64, device="cuda")
    pu, pa = torch.empty(n, dtype=torch.float64, device="cuda"), torch.empty(n, dtype=torch.float64, device="cuda")
    L = dm.lib()
    stream = torch.cuda.Stream()
    sp = C.c_void_p(stream.cuda_stream)

    def sample():
        ctx.check(L.dmap_emitter_sample(em.h, tri.data_ptr(), uni.data_ptr(), K, None, n, out.data_ptr(), sp),
                  "dmap_emitter_sample")

    def pdf():
        ctx.check(L.dmap_emitter_pdf(em.h, tri.data_ptr(), uv.data_ptr(), None, n, pu.data_ptr(), pa.data_ptr(), sp),
                  "dmap_emitter_pdf")

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(args.steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        return float(np.mean(ms))

    l0 = ctx.kernel_launches
    with Clocks(local) as clk:
        ms = timed(sample)
    launches = (ctx.kernel_launches - l0) // (args.warmup + args.steps)
    rec = np.frombuffer(out.cpu().numpy().tobytes(), dm.EMITTER_POINT)
    uv.copy_(torch.from_numpy(np.stack([rec["u"], rec["v"]], 1)))
    ms_pdf = timed(pdf)
    agree = bool(np.array_equal(pu.cpu().numpy(), rec["pdf_uv"]))
    levels = np.array([em.triangle_info(t)[0] + 1 for t in range(8)]).mean()
    byts = K * 4 + dm.EMITTER_POINT.itemsize + 4 * levels * 64
    hbm, peak_src = peaks()
    gbs = n * byts / (ms * 1e-3) / 1e9
    line = {"metric": "Msamples/s displaced-emitter samples", "value": n / (ms * 1e-3) / 1e6, "unit": "Msamples/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "gpu_launches": launches,
            "config": {"workload": f"DescentSampler (Product, beta 0.05), 4 cube-sphere patches (8 triangles) of "
                                   f"{sub.assets[0].n_leaf}^2 FP32 maps and emission tiles", "samples": n,
                       "uniforms_per_sample": K, "descent_levels_mean": float(levels), "setup_s": setup_s},
            "roofline": {"bound": "fp64 issue", "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                         "traffic": None, "peak_source": peak_src, "kernel": "sample_kernel",
                         "bytes_per_sample": byts},
            "pdf": {"ms": ms_pdf, "Mqueries/s": n / (ms_pdf * 1e-3) / 1e6, "equals_sampled_pdf": agree},
            "draws_mean": float(rec["draws"].mean()), "no_mass": int((rec["draws"] < 0).sum())}
    if not args.no_cpu:
        sys.path.insert(0, str(ROOT / "oracle"))
        import py_oracle
        cpu = py_oracle.CpuScene(py_oracle.Reference() if py_oracle.Reference.available() else py_oracle.Oracle(),
                                 sub)
        ce = py_oracle.CpuEmitter(cpu, 0, tex[0], "product", beta=0.05)
        uu = uni[:4096].cpu().numpy()
        t0 = time.perf_counter()
        for k in range(len(uu)):
            ce.sample(uu[k])
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": len(uu) / dt / 1e6, "unit": "Msamples/s", "cores": 1,
                                "kind": "reference" if isinstance(cpu.lib, py_oracle.Reference) else "port",
                                "sample": "4096 samples of triangle 0, one Python call each"}
    clk_s = clk.summary()
    if clk_s:
        line["clocks"] = clk_s
    if rank == 0:
        print(json.dumps(line), flush=True)


def serve_trace(n_req: int, interarrival_ms: float, seed: int, small: bool):
    """The arrival trace: Poisson arrivals, a seeded scene id and a ray
    count log-uniform in [1K, 4M] (4x smaller bounds with --small); mix 60%
    primary (scene 0, 1 or 2), 30% path-traced (scene 2, 4 spp, depth 3,
    ray count = camera samples), 10% shadow-only (scene 2)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = np.cumsum(rng.exponential(interarrival_ms * 1e-3, n_req))
    t -= t[0]
    hi = 1 << 20 if small else 4 << 20
    n = np.exp(rng.uniform(np.log(1024), np.log(hi), n_req)).astype(np.int64)
    u = rng.random(n_req)
    kind = np.where(u < 0.6, 0, np.where(u < 0.9, 1, 2))          # primary, path-traced, shadow
    scene = np.where(kind == 0, rng.integers(0, 3, n_req), 2)
    return [dict(t=float(t[k]), n=int(n[k]), kind=int(kind[k]), scene=int(scene[k]), seed=seed + k,
                 off=float(rng.random())) for k in range(n_req)]


def run_serve(args, rank, world, local, dist):
    """Serving: resident scenes (the quad, the cube sphere, the cube sphere +
    ground + emitter sharing the sphere's assets), an open-loop Poisson trace
    of requests, served by dmap_server (continuous batching, HBM-budget
    admission) and, on the same arrival times, by the plain path: each
    request alone, in arrival order, one launch per query (the simple
    one-thread-per-ray schedule through dmap_intersect_host / dmap_render)."""
    import torch
    import dmap_b200 as dm
    t_setup = time.perf_counter()
    small = args.small
    sph, _ = build_scene("sphere", small)
    quad = scenes.quad_scene(128 if small else 512)
    ctx = dm.Context(local)
    d_quad = dm.Scene.from_synthetic(ctx, quad)
    sph_assets = [dm.Asset(ctx, a.nodes) for a in sph.assets]
    d_sph = dm.Scene(ctx, sph_assets, sph.tris, sph.tri_asset)
    pt = scenes.with_ground_and_emitter(sph, 512 if small else 4096)
    ground = dm.Asset(ctx, pt.assets[-1].nodes)
    d_pt = dm.Scene(ctx, sph_assets + [ground], pt.tris, pt.tri_asset)   # shares the sphere's pyramids
    devs = [d_quad, d_sph, d_pt]
    resident = sum(a.device_bytes for a in sph_assets + [ground]) + sum(a.device_bytes for a in d_quad.assets)
    view = scenes.path_tracer_view(1280, 720)
    # ray pools in pinned memory: camera rays per scene, shadow rays toward the emitter
    side = 1024 if small else 2048
    pools = [scenes.quad_camera_rays(side, side),
             scenes.sphere_camera_rays(side * 5 // 4, side * 4 // 5 if small else 1638),
             scenes.pinhole_rays(view["eye"], view["target"], view["up"], view["fov_deg"], side * 5 // 4,
                                 side * 4 // 5 if small else 1638, jitter_seed=scenes.SEED + 3)]
    h = d_pt.intersect(pools[2], dm.TraversalOptions(), np.float32)
    hit = h["tri"] >= 0
    x = pools[2][hit, 0:3] + h["t"][hit, None] * pools[2][hit, 3:6]
    ng = h["ng"][hit]
    ng = np.where((np.sum(ng * pools[2][hit, 3:6], 1) > 0)[:, None], -ng, ng)
    rng = np.random.Generator(np.random.PCG64(scenes.SEED + 4))
    e = pt.emitter
    y = e[0] + rng.random((len(x), 1)) * (e[1] - e[0]) + rng.random((len(x), 1)) * (e[2] - e[0])
    xo = x + 1e-4 * ng
    w = y - xo
    dist_ = np.linalg.norm(w, axis=1)
    shadow = np.zeros((len(x), 8), np.float32)
    shadow[:, 0:3], shadow[:, 3:6], shadow[:, 7] = xo, w / dist_[:, None], dist_ - 1e-4
    pools.append(shadow)
    pinned = [torch.from_numpy(np.ascontiguousarray(p)).pin_memory() for p in pools]
    trace = serve_trace(args.requests, args.interarrival_ms, scenes.SEED + 99, small)
    ring_n = (16 << 20) if not small else (4 << 20)
    ring = torch.empty(ring_n * 48, dtype=torch.uint8).pin_memory().numpy().view(dm.HIT32)
    setup_s = time.perf_counter() - t_setup

    def request_rays(r):
        pool = pinned[3] if r["kind"] == 2 else pinned[r["scene"]]
        n = min(r["n"], len(pool))
        lo = int(r["off"] * (len(pool) - n))
        return pool.numpy()[lo:lo + n]

    def request_view(r):
        px = max(64, r["n"] // 4)
        wdt = max(8, int(round(math.sqrt(px * 16 / 9))))
        v = dict(view)
        v["width"], v["height"] = wdt, max(8, px // wdt)
        return v

    rkw = dict(spp=4, max_depth=3, rr_depth=3)
    opt = dm.TraversalOptions(schedule=args.schedule, rounds=args.rounds, blocks_per_sm=args.blocks_per_sm,
                              order=args.order, leaf_precision=args.leaf)
    # warm-up: every path once
    srv = dm.Server(ctx, hbm_budget_bytes=120 * 10 ** 9, slots=2, options=opt)
    for k in range(args.warmup):
        ids = [srv.submit_rays(devs[k % 3], pools[k % 3][:50000])[0],
               srv.submit_render(d_pt, request_view({"n": 40000}), pt.emitter, seed=k, **rkw)[0]]
        srv.drain()
    srv.close()

    # served
    srv = dm.Server(ctx, hbm_budget_bytes=120 * 10 ** 9, slots=2, options=opt, policy=args.policy)
    ring_at, outstanding = 0, []
    t0 = time.perf_counter()
    with Clocks(local) as clk:
        for r in trace:
            now = time.perf_counter() - t0
            if r["t"] > now:
                time.sleep(r["t"] - now)
            if r["kind"] == 1:
                srv.submit_render(d_pt, request_view(r), pt.emitter, seed=r["seed"], **rkw)
                continue
            rays = request_rays(r)
            n = len(rays)
            if ring_at + n > ring_n:
                ring_at = 0
            # back-pressure: the ring slice must be free
            while outstanding and any(a < ring_at + n and ring_at < b for a, b, _ in outstanding):
                a, b, rid = outstanding.pop(0)
                srv.wait(rid)
            rid, _ = srv.submit_rays(devs[r["scene"]] if r["kind"] == 0 else d_pt, rays,
                                     "occluded" if r["kind"] == 2 else "closest", hits=ring[ring_at:ring_at + n])
            outstanding.append((ring_at, ring_at + n, rid))
            ring_at += n
        srv.drain()
        wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    served = {"mrays_s": st["rays"] / st["wall_s"] / 1e6, "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
              "mean_ms": st["mean_ms"], "max_ms": st["max_ms"], "queries": st["rays"], "makespan_s": st["wall_s"],
              "busy_s": st["busy_s"], "launches": st["launches"], "peak_device_bytes": st["peak_bytes"] + resident}

    def run_plain(schedule):
        """Each request alone, in arrival order, one query launch at a time
        through the host API (dmap_intersect_host / dmap_render without a
        graph) on the given schedule."""
        popt = dm.TraversalOptions(schedule=schedule, order=args.order, rounds=args.rounds,
                                   blocks_per_sm=args.blocks_per_sm, leaf_precision=args.leaf)
        lat, queries = [], 0
        t0 = time.perf_counter()
        for r in trace:
            now = time.perf_counter() - t0
            if r["t"] > now:
                time.sleep(r["t"] - now)
            if r["kind"] == 1:
                _, rs, _ = d_pt.render(request_view(r), pt.emitter, seed=r["seed"], use_graph=False, options=popt,
                                       **rkw)
                queries += rs["extension_rays"] + rs["shadow_rays"]
            else:
                rays = request_rays(r)
                d = devs[r["scene"]] if r["kind"] == 0 else d_pt
                d.intersect(rays, dm.TraversalOptions(schedule=schedule, order=args.order, rounds=args.rounds,
                                                      blocks_per_sm=args.blocks_per_sm, leaf_precision=args.leaf,
                                                      mode="occluded" if r["kind"] == 2 else "closest"), np.float32)
                queries += len(rays)
            lat.append((time.perf_counter() - t0 - r["t"]) * 1e3)
        mk = time.perf_counter() - t0
        lat = np.sort(np.array(lat))
        return {"schedule": schedule, "mrays_s": queries / mk / 1e6,
                "p50_ms": float(np.percentile(lat, 50, method="inverted_cdf")),
                "p99_ms": float(np.percentile(lat, 99, method="inverted_cdf")), "mean_ms": float(lat.mean()),
                "makespan_s": mk, "queries": queries}

    # the plain one-launch-per-request path (one thread per ray), and the
    # same one request at a time on the wavefront kernel: the second
    # separates what continuous batching gains from what the kernel gains
    plain = None if args.no_plain else run_plain("simple")
    plain_wave = None if args.no_plain else run_plain("wavefront")
    line = {"metric": METRIC, "value": served["mrays_s"], "unit": "Mrays/s", "n_gpus": world, "steps": 1,
            "warmup": args.warmup, "ms_per_step": served["makespan_s"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"serving: {args.requests} Poisson requests (mean inter-arrival "
                                   f"{args.interarrival_ms} ms), rays log-uniform in [1K, {'1M' if small else '4M'}], "
                                   "60% primary / 30% path-traced (4 spp, depth 3) / 10% shadow-only, scenes: quad "
                                   f"{128 if small else 512}^2, cube sphere 96 x {256 if small else 2048}^2, "
                                   "cube sphere + ground + emitter (shared assets), 120 GB budget",
                       "resident_scene_bytes": resident, "policy": args.policy},
            "served": served, "plain": plain, "plain_wavefront": plain_wave,
            "served_over_plain": (served["mrays_s"] / plain["mrays_s"]) if plain else None,
            "served_over_plain_wavefront": (served["mrays_s"] / plain_wave["mrays_s"]) if plain_wave else None,
            "p50_ms": served["p50_ms"], "p99_ms": served["p99_ms"],
            "e2e": {"value": served["mrays_s"], "unit": "Mrays/s", "h2d_bytes_per_step": None,
                    "d2h_bytes_per_step": None, "note": "every request through the host API"},
            "gpu_launches": served["launches"], "setup_s": setup_s}
    clk_s = clk.summary()
    if clk_s:
        line["clocks"] = clk_s
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
