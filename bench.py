#!/usr/bin/env python
"""Benchmark of toaster's GPU path-tracing path on B200: Mpaths/s on the mixed scene.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the mixed scene (2,048 seeded triangles + 128 spheres, 50/30/20 diffuse / metal /
dielectric, 16 emissive triangles, 1024x512 FP32 sky with a 0.5-degree sun of radiance 1e4) at
1280x720, 64 samples per pixel, 8 bounces. One step = one full frame (921,600 pixels x 64 paths).

`value` is device time (CUDA events on the library's stream) over exactly K frames with the
scene resident in HBM; L2 is flushed (a 256 MiB write) before every timed frame. `e2e` is the
same metric through the public C ABI with host buffers: each step uploads the scene records
from pinned host memory (the library rebuilds the hierarchy and the environment tables),
renders, and reads the float4 image back into pinned host memory; it is timed with the host
clock. Multi-GPU runs are independent replicas (the path has no cross-rank exchange).
`--impl reference` times the oracle (a C++ restatement of the reference CPU renderer, the
reference itself being Rust that cannot be built here) on all host threads over a strided row
sample of the same frame.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mpaths/s (1280x720, 8 bounces)"
UNIT = "Mpaths/s"
WORKLOAD = ("mixed scene: 2,048 seeded triangles + 128 spheres (50/30/20 diffuse/metal/dielectric, 16 emissive "
            "triangles), 1024x512 FP32 sky + 0.5-degree sun (1e4), 1280x720, 64 spp, 8 bounces")



def ordinal(n: int) -> str:
    """1st, 2nd, 3rd, 4th, ..., 11th-13th, 21st."""
    suffix = "th" if 10 <= n % 100 <= 20 else {1: "st", 2: "nd", 3: "rd"}.get(n % 10, "th")
    return f"{n}{suffix}"

def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="target wall time of one CPU sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--spp", type=int, default=64, help="samples per pixel per frame (64 = the benchmark workload)")
    ap.add_argument("--no-equal-time", action="store_true", help="skip the guided-vs-plain equal-time comparison")
    ap.add_argument("--no-reference-suite", action="store_true",
                    help="skip the reference's own benchmark fixtures under its protocol")
    ap.add_argument("--equal-time-ref-spp", type=int, default=65536,
                    help="samples per pixel of the plain FP64 reference the equal-time RMSE is measured against")
    ap.add_argument("--equal-time-seeds", type=int, default=3, help="independent guided/plain runs (median)")
    ap.add_argument("--cpu-table", action="store_true",
                    help="only time the CPU baseline (the oracle) at 1 thread and all threads on the plain-small, "
                         "mixed, large-mesh and window-room workloads, one JSON line each")
    ap.add_argument("--batch-eval", action="store_true",
                    help="also run the batched-scenes and animated-frames evaluation (a few minutes)")
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device = device_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_sample(scene, target_seconds: float, threads: int = 0):
    """Times the oracle on evenly strided rows sized to about `target_seconds` of wall time."""
    import oracle

    o = oracle.Oracle(scene)
    h, w, spp = scene.height, scene.width, scene.samples
    t0 = time.perf_counter()
    o.render(seed=1, rows=(h // 2, h // 2 + 1), row_step=1, threads=threads)
    probe = time.perf_counter() - t0
    rows_wanted = max(2, min(h, int(target_seconds / max(probe, 1e-4))))
    step = max(1, h // rows_wanted)
    t0 = time.perf_counter()
    mean, _, counts = o.render(seed=2, rows=(0, h), row_step=step, threads=threads, counts=True)
    dt = time.perf_counter() - t0
    nrows = mean.shape[0]
    paths = nrows * w * spp
    return {
        "mpaths_s": paths / dt / 1e6,
        "seconds": dt,
        "paths": paths,
        "rows": nrows,
        "row_step": step,
        "cores": oracle.binding.num_threads() if threads <= 0 else threads,
        "counts": [int(c) for c in counts],
    }


def algorithmic_bytes_per_ray(counts):
    """Reference traversal work per ray: child boxes tested (root + 2 per interior visit) x 32 B,
    triangle tests x 36 B (v0, e1, e2), sphere tests x 16 B (centre, radius), counted by the
    oracle's ordered traversal over the frame's own ray mix (primary, bounce and shadow rays)."""
    rays, _, spheres, tris, interior, _ = counts
    return ((rays + 2 * interior) * 32 + tris * 36 + spheres * 16) / max(rays, 1)


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    from toaster_b200 import configs
    import oracle

    scene = configs.mixed()
    samples = []
    for i in range(args.warmup + args.steps):
        s = cpu_sample(scene, args.cpu_seconds if i >= args.warmup else min(2.0, args.cpu_seconds))
        if i >= args.warmup:
            samples.append(s)
    value = statistics.median([s["mpaths_s"] for s in samples])
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": statistics.median([s["seconds"] * 1e3 for s in samples]),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "width": 1280, "height": 720, "spp": 64, "max_bounces": 8},
        "cpu_baseline": {
            "value": value, "unit": UNIT, "cores": samples[0]["cores"], "kind": "port",
            "sample": f"every {ordinal(samples[0]['row_step'])} row ({samples[0]['rows']} rows x 1280 px x 64 spp) per step; "
                      "oracle = C++ restatement of crates/toaster-cpu (reference is Rust, unbuildable here)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def pinned_copy(arr, keep):
    import numpy as np
    import torch

    if arr is None:
        return None
    t = torch.empty(max(arr.nbytes, 1), dtype=torch.uint8, pin_memory=True)
    keep.append(t)
    view = t.numpy()[: arr.nbytes].view(arr.dtype).reshape(arr.shape)
    view[...] = arr
    return view


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    from toaster_b200 import build, configs
    from toaster_b200.renderer import GpuRenderer
    from toaster_b200.replicas import job_throughput, max_over_ranks
    from toaster_b200.scene import SceneGpuData, scene_to_gpu

    world, rank, local = dist_env()
    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    build.build()
    scene = configs.mixed(samples=args.spp)
    data = scene_to_gpu(scene)
    w, h, spp = scene.width, scene.height, scene.samples
    paths_per_step = w * h * spp

    from toaster_b200.native import probe_cache_read

    # The roofline's denominator: L2 read bandwidth (the scene's working set is L2-resident).
    l2_peak = statistics.median(probe_cache_read(local, 64 << 20, 50) for _ in range(3))

    r = GpuRenderer(local)
    stream = torch.cuda.Stream(device=local)
    r.set_stream(stream.cuda_stream)
    r.upload(data)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    def barrier():
        if world > 1:
            dist.barrier()

    for i in range(args.warmup):
        r.render(frame_index=0)
    torch.cuda.synchronize()

    # ---------------- device-timed steps (scene resident)
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    step_ms, kernel_ms, rays, launches = [], [], [], 0
    phases = {"trace_ms": [], "logic_ms": [], "shade_ms": [], "wf_iterations": []}
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r.render(frame_index=0, phase_timing=True)
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        st = r.stats()
        kernel_ms.append(st["kernel_ms"])
        rays.append(st["rays"])
        launches += st["kernel_launches"]
        for key in phases:
            phases[key].append(st[key])
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier()
    total_ms = max_over_ranks(sum(step_ms), device=f"cuda:{local}")
    value = job_throughput(paths_per_step, args.steps, world, total_ms * 1e-3)

    # ---------------- end-to-end through the C ABI with pinned host buffers
    keep = []
    pinned = SceneGpuData(**{k: pinned_copy(v, keep) if isinstance(v, np.ndarray) else v
                             for k, v in data.__dict__.items()})
    h2d = pinned.host_bytes()
    out = pinned_copy(np.zeros((h, w, 4), np.float32), keep)
    d2h = out.nbytes
    r2 = GpuRenderer(local)
    r2.upload(pinned)
    r2.render(frame_index=0)
    r2.readback(out)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(args.steps):
        r2.upload(pinned)
        r2.render(frame_index=0)
        r2.readback(out)
    e2e_s = time.perf_counter() - t0
    barrier()
    e2e_s = max_over_ranks(e2e_s, device=f"cuda:{local}")
    e2e_value = job_throughput(paths_per_step, args.steps, world, e2e_s)
    assert np.all(np.isfinite(out)), "non-finite pixels in the benchmark image"
    r2.close()

    line = None
    if rank == 0:
        mean_kernel_ms = statistics.mean(kernel_ms)
        mean_rays = statistics.mean(rays)
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_sample(scene, args.cpu_seconds)
        hbm_peak, peak_kind = measured_peaks()
        roofline = None
        if cpu is not None:
            # Dominant kernel: the wavefront's trace launches (one per iteration), timed live by the
            # library's per-phase CUDA events on the render stream. Their algorithmic bytes are the
            # traversal's node and primitive fetches of every ray the step traced.
            bpr = algorithmic_bytes_per_ray(cpu["counts"])
            trace_ms = statistics.mean(phases["trace_ms"])
            iterations = statistics.mean(phases["wf_iterations"])
            achieved = bpr * mean_rays / (trace_ms * 1e-3) / 1e9
            prof = kernel_profile()
            tpi = prof.get("threads_per_instruction") if prof else None
            trace_dram = prof.get("dram_bytes_per_ray_trace_kernel") if prof else None
            roofline = {"bound": "l2", "achieved": achieved, "peak": l2_peak, "unit": "GB/s",
                        "frac": achieved / l2_peak,
                        "traffic": None if trace_dram is None else trace_dram * mean_rays / iterations,
                        "traffic_note": "DRAM bytes per trace launch: ncu's dram__bytes_read + write per ray of "
                                        "the trace launches (8-spp frames of this scene) x rays per launch",
                        "peak_source": "measured live: L2 read bandwidth of a 64 MiB buffer streamed by every SM "
                                       "(tc_probe_cache_read, loads bypassing L1)",
                        "hbm_peak": hbm_peak, "hbm_peak_source": peak_kind, "frac_of_hbm": achieved / hbm_peak,
                        "issue": None if tpi is None else {
                            "threads_per_instruction": tpi, "of": 32, "frac": tpi / 32.0,
                            "source": prof.get("source")},
                        "kernel": "wf_trace_kernel<0, 0, 0> (wavefront trace launches)",
                        "launches_per_step": iterations, "bytes_per_ray": bpr,
                        "algorithmic_bytes_per_launch": bpr * mean_rays / iterations,
                        "launch_ms": trace_ms / iterations,
                        "phases_ms_per_step": {k: statistics.mean(phases[k])
                                               for k in ("trace_ms", "logic_ms", "shade_ms")},
                        "step_kernel_ms": mean_kernel_ms,
                        "frac_over_whole_step": bpr * mean_rays / (mean_kernel_ms * 1e-3) / 1e9 / l2_peak}
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "width": w, "height": h, "spp": spp, "max_bounces": scene.max_bounces,
                       "l2": "flushed before every timed step (256 MiB write)", "parallelism": f"replicas x{world}"},
            "mrays_per_s": world * mean_rays * args.steps / (total_ms * 1e-3) / 1e6,
            "kernel_ms": mean_kernel_ms,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "timing": "host clock over K steps of upload + render + readback"},
            "gpu_launches": launches,
            "clocks": clk,
        }
        if roofline is not None:
            line["roofline"] = roofline
        if world == 1 and not args.no_equal_time:
            line["equal_time"] = equal_time_block(args.equal_time_ref_spp, local, args.equal_time_seeds)
        if world == 1 and not args.no_reference_suite:
            line["reference_suite"] = reference_suite_block(local)
        if world == 1 and args.batch_eval:
            from toaster_b200 import batch_eval
            line["batched"] = batch_eval.uneven()
            line["animation"] = batch_eval.animation(frames=240)
        if cpu is not None:
            line["cpu_baseline"] = {
                "value": cpu["mpaths_s"], "unit": UNIT, "cores": cpu["cores"], "kind": "port",
                "sample": f"oracle (C++ restatement of crates/toaster-cpu) on every {ordinal(cpu['row_step'])} row "
                          f"({cpu['rows']} rows x {w} px x {spp} spp, {cpu['seconds']:.1f} s)"}
        print(json.dumps(line), flush=True)
    r.set_stream(0)
    r.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def reference_suite_block(device: int) -> dict:
    """The reference's seven benchmark fixtures (regenerated byte for byte; 320x180, 4 spp,
    4 bounces) under its own protocol (2 warm-up + 5 measured frames, seed 0, medians), beside the
    RTX 2080 Ti medians it publishes. Loaded through the native scene loader."""
    import tempfile

    from toaster_b200 import bench_fixtures

    with tempfile.TemporaryDirectory() as tmp:
        rows = bench_fixtures.run(tmp, device=device)
    keep = ("dispatch_ms", "kernel_ms", "total_ms", "published_2080ti_dispatch_ms", "published_2080ti_total_ms",
            "dispatch_speedup_vs_published", "total_speedup_vs_published")
    return {"protocol": "320x180, 4 spp, 4 bounces; median of 5 frames after 2 warm-up frames; seed 0",
            "published": "RTX 2080 Ti / Vulkan medians from the reference's README",
            "fixtures": {row["scene"].split(".")[0]: {k: row[k] for k in keep} for row in rows}}


def equal_time_block(ref_spp: int, device: int, seeds: int = 3) -> dict:
    """Guided vs plain sampling at equal GPU time on the learned-guiding workload (window room,
    8,192 clutter triangles with 30% metal, 1280x720, 8 bounces): plain accumulates 256 spp in
    16-spp batches; guided records 16 spp, trains the recipe's Adam steps on the GPU and accumulates
    guided batches, each recording its own training samples into the pool and followed by the
    recipe's online Adam steps (their time counts). RMSE is against a plain FP64 reference of ``ref_spp`` samples per pixel, taken
    over 4 evenly spaced bands of 8 rows (40,960 pixels; the reference is rendered for those rows
    only, which keeps the 65,536-spp render within a minute); the trimmed RMSE leaves out the 0.1%
    largest pixel errors. Medians over ``seeds`` independent runs, each seed's figures beside them."""
    from toaster_b200 import configs, guiding_eval

    scene = configs.room_with_window()
    t0 = time.perf_counter()
    rows, reference = guiding_eval.reference_bands(scene, ref_spp, bands=4, rows=8, device=device)
    ref_s = time.perf_counter() - t0
    keep = ["plain_seconds", "plain_rmse", "guided_seconds_to_plain_rmse", "time_fraction",
            "guided_rmse_at_plain_time", "plain_trimmed_rmse", "time_fraction_trimmed",
            "guided_trimmed_rmse_at_plain_time", "train_seconds", "samples", "pool_samples",
            "online_train_seconds"]
    runs = []
    for seed in range(seeds):
        out = guiding_eval.equal_time_comparison(scene, ref_spp=ref_spp, plain_spp=256, batch=16, record_spp=16,
                                                 train_steps=guiding_eval.TRAIN_STEPS, train_batch=8192, seed=seed,
                                                 device=device, reference=reference, rows=rows)
        runs.append({k: out.get(k) for k in keep})

    def median(key):
        vals = [r[key] for r in runs if r[key] is not None]
        return statistics.median(vals) if len(vals) == len(runs) else None

    return {"workload": "window room, 8,192 clutter triangles (30% metal), 1280x720, 8 bounces",
            "reference_spp": ref_spp, "reference_rows": "4 bands of 8 rows (40,960 pixels)",
            "reference_seconds": ref_s, "plain_spp": 256, "record_spp": 16,
            "train_steps": guiding_eval.TRAIN_STEPS, "online_steps": guiding_eval.ONLINE_STEPS,
            "online_batch": guiding_eval.ONLINE_BATCH, "seeds": seeds,
            "time_fraction": median("time_fraction"), "time_fraction_trimmed": median("time_fraction_trimmed"),
            "plain_rmse": median("plain_rmse"), "plain_trimmed_rmse": median("plain_trimmed_rmse"),
            "per_seed": runs, "wall_seconds": time.perf_counter() - t0}


def kernel_profile():
    """The committed ncu figures of the bench's dominant kernel (DRAM bytes per ray, threads per
    executed instruction), or None."""
    p = ROOT / "profiles" / "bench_frame_figures.json"
    if not p.exists():
        return None
    try:
        return json.loads(p.read_text())
    except Exception:
        return None


def cpu_table(args) -> int:
    """The CPU baseline beside every GPU workload: the oracle at 1 thread and at all host threads,
    on the whole plain-small frame and on strided row samples of the others."""
    from toaster_b200 import configs

    workloads = [("plain_small", configs.plain_small), ("mixed", configs.mixed),
                 ("large_mesh", configs.large_mesh), ("room", configs.room_with_window)]
    for name, make in workloads:
        scene = make()
        for threads in (1, 0):
            t = cpu_sample(scene, args.cpu_seconds, threads=threads)
            rays = t["counts"][0]
            print(json.dumps({"workload": name, "width": scene.width, "height": scene.height, "spp": scene.samples,
                              "max_bounces": scene.max_bounces, "threads": t["cores"], "mpaths_per_s": t["mpaths_s"],
                              "mrays_per_s": rays / t["seconds"] / 1e6, "rows": t["rows"],
                              "row_step": t["row_step"], "seconds": t["seconds"]}), flush=True)
    return 0


def main():
    args = parse_args()
    if args.cpu_table:
        return cpu_table(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
