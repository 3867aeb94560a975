#!/usr/bin/env python
"""Benchmark of the plain per-frame GI path (trace + temporal + 3x a-trous +
present) on the full-size workload: 256^3 world (seed 2), 1920x1080, 1 spp,
2 indirect bounces, firefly clamp 10, along the 120-frame camera spline.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one frame.  Device time per frame comes from CUDA events the
library records on its own stream around its kernels; the L2 is flushed (a
256 MB write) before every timed frame, outside the events.  `value` is
Mrays/s over all ranks (rays = trace invocations: primary + bounce + shadow).
N > 1 runs independent replicas (one per GPU, no collective on the data
path); the reported time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mrays/s & 1080p frame ms, plain vs batched+cache at equal MSE; p50/p99 latency"
WORKLOAD = dict(kind=2, n=256, seed=2, W=1920, H=1080, bounces=2, fclamp=10.0, maxhist=64.0, flags=3, path_frames=120)
WORKLOAD_NAME = ("plain GI frame (pathtrace+temporal+3x a-trous+present): 256^3 procedural world seed 2, "
                 "1920x1080, 1 spp, 2 bounces, clamp 10, 120-frame camera spline")
ALG_BYTES_PER_PX = 28          # pathtrace writes: radiance 8 + albedo 4 + G-buffer 16
FRAME_BYTES_PER_PX = 196       # all passes, compulsory (pathtrace 28, temporal 56, a-trous 96, present 16)
L2_FLUSH_BYTES = 256 << 20


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-cache-compare", action="store_true",
                    help="frame mode: skip the plain vs batched+cache comparison in the output line")
    ap.add_argument("--path-kernel", default="wavefront", choices=["wavefront", "megakernel"])
    ap.add_argument("--mode", default="frame", choices=["frame", "batched", "serve", "cache", "cache-frame", "lights",
                                                        "restir", "restir-scenes", "voxelbench", "correctness",
                                                        "wave-sweep"],
                    help="frame: the full-size plain frame (default); batched: 64 mixed jobs in one launch; "
                         "serve: Poisson request stream over 32 sessions; cache: cache-assisted vs plain "
                         "path tracing at matched MSE; restir: the ReSTIR presets beside the plain frame; "
                         "restir-scenes: `ours` on the reference's own scenarios with its capture settings; "
                         "correctness: the reference's estimator-correctness captures against its recorded "
                         "channel means and HDR errors; cache-frame: one cache-assisted 1080p frame (for "
                         "profiling); wave-sweep: the plain frame over refill thresholds and tracer variants "
                         "(for per-wave launch lists)")
    ap.add_argument("--rates", default="200,500,1000,2000", help="serve: arrival rates (requests/s)")
    ap.add_argument("--duration", type=float, default=1.5, help="serve: seconds of arrivals per rate")
    ap.add_argument("--jobs", type=int, default=64)
    ap.add_argument("--cache", action="store_true", help="serve: also run the sweep with the cache-assisted path")
    ap.add_argument("--no-extras", action="store_true",
                    help="frame mode: skip the ReSTIR and VoxelBench summaries in the output line")
    ap.add_argument("--runs", default="", help="restir: comma-separated subset of plain,gi,ours,ours_b6_nodenoise")
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(kernel: str):
    """DRAM bytes (read + write) per launch of `kernel` from the committed
    ncu summary of this workload (profiles/<kernel>_1080p_256.md)."""
    p = ROOT / "profiles" / f"{kernel}_1080p_256.md"
    if not p.exists():
        return None
    m = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", p.read_text())
    return float(m.group(1)) if m else None


def profiled_l2(kernel: str):
    """L2 throughput of `kernel` as a fraction of its peak, from the committed
    ncu summary (profiles/<kernel>_1080p_256.md, `l2_throughput_pct:` line)."""
    p = ROOT / "profiles" / f"{kernel}_1080p_256.md"
    if not p.exists():
        return None
    m = re.search(r"l2_throughput_pct:\s*([0-9.eE+]+)", p.read_text())
    return {"frac": round(float(m.group(1)) / 100.0, 4),
            "source": f"ncu lts__t_sectors throughput, % of peak (profiles/{p.name})"} if m else None


class ClockSampler:
    """nvidia-smi clocks + throttle reasons sampled every 20 ms while the timed
    region runs.  start() returns once the sampler has produced its first line
    (nvidia-smi's own startup can outlast a short timed region); stop() keeps
    the samples taken between start() and stop()."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []
        self.t0 = 0.0

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line))

    def start(self):
        import threading

        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "20", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.th = threading.Thread(target=self._read, daemon=True)
        self.th.start()
        deadline = time.perf_counter() + 5.0
        while not self.lines and time.perf_counter() < deadline and self.proc.poll() is None:
            time.sleep(0.005)
        self.t0 = time.perf_counter()

    def stop(self):
        if self.proc is None:
            return None
        t1 = time.perf_counter()
        time.sleep(0.03)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            self.proc.wait()
        self.th.join(timeout=5)
        inside = [ln for t, ln in self.lines if self.t0 <= t <= t1 + 0.03]
        if not inside and self.lines:
            inside = [self.lines[-1][1]]
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in inside:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def reduce_over_ranks(dist, device, seconds_or_ms: float, count: float):
    """Replica aggregation: the job's time is the slowest rank's, the work is
    the sum over ranks.  Returns (max time, summed count)."""
    if dist is None:
        return float(seconds_or_ms), float(count)
    import torch
    t = torch.tensor([float(seconds_or_ms)], dtype=torch.float64, device=device)
    c = torch.tensor([float(count)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), float(c.item())


def workload_config() -> dict:
    """The `config` of the plain-frame line, identical in both arms; how each
    arm runs it is under `impl_details`."""
    return {"workload": WORKLOAD_NAME, "grid": WORKLOAD["n"], "width": WORKLOAD["W"], "height": WORKLOAD["H"],
            "spp": 1, "bounces": WORKLOAD["bounces"], "history": "rgba16f, cap 64", "denoise": "a-trous 1/2/4",
            "l2": "GPU arm: flushed before every timed frame (256 MB write), outside the timed events; "
                  "CPU arm: not applicable"}


def frame_uniforms(vrt, spawn, f):
    W, H = WORKLOAD["W"], WORKLOAD["H"]
    k = f % WORKLOAD["path_frames"]
    pose = vrt.camera_spline(spawn, k)
    prev = vrt.camera_spline(spawn, k - 1) if k > 0 else None
    return vrt.make_uniforms(pose, prev, vrt.Lighting(), f, WORKLOAD["bounces"], WORKLOAD["flags"], W, H, 1.0,
                             WORKLOAD["maxhist"])


def cpu_baseline_port(vox, spawn, vrt):
    """The CPU oracle (scalar restatement of the same path, OpenMP over rows)
    on one full frame of the workload: pathtrace + temporal + 3x a-trous + present."""
    import numpy as np

    import oracle
    n, W, H = WORKLOAD["n"], WORKLOAD["W"], WORKLOAD["H"]
    b, m = oracle.build_bricks(vox, n)
    u = frame_uniforms(vrt, spawn, 0)
    acc = np.zeros((H, W, 4), np.uint16)
    g = np.zeros((H, W, 4), np.float32)
    t0 = time.perf_counter()
    r = oracle.frame(vox, b, m, n, vrt.uniforms_bytes(u), WORKLOAD["fclamp"], W, H, acc, g)
    dt = time.perf_counter() - t0
    rays = r["stats"]["rays"]
    return {"value": round(rays / dt / 1e6, 3), "unit": "Mrays/s", "cores": oracle.num_threads(), "kind": "port",
            "sample": f"1 full frame ({rays} rays) of the workload through the CPU oracle "
                      f"(pathtrace+temporal+3x a-trous+present), {dt:.2f} s",
            "frame_ms": round(dt * 1e3, 1)}


def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    import voxelrt_b200 as vrt
    from voxelrt_b200._lib import lib as vlib

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    n, W, H = WORKLOAD["n"], WORKLOAD["W"], WORKLOAD["H"]
    vox, spawn = vrt.generate_scene(WORKLOAD["kind"], n, WORKLOAD["seed"])
    ctx = vrt.Context(local)
    scene = vrt.Scene(ctx, vox, n)
    sess = vrt.Session(ctx, scene, W, H, firefly_clamp=WORKLOAD["fclamp"], accum_f32=False,
                       path_kernel=args.path_kernel)
    sess.set_timing(True)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=f"cuda:{local}")

    for i in range(args.warmup):
        sess.frame(frame_uniforms(vrt, spawn, i))
        sess.stats()
    ctx.synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    frame_ms, pt_ms, rays, dda_bytes, pixels, launches = [], [], 0, 0, 0, 0
    trace_ms, trace_launches, lane_steps, step_slots = 0.0, 0, 0, 0
    for i in range(args.steps):
        f = args.warmup + i
        u = frame_uniforms(vrt, spawn, f)
        flush.zero_()
        torch.cuda.synchronize()
        sess.frame(u)
        st = sess.stats()
        frame_ms.append(st.ms_total)
        pt_ms.append(st.ms_pathtrace)
        rays += st.rays
        dda_bytes += 4 * (st.dda_outer + st.dda_inner + st.voxel_reads)
        pixels += st.pixels
        launches += st.launches
        trace_ms += st.ms_trace
        trace_launches += st.trace_launches
        lane_steps += st.dda_outer + st.dda_inner
        step_slots += st.trace_step_slots
    ctx.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = sum(frame_ms)
    if dist:
        dist.barrier()
    total_ms_max, rays_all = reduce_over_ranks(dist, f"cuda:{local}", total_ms, rays)

    # ---- end to end through the C ABI: host uniforms in, LDR frame out ----
    ldr_host = torch.empty(W * H * 4, dtype=torch.uint8, pin_memory=True)
    e2e_rays, e2e_s = 0, 0.0
    for i in range(args.steps):
        u = frame_uniforms(vrt, spawn, args.warmup + args.steps + i)
        t0 = time.perf_counter()
        sess.frame(u)
        code = vlib.vrt_read_ldr(sess.h, ldr_host.data_ptr(), W * H * 4)
        e2e_s += time.perf_counter() - t0
        if code:
            raise RuntimeError(vlib.vrt_last_error_string().decode())
        e2e_rays += sess.stats().rays
    e2e_s, e2e_rays = reduce_over_ranks(dist, f"cuda:{local}", e2e_s, e2e_rays)

    peak, peak_kind = measured_peaks()
    if args.path_kernel == "wavefront" and trace_launches:
        # dominant kernel: the persistent queue tracer (one launch per wave)
        kernel, n_launch, kernel_ms = "k_wf_trace", trace_launches, trace_ms
        alg_bytes = dda_bytes
        alg_note = ("algorithmic bytes = 4*(brick words + mask words + voxel words read) per traced ray, "
                    "summed over the launch; duration from CUDA events around each launch")
    else:
        kernel, n_launch, kernel_ms = "k_pathtrace", args.steps, sum(pt_ms)
        alg_bytes = dda_bytes + ALG_BYTES_PER_PX * pixels
        alg_note = ("algorithmic bytes = 4*(brick words + mask words + voxel words read) per traced ray "
                    "+ 28 B/pixel written; duration from CUDA events around the launch")
    achieved = alg_bytes / (kernel_ms / 1e3) / 1e9
    traffic = profiled_traffic(kernel)
    line = {
        "metric": METRIC,
        "value": round(rays_all / (total_ms_max / 1e3) / 1e6, 2),
        "unit": "Mrays/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(total_ms_max / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded procedural voxel world and camera path)",
        "config": workload_config(),
        "impl_details": {"parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                         "path_kernel": args.path_kernel,
                         "timing": "CUDA events on the library's stream around its kernels, per frame"},
        "frame_ms": {"mean": round(statistics.mean(frame_ms), 4),
                     "p50": round(statistics.median(frame_ms), 4),
                     "p99": round(float(np.percentile(frame_ms, 99)), 4)},
        "pass_ms_mean": {"pathtrace": round(statistics.mean(pt_ms), 4),
                         "trace_kernels": round(trace_ms / args.steps, 4)},
        "rays_per_frame": round(rays / args.steps),
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": kernel, "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                     "traffic": traffic,
                     "algorithmic_bytes_per_launch": round(alg_bytes / n_launch),
                     "launch_ms_mean": round(kernel_ms / n_launch, 4), "launches": n_launch,
                     "warp_exec_efficiency": round(lane_steps / step_slots, 4) if step_slots else None,
                     "warp_exec_efficiency_note": "brick + voxel iterations of all rays over the tracer's lane "
                                                  "slots (32 x DDA steps per pass x warp passes), counted in the "
                                                  "kernel",
                     "l2": profiled_l2(kernel),
                     "note": alg_note + "; the DDA working set (2 MB masks, 64 MB voxels) is L2-resident, "
                             "so the kernel is issue-bound, not HBM-bound"},
        "e2e": {"value": round(e2e_rays / e2e_s / 1e6, 2), "unit": "Mrays/s", "h2d_bytes_per_step": 304,
                "d2h_bytes_per_step": W * H * 4,
                "note": "vrt_frame (uniform block from the host) + vrt_read_ldr into pinned host memory, "
                        "host wall clock per frame"},
    }
    if clk:
        line["clocks"] = clk
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_port(vox, spawn, vrt)
    sess.close()
    scene.close()
    ctx.close()
    if rank == 0 and world == 1 and not args.no_cache_compare:
        # the metric's second half: plain vs batched + cache at equal MSE
        import copy
        a2 = copy.copy(args)
        a2.steps = min(args.steps, 10)
        cc = cache_comparison(a2, local)
        line["plain_vs_batched_cache"] = cache_summary(cc)
        try:
            line["served_c5"] = served_summary(served_comparison(a2, local), cc)
        except Exception as e:   # the headline line must still print
            line["served_c5"] = {"error": str(e)[:300]}
        try:
            a4 = copy.copy(args)
            a4.steps, a4.warmup, a4.jobs = 5, 3, 64
            bl = batched_line(a4, local)
            line["batched_c3"] = {"metric": bl["metric"], "batched_mrays_s": bl["value"],
                                  "sequential_mrays_s": bl["sequential"]["value"],
                                  "speedup_vs_sequential": bl["speedup_vs_sequential"],
                                  "batch_frame_ms": bl["frame_ms"], "sequential_ms_per_step":
                                      bl["sequential"]["ms_per_step"], "pixels_per_step": bl["config"]["pixels_per_step"],
                                  "tuning": bl["config"]["tuning"], "details": "bench.py --mode batched"}
        except Exception as e:
            line["batched_c3"] = {"error": str(e)[:300]}
    if rank == 0 and world == 1 and not args.no_extras:
        # measured on the same box: the ReSTIR presets, `ours` on the reference's scenarios, the VoxelBench adapter
        import copy
        a3 = copy.copy(args)
        a3.steps, a3.warmup, a3.no_cpu_baseline, a3.runs = 10, 3, True, "gi,ours_b6_nodenoise"
        try:
            r = restir_line(a3, local)
            line["restir"] = {k: {"preset": v["preset"], "bounces": v["bounces"], "frame_ms": v["frame_ms_mean"],
                                  "rays_per_frame": v["rays_per_frame"]} for k, v in r["runs"].items()}
            line["restir"]["details"] = "bench.py --mode restir"
        except Exception as e:   # the headline line must still print
            line["restir"] = {"error": str(e)[:300]}
        try:
            rs = restir_scenes_line(a3, local)
            line["restir_reference_scenarios"] = {
                k: {"frame_ms_p50": v["frame_ms_p50"], "reference_published_ms": v["reference_published_ms"]}
                for k, v in rs["scenarios"].items()}
            line["restir_reference_scenarios"]["details"] = "bench.py --mode restir-scenes"
        except Exception as e:
            line["restir_reference_scenarios"] = {"error": str(e)[:300]}
        try:
            v = voxelbench_line(a3, local, 10, 32)
            line["voxelbench"] = {sc: {"vrt_ms": x["vrt_ms"], "pt_ms": x["pt_ms"], "psnr_pt_vrt": x["psnr"]}
                                  for sc, x in v.get("scenes", {}).items()} or v
            if v.get("scenes"):
                line["voxelbench"]["details"] = "bench.py --mode voxelbench"
        except Exception as e:
            line["voxelbench"] = {"error": str(e)[:300]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args, world, rank):
    """The reference's own CPU traversal (VoxelBench/pipeline/core.cpp:52-130
    `trace`, compiled from the reference sources into oracle/_ref at the
    host's ISA level) replaying every ray of each frame of this workload
    (primary, bounce, sun shadow; collected untimed by the CPU oracle) on all
    host cores.  The WGSL path has no CPU implementation in the reference, and
    its traversal is the frame's dominant step; shading, temporal, denoise
    and present are not part of the timed region, so the arm's rays/s is an
    upper bound for a CPU frame.  The process loads only oracle libraries:
    the world, camera path and uniforms are the oracle's restatements.  The
    CPU oracle's full path stands in when the traversal library is absent."""
    if rank != 0:
        return
    import ctypes as C

    import numpy as np

    import oracle
    n, W, H = WORKLOAD["n"], WORKLOAD["W"], WORKLOAD["H"]
    vox, spawn = oracle.generate_scene(WORKLOAD["kind"], n, WORKLOAD["seed"])

    def uni(f):
        k = f % WORKLOAD["path_frames"]
        pose = oracle.camera_spline(spawn, k)
        prev = oracle.camera_spline(spawn, k - 1) if k > 0 else None
        return oracle.uniforms(pose, prev, f, WORKLOAD["bounces"], WORKLOAD["flags"], W, H, 1.0,
                               WORKLOAD["maxhist"])

    threads = os.cpu_count() or 1
    vb, vb_build = oracle.ref_lib_best()
    base = {"impl": "reference", "metric": METRIC, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural voxel world and camera path)", "config": workload_config()}
    b, m = oracle.build_bricks(vox, n)
    if vb is not None:
        occ = (vox != 0).astype(np.uint8)
        assert vb.vb_set_grid(n, n, n, C.c_void_p(occ.ctypes.data)) == 0
        per_step = []
        nrays = 0
        for i in range(args.warmup + args.steps):
            rays = oracle.collect_rays(vox, b, m, n, uni(i), WORKLOAD["fclamp"], W, H)
            o = np.ascontiguousarray(rays[:, 0:3])
            d = np.ascontiguousarray(rays[:, 3:6])
            t = np.ascontiguousarray(rays[:, 6])
            secs = vb.vb_time_trace(C.c_void_p(o.ctypes.data), C.c_void_p(d.ctypes.data), C.c_void_p(t.ctypes.data),
                                    C.c_int(len(o)), C.c_int(threads))
            if i >= args.warmup:
                per_step.append(secs)
                nrays += len(o)
        secs = sum(per_step)
        value = nrays / secs / 1e6
        sample = (f"VoxelBench trace() (4^3 brickmap DDA, core.cpp:52-130; built {vb_build}) on the workload's "
                  f"occupancy grid, replaying every ray of each frame ({nrays // args.steps} rays per step); "
                  f"the frame's shading, temporal, denoise and present are not timed")
        kind = "reference"
    else:
        per_step = []
        nrays = 0
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            r = oracle.pathtrace(vox, b, m, n, uni(i), WORKLOAD["fclamp"], W, H, i % 8, H, 8)
            if i >= args.warmup:
                per_step.append(time.perf_counter() - t0)
                nrays += r["stats"]["rays"]
        secs = sum(per_step)
        value = nrays / secs / 1e6
        sample = "CPU oracle path trace of every 8th row per step (reference traversal library not built)"
        kind = "port"
    line = dict(base)
    line.update({"value": round(value, 3), "ms_per_step": round(secs * 1e3 / args.steps, 3),
                 "impl_details": {"parallelism": f"host CPU, {threads} threads",
                                  "timing": "host wall clock around the traversal of each step's rays"},
                 "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s", "cores": threads, "kind": kind,
                                  "sample": sample},
                 "e2e": {"value": round(value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": 0}})
    print(json.dumps(line), flush=True)


def batched_jobs(n_jobs: int, seed: int = 3):
    """Seeded mixed workload: grid from {64,128,256,512}^3 (random worlds with
    0.1% emissive voxels of intensity U(1,20); 4 worlds per grid size),
    resolution log-uniform 320x180 .. 2560x1440, bounces U{1..6}, camera at a
    seeded pose inside its grid."""
    import random
    rnd = random.Random(seed)
    jobs = []
    for j in range(n_jobs):
        n = rnd.choice([64, 128, 256, 512])
        s = 2.0 ** rnd.uniform(0.0, 3.0)
        w, h = max(8, round(320 * s)), max(8, round(180 * s))
        jobs.append(dict(n=n, world=rnd.randrange(4), w=w, h=h, bounces=rnd.randint(1, 6),
                         yaw=rnd.uniform(0, 6.283), frame0=rnd.randrange(1 << 20)))
    return jobs


def run_batched(args, local):
    print(json.dumps(batched_line(args, local)), flush=True)


def batched_line(args, local):
    """64 independent jobs rendered (a) in one batch frame (one launch
    sequence, CUDA graph, autotuned launch shape) and (b) as 64 sequential
    plain frames, one session after another.  Device time from CUDA events;
    L2 flushed before every timed batch frame / sequential round."""
    import numpy as np
    import torch

    import voxelrt_b200 as vrt
    torch.cuda.set_device(local)
    ctx = vrt.Context(local)
    jobs = batched_jobs(args.jobs)
    worlds = {}
    for jb in jobs:
        key = (jb["n"], jb["world"])
        if key not in worlds:
            vox, spawn = vrt.generate_scene(vrt.VRT_SCENE_RANDOM, jb["n"], 1000 * jb["n"] + jb["world"])
            worlds[key] = (vrt.Scene(ctx, vox, jb["n"]), spawn)
            del vox
    light = vrt.Lighting()
    alone, inb, poses = [], [], []
    for jb in jobs:
        sc, spawn = worlds[(jb["n"], jb["world"])]
        alone.append(vrt.Session(ctx, sc, jb["w"], jb["h"], firefly_clamp=10.0))
        inb.append(vrt.Session(ctx, sc, jb["w"], jb["h"], firefly_clamp=10.0, path_kernel="batch_only"))
        poses.append(vrt.CameraPose(spawn.pos, jb["yaw"], spawn.pitch, spawn.fov_y))
    batch = vrt.Batch(ctx, inb)
    pixels = sum(jb["w"] * jb["h"] for jb in jobs)

    def uniforms(f):
        return [vrt.make_uniforms(poses[i], None, light, jobs[i]["frame0"] + f, jobs[i]["bounces"], 3,
                                  jobs[i]["w"], jobs[i]["h"]) for i in range(len(jobs))]

    t0 = time.perf_counter()
    tune, tune_ms = batch.autotune(uniforms(0), frames=1)
    tune_s = time.perf_counter() - t0
    for s in alone:
        s.set_tuning(*tune)
        s.set_timing(True)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=f"cuda:{local}")
    for f in range(args.warmup):
        u = uniforms(f)
        batch.frame(u)
        batch.stats()
        for i, s in enumerate(alone):
            s.frame(u[i])
    b_ms, b_rays, s_ms, s_rays = [], 0, [], 0
    for f in range(args.steps):
        u = uniforms(args.warmup + f)
        flush.zero_()
        torch.cuda.synchronize()
        batch.frame(u)
        st = batch.stats()
        b_ms.append(st.ms_total)
        b_rays += st.rays
        flush.zero_()
        torch.cuda.synchronize()
        tot = 0.0
        for i, s in enumerate(alone):
            s.frame(u[i])
            stj = s.stats()
            tot += stj.ms_total
            s_rays += stj.rays
        s_ms.append(tot)
    b_val = b_rays / (sum(b_ms) / 1e3) / 1e6
    s_val = s_rays / (sum(s_ms) / 1e3) / 1e6
    line = {
        "metric": "aggregate Mrays/s of 64 mixed render jobs: one batched launch vs 64 sequential plain launches",
        "mode": "batched", "value": round(b_val, 2), "unit": "Mrays/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(statistics.mean(b_ms), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded random voxel worlds, poses, sizes, bounce counts)",
        "config": {"workload": "64 jobs: grids {64,128,256,512}^3 (0.1% emissive, I~U(1,20)), "
                               "log-uniform 320x180..2560x1440, bounces U{1..6}, 1 spp, temporal+a-trous+present",
                   "jobs": len(jobs), "pixels_per_step": pixels, "worlds": len(worlds),
                   "graph": True, "tuning": dict(zip(["refill_min", "trace_blocks_per_sm", "shade_blocks_per_sm",
                                                      "trace_variant", "atrous_tile_rows", "tail_wave"], tune)),
                   "autotune_s": round(tune_s, 2),
                   "l2": "flushed before every timed batch frame and every sequential round"},
        "sequential": {"value": round(s_val, 2), "unit": "Mrays/s", "ms_per_step": round(statistics.mean(s_ms), 3)},
        "speedup_vs_sequential": round(b_val / s_val, 3),
        "rays_per_step": round(b_rays / args.steps),
        "frame_ms": {"p50": round(statistics.median(b_ms), 3), "p99": round(float(np.percentile(b_ms, 99)), 3)},
        "gpu_launches_per_step": batch.stats().launches,
    }
    batch.close()
    for s in alone + inb:
        s.close()
    for sc, _ in worlds.values():
        sc.close()
    ctx.close()
    return line


CACHE_SCENES = [
    # (label, scene kind, grid, seed, width, height, reference image)
    ("64^3 test scene (Cornell room on terrain, seed 1)", 1, 64, 1, 256, 144, "cache_reference_64_256x144.npz"),
    ("256^3 world (seed 2)", 2, 256, 2, 480, 270, "cache_reference_256_480x270.npz"),
]
CACHE_CFG = dict(train_bounces=6, train_vertices=3, train_batch=65536, train_steps=1, learning_rate=1e-2, seed=1)


def cache_quality(vrt, ctx, scene, spawn, W, H, ref, bounces, cache, warm, K):
    """MSE against the FP64 reference of K consecutive 1-spp frames (static
    camera at the spawn pose) after `warm` frames: the mean per-frame MSE,
    the MSE of the K-frame average, and the implied per-frame variance and
    squared bias (MSE_K = bias^2 + var / K)."""
    import numpy as np

    from voxelrt_b200.quality import hdr_image, mse
    s = vrt.Session(ctx, scene, W, H, firefly_clamp=10.0, keep_radiance_f32=True)
    if cache:
        s.set_cache(**cache)
    light = vrt.Lighting()
    for f in range(warm):
        s.pathtrace(vrt.make_uniforms(spawn, None, light, f, bounces, 0, W, H))
        s.end_frame()
    per, acc = [], np.zeros_like(ref)
    for f in range(warm, warm + K):
        s.pathtrace(vrt.make_uniforms(spawn, None, light, f, bounces, 0, W, H))
        s.end_frame()
        img = hdr_image(s)
        per.append(mse(img, ref))
        acc += img
    s.close()
    m1, mk = float(np.mean(per)), mse(acc / K, ref)
    var = max(m1 - mk, 0.0) * K / (K - 1)
    return {"mse_1spp": round(m1, 6), f"mse_{K}frame_mean": round(mk, 6), "var": round(var, 6),
            "bias2": round(mk - var / K, 7)}


def run_wave_sweep(args, local):
    """The bench frame (1080p / 256^3 / 2 bounces) at each refill threshold
    (4, 8, 12, 16, 24, 32 idle lanes) and then each tracer variant (0, 1, 2,
    3, 7), five frames per setting in that order: a command for per-wave launch
    lists (`ncu --metrics gpu__time_duration.sum -k regex:k_wf_trace`); the
    images do not depend on the settings."""
    import torch

    import voxelrt_b200 as vrt
    torch.cuda.set_device(local)
    n, W, H = WORKLOAD["n"], WORKLOAD["W"], WORKLOAD["H"]
    vox, spawn = vrt.generate_scene(WORKLOAD["kind"], n, WORKLOAD["seed"])
    ctx = vrt.Context(local)
    sc = vrt.Scene(ctx, vox, n)
    s = vrt.Session(ctx, sc, W, H, firefly_clamp=WORKLOAD["fclamp"])
    settings = [dict(refill_min=r) for r in (4, 8, 12, 16, 24, 32)] + [dict(trace_variant=v) for v in (0, 1, 2, 3, 7)]
    for st in settings:
        s.set_tuning(**st)
        for i in range(5):
            s.frame(frame_uniforms(vrt, spawn, 10 + i))
        ctx.synchronize()
    print(json.dumps({"mode": "wave-sweep", "settings": settings, "frames_per_setting": 5}), flush=True)
    s.close()
    sc.close()
    ctx.close()


def run_cache_frame(args, local):
    """The cache-assisted 1080p frame of the 256^3 world alone (static spawn
    camera): `warmup` training frames, then `steps` timed frames.  A small
    command for profiling the cache kernels."""
    import numpy as np
    import torch

    import voxelrt_b200 as vrt
    torch.cuda.set_device(local)
    ctx = vrt.Context(local)
    vox, spawn = vrt.generate_scene(2, 256, 2)
    sc = vrt.Scene(ctx, vox, 256)
    W, H = 1920, 1080
    s = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0)
    s.set_cache(**CACHE_CFG)
    s.set_timing(True)
    light = vrt.Lighting()
    for f in range(max(args.warmup, 3)):
        s.frame(vrt.make_uniforms(spawn, None, light, f, 2, 3, W, H, 1.0, 64.0))
    rows = []
    for f in range(args.steps):
        s.frame(vrt.make_uniforms(spawn, None, light, args.warmup + f, 2, 3, W, H, 1.0, 64.0))
        st = s.stats()
        rows.append((st.ms_total, st.ms_pathtrace, st.ms_cache, st.rays, st.cache_queries, st.cache_samples,
                     st.launches))
    a = np.array(rows, np.float64)
    print(json.dumps({"mode": "cache-frame", "frame_ms": round(float(a[:, 0].mean()), 4),
                      "pathtrace_ms": round(float(a[:, 1].mean()), 4), "cache_ms": round(float(a[:, 2].mean()), 4),
                      "rays": int(a[:, 3].mean()), "queries": int(a[:, 4].mean()), "samples": int(a[:, 5].mean()),
                      "launches": int(a[:, 6].mean())}), flush=True)
    s.close()
    sc.close()
    ctx.close()


def served_views(vrt, ctx, sc, spawn, flush, args, K, warm_train, views=16):
    """`views` sessions of one scene at 480x270 (the reference image's view,
    each with its own frame-index stream): batched with a cache per view
    (quality + time), batched plain, and plain views one after another."""
    import numpy as np
    import torch

    from voxelrt_b200.quality import hdr_image, mse
    W, H = 480, 270
    ref = np.load(ROOT / "tests" / "golden" / "cache_reference_256_480x270.npz")["ref"].astype(np.float64)
    light = vrt.Lighting()

    def uni(i, f, b, flags):
        return vrt.make_uniforms(spawn, None, light, 100000 * i + f, b, flags, W, H, 1.0, 64.0)

    out = {"views": views, "resolution": f"{W}x{H}"}
    # batched with caches: quality (pass-level calls, no temporal) then timing (full frames)
    ss = [vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, keep_radiance_f32=True, path_kernel="batch_only")
          for _ in range(views)]
    for i, s in enumerate(ss):
        s.set_cache(**dict(CACHE_CFG, seed=i + 1))
    batch = vrt.Batch(ctx, ss)
    for f in range(warm_train):
        batch.frame([uni(i, f, 2, 0) for i in range(views)])
    acc = [np.zeros_like(ref) for _ in range(views)]
    for f in range(warm_train, warm_train + K):
        batch.frame([uni(i, f, 2, 0) for i in range(views)])
        for i, s in enumerate(ss):
            acc[i] += hdr_image(s)
    m = [mse(a / K, ref) for a in acc]

    def time_batch(b, bounces, f0):
        ms = []
        for f in range(f0, f0 + args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            b.frame([uni(i, f, bounces, 3) for i in range(views)])
            ms.append(b.stats().ms_total)
        return float(np.mean(ms))

    ms_c = time_batch(batch, 2, warm_train + K)
    out["batched_cache"] = {"mse_64frame_mean": round(float(np.mean(m)), 6), "mse_spread": [round(min(m), 6), round(max(m), 6)],
                            "ms_per_batch": round(ms_c, 4), "views_per_s": round(views * 1e3 / ms_c, 1)}
    batch.close()
    for s in ss:
        s.close()
    # batched plain 2-bounce
    ss = [vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, path_kernel="batch_only") for _ in range(views)]
    batch = vrt.Batch(ctx, ss)
    for f in range(max(args.warmup, 3)):
        batch.frame([uni(i, f, 2, 3) for i in range(views)])
    ms_p = time_batch(batch, 2, 100)
    out["batched_plain_2bounce"] = {"ms_per_batch": round(ms_p, 4), "views_per_s": round(views * 1e3 / ms_p, 1)}
    batch.close()
    for s in ss:
        s.close()
    # plain views one after another
    for b in (2, 6):
        ss = [vrt.Session(ctx, sc, W, H, firefly_clamp=10.0) for _ in range(views)]
        for s in ss:
            s.set_timing(True)
        for f in range(max(args.warmup, 3)):
            for i, s in enumerate(ss):
                s.frame(uni(i, f, b, 3))
        tot, pt = [], []
        for f in range(100, 100 + args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t_all, p_all = 0.0, 0.0
            for i, s in enumerate(ss):
                s.frame(uni(i, f, b, 3))
                st = s.stats()
                t_all += st.ms_total
                p_all += st.ms_pathtrace
            tot.append(t_all)
            pt.append(p_all)
        out[f"sequential_plain_{b}bounce"] = {"ms_per_view": round(float(np.mean(tot)) / views, 4),
                                              "pathtrace_ms_per_view": round(float(np.mean(pt)) / views, 4),
                                              "views_per_s": round(views * 1e3 / float(np.mean(tot)), 1)}
        for s in ss:
            s.close()
    return out


def run_cache(args, local):
    """`--mode cache`: prints cache_comparison's full result."""
    print(json.dumps(cache_comparison(args, local)), flush=True)


def quality_1080p(vrt, ctx, sc, spawn, forms, K, warm_train, ref_spp=4096):
    """MSE of each form at the full workload size (1920x1080, 256^3 world,
    static spawn camera) against a 4096-spp plain 6-bounce reference
    accumulated in FP64 on the GPU (vrt_hdr_accumulate: bit-identical to the
    CPU oracle's FP64 accumulation, tests/test_hdr.py).  Errors are summed on
    the device."""
    W, H = 1920, 1080
    light = vrt.Lighting()
    r = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, keep_radiance_f32=True)
    t0 = time.perf_counter()
    r.hdr_accum_reset()
    r.hdr_accumulate(vrt.make_uniforms(spawn, None, light, 0, 6, 0, W, H), 1 << 20, ref_spp)
    ref, count = r.hdr_accum()
    ref_s = time.perf_counter() - t0
    r.close()
    ref32 = ref.astype("float32")
    out = {"resolution": f"{W}x{H}", "reference": {"spp": count, "bounces": 6, "seconds": round(ref_s, 2)}}
    for name, b, c in forms:
        s = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0, keep_radiance_f32=True)
        if c:
            s.set_cache(**c)
        s.set_hdr_reference(ref32)
        w = warm_train if c else 0
        for f in range(w):
            s.pathtrace(vrt.make_uniforms(spawn, None, light, f, b, 0, W, H))
            s.end_frame()
        s.hdr_accum_reset()
        per = []
        for f in range(w, w + K):
            s.pathtrace(vrt.make_uniforms(spawn, None, light, f, b, 0, W, H))
            s.end_frame()
            per.append(s.hdr_frame_mse())
            s.hdr_accum_add()
        m1, mk = sum(per) / K, s.hdr_accum_mse()
        var = max(m1 - mk, 0.0) * K / (K - 1)
        out[name] = {"mse_1spp": round(m1, 6), f"mse_{K}frame_mean": round(mk, 6), "var": round(var, 6),
                     "bias2": round(mk - var / K, 7)}
        s.close()
    return out


def cache_summary(c):
    """The headline figures of cache_comparison for the default bench line."""
    q1 = c["quality"]["256^3 world (seed 2), 1920x1080, GPU FP64 reference"]
    sv = c["served_16_views"]
    return {
        "metric": "frames/s at matched MSE (64-frame accumulation vs a 4096-spp FP64 plain 6-bounce reference), "
                  "cache-assisted over plain; 1080p quality against a GPU-accumulated reference",
        "mse_64frame_256world_1080p": {k: q1[k]["mse_64frame_mean"] for k in ("plain_2bounce", "plain_6bounce",
                                                                               "cache")},
        "single_1080p": {"fps": {k: c["speed_1080p"][k]["fps"] for k in c["speed_1080p"]},
                         "speedup_at_matched_mse": {k: v.get("cache_speedup") for k, v in
                                                    c["matched_mse_64frame"].items()}},
        "served_16_views_batched": {"views_per_s": sv["batched_cache"]["views_per_s"],
                                    "mse_64frame": sv["batched_cache"]["mse_64frame_mean"],
                                    "speedup_at_matched_mse_vs_views_one_after_another": {
                                        k: sv["matched_" + k].get("batched_cache_speedup")
                                        for k in ("plain_2bounce", "plain_6bounce")}},
        "details": "bench.py --mode cache",
    }


def served_summary(sc, cc):
    """The serving block of the default line: each form's capacity and
    latency, its 64-frame MSE against the 4096-spp FP64 reference (the 1080p
    statistics of the same estimators), and the cache-assisted served form
    against the plain form, raw and at matched MSE (the plain form at the
    samples per frame that reach the cache form's MSE)."""
    f = sc["forms"]
    q = cc["quality"]["256^3 world (seed 2), 1920x1080, GPU FP64 reference"]
    sp, m = cc["speed_1080p"]["plain_2bounce"], cc["matched_mse_64frame"]["plain_2bounce"]
    cost = (m["frame_ms_at_matched_mse"] / sp["frame_ms"]) if m.get("frame_ms_at_matched_mse") else None
    seq = f["plain_sequential"]["capacity"]["frames_per_s"]
    best = max((k for k in f if k.startswith("cache_")), key=lambda k: f[k]["capacity"]["frames_per_s"])
    cb = f[best]["capacity"]["frames_per_s"]
    out = {"metric": "served frames/s (capacity, queue never empty) and p50/p99 latency under Poisson arrivals; "
                     "cache-assisted continuous batching vs the plain form (requests one after another, unbatched)",
           "sessions": sc["sessions"], "session_pixels": sc["session_pixels"],
           "mse_64frame_vs_4096spp": {"plain": q["plain_2bounce"]["mse_64frame_mean"],
                                      "cache": q["cache"]["mse_64frame_mean"]},
           "forms": {k: {"frames_per_s": v["capacity"]["frames_per_s"],
                         "latency_ms": {str(int(r["rate_rps"])): [r["latency_ms_p50"], r["latency_ms_p99"]]
                                        for r in v["poisson"]}} for k, v in f.items()},
           "served_form": best,
           "forms_note": f"sequential: one request per launch through the session's own frame path; batched: "
                         f"continuous batching of every request; hybrid: continuous batching of views below "
                         f"{sc['solo_pixels']} pixels, larger views alone; every form serves the same request "
                         f"stream (sessions, edits, arrival times, camera paths)",
           "speedup_cache_served_vs_plain_sequential": round(cb / seq, 3),
           "speedup_plain_batched_vs_plain_sequential": round(f["plain_batched"]["capacity"]["frames_per_s"] / seq, 3),
           "speedup_plain_hybrid_vs_plain_sequential": round(f["plain_hybrid"]["capacity"]["frames_per_s"] / seq, 3),
           "plain_cost_factor_at_matched_mse": round(cost, 3) if cost else None,
           "speedup_at_matched_mse": round(cb / seq * cost, 3) if cost else None,
           "latency_note": "latency_ms: rate (req/s) -> [p50, p99]",
           "details": "bench.py --mode serve"}
    return out


def cache_comparison(args, local):
    """Cache-assisted path tracing against plain 2- and 6-bounce tracing.

    Quality: MSE against 4096-spp FP64 plain 6-bounce references -- the
    committed CPU-oracle fixtures of two scenes at small sizes, and the 256^3
    world at 1920x1080 against a reference accumulated on the GPU.  Speed:
    full frames (trace + temporal + 3x a-trous + present) of the 256^3 world
    at 1920x1080 from its spawn pose, after the cache trained on the preceding
    frames.  Matched MSE: the MSE of a 64-frame accumulation (the temporal
    history cap) of the cache form; the plain form needs
    s* = var / (64 (MSE_cache - bias^2)) samples per frame to reach it, i.e.
    s* times its path-tracing pass per frame."""
    import numpy as np
    import torch

    import voxelrt_b200 as vrt
    torch.cuda.set_device(local)
    ctx = vrt.Context(local)
    K, WARM_TRAIN = 64, 256
    forms = [("plain_2bounce", 2, None), ("plain_6bounce", 6, None), ("cache", 2, CACHE_CFG)]
    quality = {}
    for label, kind, n, seed, W, H, refname in CACHE_SCENES:
        ref = np.load(ROOT / "tests" / "golden" / refname)["ref"].astype(np.float64)
        vox, spawn = vrt.generate_scene(kind, n, seed)
        sc = vrt.Scene(ctx, vox, n)
        quality[label] = {name: cache_quality(vrt, ctx, sc, spawn, W, H, ref, b, c, WARM_TRAIN if c else 0, K)
                          for name, b, c in forms}
        quality[label]["resolution"] = f"{W}x{H}"
        sc.close()
    # speed at 1080p on the 256^3 world
    W, H = 1920, 1080
    vox, spawn = vrt.generate_scene(2, 256, 2)
    sc = vrt.Scene(ctx, vox, 256)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=f"cuda:{local}")
    light = vrt.Lighting()
    speed = {}
    for name, b, c in forms:
        s = vrt.Session(ctx, sc, W, H, firefly_clamp=10.0)
        if c:
            s.set_cache(**c)
        s.set_timing(True)
        warm = max(args.warmup, 3) + (64 if c else 0)
        for f in range(warm):
            s.frame(vrt.make_uniforms(spawn, None, light, f, b, 3, W, H, 1.0, 64.0))
        rows = []
        for f in range(warm, warm + args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            s.frame(vrt.make_uniforms(spawn, None, light, f, b, 3, W, H, 1.0, 64.0))
            st = s.stats()
            rows.append((st.ms_total, st.ms_pathtrace, st.ms_cache, st.rays, st.launches, st.cache_queries,
                         st.cache_samples))
        a = np.array(rows, np.float64)
        speed[name] = {"frame_ms": round(float(a[:, 0].mean()), 4), "frame_ms_p50": round(float(np.median(a[:, 0])), 4),
                       "frame_ms_p99": round(float(np.percentile(a[:, 0], 99)), 4),
                       "pathtrace_ms": round(float(a[:, 1].mean()), 4), "cache_ms": round(float(a[:, 2].mean()), 4),
                       "fps": round(1e3 / float(a[:, 0].mean()), 1), "rays_per_frame": round(float(a[:, 3].mean())),
                       "mrays_s": round(float(a[:, 3].sum()) / (float(a[:, 0].sum()) / 1e3) / 1e6, 1),
                       "launches_per_frame": round(float(a[:, 4].mean()), 1)}
        if c:
            speed[name]["queries_per_frame"] = round(float(a[:, 5].mean()))
            speed[name]["training_samples_per_frame"] = round(float(a[:, 6].mean()))
        s.close()
    q1080 = quality_1080p(vrt, ctx, sc, spawn, forms, K, WARM_TRAIN)
    # served form: 16 views of the 256^3 world at the reference's 480x270, one
    # batch frame for all of them, each view with its own cache; against the
    # same views rendered one after another by plain sessions
    served = served_views(vrt, ctx, sc, spawn, flush, args, K, WARM_TRAIN)
    sc.close()
    ctx.close()
    # matched MSE at 1080p: quality and speed of the same view at the same size
    quality["256^3 world (seed 2), 1920x1080, GPU FP64 reference"] = q1080
    q = q1080
    target = q["cache"][f"mse_{K}frame_mean"]
    matched = {}
    for name in ("plain_2bounce", "plain_6bounce"):
        var, bias2 = q[name]["var"], q[name]["bias2"]
        sp = speed[name]
        if target <= bias2:
            matched[name] = {"spp_needed": None, "note": "the plain form's bias alone exceeds the cache form's MSE"}
            continue
        s_star = max(1.0, var / (K * (target - bias2)))
        ms = s_star * sp["pathtrace_ms"] + (sp["frame_ms"] - sp["pathtrace_ms"])
        matched[name] = {"spp_needed": round(s_star, 3), "frame_ms_at_matched_mse": round(ms, 4),
                         "cache_speedup": round(ms / speed["cache"]["frame_ms"], 3)}
    # served form at matched MSE: plain views one after another at s* spp
    # (the 480x270 views' own statistics)
    sv = served
    q480 = quality[CACHE_SCENES[1][0]]
    target_b = sv["batched_cache"]["mse_64frame_mean"]
    for name in ("plain_2bounce", "plain_6bounce"):
        var, bias2 = q480[name]["var"], q480[name]["bias2"]
        seq = sv["sequential_" + name]
        if target_b <= bias2:
            sv["matched_" + name] = {"spp_needed": None}
            continue
        s_star = max(1.0, var / (K * (target_b - bias2)))
        per_view = s_star * seq["pathtrace_ms_per_view"] + (seq["ms_per_view"] - seq["pathtrace_ms_per_view"])
        sv["matched_" + name] = {"spp_needed": round(s_star, 3), "ms_per_view": round(per_view, 4),
                                 "views_per_s": round(1e3 / per_view, 1),
                                 "batched_cache_speedup": round(sv["batched_cache"]["views_per_s"] * per_view / 1e3, 3)}
    line = {
        "metric": "1080p frames/s of cache-assisted vs plain path tracing at matched MSE (FP64 4096-spp reference)",
        "mode": "cache", "value": speed["cache"]["fps"], "unit": "frames/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": speed["cache"]["frame_ms"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 path tracing; bf16 MLP with f32 accumulation",
        "data": "synthetic (seeded procedural voxel worlds, static spawn camera)",
        "config": {"workload": "256^3 world seed 2, 1920x1080, 1 spp, full frame (trace + temporal + 3x a-trous "
                               "+ present), static spawn camera; quality on two scenes at the stated resolutions",
                   "cache": CACHE_CFG, "quality_frames": K, "cache_training_frames_before_quality": WARM_TRAIN,
                   "reference": "plain 6-bounce path, 4096 spp, FP64 accumulation (tests/golden)",
                   "l2": "flushed before every timed frame (256 MB write), outside the timed events"},
        "quality": quality, "speed_1080p": speed, "matched_mse_64frame": matched, "served_16_views": sv,
    }
    return line


def run_lights(args, local):
    """Scene light structures (emissive-face list, power alias table, top-16
    per-brick light grid; scene.js builds them once on the CPU) rebuilt on the
    GPU after an edit, against the CPU restatement on all host cores."""
    import numpy as np
    import torch

    import oracle
    import voxelrt_b200 as vrt
    torch.cuda.set_device(local)
    ctx = vrt.Context(local)
    rows = []
    for label, kind, n, seed, extra in (("256^3 world (lanterns)", 2, 256, 2, 0),
                                        ("256^3 world + 5000 emissive surface voxels", 2, 256, 2, 5000)):
        vox, _ = vrt.generate_scene(kind, n, seed)
        if extra:
            # seeded emissive voxels on solid voxels with air above (visible surfaces)
            v3 = vox.reshape(n, n, n)
            top = (v3[:, :-1, :] != 0) & (v3[:, 1:, :] == 0)
            zz, yy, xx = np.nonzero(top)
            pick = np.random.default_rng(11).choice(len(zz), extra, replace=False)
            e = np.random.default_rng(12).integers(11, 213, extra).astype(np.uint32)   # I ~ U(1, 20)
            v3[zz[pick], yy[pick], xx[pick]] = (v3[zz[pick], yy[pick], xx[pick]] & 0x00FFFFFF) | (e << 24)
            vox = v3.ravel()
        sc = vrt.Scene(ctx, vox, n)
        sc.build_lights()                          # warm-up (allocations)
        ms = []
        for k in range(max(args.steps, 3)):
            sc.edit_box(8 * k, 8, 8, 8 * k + 15, 23, 23, 0)   # remove a box, then rebuild
            t0 = time.perf_counter()
            st = sc.build_lights()
            ms.append((time.perf_counter() - t0) * 1e3)
        v, _, _ = sc.read()
        t0 = time.perf_counter()
        ow, owt = oracle.light_list(v, n)
        oracle.light_alias(owt)
        oracle.light_grid(n, ow, owt)
        cpu_ms = (time.perf_counter() - t0) * 1e3
        rows.append({"scene": label, "lights": int(st.count), "gpu_ms_wall": round(float(np.median(ms)), 2),
                     "gpu_ms_list": round(st.ms_list, 3), "host_ms_alias": round(st.ms_alias, 3),
                     "gpu_ms_grid": round(st.ms_grid, 3), "cpu_ms": round(cpu_ms, 1),
                     "cpu_threads": oracle.num_threads(), "speedup": round(cpu_ms / float(np.median(ms)), 1)})
        sc.close()
    ctx.close()
    print(json.dumps({"metric": "scene light structures rebuilt after an edit (ms)", "mode": "lights",
                      "value": rows[-1]["gpu_ms_wall"], "unit": "ms", "higher_is_better": False, "n_gpus": 1,
                      "data": "synthetic (seeded procedural worlds)", "rows": rows}), flush=True)


SERVE_RES = [((640, 360), 0.40), ((1280, 720), 0.35), ((1920, 1080), 0.20), ((2560, 1440), 0.05)]
SERVE_MIN_BATCH = 1    # batched forms: fewer sessions waiting than this render one request at a time
# (measured on the serving mix with the cache: 1 / 4 / 8 / 16 -> 930 / 931 / 926 / 912 frames/s, so none)


def run_serve(args, local):
    """Poisson arrivals of frame requests over 32 device-resident sessions
    (resolution mix 360p 40% / 720p 35% / 1080p 20% / 1440p 5%, grids 128^3 or
    256^3, each request carrying one seeded voxel-box edit of 1-4096 voxels),
    admitted by a 150 GB HBM budget, served by continuous batching.  Latency =
    device completion - arrival on the server clock."""
    import numpy as np
    import torch

    import voxelrt_b200 as vrt
    torch.cuda.set_device(local)
    rng = np.random.default_rng(5)
    ctx = vrt.Context(local, hbm_budget_bytes=150 * (1 << 30))
    sessions, scenes, spawns, meta = [], [], [], []
    for k in range(32):
        n = 128 if rng.random() < 0.5 else 256
        (w, h), = [SERVE_RES[int(rng.choice(4, p=[p for _, p in SERVE_RES]))][0]]
        vox, spawn = vrt.generate_scene(vrt.VRT_SCENE_FULL, n, 100 + k)
        try:
            sc = vrt.Scene(ctx, vox, n)
            s = vrt.Session(ctx, sc, w, h, firefly_clamp=10.0, path_kernel="batch_only")
        except vrt.VrtError as e:      # admission refused by the budget
            if e.code != 5:
                raise
            break
        scenes.append(sc)
        sessions.append(s)
        spawns.append(spawn)
        meta.append((n, w, h))
    server = vrt.Server(ctx, sessions, max_in_flight=2)
    light = vrt.Lighting()
    frames = [0] * len(sessions)

    def make_request(k):
        n, w, h = meta[k]
        f = frames[k]
        frames[k] += 1
        pose = vrt.camera_spline(spawns[k], f % 120)
        prev = vrt.camera_spline(spawns[k], (f - 1) % 120) if f % 120 else None
        u = vrt.make_uniforms(pose, prev, light, f, 2, 3, w, h)
        size = rng.integers(1, 17, 3)
        lo = rng.integers(0, n - 16, 3)
        val = 0 if rng.random() < 0.5 else int(rng.integers(1, 1 << 24))
        return u, [(int(lo[0]), int(lo[1]), int(lo[2]), int(lo[0] + size[0] - 1), int(lo[1] + size[1] - 1),
                    int(lo[2] + size[2] - 1), val)]

    def warm(rounds):
        for _ in range(rounds):
            for k in range(len(sessions)):
                u, e = make_request(k)
                server.submit(k, u, e)
            server.drain()

    warm(1)
    results = sweep(args, server, sessions, make_request, rng)
    forms = {"plain": results}
    if args.cache:
        # the same sessions switched to the cache-assisted path (one network each),
        # trained on 32 frames per session before the sweep
        for k, s in enumerate(sessions):
            s.set_cache(**dict(CACHE_CFG, seed=k + 1))
        warm(32)
        forms["cache"] = sweep(args, server, sessions, make_request, rng)
    px = sum(w * h for _, w, h in meta)
    line = {
        "metric": "served frames/s and p50/p99 frame latency under Poisson arrivals"
                  + (" (plain and cache-assisted path)" if args.cache else " (plain path)"),
        "mode": "serve", "value": max(r["frames_per_s"] for r in forms["cache" if args.cache else "plain"]),
        "unit": "frames/s", "n_gpus": 1,
        "higher_is_better": True, "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded worlds, cameras, edits, arrival times)",
        "config": {"workload": "32 sessions, 360p 40% / 720p 35% / 1080p 20% / 1440p 5%, grids {128,256}^3, "
                               "2 bounces, temporal+a-trous+present, one 1-4096 voxel box edit per request",
                   "sessions": len(sessions), "session_pixels": px, "hbm_budget_gb": 150,
                   "hbm_in_use_gb": round(ctx.bytes_in_use / 2 ** 30, 2), "max_in_flight": 2,
                   "duration_s_per_rate": args.duration,
                   "cache": CACHE_CFG if args.cache else None,
                   "quality": "per-view MSE of both forms: bench.py --mode cache (FP64 4096-spp references)"},
        "rates": results,
    }
    if args.cache:
        line["forms"] = forms
    print(json.dumps(line), flush=True)
    server.close()
    for s_ in sessions:
        s_.close()
    for sc in scenes:
        sc.close()
    ctx.close()
    line["churn"] = churn_line(args, local)
    print(json.dumps({"mode": "serve-churn", **line["churn"]}), flush=True)


def serve_mix(vrt, ctx, rng, path_kernel="batch_only", count=32):
    """The serving workload's sessions: grids 128^3 or 256^3 (seeded benchmark
    worlds), resolutions 360p 40% / 720p 35% / 1080p 20% / 1440p 5%, each
    session with its own scene (its requests edit it); stops at the first
    session the context's HBM budget refuses."""
    sessions, scenes, spawns, meta = [], [], [], []
    for k in range(count):
        n = 128 if rng.random() < 0.5 else 256
        (w, h), = [SERVE_RES[int(rng.choice(4, p=[p for _, p in SERVE_RES]))][0]]
        vox, spawn = vrt.generate_scene(vrt.VRT_SCENE_FULL, n, 100 + k)
        try:
            sc = vrt.Scene(ctx, vox, n)
            s = vrt.Session(ctx, sc, w, h, firefly_clamp=10.0, path_kernel=path_kernel)
        except vrt.VrtError as e:      # admission refused by the budget
            if e.code != 5:
                raise
            break
        scenes.append(sc)
        sessions.append(s)
        spawns.append(spawn)
        meta.append((n, w, h))
    return sessions, scenes, spawns, meta


def serve_requests(vrt, rng, spawns, meta, frames):
    """make_request(k): the next frame of session k on its camera path with one
    seeded voxel-box edit of 1..16^3 voxels (carve or fill)."""
    light = vrt.Lighting()

    def make_request(k):
        n, w, h = meta[k]
        f = frames[k]
        frames[k] += 1
        pose = vrt.camera_spline(spawns[k], f % 120)
        prev = vrt.camera_spline(spawns[k], (f - 1) % 120) if f % 120 else None
        u = vrt.make_uniforms(pose, prev, light, f, 2, 3, w, h)
        size = rng.integers(1, 17, 3)
        lo = rng.integers(0, n - 16, 3)
        val = 0 if rng.random() < 0.5 else int(rng.integers(1, 1 << 24))
        return u, [(int(lo[0]), int(lo[1]), int(lo[2]), int(lo[0] + size[0] - 1), int(lo[1] + size[1] - 1),
                    int(lo[2] + size[2] - 1), val)]
    return make_request


def capacity(server, n_sessions, make_request, rng, n_req):
    """Frames/s with the queue never empty: n_req requests (uniform over the
    sessions) submitted at once, served to completion; device completion
    times on the server clock."""
    import numpy as np
    t0 = server.now()
    for _ in range(n_req):
        k = int(rng.integers(0, n_sessions))
        u, e = make_request(k)
        server.submit(k, u, e, t_arrival=t0)
    done = server.drain()
    t_end = max(td for *_, td in done)
    lat = np.array([(td - ta) * 1e3 for _, _, ta, td in done])
    return {"requests": n_req, "frames_per_s": round(n_req / (t_end - t0), 1),
            "mean_frame_ms": round((t_end - t0) * 1e3 / n_req, 4), "queue_drain_ms_p99": round(float(np.percentile(lat, 99)), 2)}


def served_comparison(args, local, rates=(200.0, 500.0), duration=1.0, n_sat=320):
    """The serving mix (32 sessions, edits between frames) served six ways
    over the same device-resident sessions: `plain_sequential`, the plain
    form -- requests one after another through each session's own frame path,
    unbatched; `plain_batched` -- continuous batching of every request;
    `plain_hybrid` -- continuous batching of views below 720p, larger views
    alone; `cache_sequential`, `cache_batched` and `cache_hybrid` -- the same
    with each session's radiance cache (trained on 32 frames per session
    first).  Per form: capacity (the queue never empty) and p50/p99 latency
    under Poisson arrivals at each rate."""
    import numpy as np
    import torch

    import voxelrt_b200 as vrt
    torch.cuda.set_device(local)
    rng = np.random.default_rng(5)
    ctx = vrt.Context(local, hbm_budget_bytes=150 * (1 << 30))
    sessions, scenes, spawns, meta = serve_mix(vrt, ctx, rng, path_kernel="wavefront")
    server = vrt.Server(ctx, sessions, max_in_flight=2)
    frames = [0] * len(sessions)
    make_request = serve_requests(vrt, rng, spawns, meta, frames)
    a2 = argparse.Namespace(**vars(args))
    a2.rates, a2.duration = ",".join(str(r) for r in rates), duration

    def warm(rounds):
        for _ in range(rounds):
            for k in range(len(sessions)):
                u, e = make_request(k)
                server.submit(k, u, e)
            server.drain()

    out = {}
    solo = 1280 * 720      # views of 720p and up fill the GPU alone; smaller ones are batched
    for form in ("plain_sequential", "plain_batched", "plain_hybrid", "cache_sequential", "cache_batched",
                 "cache_hybrid"):
        server.set_sequential(form.endswith("sequential"))
        server.set_solo_pixels(solo if form.endswith("hybrid") else 0)
        server.set_min_batch(SERVE_MIN_BATCH if not form.endswith("sequential") else 1)
        if form == "cache_sequential":
            for k, s in enumerate(sessions):
                s.set_cache(**dict(CACHE_CFG, seed=k + 1))
            warm(32)
        else:
            warm(1)
        # every form serves the same request stream: sessions, edits and arrival times from the same seeds,
        # each session's camera path from the same frame on
        rq = np.random.default_rng(77)
        mr = serve_requests(vrt, rq, spawns, meta, [1000] * len(sessions))
        out[form] = {"capacity": capacity(server, len(sessions), mr, rq, n_sat),
                     "poisson": sweep(a2, server, sessions, mr, np.random.default_rng(78))}
    out["solo_pixels"] = solo
    px = sum(w * h for _, w, h in meta)
    server.close()
    for s_ in sessions:
        s_.close()
    for sc in scenes:
        sc.close()
    ctx.close()
    solo = out.pop("solo_pixels")
    return {"sessions": len(sessions), "session_pixels": px, "forms": out, "solo_pixels": solo}


def churn_line(args, local, slots=32, close_p=0.02):
    """Serving with sessions that come and go: a dynamic server with 32
    session slots and a launch pool for 32 sessions of the largest size, under
    the 150 GB HBM budget.  Sessions open through the admission queue; after
    each request its session closes with probability close_p and a new session
    (new world, resolution from the mix) asks for admission, waiting until a
    slot and memory free up -- the old session's requests drain first.
    Poisson arrivals over the open sessions at each rate."""
    import numpy as np
    import torch

    import voxelrt_b200 as vrt
    torch.cuda.set_device(local)
    rng = np.random.default_rng(11)
    ctx = vrt.Context(local, hbm_budget_bytes=150 * (1 << 30))
    max_px = SERVE_RES[-1][0][0] * SERVE_RES[-1][0][1]
    server = vrt.Server(ctx, None, max_in_flight=2, max_sessions=slots, max_pixels=slots * max_px)
    light = vrt.Lighting()
    state = {}            # slot -> dict(n, w, h, spawn, frame)
    waiting = {}          # ticket -> (t_open, n, w, h, spawn)
    scenes = []
    opened = [0]
    waits = []

    def open_one():
        k = opened[0]
        opened[0] += 1
        n = 128 if rng.random() < 0.5 else 256
        (w, h), = [SERVE_RES[int(rng.choice(4, p=[p_ for _, p_ in SERVE_RES]))][0]]
        vox, spawn = vrt.generate_scene(vrt.VRT_SCENE_FULL, n, 500 + k)
        sc = vrt.Scene(ctx, vox, n)
        scenes.append(sc)
        t = server.open_session(sc, w, h, firefly_clamp=10.0)
        waiting[t] = (server.now(), n, w, h, spawn)

    def admit():
        for t in list(waiting):
            slot = server.session_of(t)
            if slot is None:
                continue
            t0, n, w, h, spawn = waiting.pop(t)
            waits.append((server.now() - t0) * 1e3)
            state[slot] = dict(n=n, w=w, h=h, spawn=spawn, frame=0)

    def request(slot):
        st = state[slot]
        f = st["frame"]
        st["frame"] += 1
        pose = vrt.camera_spline(st["spawn"], f % 120)
        prev = vrt.camera_spline(st["spawn"], (f - 1) % 120) if f % 120 else None
        u = vrt.make_uniforms(pose, prev, light, f, 2, 3, st["w"], st["h"])
        n = st["n"]
        size = rng.integers(1, 17, 3)
        lo = rng.integers(0, n - 16, 3)
        val = 0 if rng.random() < 0.5 else int(rng.integers(1, 1 << 24))
        return u, [(int(lo[0]), int(lo[1]), int(lo[2]), int(lo[0] + size[0] - 1), int(lo[1] + size[1] - 1),
                    int(lo[2] + size[2] - 1), val)]

    for _ in range(slots):
        open_one()
    admit()
    results = []
    closes = 0
    for rate in [float(x) for x in args.rates.split(",")]:
        n_req = max(1, int(rate * args.duration))
        gaps = rng.exponential(1.0 / rate, n_req)
        t_start = server.now() + 0.01
        arrivals = t_start + np.cumsum(gaps)
        done, i = [], 0
        while i < n_req:
            now = server.now()
            while i < n_req and arrivals[i] <= now:
                admit()
                slot = int(rng.choice(list(state)))
                u, e = request(slot)
                server.submit(slot, u, e, t_arrival=float(arrivals[i]))
                i += 1
                if rng.random() < close_p and len(state) > 1:
                    server.close_session(slot)
                    del state[slot]
                    closes += 1
                    open_one()
            done += server.poll()
            admit()
            if i < n_req and arrivals[i] > server.now():
                time.sleep(min(2e-4, max(0.0, arrivals[i] - server.now())))
        done += server.drain()
        admit()
        lat = np.array([(td - ta) * 1e3 for _, _, ta, td in done])
        t_end = max(td for *_, td in done)
        results.append({"rate_rps": rate, "requests": n_req, "frames_per_s": round(n_req / (t_end - t_start), 1),
                        "latency_ms_p50": round(float(np.percentile(lat, 50)), 3),
                        "latency_ms_p99": round(float(np.percentile(lat, 99)), 3)})
    open_, wait_ = server.session_counts()
    out = {"rates": results, "sessions_opened": opened[0], "sessions_closed": closes, "open_at_end": open_,
           "waiting_at_end": wait_,
           "admission_wait_ms": {"p50": round(float(np.percentile(waits, 50)), 3) if waits else None,
                                  "p99": round(float(np.percentile(waits, 99)), 3) if waits else None,
                                  "admitted": len(waits)},
           "hbm_in_use_gb": round(ctx.bytes_in_use / 2 ** 30, 2),
           "note": "dynamic server: a session closes after a request with probability 0.02 and a new one waits "
                   "in the admission queue for a slot and memory (150 GB budget)"}
    server.close()
    for sc in scenes:
        sc.close()
    ctx.close()
    return out


def sweep(args, server, sessions, make_request, rng):
    """One run of Poisson arrivals per rate; latency = device completion -
    arrival on the server clock."""
    import numpy as np
    results = []
    for rate in [float(x) for x in args.rates.split(",")]:
        n_req = max(1, int(rate * args.duration))
        gaps = rng.exponential(1.0 / rate, n_req)
        reqs = [(int(rng.integers(0, len(sessions))),) for _ in range(n_req)]
        done = []
        t_start = server.now() + 0.01
        arrivals = t_start + np.cumsum(gaps)
        i = 0
        while i < n_req:
            now = server.now()
            while i < n_req and arrivals[i] <= now:
                k = reqs[i][0]
                u, e = make_request(k)
                server.submit(k, u, e, t_arrival=float(arrivals[i]))
                i += 1
            done += server.poll()
            if i < n_req and arrivals[i] > server.now():
                time.sleep(min(2e-4, max(0.0, arrivals[i] - server.now())))
        done += server.drain()
        lat = np.array([(td - ta) * 1e3 for _, _, ta, td in done])
        t_end = max(td for *_, td in done)
        results.append({"rate_rps": rate, "requests": n_req, "frames_per_s": round(n_req / (t_end - t_start), 1),
                        "latency_ms_p50": round(float(np.percentile(lat, 50)), 3),
                        "latency_ms_p99": round(float(np.percentile(lat, 99)), 3),
                        "latency_ms_mean": round(float(lat.mean()), 3)})
    return results


RESTIR_RUNS = [   # (label, preset, bounces, params0.z flags: bit0 temporal, bit1 denoise)
    ("plain", "base", 2, 3),
    ("gi", "gi", 2, 3),
    ("ours", "ours", 2, 3),
    ("ours_b6_nodenoise", "ours", 6, 1),
]


def run_restir(args, local):
    print(json.dumps(restir_line(args, local)), flush=True)


def restir_line(args, local):
    """`--mode restir`: the reference's ReSTIR presets -- `gi` (RF_RESTIR |
    RF_TEMPORAL | RF_SPATIAL) and its default `ours` (paired reuse, duplication
    map, vector weights, unified light-list NEE with power sampling, plane,
    rescue, full visibility, clamp) -- on the full-size workload, timed like
    the plain frame, with the plain frame measured beside them.  `value` is
    `ours` at 6 bounces with the denoiser off, the configuration of the
    reference's published GPU timings (docs/STATUS.md:79-81, RTX 3080)."""
    import numpy as np
    import torch

    import voxelrt_b200 as vrt

    torch.cuda.set_device(local)
    n, W, H = WORKLOAD["n"], WORKLOAD["W"], WORKLOAD["H"]
    vox, spawn = vrt.generate_scene(WORKLOAD["kind"], n, WORKLOAD["seed"])
    ctx = vrt.Context(local)
    scene = vrt.Scene(ctx, vox, n)
    nlights = int(scene.build_lights().count)
    sess = vrt.Session(ctx, scene, W, H, firefly_clamp=WORKLOAD["fclamp"], accum_f32=False,
                       path_kernel=args.path_kernel)
    sess.set_timing(True)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=f"cuda:{local}")

    def uni(f, preset, bounces, flags):
        k = f % WORKLOAD["path_frames"]
        pose = vrt.camera_spline(spawn, k)
        prev = vrt.camera_spline(spawn, k - 1) if k > 0 else None
        return vrt.make_uniforms(pose, prev, vrt.Lighting(), f, bounces, flags, W, H, 1.0, WORKLOAD["maxhist"],
                                 preset=preset, light_count=nlights)

    res, clk = {}, None
    runs = [r for r in RESTIR_RUNS if not args.runs or r[0] in args.runs.split(",")]
    for label, preset, bounces, flags in runs:
        sess.reset()
        for i in range(args.warmup):
            sess.frame(uni(i, preset, bounces, flags))
            sess.stats()
        ctx.synchronize()
        clocks = ClockSampler(local)
        clocks.start()
        fm, pt, ru, rays, launches = [], [], [], 0, 0
        for i in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            sess.frame(uni(args.warmup + i, preset, bounces, flags))
            st = sess.stats()
            fm.append(st.ms_total)
            pt.append(st.ms_pathtrace)
            ru.append(st.ms_reuse)
            rays += st.rays
            launches += st.launches
        ctx.synchronize()
        c = clocks.stop()
        if label == runs[-1][0]:
            clk = c
        res[label] = {"preset": preset, "bounces": bounces, "denoise": bool(flags & 2),
                      "frame_ms_mean": round(statistics.mean(fm), 4), "frame_ms_p50": round(statistics.median(fm), 4),
                      "frame_ms_p99": round(float(np.percentile(fm, 99)), 4),
                      "pathtrace_ms_mean": round(statistics.mean(pt), 4),
                      "reuse_ms_mean": round(statistics.mean(ru), 4),
                      "rays_per_frame": round(rays / args.steps), "launches": launches,
                      "mrays_s": round(rays / (sum(fm) / 1e3) / 1e6, 2)}
    sess.close()
    scene.close()
    ctx.close()
    head = res[runs[-1][0]]
    line = {
        "metric": "ReSTIR `ours` frame ms at 1080p, 6 bounces, denoiser off (initial + reuse + temporal + present)",
        "value": head["frame_ms_mean"], "unit": "ms/frame", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["frame_ms_mean"], "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded procedural voxel world and camera path)",
        "config": {"workload": "ReSTIR presets on " + WORKLOAD_NAME, "lights": nlights, "taps": 3, "radius_px": 30,
                   "ccap": 20, "pairing_sigma": 16, "path_kernel": args.path_kernel,
                   "l2": "flushed before every timed frame (256 MB write), outside the timed events"},
        "runs": res,
        "reference_published_ms": {"ours_b6_nodenoise_1080p_rtx3080_webgpu": {
            "exterior": 22.56, "lamps": 33.31, "interior": 33.96,
            "note": "other hardware and scenes (docs/STATUS.md:79-81); context, not a like-for-like ratio"}},
        "gpu_launches": head["launches"],
    }
    if clk:
        line["clocks"] = clk
    if not args.no_cpu_baseline:
        import oracle
        b, m = oracle.build_bricks(vox, n)
        u = uni(0, "gi", 2, 3)
        t0 = time.perf_counter()
        r = oracle.frame(vox, b, m, n, vrt.uniforms_bytes(u), WORKLOAD["fclamp"], W, H,
                         np.zeros((H, W, 4), np.uint16), np.zeros((H, W, 4), np.float32))
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": round(dt * 1e3, 1), "unit": "ms/frame", "cores": oracle.num_threads(),
                                "kind": "port", "rays": r["stats"]["rays"],
                                "sample": "1 full ReSTIR gi frame (2 bounces) of the workload through the CPU oracle"}
    return line


# The scenarios of the reference's published `ours` timings
# (test/eval/claim-manifest.v1.json: poses in metres / radians; the moving runs
# strafe along x by sin(0.07 frame) * 0.6 m, main.js:687-691; capture 1920x1080,
# 6 bounces, denoiser off, firefly clamp 0, rgba32f history) on the reference's
# world (scene.js generateScene(256, 'default' or 'lamps'), noise seed 1337).
REF_SCENARIOS = {
    "exterior": {"pos": (8.0, 4.9, 4.6), "yaw": 0.85, "pitch": -0.1, "world": 0, "published_ms": 22.56},
    "lamps": {"pos": (6.6, 4.9, 6.9), "yaw": 0.55, "pitch": 0.0, "world": 4, "published_ms": 33.31},
    "interior": {"pos": (8.8, 4.7, 7.0), "yaw": -0.45, "pitch": 0.02, "world": 0, "published_ms": 33.96},
}
REF_SCENARIO_FRAMES = 96
REF_SCENARIO_MOVE = (0.6, 0.07)


def run_restir_scenes(args, local):
    print(json.dumps(restir_scenes_line(args, local)), flush=True)


def restir_scenes_line(args, local):
    """`--mode restir-scenes`: the reference's `ours` preset on its own default
    world and the exterior / interior scenario poses, with the capture settings
    of its published GPU timings (docs/STATUS.md:75-81: median GPU ms of the
    96-frame moving runs, RTX 3080, Chromium WebGPU): 1920x1080, 6 bounces,
    denoiser off, firefly clamp 0, rgba32f history, the reference's sun and
    70-degree camera.  Frames 1..96 of the strafe are rendered; the first
    `--warmup` are untimed; the median and mean of the rest are reported."""
    import numpy as np
    import torch

    import voxelrt_b200 as vrt

    torch.cuda.set_device(local)
    n, W, H = 256, 1920, 1080
    ctx = vrt.Context(local)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=f"cuda:{local}")
    light = vrt.Lighting.reference_default()
    amp, step = REF_SCENARIO_MOVE

    def pose_at(sc, f):
        x, y, z = sc["pos"]
        return vrt.CameraPose((x + math.sin(f * step) * amp, y, z), sc["yaw"], sc["pitch"])

    out, clk, lights = {}, None, {}
    warm = max(args.warmup, 3)
    for name, sc in REF_SCENARIOS.items():
        vox, _ = vrt.generate_scene(sc["world"], n, 1337)
        scene = vrt.Scene(ctx, vox, n)
        nlights = int(scene.build_lights().count)
        lights[name] = nlights
        sess = vrt.Session(ctx, scene, W, H, firefly_clamp=0.0, accum_f32=True, path_kernel=args.path_kernel)
        sess.set_timing(True)
        fm, rays = [], 0
        clocks = None
        for f in range(REF_SCENARIO_FRAMES):
            if f == warm:
                ctx.synchronize()
                clocks = ClockSampler(local)
                clocks.start()
            u = vrt.make_uniforms(pose_at(sc, f), pose_at(sc, f - 1) if f > 0 else None, light, f, 6, 1, W, H,
                                  1.0, 64.0, preset="ours", light_count=nlights)
            flush.zero_()
            torch.cuda.synchronize()
            sess.frame(u)
            st = sess.stats()
            if f >= warm:
                fm.append(st.ms_total)
                rays += st.rays
        ctx.synchronize()
        c = clocks.stop() if clocks else None
        clk = c or clk
        sess.close()
        scene.close()
        out[name] = {"frame_ms_p50": round(statistics.median(fm), 4), "frame_ms_mean": round(statistics.mean(fm), 4),
                     "frame_ms_p99": round(float(np.percentile(fm, 99)), 4), "frames_timed": len(fm),
                     "rays_per_frame": round(rays / len(fm)),
                     "reference_published_ms": sc["published_ms"],
                     "ratio_published_over_ours": round(sc["published_ms"] / statistics.median(fm), 2)}
    ctx.close()
    line = {"mode": "restir-scenes", "metric": "ReSTIR `ours` median frame ms on the reference's scenarios "
            "(1920x1080, 6 bounces, denoiser off, fclamp 0)", "unit": "ms/frame", "higher_is_better": False,
            "lights": lights, "world": "scene.js world ('default', or 'lamps' for the lamps scenario), 256^3, "
                                        "noise seed 1337",
            "scenarios": out,
            "note": "the published numbers are an RTX 3080 in Chromium WebGPU (docs/STATUS.md:75-81); same scene, "
                    "pose, resolution, bounces and preset, different hardware and runtime."}
    if clk:
        line["clocks"] = clk
    return line


def correctness_line(args, local, configs=None):
    """`--mode correctness`: the reference's estimator-correctness gate
    (test/eval/correctness-manifest.v1.json; its record
    test/eval/estimator-correctness.v1.json read into
    tests/golden/estimator_correctness_rows.json) rendered by this library:
    per scenario a 1600-frame, 12-bounce plain reference capture and, per
    configuration, an 800-frame, 8-bounce test capture (1920x1080,
    maxhist=1e6, fclamp=0, denoiser off, fseed=0), each compared with the
    channel means the reference recorded for the same capture, and the HDR
    error between this library's two captures beside the reference's."""
    import numpy as np
    import torch

    import voxelrt_b200 as vrt
    from voxelrt_b200 import quality

    torch.cuda.set_device(local)
    rows = json.loads((ROOT / "tests" / "golden" / "estimator_correctness_rows.json").read_text())
    W, H = rows["resolution"]["width"], rows["resolution"]["height"]
    rf, rb = rows["reference"]["frames"], rows["reference"]["bounces"]
    configs = configs or list(rows["configurations"])
    ctx = vrt.Context(local)
    light = vrt.Lighting.reference_default()
    out, worst = [], 0.0
    t0 = time.perf_counter()
    for name, sc_def in rows["scenarios"].items():
        kind = vrt.VRT_SCENE_VOXELRT_LAMPS if sc_def["scene"] == "lamps" else vrt.VRT_SCENE_VOXELRT
        vox, _ = vrt.generate_scene(kind, 256, 1337)
        scene = vrt.Scene(ctx, vox, 256)
        nl = int(scene.build_lights().count)
        p = sc_def["pose"]
        pose = vrt.CameraPose((p["px"], p["py"], p["pz"]), p["yaw"], p["pitch"])
        sess = vrt.Session(ctx, scene, W, H, firefly_clamp=0.0, accum_f32=True)
        ref = quality.accumulated_capture(ctx, scene, pose, light, W, H, rf, rb, 0, nl, session=sess)
        for cfg in configs:
            row = next(r for r in rows["rows"] if r["scenario"] == name and r["config"] == cfg)
            test = quality.accumulated_capture(ctx, scene, pose, light, W, H, row["frames"], row["bounces"],
                                               quality.config_flags(cfg), nl, session=sess)
            m = quality.hdr_metrics(ref, test)
            dref = [abs(a - b) / abs(b) for a, b in zip(m["referenceMeanRgb"], row["referenceMeanRgb"])]
            dtest = [abs(a - b) / abs(b) for a, b in zip(m["testMeanRgb"], row["testMeanRgb"])]
            worst = max(worst, max(dref), max(dtest))
            out.append({"scenario": name, "config": cfg,
                        "reference_mean_rgb": [round(v, 5) for v in m["referenceMeanRgb"]],
                        "reference_mean_rgb_recorded": [round(v, 5) for v in row["referenceMeanRgb"]],
                        "reference_mean_max_rel_delta": float(f"{max(dref):.3e}"),
                        "test_mean_rgb": [round(v, 5) for v in m["testMeanRgb"]],
                        "test_mean_rgb_recorded": [round(v, 5) for v in row["testMeanRgb"]],
                        "test_mean_max_rel_delta": float(f"{max(dtest):.3e}"),
                        "hdr_mse": round(m["hdrMse"], 5), "hdr_mse_recorded": round(row["hdrMse"], 5),
                        "hdr_psnr_peak_db": round(m["hdrPsnrPeak"], 2),
                        "hdr_psnr_peak_db_recorded": round(row["hdrPsnrPeak"], 2)})
        sess.close()
        scene.close()
    ctx.close()
    return {"mode": "correctness", "metric": "channel-mean relative delta vs the reference's recorded captures "
            "(gate: 1%) and HDR MSE test-vs-reference beside the recorded one",
            "resolution": [W, H], "reference_capture": {"frames": rf, "bounces": rb},
            "max_channel_mean_rel_delta": float(f"{worst:.3e}"), "pass": worst <= rows["thresholds"][
                "maxChannelMeanRelativeDelta"], "rows": out, "seconds": round(time.perf_counter() - t0, 1)}


VB_SCENES = ["bunker", "cavern", "courtyard", "town"]
VB_PUBLISHED_PT_MS = {"bunker": 115.7, "cavern": 123.5, "courtyard": 36.4, "town": 34.6}


def run_voxelbench(args, local):
    print(json.dumps(voxelbench_line(args, local, max(args.steps, 5), 64)), flush=True)


def voxelbench_line(args, local, frames, ref_spp):
    """`--mode voxelbench`: the VoxelBench harness protocol (240x135, ray budget
    4*W*H per frame, the reference's scenes and metrics) with the library's
    Technique adapter MethodVRT on the GPU beside the reference's own baseline
    MethodPT on the CPU (the harness's 2 OpenMP threads), same estimator and
    budget.  Runs oracle/_ref/vb_vrt (built from the reference sources)."""
    import oracle

    if not oracle.VB_VRT.exists():
        return {"mode": "voxelbench", "unavailable": "oracle/_ref/vb_vrt not built (needs the reference sources "
                "at build time)"}
    out = {}
    for sc in VB_SCENES:
        r = subprocess.run([str(oracle.VB_VRT), sc, "1.0", str(frames), str(ref_spp), "1"], capture_output=True, text=True,
                           timeout=1800, env={**os.environ, "CUDA_VISIBLE_DEVICES": os.environ.get(
                               "CUDA_VISIBLE_DEVICES", str(local))})
        if r.returncode != 0:
            raise RuntimeError(f"vb_vrt {sc}: {r.stderr[-2000:]}")
        rows = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
        summ = {x["summary"]: x for x in rows if "summary" in x}
        ref = [x for x in rows if "reference" in x][0]
        vrt_ms = [x["ms"] for x in rows if x.get("method") == "VRT"][1:]   # the first frame uploads
        out[sc] = {"vrt_ms": round(statistics.mean(vrt_ms), 4), "pt_ms": round(summ["PT"]["mean_ms"], 2),
                   "speedup": round(summ["PT"]["mean_ms"] / statistics.mean(vrt_ms), 1),
                   "rays_per_frame": round(summ["VRT"]["rays_per_frame"]),
                   "psnr": [summ["PT"]["psnr"], summ["VRT"]["psnr"]], "ssim": [summ["PT"]["ssim"], summ["VRT"]["ssim"]],
                   "gpsnr": [summ["PT"]["gpsnr"], summ["VRT"]["gpsnr"]],
                   "mean_luma": [summ["PT"]["mean_luma"], summ["VRT"]["mean_luma"], ref["mean_luma"]],
                   "published_pt_ms_author_cpu": VB_PUBLISHED_PT_MS[sc]}
    line = {
        "metric": "VoxelBench PT@1.0x frame ms (240x135, budget 4*W*H rays): MethodVRT (GPU) vs the reference MethodPT",
        "value": round(statistics.mean(v["vrt_ms"] for v in out.values()), 4), "unit": "ms/frame", "n_gpus": 1,
        "steps": frames, "warmup": 1, "ms_per_step": round(statistics.mean(v["vrt_ms"] for v in out.values()), 4),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "the reference's procedural VoxelBench scenes (pre-event state)",
        "config": {"workload": "VoxelBench harness run protocol, 4 scenes", "frames": frames, "ref_spp": ref_spp,
                   "pt_threads": 1, "note": "host wall clock per Technique::frame (upload of the G-buffer excluded "
                   "after the first frame); quality pairs are [PT, VRT] against the same reference"},
        "scenes": out,
    }
    return line


def main():
    args = parse_args()
    world, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, world, rank)
    elif args.mode == "batched":
        if rank == 0:
            run_batched(args, local)
    elif args.mode == "serve":
        if rank == 0:
            run_serve(args, local)
    elif args.mode == "cache":
        if rank == 0:
            run_cache(args, local)
    elif args.mode == "cache-frame":
        if rank == 0:
            run_cache_frame(args, local)
    elif args.mode == "wave-sweep":
        if rank == 0:
            run_wave_sweep(args, local)
    elif args.mode == "lights":
        if rank == 0:
            run_lights(args, local)
    elif args.mode == "restir":
        if rank == 0:
            run_restir(args, local)
    elif args.mode == "restir-scenes":
        if rank == 0:
            run_restir_scenes(args, local)
    elif args.mode == "voxelbench":
        if rank == 0:
            run_voxelbench(args, local)
    elif args.mode == "correctness":
        if rank == 0:
            print(json.dumps(correctness_line(args, local)), flush=True)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
