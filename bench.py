"""Benchmark of the strand software-raster path on B200.

One step = one frame of the seeded "medium" plain-pipeline workload (100,000
strands x 32 points = 3.1 M segments, 1920x1080 camera orbiting 360 degrees over
200 frames, one directional light with a 2048^2 x 8-layer deep-opacity map):
prepass -> deep shadow + stampback -> shading -> raster -> composite, replayed
from one CUDA graph per frame.

Prints one JSON line. `value` is whole-job segments/s with the scene resident in
HBM; `e2e` is the same metric through fiber_render_host with the scene image
copied in from pinned host memory and the composited RGBA16F frame copied back
every step. `--impl reference` times the CPU restatement of the reference path
(the reference itself is Rust + WGSL over wgpu and cannot run here) on every
host thread. With torchrun (N > 1) every rank renders its own frames: replicas,
weak scaling, no collective on the data path.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "segments/s & frames/s at 1080p; served p50/p99 latency vs plain loop, 1 B200"
UNIT = "segments/s"


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=30)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="fiber", choices=["fiber", "reference"])
    p.add_argument("--workload", default="medium")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--profile", action="store_true",
                   help="render warmup + steps frames only (no timing extras); the command profiled under ncu")
    p.add_argument("--no-served", action="store_true", help="skip the served-mode measurement")
    p.add_argument("--served-rate", type=float, default=200.0, help="Poisson arrival rate, requests/s")
    p.add_argument("--served-seconds", type=float, default=5.0, help="length of the 200 req/s arrival stream")
    p.add_argument("--served-sustain-seconds", type=float, default=20.0,
                   help="length of the stream at 80%% of the plain loop's throughput (p50/p99 of service)")
    p.add_argument("--served-saturate", type=int, default=256, help="requests submitted at once for throughput")
    p.add_argument("--no-batched", action="store_true", help="skip the batched-mode measurement")
    p.add_argument("--binning-backend", default="segment", choices=["segment", "page-csr"],
                   help="FineBinningBackend: segment-owned scatter (default) or the page CSR")
    p.add_argument("--dom-page-pool", type=int, default=0,
                   help="sparse deep-opacity residency in this many 256^2 pages (0: dense layers)")
    p.add_argument("--batched-views", type=int, default=64, help="independent views in one batch launch")
    return p.parse_args()


# ---------------------------------------------------------------------------
# Clock sampling during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# Scene setup shared by the arms
# ---------------------------------------------------------------------------
def make_scene(name: str):
    from bevy_strand_rasterizer_b200.plugin import FroxelConfig, StrandMaterial, pack_strand_set
    from bevy_strand_rasterizer_b200.scene import LightSpec, scalp_hair, workload
    w = workload(name)
    strands = scalp_hair(w.strands, w.points, w.seed, curly=w.curly)
    packed = pack_strand_set(strands)
    cam_cfg = FroxelConfig(w.width, w.height, w.froxel, w.froxel, w.depth_slices)
    lights = [(FroxelConfig(w.dom_size, w.dom_size, w.froxel, w.froxel, w.depth_slices), LightSpec(d, size=w.dom_size))
              for d in w.lights]
    return w, packed, StrandMaterial(), cam_cfg, lights


def frame_structs(w, packed, frame, lights):
    from bevy_strand_rasterizer_b200 import abi
    spec = w.camera(frame)
    cam = abi.Camera()
    cam.clip_from_world[:] = [float(x) for x in spec.clip_from_world()]
    cam.world_position[:] = [float(x) for x in spec.eye]
    lc = (abi.Light * max(1, len(lights)))()
    for i, (_, ls) in enumerate(lights):
        lc[i].clip_from_world[:] = [float(x) for x in ls.clip_from_world(packed.aabb_min, packed.aabb_max)]
        lc[i].direction_to_light[:] = [float(x) for x in ls.direction()]
        lc[i].color[:] = [float(x) for x in ls.color4()]
    return cam, lc


def algorithmic_bytes(st, w, n_lights: int, K: int, D: int) -> dict:
    """B_alg of the frame and of each kernel, from the frame's own counts.

    Per unit: 20 B / point + 16 B / strand (vertex float4 + index, meta), 28 B per
    binning task written and read (BinningTask 16 + ProjectedSegment 12), 8 B per
    allocated cell (count + offset), 24 B per fine ref (written + read), 12 B per
    binning task of cell-order key + material (written by k_visit), per visit
    (counted as fine refs): 8 B record written by k_visit, 16 B read/written by
    k_count_visits (record, rank, count), 20 B by k_fill_visits (record, rank,
    task, offset read; task index written), 32 B by k_sort_cells (task index,
    12 B key + material gathered, 16 B reference + key written); 64 B per work
    item / tile run (written + read), 40 B per ref of endpoint gather in the
    rasters, 40 + 8 L B per camera segment in shading, 12 B per camera pixel
    (RGBA16F + R32F), 4 (K + 1) B per deep-opacity texel.
    """
    F = st.frustum_count
    P, S = st.total_points, st.total_strands
    tasks = [st.frustum_tasks[f] for f in range(F)]
    pages = [st.frustum_pages[f] for f in range(F)]
    refs = [st.frustum_refs[f] for f in range(F)]
    work = [st.frustum_work[f] for f in range(F)]
    runs = [st.frustum_runs[f] for f in range(F)]
    WH = w.width * w.height
    dom = n_lights * 4 * (K + 1) * D * D
    per = {
        "k_fine": 20 * P + 16 * S + sum(60 * n for n in tasks),  # + 32 B projected end points per task
        "k_visit": sum(40 * n for n in tasks) + sum(8 * r for r in refs),
        "k_count_visits": sum(16 * r for r in refs),
        "k_fill_visits": sum(20 * r for r in refs),
        "k_prefix_pages": sum(8 * 256 * p for p in pages),
        "k_emit+k_sort_cells": sum(32 * (wk + t) + 36 * r for wk, t, r in zip(work, runs, refs)),
        # the rasters stage a reference from its 12 B record, its task index
        # and the task's 32 B of projected end points
        "k_shadow": sum(48 * refs[f] + 32 * (work[f] + runs[f]) for f in range(1, F)) + dom,
        "k_shade": st.camera_tasks * (40 + 8 * n_lights),
        "k_raster": 48 * refs[0] + 32 * (work[0] + runs[0]) + 12 * WH,
    }
    # The frame's B_alg is the path's own formula (fixed before any kernel was
    # written); the per-kernel figures above add this implementation's records.
    total = (20 * P + 16 * S + sum(56 * n + 8 * 256 * p + 24 * r + 64 * (wk + t) + 40 * r
                                   for n, p, r, wk, t in zip(tasks, pages, refs, work, runs))
             + st.camera_tasks * (40 + 8 * n_lights) + 12 * WH + dom)
    b_min = 20 * P + 16 * S + 12 * WH + dom
    return {"per_kernel": per, "frame": total, "min": b_min}


# Kernels one fused frame launches: broad, lut, fine, visit, alloc, zero_pages,
# count_visits, traverse<count> (returns at once unless the visit records did
# not fit), prefix_pages, fill_visits, traverse<fill> (likewise),
# compact_active, emit, sort_cells, sort_big_cells, shadow, shade, raster,
# composite.
KERNELS_PER_FRAME = 19

SPAN_TO_KERNEL = {
    "strand_prepass/fine": "k_fine",
    "strand_prepass/mark_count_pages": "k_visit",
    "strand_prepass/binning": "k_count_visits",
    "strand_prepass/prefix_fine_pages": "k_prefix_pages",
    "strand_prepass/fill_segment_refs": "k_fill_visits",
    "strand_prepass/emit_raster_work": "k_emit+k_sort_cells",
    "strand_shadow_rasterizer/rasterize": "k_shadow",
    "strand_shading/shade": "k_shade",
    "strand_rasterizer/rasterize": "k_raster",
}


def load_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def load_traffic() -> dict:
    p = ROOT / "profiles" / "ncu_traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            return {}
    return {}


def bench_config(w, segs: int, n_lights: int, args, world: int) -> dict:
    """The workload both arms run (the same text, so the lines compare)."""
    return {"workload": f"{w.name}: {w.strands} strands x {w.points} points ({segs} segments), {w.width}x{w.height} "
                        f"camera orbiting over {w.orbit_frames} frames, {n_lights} light(s) with {w.dom_size}^2 x "
                        f"{w.dom_layers} deep-opacity maps",
            "tile_px": w.froxel, "parallelism": f"replicas x{world}",
            "l2": "per-frame working set (tasks, refs, pages, DOM) > 126 MB L2",
            "stochastic_cull": "on (reference default)", "ref_capacity_factor": w.ref_capacity_factor,
            "fine_binning_backend": args.binning_backend, "dom_page_pool": args.dom_page_pool}


# ---------------------------------------------------------------------------
# CPU arm (oracle restatement on the host cores)
# ---------------------------------------------------------------------------
def cpu_frame_time(w, packed, material, cam_cfg, lights, frame=0, max_strands=None):
    """Times one oracle frame on every host thread; returns (seconds, segments, sample text)."""
    sys.path.insert(0, str(ROOT / "tests"))
    from bevy_strand_rasterizer_b200 import abi
    from bevy_strand_rasterizer_b200.plugin import pack_indexed_strands
    from oracle_bridge import run_oracle
    sample = packed
    note = f"one full {w.name} frame"
    if max_strands and packed.strand_count > max_strands:
        n = max_strands
        meta = packed.meta[:n]
        end = int(meta["offset"][-1] + meta["count"][-1])
        sample = pack_indexed_strands(packed.vertices[:, :3], meta["count"], meta["offset"], packed.indices[:end])
        note = f"one {w.name} frame over the first {n} of {packed.strand_count} strands"
    cam, lc = frame_structs(w, packed, frame, lights)
    st = abi.default_settings()
    st.dom_slices = w.dom_layers
    st.ref_capacity_factor = w.ref_capacity_factor
    segs = int(np.maximum(sample.meta["count"].astype(np.int64) - 1, 0).sum())
    t0 = time.perf_counter()
    fr = run_oracle([(sample, material, np.eye(4, dtype=np.float32).reshape(16))], cam_cfg, cam,
                    [c for c, _ in lights], lc, st, threads=os.cpu_count() or 1)
    dt = time.perf_counter() - t0
    fr.free()
    return dt, segs, note


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w, packed, material, cam_cfg, lights = make_scene(args.workload)
    # Each step is one whole frame of the workload (the same strands, camera
    # orbit and light as the GPU arm), a few seconds of host work.
    for i in range(args.warmup):
        cpu_frame_time(w, packed, material, cam_cfg, lights, frame=i)
    times, segs, note = [], 0, ""
    for k in range(args.steps):
        dt, segs, note = cpu_frame_time(w, packed, material, cam_cfg, lights, frame=args.warmup + k)
        times.append(dt)
    total = sum(times)
    value = segs * args.steps / total
    cores = os.cpu_count() or 1
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": dict(bench_config(w, segs, len(lights), args, args.gpus), sample=note),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": note},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference is Rust + WGSL over wgpu/Vulkan with no CPU implementation; its CPU arm is the "
                "oracle restatement (oracle/fiber_ref.cpp) on every host thread",
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def fiber_arm(args):
    import torch
    import torch.distributed as dist
    from bevy_strand_rasterizer_b200 import abi, replicas
    from bevy_strand_rasterizer_b200.plugin import StrandRasterizerPlugin, image_from_tensor

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    w, packed, material, cam_cfg, lights = make_scene(args.workload)
    from bevy_strand_rasterizer_b200.plugin import FineBinningBackend
    backend = FineBinningBackend.PageCsr if args.binning_backend == "page-csr" else FineBinningBackend.SegmentScatter
    plugin = StrandRasterizerPlugin(device=local, dom_slices=w.dom_layers, ref_capacity_factor=w.ref_capacity_factor,
                                    backend=backend, dom_page_pool=args.dom_page_pool)
    plugin.add_geometry(packed, material)
    stream = torch.cuda.Stream()
    H, W = w.height, w.width
    scene = torch.empty((H, W, 4), dtype=torch.float16, device="cuda")
    scene[...] = torch.tensor([0.08, 0.09, 0.11, 1.0], dtype=torch.float16)
    out = torch.empty_like(scene)
    scene_img = image_from_tensor(scene, abi.FMT_RGBA16F)
    out_img = image_from_tensor(out, abi.FMT_RGBA16F)
    light_cfgs = [c for c, _ in lights]

    def step(k):
        cam, lc = frame_structs(w, packed, replicas.frame_index(rank, k), lights)
        plugin.frame_begin_raw(cam_cfg, cam, light_cfgs, lc, stream)
        # The scene is opaque (alpha 1), so the blend onto `out` does not
        # depend on what `out` held before.
        plugin.frame_fused(scene_img, None, out_img, stream)

    with torch.cuda.stream(stream):
        for i in range(args.warmup):
            step(i)
    stream.synchronize()
    st = plugin.stats()
    if args.profile:
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                step(args.warmup + k)
        stream.synchronize()
        print(json.dumps({"profile": w.name, "frames": args.warmup + args.steps, "tasks": st.binning_tasks,
                          "refs": st.fine_refs}), flush=True)
        plugin.close()
        return
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for k in range(args.steps):
            step(args.warmup + k)
        e1.record(stream)
    stream.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    elapsed = replicas.max_over_ranks(e0.elapsed_time(e1), device="cuda")
    if world > 1:
        dist.barrier()
    segs = st.total_segments
    value = replicas.job_rate(segs * args.steps, world, elapsed / 1000.0)
    ms_per_step = elapsed / args.steps

    # Per-stage device times (events recorded inside the frame graph).
    spans = {}
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            step(args.warmup + args.steps + k)
            stream.synchronize()
            for name, ms in plugin.span_times().items():
                spans.setdefault(name, []).append(ms)
    span_med = {k: statistics.median(v) for k, v in spans.items()}
    # Per-frame device times of the same frames (each synchronised on its own):
    # median / p95 / p99, as the reference's bench summarises its frames.
    per_frame = sorted(spans.get("frame/total", []))
    frame_pct = None
    if per_frame:
        def pct(q):
            return per_frame[min(len(per_frame) - 1, int(round(q * (len(per_frame) - 1))))]
        frame_pct = {"frames": len(per_frame), "median": statistics.median(per_frame), "p95": pct(0.95),
                     "p99": pct(0.99)}

    # End to end through fiber_render_host: pinned host scene in, composited frame out.
    host_in = torch.empty((H, W, 4), dtype=torch.float16, pin_memory=True)
    host_in.copy_(scene.cpu())
    host_out = torch.empty((H, W, 4), dtype=torch.float16, pin_memory=True)
    lib = plugin.lib
    h2d = H * W * 8 + 4096  # scene image + frame tables (FrameParams, instance rows)
    d2h = H * W * 8
    sh = C.c_void_p(stream.cuda_stream)
    with torch.cuda.stream(stream):
        for k in range(max(1, args.warmup)):
            cam, lc = frame_structs(w, packed, replicas.frame_index(rank, k), lights)
            plugin.frame_begin_raw(cam_cfg, cam, light_cfgs, lc, stream)
            abi.check(lib.fiber_render_host(plugin.ctx, C.c_void_p(host_in.data_ptr()), None,
                                            C.c_void_p(host_out.data_ptr()), sh), "fiber_render_host")
        stream.synchronize()
        e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2.record(stream)
        for k in range(args.steps):
            cam, lc = frame_structs(w, packed, replicas.frame_index(rank, k), lights)
            plugin.frame_begin_raw(cam_cfg, cam, light_cfgs, lc, stream)
            abi.check(lib.fiber_render_host(plugin.ctx, C.c_void_p(host_in.data_ptr()), None,
                                            C.c_void_p(host_out.data_ptr()), sh), "fiber_render_host")
        e3.record(stream)
    stream.synchronize()
    e2e_ms = replicas.max_over_ranks(e2.elapsed_time(e3), device="cuda")
    e2e_value = replicas.job_rate(segs * args.steps, world, e2e_ms / 1000.0)
    assert np.isfinite(host_out.float().numpy()).all()

    # PrepassTelemetrySettings counters over a few more orbit frames (telemetry
    # adds atomics to the prepass, so it is switched on only after the timing).
    tel_samples = {}
    if not args.profile:
        plugin.settings.telemetry_enabled = 1
        abi.check(plugin.lib.fiber_settings_set(plugin.ctx, C.byref(plugin.settings)), "fiber_settings_set")
        with torch.cuda.stream(stream):
            for k in range(min(args.steps, 10)):
                step(k)
                stream.synchronize()
                for name, v in telemetry_words(plugin.telemetry()).items():
                    tel_samples.setdefault(name, []).append(float(v))

    # Roofline of the dominant kernel (HBM-bound dataflow; no dense contraction).
    ab = algorithmic_bytes(st, w, len(lights), w.dom_layers, w.dom_size)
    kernel_ms = {SPAN_TO_KERNEL[k]: v for k, v in span_med.items() if k in SPAN_TO_KERNEL}
    dom_kernel = max(kernel_ms, key=kernel_ms.get)
    peak, peak_kind = load_peaks()
    achieved = ab["per_kernel"][dom_kernel] / (kernel_ms[dom_kernel] / 1000.0) / 1e9
    traffic = load_traffic().get(dom_kernel, {}).get("bytes_per_launch")
    frame_ms = span_med.get("frame/total", ms_per_step)
    frame_gbs = ab["frame"] / (ms_per_step / 1000.0) / 1e9

    line = None
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            cpu_frame_time(w, packed, material, cam_cfg, lights, frame=0)
            dts = []
            for k in range(2):
                dt, csegs, note = cpu_frame_time(w, packed, material, cam_cfg, lights, frame=1 + k)
                dts.append(dt)
            cpu = {"value": csegs * len(dts) / sum(dts), "unit": UNIT, "cores": os.cpu_count() or 1,
                   "kind": "port", "sample": f"{note}: two orbit frames after one warm-up frame"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "frames_per_s": 1000.0 * world / ms_per_step,
            "config": bench_config(w, segs, len(lights), args, world),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "entry_point": "fiber_render_host", "ms_per_step": e2e_ms / args.steps},
            "roofline": {"bound": "hbm", "kernel": dom_kernel, "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "alg_bytes_per_launch": ab["per_kernel"][dom_kernel],
                         "launch_ms": kernel_ms[dom_kernel]},
            "frame_roofline": {"b_alg": ab["frame"], "b_min": ab["min"], "achieved_gbs": frame_gbs,
                               "frac": frame_gbs / peak},
            "cpu_baseline": cpu,
            "clocks": clk,
            "gpu_launches": KERNELS_PER_FRAME * args.steps,
            "spans_ms": span_med,
            "frame_ms": frame_pct,
            "report": bench_report(args, w, packed, spans, tel_samples),
            "counts": {"binning_tasks": st.binning_tasks, "camera_tasks": st.camera_tasks,
                       "pages": st.allocated_pages, "fine_refs": st.fine_refs, "work_items": st.work_items,
                       "camera_runs": st.camera_runs, "shadow_runs": st.shadow_runs},
        }
    plugin.close()
    if line is not None and world == 1 and not args.no_served:
        line["served"] = served_section(args)
    if line is not None and world == 1 and not args.no_batched:
        line["batched"] = batched_section(args)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


def summarize(values) -> dict:
    """min / mean / median / p90 / p95 / p99 / max of samples, nearest-rank on
    (n - 1) * q as the reference's strand_bench summarises them
    (examples/strand_bench.rs:931-947)."""
    v = sorted(values)
    def pct(q):
        return v[int(round((len(v) - 1) * q))]
    return {"samples": len(v), "min": v[0], "mean": sum(v) / len(v), "median": pct(0.5), "p90": pct(0.9),
            "p95": pct(0.95), "p99": pct(0.99), "max": v[-1]}


def telemetry_words(t) -> dict:
    """The telemetry image as the reference names its diagnostics
    (src/pipelines/prepass.rs:1345-1396)."""
    out = {}
    for name in ("allocated_pages", "binning_tasks", "page_candidates", "fine_cell_hits", "active_candidate_pages",
                 "max_candidates_per_page"):
        out[name] = getattr(t, name)
    for b in range(len(t.candidate_histogram)):
        out[f"candidate_histogram/{b}"] = t.candidate_histogram[b]
    for f in range(min(t.frustum_count, len(t.frustum))):
        for name, _ in t.frustum[f]._fields_:
            out[f"frustum/{f}/{name}"] = getattr(t.frustum[f], name)
    return out


def bench_report(args, w, packed, spans: dict, tel_samples: dict) -> dict:
    """The reference benchmark's report (examples/strand_bench.rs:859-913):
    schema version, case, shape, per-span GPU time summaries and the prepass
    telemetry summaries."""
    import torch
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    return {
        "schema_version": 1, "case": w.name, "mode": "headless",
        "resolution": {"width": w.width, "height": w.height},
        "warmup_frames": args.warmup, "sample_frames": len(spans.get("frame/total", [])),
        "telemetry_enabled": bool(tel_samples),
        "fine_binning_backend": args.binning_backend, "seed": w.seed,
        "workload": {"geometry_count": 1, "strand_count": int(packed.strand_count),
                     "vertex_count": int(packed.vertices.shape[0]), "points_per_strand": w.points,
                     "asset": "synthetic scalp hair"},
        "adapter": {"name": props.name, "backend": "cuda", "driver": torch.version.cuda},
        "timings_ms": {f"render/{k}/elapsed_gpu": summarize(v) for k, v in sorted(spans.items()) if v},
        "telemetry": {k: summarize(v) for k, v in sorted(tel_samples.items())},
    }


SERVED_BUDGET = 150 * 10**9  # bytes of HBM the served configuration may hold
SERVED_REF_FACTOR = 8


def served_section(args) -> dict:
    """The served configuration: 8 resident scenes (5k-500k strands), a seeded
    Poisson stream of requests of mixed scenes, resolutions (256^2 to 1080p)
    and shadow-map sizes. The server admits requests into as many slots as the
    HBM budget holds and overlaps them on the GPU; the plain per-request loop
    is the same server with one slot (each request runs alone, in arrival
    order). Latency is arrival to image in pinned host memory. A second pass
    submits a batch at once to measure throughput when every slot is busy."""
    import torch

    from bevy_strand_rasterizer_b200 import served
    from bevy_strand_rasterizer_b200.server import FiberServer

    t = time.time()
    scenes = served.served_scenes()
    gen_s = time.time() - t
    outputs = {(w, h): torch.empty((h, w, 4), dtype=torch.float16, pin_memory=True) for (w, h) in served.RESOLUTIONS}
    n_stream = max(1, int(args.served_rate * args.served_seconds))
    arrivals, reqs = served.request_stream(n_stream, args.served_rate, scenes, seed=7)
    _, batch = served.request_stream(args.served_saturate, 0.0, scenes, seed=8)
    _, warm = served.request_stream(32, 0.0, scenes, seed=9)
    result = {"scenes": [int(s.strand_count) for s in scenes], "points_per_strand": served.SCENE_POINTS,
              "resolutions": [f"{w}x{h}" for w, h in served.RESOLUTIONS], "dom_sizes": list(served.DOM_SIZES),
              "offered_rps": args.served_rate, "stream_s": args.served_seconds,
              "sustain_stream_s": args.served_sustain_seconds, "hbm_budget": SERVED_BUDGET,
              "ref_capacity_factor": SERVED_REF_FACTOR,
              "scene_gen_s": gen_s}
    # The plain loop runs first: its batch throughput sets the second, sustainable
    # arrival rate (80 % of what one request at a time can serve), at which
    # latency is service time rather than queue growth.
    sustain = None
    from bevy_strand_rasterizer_b200 import abi
    st = abi.default_settings()
    # Slots are sized once at start; a reference capacity factor of 8 (the
    # large workload's) leaves room for close-up views of the 500k-strand
    # scenes, so almost no request has to grow its slot (a growth reallocates
    # and synchronises the device) and none is truncated either way.
    st.ref_capacity_factor = SERVED_REF_FACTOR
    for label, slots in (("plain", 1), ("served", 0)):
        t = time.time()
        srv = FiberServer(slots=slots, max_width=1920, max_height=1080, max_lights=1, max_dom=2048,
                          hbm_budget=SERVED_BUDGET, settings=st)
        ids = [srv.add_scene(p) for p in scenes]
        n = srv.start()
        setup_s = time.time() - t
        served.replay(srv, ids, np.zeros(len(warm)), warm, outputs)
        sat = served.replay(srv, ids, np.zeros(len(batch)), batch, outputs)
        if sustain is None:
            rate = 0.8 * sat["frames_per_s"]
            sustain = (rate,) + served.request_stream(max(1, int(rate * args.served_sustain_seconds)), rate, scenes,
                                                      seed=10)
        stream = served.replay(srv, ids, arrivals, reqs, outputs)
        stream_s = served.replay(srv, ids, sustain[1], sustain[2], outputs)
        srv.close()
        result[label] = {"slots": n, "setup_s": setup_s, "batch": sat, "stream": stream,
                         "stream_sustainable": stream_s}
    result["sustainable_rps"] = sustain[0]
    result["frames_per_s_ratio"] = result["served"]["batch"]["frames_per_s"] / result["plain"]["batch"]["frames_per_s"]
    return result


def batched_section(args, reps: int = 5) -> dict:
    """The batched configuration: independent views (strands log-uniform in
    [1k, 200k] at 16 or 32 points, 256^2 to 1080p, one light with a 512^2 to
    2048^2 deep-opacity map) rendered two ways: multi-view frames whose kernels
    cover every view of the frame (fiber_frame_begin_views, replayed from one
    graph; the tuner picks 1, 2 or 4 such frames on concurrent streams), and
    one graph launch of the views' own frames over concurrent branches after
    the autotuner picked the branch count and view order; the faster is the
    batch. Compared with the same views as a loop of plain frames
    (per view: frame tables, then its own frame graph). All are timed with CUDA
    events on one stream over `reps` passes, after a warm-up pass, inputs
    resident on the device."""
    import torch

    from bevy_strand_rasterizer_b200 import batched

    t = time.time()
    specs = batched.batched_views(args.batched_views)
    packed = [batched.view_strands(v) for v in specs]
    gen_s = time.time() - t
    t = time.time()
    plugins = [batched.view_plugin(v, p) for v, p in zip(specs, packed)]
    setup_s = time.time() - t
    segments = int(sum(int(np.maximum(p.meta["count"].astype(np.int64) - 1, 0).sum()) for p in packed))
    stream = torch.cuda.Stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn) -> float:
        fn()  # warm-up pass (captures the graphs)
        stream.synchronize()
        ev0.record(stream)
        for _ in range(reps):
            fn()
        ev1.record(stream)
        ev1.synchronize()
        return ev0.elapsed_time(ev1) / reps

    def plain_pass():
        for v, p in zip(specs, plugins):
            batched.plain_frame(p, v, stream)

    plain_ms = timed(plain_pass)
    batch = batched.FiberBatch(plugins)
    t = time.time()
    best = batch.tune(stream)
    tune_s = time.time() - t
    branches_ms = timed(lambda: batch.launch(stream))
    batch.close()
    for p in plugins:
        p.close()
    # Multi-view frames: every kernel of a frame covers all of its views; the
    # tuner times the views as 1, 2 and 4 such frames on concurrent streams.
    t = time.time()
    group_ms = {}
    for g in (1, 2, 4):
        merged = batched.MultiViewGroups(specs, packed, g)
        group_ms[g] = timed(lambda: merged.launch(stream))
        merged.close()
    merged_setup_s = time.time() - t
    groups = min(group_ms, key=group_ms.get)
    merged_ms = group_ms[groups]
    n = len(specs)

    def rates(ms):
        return {"ms_per_pass": ms, "frames_per_s": n * 1e3 / ms, "segments_per_s": segments * 1e3 / ms}

    # The tuner's choice between the two batched forms: the faster one.
    mode = "multi_view_frame" if merged_ms <= branches_ms else "graph_branches"
    batch_ms = min(merged_ms, branches_ms)
    return {"views": n, "segments_per_pass": segments, "strands": [v.strands for v in specs],
            "resolutions": sorted({f"{v.camera.width}x{v.camera.height}" for v in specs}),
            "scene_gen_s": gen_s, "setup_s": setup_s, "tune_s": tune_s, "merged_setup_s": merged_setup_s,
            "passes": reps,
            "plain": rates(plain_ms),
            "multi_view_frame": dict(rates(merged_ms), groups=groups,
                                     ms_by_groups={str(k): v for k, v in group_ms.items()}),
            "graph_branches": dict(rates(branches_ms), tuning={"branches": int(best.branches),
                                                               "order": "lpt" if best.order else "index",
                                                               "tuned_ms": float(best.ms)}),
            "batch": dict(rates(batch_ms), mode=mode),
            "frames_per_s_ratio": plain_ms / batch_ms}


def main():
    args = parse_args()
    if args.impl == "reference":
        reference_arm(args)
    else:
        fiber_arm(args)


if __name__ == "__main__":
    main()
