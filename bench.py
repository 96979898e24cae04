#!/usr/bin/env python
"""Benchmark of the B200 path-tracing hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload rays|cornell|ggx] [--impl ours|reference]

Default workload (the ray-query configuration): 2^22 FP32 rays, origins uniform in the scene
box and directions uniform on the sphere (seeded), against a 1,310,720-triangle displaced
icosphere (level 8, radius 10, 4-octave value noise of amplitude 0.1); closest hit through the
8-wide quantised BVH. A step = one closest-hit launch over all rays; the metric is Mrays/s.

One JSON line on rank 0. `value`: device-timed (CUDA events) throughput with rays resident in
HBM; `e2e`: the same rays through the host-buffer C-ABI entry point rbr_trace_host (pinned
host rays in, hits out, copies inside the timed region); `roofline`: algorithmic bytes of the
traversal kernel (rays + hits + nodes and leaf records the traversal fetches, counted by
rbr_trace_counts) per launch over its event-timed duration, against the measured HBM copy
bandwidth; `cpu_baseline`: the reference's own BVH (oracle/_ref, built from the reference
sources) on the host cores over a bounded sample of the same rays.

With --impl reference the reference's CPU implementation is timed instead (rank 0 only).
Multi-GPU: every rank traces its own 2^22 rays (weak scaling, no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "ray-based-rendering_b200"))

RAYS_LOG2 = 22
ICO_LEVEL = 8


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=None, help="timed steps (default 200; cache workload: 256 frames)")
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", choices=["rays", "cornell", "ggx", "fog", "cache", "batch"], default="rays")
    p.add_argument("--ref-spp", type=int, default=4096, help="cache workload: spp of the converged GPU reference")
    p.add_argument("--cpu-ref-crop", type=int, default=0,
                   help="cache workload: also compare against the reference CPU integrator on a central crop of "
                        "this many pixels square")
    p.add_argument("--cpu-ref-spp", type=int, default=4096, help="cache workload: spp of the CPU reference crop")
    p.add_argument("--no-sub", action="store_true",
                   help="rays workload: skip the path-tracer and cache sub-measurements after the headline")
    p.add_argument("--cache-suffix", type=int, default=None,
                   help="cache workload: rbr_cache_config.train_suffix (default: the library's)")
    p.add_argument("--cache-config", action="append", default=[],
                   help="cache workload: NAME=INT field of rbr_cache_config (e.g. termination_depth=2)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true", help="skip the host-buffer measurement (profiling runs)")
    p.add_argument("--param", action="append", default=[], help="NAME=VALUE context tunable (rbr_param_set)")
    p.add_argument("--cpu-seconds", type=float, default=8.0, help="target length of the CPU-baseline sample")
    return p.parse_args()


# ------------------------------------------------------------------------------------------
def measured_peaks():
    f = REPO / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
            t0 = time.time()  # wait until sampling is live so that it covers the timed region
            while time.time() - t0 < 10 and Path(self.path).stat().st_size == 0:
                time.sleep(0.05)
        except Exception:
            self.proc = None

    def stop(self, gpu_indices=None):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                idx, sm, smax = int(c[0]), float(c[1]), float(c[2])
            except ValueError:
                continue
            if gpu_indices is not None and idx not in gpu_indices:
                continue
            rows.append((idx, sm, smax, c[5:9]))
        os.unlink(self.path)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i, v in enumerate(r[3]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[1] for r in rows), "sm_max_mhz": max(r[2] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def visible_gpu_indices(local_rank):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        try:
            return [int(vis.split(",")[local_rank])]
        except (ValueError, IndexError):
            return None
    return [local_rank]


# ------------------------------------------------------------------------------------------
# multi-rank plumbing (one process per GPU, replicas: no data-path collective)
def max_over_ranks(x: float, dist, device) -> float:
    """The largest of the ranks' values (a device time or a wall time): the job's time."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_scaling_rate(units_per_rank: int, world: int, seconds: float) -> float:
    """Whole-job throughput in millions of units per second: every rank processed
    units_per_rank, the job took the slowest rank's time."""
    return units_per_rank * world / seconds / 1e6


def workload(rank):
    from rbr_b200 import scenes

    scene = scenes.ray_query_scene(level=ICO_LEVEL, radius=10.0, seed=0)
    lo, hi = scenes.scene_bounds(scene)
    rays = scenes.uniform_rays(1 << RAYS_LOG2, lo, hi, seed=rank)
    return scene, rays


def cpu_baseline(scene, rays, target_s):
    """The reference BVH (oracle/_ref) over a bounded sample of the rays, all host threads."""
    sys.path.insert(0, str(REPO / "oracle"))
    from oracle import Reference, have_reference

    if not have_reference():
        return None
    ref = Reference()
    h = ref.scene(scene)
    threads = ref.max_threads()
    n = 1 << 14
    t0 = time.perf_counter()
    ref.trace_closest(h, rays[:n], threads=threads)
    dt = max(time.perf_counter() - t0, 1e-4)
    n = int(min(len(rays), max(1 << 15, n / dt * target_s)))
    t0 = time.perf_counter()
    ref.trace_closest(h, rays[:n], threads=threads)
    dt = time.perf_counter() - t0
    return {"value": n / dt / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "reference",
            "sample": f"first {n} of the 2^22 rays, reference BVH::intersect (src/acceleration/bvh.cpp) "
                      f"in an OpenMP loop, {dt:.1f} s; BVH build not timed"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    sys.path.insert(0, str(REPO / "oracle"))
    from oracle import Reference, have_reference

    if not have_reference():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/librbr_ref.so was not built"}))
        return
    scene, rays = workload(0)
    ref = Reference()
    h = ref.scene(scene)
    threads = ref.max_threads()
    n = 1 << 14
    t0 = time.perf_counter()
    ref.trace_closest(h, rays[:n], threads=threads)
    rate = n / max(time.perf_counter() - t0, 1e-4)
    # each step: a bounded sample so that the whole run stays within a few minutes
    n = int(min(len(rays), max(1 << 15, rate * 120.0 / max(1, args.steps + args.warmup))))
    for i in range(args.warmup):
        ref.trace_closest(h, rays[:n], threads=threads)
    t0 = time.perf_counter()
    for i in range(args.steps):
        ref.trace_closest(h, rays[:n], threads=threads)
    dt = time.perf_counter() - t0
    value = n * args.steps / dt / 1e6
    sample = f"{n} of the 2^22 rays per step, reference BVH::intersect in an OpenMP loop over {threads} threads"
    print(json.dumps({
        "impl": "reference", "metric": "Mrays/s traversal (closest hit)", "value": value, "unit": "Mrays/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": config_block(),
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def config_block():
    return {"workload": "ray-query: 2^22 rays (origins uniform in the scene box, directions uniform on the sphere, "
                        "seed 0) vs a 1,310,720-triangle displaced icosphere (level 8, radius 10, 4-octave value "
                        "noise, amplitude 0.1); closest hit",
            "rays_per_step": 1 << RAYS_LOG2, "triangles": 20 * 4 ** ICO_LEVEL,
            "l2": "inputs larger than L2: 134 MB of rays per step (the 70 MB BVH stays L2-resident by design)",
            "parallelism": "replicas (each GPU its own rays)"}


# ------------------------------------------------------------------------------------------
# path-tracer workloads: a step = one rbr_render of the whole image
RENDER_CONFIGS = {
    "cornell": dict(spp=16, max_depth=8, desc="Cornell box (18 quads, quad light 0.5x0.5 emission (17,12,4), two "
                                               "boxes rotated +-17 deg), pinhole fov 40, 256x256, 16 spp, max depth 8, "
                                               "NEE+MIS, RR after depth 3, FP32 RGB film, seed 0"),
    "ggx": dict(spp=64, max_depth=16, desc="GGX material scene: 256 spheres + 2M-triangle mound on a ground quad, "
                                           "random per-object materials (20% glass), 2 quad area lights + 1 point "
                                           "light, thin-lens camera, 1920x1080, 64 spp, max depth 16"),
    "fog": dict(spp=16, max_depth=8, volumetric=True,
                desc="foggy Cornell box: the Cornell box in a homogeneous medium (sigma_t 0.1, albedo 0.8, "
                     "Henyey-Greenstein g 0.5) plus a point light under the lamp, volumetric path integrator, "
                     "256x256, 16 spp, max depth 8"),
}


def render_scene(which):
    from rbr_b200 import scenes

    if which == "fog":
        return scenes.foggy_cornell_box()
    return scenes.cornell_box() if which == "cornell" else scenes.ggx_scene()


# Algorithmic bytes of the wavefront path tracer, per event (the fixed record sizes its kernels
# read and write; traversal bytes come from counted nodes and leaf records, 80 B and 48 B):
#   camera path (k_raygen: ray 32 + throughput 16 + radiance 16 + queue 4; k_film: radiance 16)
#   extension ray (k_extend: queue 4 + ray 32 + hit 8 + class queue 4)
#   shaded vertex (k_shade: class queue 4 + hit 8 + ray 32 + throughput 16 + leaf record 48 +
#                  material index 4 + material 44)
#   continuation (k_shade: next ray 32 + throughput 16 + queue 4)
#   shadow ray (k_shade writes and k_shadow reads its 48 B record)
#   pixel (k_film: 12 B of RGB film written)
PT_BYTES = {"path": 68 + 16, "extension_ray": 48, "shaded_vertex": 156, "continuation": 52, "shadow_ray": 96,
            "pixel": 12, "node": 80, "leaf_record": 48}


def path_tracer_bytes(st, pixels):
    """Algorithmic bytes of one render from its counted events (rbr_render_stats)."""
    b = PT_BYTES
    return (st.paths * b["path"] + st.extension_rays * b["extension_ray"] + st.shaded_vertices * b["shaded_vertex"]
            + (st.extension_rays - st.paths) * b["continuation"] + st.shadow_rays * b["shadow_ray"]
            + pixels * b["pixel"] + (st.ext_nodes + st.shadow_nodes) * b["node"]
            + (st.ext_records + st.shadow_records) * b["leaf_record"])


def cpu_render_baseline(scene, cam, spp, max_depth, volumetric, row_frac):
    """The reference's own Integrator::render (oracle/_ref) on a central band of the image."""
    sys.path.insert(0, str(REPO / "oracle"))
    from oracle import Reference, have_reference

    from rbr_b200 import render_params

    if not have_reference():
        return None
    import ctypes

    ref = Reference()
    h = ref.scene(scene)
    small = type(cam)()
    ctypes.memmove(ctypes.byref(small), ctypes.byref(cam), ctypes.sizeof(cam))
    small.height = max(8, int(cam.height * row_frac))
    small.cy = small.cy - (cam.height - small.height) / 2.0
    t0 = time.perf_counter()
    ref.render(h, small, render_params(spp=spp, max_depth=max_depth), volumetric=volumetric, threads=0)
    dt = time.perf_counter() - t0
    return {"value": cam.width * small.height * spp / dt / 1e6, "unit": "Mpaths/s", "cores": ref.max_threads(),
            "kind": "reference",
            "sample": f"central {cam.width}x{small.height} band of the image, the reference's own Integrator::render "
                      f"with {'VolumetricPathIntegrator' if volumetric else 'PathTracingIntegrator'} (OpenMP rows), "
                      f"{dt:.1f} s"}


def set_params(ctx, params, bvh=False):
    """Applies NAME=INT context parameters: only the BVH build ones (bvh.*, read at the next
    upload) with bvh=True, all of them otherwise."""
    for kv in params:
        k, v = kv.split("=")
        if not bvh or k.startswith("bvh."):
            ctx.set_param(k, int(v))


def measure_render(which, ctx, local_rank, rank, world, steps, warmup, e2e_steps, cpu_row_frac, params=()):
    """Mpaths/s of the path tracer on one configuration: device-timed steps (one rbr_render of the
    whole image each), end to end through rbr_render_host, the reference CPU integrator on a band
    of the image, and the algorithmic-bytes roofline of one step from a counted render."""
    import torch

    from rbr_b200 import abi, render_params

    cfg = RENDER_CONFIGS[which]
    scene = render_scene(which)
    cam = scene.camera
    W, H = cam.width, cam.height
    set_params(ctx, params, bvh=True)  # build parameters apply at the upload
    ctx.upload(scene)
    set_params(ctx, params)
    film = torch.empty(W * H * 3, dtype=torch.float32, device=f"cuda:{local_rank}")
    stream = torch.cuda.current_stream()
    paths = W * H * cfg["spp"]
    flags = abi.RBR_RENDER_VOLUMETRIC if cfg.get("volumetric") else 0

    def step(k, extra=0):
        p = render_params(spp=cfg["spp"], max_depth=cfg["max_depth"], seed=rank * 1000003 + k, flags=flags | extra)
        ctx.render_dev(cam, p, film.data_ptr(), 0, stream.cuda_stream)

    for k in range(max(3, warmup)):
        step(k)
    torch.cuda.synchronize()
    clocks = Clocks() if rank == 0 else None
    if clocks:
        clocks.start()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    evs[0].record(stream)
    for k in range(steps):
        step(1000 + k)
    evs[1].record(stream)
    torch.cuda.synchronize()
    total_ms = evs[0].elapsed_time(evs[1])
    clk = clocks.stop(visible_gpu_indices(local_rank)) if clocks else None
    st = ctx.render_stats()
    launches = st.launches
    # one counted render of the first timed step's samples: nodes and records per ray
    step(1000, abi.RBR_RENDER_COUNT_TRAFFIC)
    torch.cuda.synchronize()
    cst = ctx.render_stats()
    alg = path_tracer_bytes(cst, W * H)
    ms_step = total_ms / steps
    peak, peak_kind = measured_peaks()
    achieved = alg / (ms_step / 1e3) / 1e9
    e2e = None
    if e2e_steps:
        host_film = torch.empty(W * H * 3, dtype=torch.float32).pin_memory().numpy()
        ctx.render_host(cam, render_params(spp=cfg["spp"], max_depth=cfg["max_depth"], seed=0, flags=flags),
                        out=host_film)  # warm-up: staging buffers
        t0 = time.perf_counter()
        for k in range(e2e_steps):
            ctx.render_host(cam, render_params(spp=cfg["spp"], max_depth=cfg["max_depth"], seed=k, flags=flags),
                            out=host_film)
        e2e_s = time.perf_counter() - t0
        e2e = {"value": paths * e2e_steps / e2e_s / 1e6, "unit": "Mpaths/s", "h2d_bytes_per_step": 0,
               "d2h_bytes_per_step": W * H * 12, "steps": e2e_steps,
               "path": "rbr_render_host: render + film -> pinned host"}
    base = None
    if rank == 0 and world == 1 and cpu_row_frac:
        base = cpu_render_baseline(scene, cam, cfg["spp"], cfg["max_depth"], bool(flags), cpu_row_frac)
    n = cst.extension_rays + cst.shadow_rays
    return {
        "metric": "Mpaths/s (camera samples per second), " + (
            "GPU volumetric path tracer" if flags else "plain GPU path tracer"),
        "value": paths * world * steps / (total_ms / 1e3) / 1e6, "unit": "Mpaths/s", "steps": steps,
        "warmup": max(3, warmup), "ms_per_step": ms_step, "workload": cfg["desc"], "paths_per_step": paths,
        "e2e": e2e, "cpu_baseline": base, "clocks": clk, "gpu_launches": launches * steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_source": f"{peak_kind} HBM copy bandwidth",
                     "algorithmic_bytes_per_step": alg, "bytes_per_path": alg / paths,
                     "record_bytes": PT_BYTES,
                     "per_path": {"extension_rays": cst.extension_rays / paths, "shadow_rays": cst.shadow_rays / paths,
                                  "shaded_vertices": cst.shaded_vertices / paths},
                     "per_ray": {"nodes": (cst.ext_nodes + cst.shadow_nodes) / max(1, n),
                                 "leaf_records": (cst.ext_records + cst.shadow_records) / max(1, n)},
                     "counted": "nodes and records of one render with RBR_RENDER_COUNT_TRAFFIC, same samples as the "
                                "first timed step"},
        "render": {"waves": st.waves, "launches_per_step": st.launches},
    }


def run_render(args, rank, world, local_rank):
    import torch

    from rbr_b200 import Context

    torch.cuda.set_device(local_rank)
    ctx = Context(local_rank)
    r = measure_render(args.workload, ctx, local_rank, rank, world, args.steps, args.warmup,
                       0 if args.no_e2e else max(3, min(args.steps, 20)), 0 if args.no_cpu_baseline else 1.0 / 8,
                       args.param)
    ctx.close()
    if rank == 0:
        line = {"metric": r["metric"], "value": r["value"], "unit": r["unit"], "n_gpus": world, "steps": r["steps"],
                "warmup": r["warmup"], "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
                "config": {"workload": r["workload"], "paths_per_step": r["paths_per_step"],
                           "l2": "working set of the two waves in flight (path state + 48 B per shadow record) larger "
                                 "than L2; the film is written once"}}
        for k in ("e2e", "cpu_baseline", "roofline", "clocks", "gpu_launches", "render"):
            line[k] = r[k]
        print(json.dumps(line))


def relmse(x, ref, ref_var=None):
    """mean((x - ref)^2 / (ref^2 + 1e-2)) over pixels and channels. With ref_var (the variance of
    the reference's per-pixel mean) the reference's own Monte-Carlo noise, which inflates the
    squared difference by ref_var on average, is subtracted: an estimate of the error against
    the converged image."""
    d2 = (x.astype(np.float64) - ref) ** 2
    if ref_var is not None:
        d2 = d2 - ref_var
    return float(np.mean(d2 / (ref.astype(np.float64) ** 2 + 1e-2)))


def measure_cache(ctx, local_rank, rank, frames, warmup, ref_spp, cache_kw, e2e_frames=8, cpu_crop=0, cpu_spp=0):
    """Learned radiance cache vs the plain GPU path tracer at equal time on the GGX scene
    (1920x1080, 1 spp per frame). A step is one frame: 1 spp with paths ending into the cache,
    plus the frame's 4 optimiser steps on 2^16 training paths. Converged reference: the plain
    GPU path tracer at ref_spp samples per pixel (independent seed) with its per-pixel variance,
    which the corrected RelMSE subtracts; optionally the reference's own CPU integrator on a
    central crop of cpu_crop^2 pixels at cpu_spp samples per pixel."""
    import torch

    from rbr_b200 import abi, render_params, scenes

    scene = scenes.ggx_scene()
    cam = scene.camera
    W, H = cam.width, cam.height
    ctx.upload(scene)
    depth = 16
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    film = torch.zeros(W * H * 3, dtype=torch.float32, device=f"cuda:{local_rank}")
    film2 = torch.zeros(W * H * 3, dtype=torch.float32, device=f"cuda:{local_rank}")

    def plain(spp, seed, var=False):
        """The plain path tracer at `spp`, in calls of at most 1024 spp (one call takes at most
        2^32 camera samples) with consecutive sample ranges; film = the sample-weighted mean, and
        with var the variance of that mean from the per-pixel second moments."""
        img, sq, total_ms, done = 0.0, 0.0, 0.0, 0
        while done < spp:
            n = min(1024, spp - done)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            ev[0].record(stream)
            ctx.render_dev(cam, render_params(spp=n, max_depth=depth, seed=seed, sample_offset=done,
                                              flags=abi.RBR_RENDER_SECOND_MOMENT if var else 0),
                           film.data_ptr(), film2.data_ptr() if var else 0, sp)
            ev[1].record(stream)
            torch.cuda.synchronize()
            img = img + film.cpu().numpy().reshape(H, W, 3).astype(np.float64) * n
            if var:
                sq = sq + film2.cpu().numpy().reshape(H, W, 3).astype(np.float64)
            total_ms += ev[0].elapsed_time(ev[1])
            done += n
        mean = img / spp
        if not var:
            return mean, total_ms
        return mean, total_ms, np.maximum(sq / spp - mean ** 2, 0.0) / (spp - 1)

    ref, ref_ms, ref_var = plain(ref_spp, 777, var=True)  # converged reference, independent seed
    # warm-up of both paths (kernels loaded, buffers allocated)
    plain(1, 1)
    ctx.cache_create(seed=3, **cache_kw)
    ctx.cache_render_dev(cam, render_params(spp=1, max_depth=depth, seed=2), max(3, warmup), film.data_ptr(), 0,
                         True, sp)
    torch.cuda.synchronize()
    # the timed cached run starts from a fresh cache
    ctx.cache_create(seed=3, **cache_kw)
    clocks = Clocks() if rank == 0 else None
    if clocks:
        clocks.start()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(stream)
    ctx.cache_render_dev(cam, render_params(spp=1, max_depth=depth, seed=11), frames, film.data_ptr(), 0, True, sp)
    ev[1].record(stream)
    torch.cuda.synchronize()
    cache_ms = ev[0].elapsed_time(ev[1])
    clk = clocks.stop(visible_gpu_indices(local_rank)) if clocks else None
    launches = ctx.render_stats().launches
    cached = film.cpu().numpy().reshape(H, W, 3).astype(np.float64)
    info = ctx.cache_info()
    # plain path tracer: equal samples, then equal time
    plain_same, plain_same_ms = plain(frames, 11)
    eq_spp = max(1, int(round(frames * cache_ms / plain_same_ms)))
    plain_eq, plain_eq_ms = plain(eq_spp, 11)
    r = {k: relmse(x, ref) for k, x in (("cache", cached), ("plain_equal_time", plain_eq),
                                         ("plain_equal_samples", plain_same))}
    rc = {k: relmse(x, ref, ref_var) for k, x in (("cache", cached), ("plain_equal_time", plain_eq),
                                                   ("plain_equal_samples", plain_same))}
    out = {
        "metric": "Mpaths/s & RelMSE at equal time: MLP cache vs plain GPU PT",
        "value": W * H * frames / (cache_ms / 1e3) / 1e6, "unit": "Mpaths/s", "steps": frames,
        "warmup": max(3, warmup), "ms_per_step": cache_ms / frames,
        "workload": "learned radiance cache on the GGX scene: 1920x1080, 1 spp per frame, "
                    f"{frames} frames; hash grid 16 levels x 2^19 x 2 FP16, MLP 5x64 BF16; "
                    "2^16 training paths per frame, 4 Adam steps of 16384 samples, lr 1e-2",
        "reference": f"plain GPU path tracer, {ref_spp} spp, independent seed ({ref_ms / 1e3:.1f} s)",
        "relmse": {**r, "gain_equal_time": r["plain_equal_time"] / r["cache"], "plain_equal_time_spp": eq_spp,
                   "plain_equal_time_ms": plain_eq_ms, "cache_ms": cache_ms,
                   "mean_bias": float(cached.mean() / ref.mean() - 1.0)},
        "relmse_noise_corrected": {**rc, "gain_equal_time": rc["plain_equal_time"] / max(rc["cache"], 1e-12),
                                   "reference_noise": float(np.mean(ref_var / (ref ** 2 + 1e-2))),
                                   "note": "the reference's per-pixel variance of its mean subtracted from the "
                                           "squared differences"},
        "cache": {"optimiser_steps": info.optimiser_steps, "last_loss": info.last_loss,
                  "queries_last_frame": info.last_queries, "train_records_last_frame": info.last_train_records,
                  "train_suffix": ctx.cache_config(**cache_kw).train_suffix,
                  "termination_depth": ctx.cache_config(**cache_kw).termination_depth},
        "clocks": clk, "gpu_launches": launches,
    }
    if cpu_crop and cpu_spp:
        sys.path.insert(0, str(REPO / "oracle"))
        from oracle import Reference, have_reference

        if have_reference():
            import ctypes

            cref = Reference()
            crop = type(cam)()
            ctypes.memmove(ctypes.byref(crop), ctypes.byref(cam), ctypes.sizeof(cam))
            x0, y0 = (W - cpu_crop) // 2, (H - cpu_crop) // 2
            crop.width = crop.height = cpu_crop
            crop.cx, crop.cy = cam.cx - x0, cam.cy - y0
            t0 = time.perf_counter()
            acc = cref.render_moments(cref.scene(scene), crop, render_params(spp=cpu_spp, max_depth=depth), batch=1)
            cpu_s = time.perf_counter() - t0
            cmean = acc[0] / cpu_spp
            cvar = np.maximum(acc[1] / cpu_spp - cmean ** 2, 0.0) / (cpu_spp - 1)
            sl = (slice(y0, y0 + cpu_crop), slice(x0, x0 + cpu_crop))
            out["relmse_cpu_reference"] = {
                "reference": f"the reference's own PathTracingIntegrator::Li, central {cpu_crop}x{cpu_crop} crop, "
                             f"{cpu_spp} spp, {cpu_s:.0f} s on {cref.max_threads()} host threads",
                "cache": relmse(cached[sl], cmean, cvar), "plain_equal_time": relmse(plain_eq[sl], cmean, cvar),
                "gpu_reference": relmse(ref[sl], cmean, cvar),
                "mean_bias_cache": float(cached[sl].mean() / cmean.mean() - 1.0),
                "mean_bias_gpu_reference": float(ref[sl].mean() / cmean.mean() - 1.0),
                "note": "noise-corrected by the CPU reference's variance of its mean"}
            out["relmse_cpu_reference"]["gain_equal_time"] = (out["relmse_cpu_reference"]["plain_equal_time"] /
                                                              max(out["relmse_cpu_reference"]["cache"], 1e-12))
    if e2e_frames:
        t0 = time.perf_counter()
        ctx.cache_render_dev(cam, render_params(spp=1, max_depth=depth, seed=12), e2e_frames, film.data_ptr(), 0,
                             True, sp)
        host = film.cpu()
        e2e_s = time.perf_counter() - t0
        del host
        out["e2e"] = {"value": W * H * e2e_frames / e2e_s / 1e6, "unit": "Mpaths/s", "h2d_bytes_per_step": 0,
                      "d2h_bytes_per_step": W * H * 12 // e2e_frames,
                      "path": f"rbr_cache_render of {e2e_frames} frames + film to host"}
    return out


def run_cache(args, rank, world, local_rank):
    import torch

    from rbr_b200 import Context

    torch.cuda.set_device(local_rank)
    cache_kw = {} if args.cache_suffix is None else {"train_suffix": args.cache_suffix}
    for kv in args.cache_config:
        k, v = kv.split("=")
        cache_kw[k] = int(v)
    ctx = Context(local_rank)
    set_params(ctx, args.param)
    r = measure_cache(ctx, local_rank, rank, args.steps, args.warmup, args.ref_spp, cache_kw,
                      cpu_crop=args.cpu_ref_crop, cpu_spp=args.cpu_ref_spp)
    ctx.close()
    if rank == 0:
        line = {"metric": r["metric"], "value": r["value"], "unit": r["unit"], "n_gpus": world, "steps": r["steps"],
                "warmup": r["warmup"], "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "bf16 (MLP) / f32 (path tracer)", "data": "synthetic (seeded)",
                "config": {"workload": r["workload"], "reference": r["reference"],
                           "l2": "path state per frame (2M paths x ~100 B) and hash grid (34 MB FP16) + Adam state "
                                 "and gradients (268 + 67 MB) exceed L2"}}
        for k in ("relmse", "relmse_noise_corrected", "relmse_cpu_reference", "cache", "e2e", "clocks",
                  "gpu_launches"):
            if k in r:
                line[k] = r[k]
        print(json.dumps(line))


def measure_batch(ctx, local_rank, rank, steps, warmup, e2e=True, autotune=True):
    """Batched request loop (config 5): 64 seeded requests, resolution uniform over {128^2,
    256^2, 512^2, 1024^2}, spp U{1..64}; scenes: 7 seeded material/light variants of the GGX
    scene sharing its geometry and BVH, and the foggy Cornell box (volumetric path, 1 in 8
    requests). Throughput with every request present at the start; then p50/p99 latency under
    staggered arrivals: a seeded Poisson process whose mean gap is 1.25 x (all-at-once run time
    / 64), i.e. about 80 % load, for the graph-replayed waves and for the persistent launch
    (cache off), and for the graph path with the radiance cache on (GGX variants end paths into
    their scene's cache and train it). Latency of a request = device time from its arrival to
    the end of its last wave."""
    import torch

    from rbr_b200 import Batch, abi, render_params, scenes

    rng = np.random.default_rng(5 + rank)
    base = scenes.ggx_scene()
    variants = [scenes.ggx_variant(base, v) for v in range(1, 7)]
    fog = scenes.foggy_cornell_box()
    sizes = [128, 256, 512, 1024]
    reqs = []
    for i in range(64):
        size = int(rng.choice(sizes))
        spp = int(rng.integers(1, 65))
        if i % 8 == 7:
            reqs.append(("fog", scenes.square_camera(fog.camera, size), spp, 8, abi.RBR_RENDER_VOLUMETRIC))
        else:
            reqs.append((int(rng.integers(0, 7)), scenes.square_camera(base.camera, size), spp, 16, 0))
    films = [torch.zeros(c.width * c.height * 3, device=f"cuda:{local_rank}") for _, c, _, _, _ in reqs]
    stream = torch.cuda.current_stream().cuda_stream
    total_paths = sum(c.width * c.height * spp for _, c, spp, _, _ in reqs)

    def make(**cfg):
        b = Batch(ctx, **cfg)
        ids = [b.add_scene(base)] + [None] * 6
        for v in range(1, 7):
            ids[v] = b.add_scene_variant(ids[0], variants[v - 1])
        fid = b.add_scene(fog)
        for sid in ids:
            b.cache_create(sid, seed=1)
        return b, ids, fid

    def submit(b, ids, fid, use_cache, arrivals=None, subset=None):
        rid = []
        for i, (sk, cam, spp, depth, flags) in enumerate(reqs if subset is None else reqs[:subset]):
            cache = use_cache and not flags
            rid.append(b.submit(fid if sk == "fog" else ids[sk], cam,
                                render_params(spp=spp, max_depth=depth, seed=1000 + i, flags=flags),
                                films[i].data_ptr(), use_cache=cache, train_cache=cache,
                                arrival_us=0 if arrivals is None else int(arrivals[i])))
        return rid

    def timed(b, ids, fid, use_cache, arrivals, n):
        lat, qlat, total_ms, paths, st, wall = [], [], 0.0, 0, None, 0.0
        for _ in range(n):
            rid = submit(b, ids, fid, use_cache, arrivals)
            t0 = time.perf_counter()
            b.run(stream)
            st = b.stats()
            wall = time.perf_counter() - t0
            total_ms += st.milliseconds
            paths += st.paths
            rs = [b.request_stats(r) for r in rid]
            lat += [r.latency_ms for r in rs]
            qlat += [r.start_ms for r in rs]
        return {"mpaths_per_s": paths / (total_ms / 1e3) / 1e6, "ms_per_run": total_ms / n,
                "latency_ms_p50": float(np.percentile(lat, 50)), "latency_ms_p99": float(np.percentile(lat, 99)),
                "queueing_ms_p50": float(np.percentile(qlat, 50)), "waves_per_run": st.waves,
                "segments_per_run": st.segments, "graph_launches_per_run": st.graph_launches,
                "kernel_launches_per_run": st.kernel_launches, "persistent_launches_per_run": st.persistent_launches,
                "wave_paths": st.wave_paths, "blocks_per_sm": st.blocks_per_sm, "host_wall_s_last_run": wall}

    out = {"workload": "64 seeded requests: resolution uniform over {128^2, 256^2, 512^2, 1024^2}, spp U{1..64}; "
                       "7 material/light variants of the GGX scene (shared geometry, depth 16) and the foggy Cornell "
                       "box (volumetric, depth 8, every 8th request)", "paths_per_run": total_paths}
    clocks = Clocks() if rank == 0 else None
    b, ids, fid = make()
    if autotune:  # wave size and grid on a calibration subset, then warm up (graphs captured)
        submit(b, ids, fid, False, subset=8)
        b.autotune(stream)
        b.run(stream)
    for _ in range(max(1, warmup)):
        submit(b, ids, fid, False)
        b.run(stream)
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
    out["all_at_once"] = timed(b, ids, fid, False, None, steps)
    gap_us = 1.25 * out["all_at_once"]["ms_per_run"] * 1000.0 / len(reqs)
    arrivals = np.cumsum(np.random.default_rng(77 + rank).exponential(gap_us, len(reqs))) - gap_us
    arrivals = np.clip(arrivals, 0, None).astype(np.int64)
    out["arrivals"] = {"process": "Poisson, seeded", "mean_gap_us": gap_us, "span_ms": float(arrivals[-1] / 1e3),
                       "load": "about 80 % of the all-at-once throughput"}
    out["staggered_graphs"] = timed(b, ids, fid, False, arrivals, steps)
    out["staggered_graphs_cache_on"] = timed(b, ids, fid, True, arrivals, steps)
    cfg = dict(wave_paths=out["all_at_once"]["wave_paths"], persistent=1)
    bp, pids, pfid = make(**cfg)
    submit(bp, pids, pfid, False)
    bp.run(stream)  # warm-up
    out["all_at_once_persistent"] = timed(bp, pids, pfid, False, None, steps)
    out["staggered_persistent"] = timed(bp, pids, pfid, False, arrivals, steps)
    out["clocks"] = clocks.stop(visible_gpu_indices(local_rank)) if clocks else None
    if e2e:  # submit, run and have every film copied to page-locked host memory
        host = [torch.empty(f.numel(), dtype=torch.float32).pin_memory() for f in films]
        t0 = time.perf_counter()
        rid = submit(b, ids, fid, False)
        for r, hb in zip(rid, host):
            b.set_host_film(r, hb.data_ptr())  # copied after the request's last wave
        b.run(stream)
        torch.cuda.current_stream().synchronize()
        e2e_s = time.perf_counter() - t0
        assert all(torch.equal(hb, f.cpu()) for hb, f in zip(host[:4], films[:4])), "host films differ"
        del host
        out["e2e"] = {"value": total_paths / e2e_s / 1e6, "unit": "Mpaths/s", "h2d_bytes_per_step": 0,
                      "d2h_bytes_per_step": sum(c.width * c.height * 12 for _, c, _, _, _ in reqs),
                      "path": "rbr_batch_submit x64 + rbr_batch_set_host_film x64 + rbr_batch_run, every film "
                              "copied to pinned host memory after its request's last wave"}
    bp.close()
    b.close()
    return out


def run_batch(args, rank, world, local_rank):
    import torch

    from rbr_b200 import Context

    torch.cuda.set_device(local_rank)
    ctx = Context(local_rank)
    set_params(ctx, args.param)
    r = measure_batch(ctx, local_rank, rank, args.steps, args.warmup, e2e=not args.no_e2e)
    ctx.close()
    if rank == 0:
        a = r["all_at_once"]
        print(json.dumps({
            "metric": "Mpaths/s & p50/p99 request latency, batched request loop (64 requests)",
            "value": a["mpaths_per_s"] * world, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(1, args.warmup), "ms_per_step": a["ms_per_run"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": r["workload"], "paths_per_run": r["paths_per_run"], "arrivals": r["arrivals"],
                       "l2": "path state of a wave (up to 8M paths x ~250 B, two waves in flight) larger than L2"},
            "latency": {k: r[k] for k in ("all_at_once", "staggered_graphs", "staggered_graphs_cache_on",
                                          "all_at_once_persistent", "staggered_persistent")},
            "e2e": r.get("e2e"), "clocks": r["clocks"], "gpu_launches": a["kernel_launches_per_run"] * args.steps,
        }))


def main():
    args = parse()
    if args.steps is None:
        args.steps = {"cache": 256, "batch": 3}.get(args.workload, 200)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "cache":
        return run_cache(args, rank, world, local_rank)
    if args.workload == "batch":
        return run_batch(args, rank, world, local_rank)
    if args.workload != "rays":
        return run_render(args, rank, world, local_rank)

    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local_rank)

    from rbr_b200 import Context, abi

    scene, rays = workload(rank)
    ctx = Context(local_rank)
    set_params(ctx, args.param, bvh=True)  # build parameters apply at the upload
    stats = ctx.upload(scene)
    set_params(ctx, args.param)
    n = len(rays)
    d_rays = torch.from_numpy(rays.view(np.uint8)).to(f"cuda:{local_rank}")
    d_hits = torch.empty(n * 8, dtype=torch.uint8, device=f"cuda:{local_rank}")
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream

    tuned = ctx.autotune_trace(d_rays.data_ptr(), n) if not args.param else {k: ctx.get_param(k) for k in
                                                                           ("trace.kernel", "trace.min_blocks",
                                                                            "trace.order")}
    tuned["trace.node_test"] = ctx.get_param("trace.node_test")

    def step():
        ctx.trace_closest_dev(d_rays.data_ptr(), n, d_hits.data_ptr(), sp)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    clocks = Clocks() if rank == 0 else None
    if clocks:
        clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    evs[0].record(stream)
    for k in range(args.steps):
        step()
        evs[k + 1].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launch_ms = [evs[k].elapsed_time(evs[k + 1]) for k in range(args.steps)]
    total_ms = evs[0].elapsed_time(evs[-1])
    total_ms = max_over_ranks(total_ms, dist, f"cuda:{local_rank}")
    clk = clocks.stop(visible_gpu_indices(local_rank)) if clocks else None

    l2_peak = ctx.l2_read_bandwidth(32 << 20, 50)
    # algorithmic traffic of one launch
    nodes, recs = ctx.trace_counts_dev(d_rays.data_ptr(), n)
    alg_bytes = n * (32 + 8) + nodes * 80 + recs * 48
    avg_launch_s = statistics.mean(launch_ms) / 1e3
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / avg_launch_s / 1e9
    # DRAM bytes per launch of this very variant from an ncu capture (profiles/traffic.json)
    traffic = None
    traffic_key = "trace_closest_icosphere8_k{}_b{}_o{}_n{}".format(
        tuned.get("trace.kernel", 0), ctx.get_param("trace.min_blocks"), tuned.get("trace.order", 0),
        tuned["trace.node_test"])
    tf = REPO / "profiles" / "traffic.json"
    if tf.exists():
        traffic = json.loads(tf.read_text()).get(traffic_key)

    # end to end through the host-buffer entry point
    e2e = None
    if not args.no_e2e:
        host_rays = torch.from_numpy(rays.view(np.uint8)).pin_memory()
        host_hits = torch.empty(n * 8, dtype=torch.uint8).pin_memory()
        hr = host_rays.numpy().view(abi.RAY_DTYPE)
        hh = host_hits.numpy().view(abi.HIT_DTYPE)
        for _ in range(2):
            ctx.trace_host(hr, out=hh)
        e2e_steps = max(3, min(args.steps, 20))
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            ctx.trace_host(hr, out=hh)
        e2e_s = time.perf_counter() - t0
        e2e_s = max_over_ranks(e2e_s, dist, f"cuda:{local_rank}")
        got = d_hits.cpu().numpy().view(abi.HIT_DTYPE)
        assert np.array_equal(got["prim"], hh["prim"]), "device and host entry points disagree"
        e2e = {"value": weak_scaling_rate(n * e2e_steps, world, e2e_s), "unit": "Mrays/s",
               "h2d_bytes_per_step": n * 32, "d2h_bytes_per_step": n * 8,
               "path": "rbr_trace_host: pinned host rays -> device, closest hit, hits -> pinned host"}

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(scene, rays, args.cpu_seconds)

    if rank == 0:
        value = weak_scaling_rate(n * args.steps, world, total_ms / 1e3)
        line = {
            "metric": "Mrays/s traversal (closest hit)", "value": value, "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)", "config": config_block(),
            "e2e": e2e,
            "roofline_l2": {"achieved": achieved, "peak": l2_peak, "unit": "GB/s", "frac": achieved / l2_peak,
                            "peak_source": "read bandwidth of a 32 MiB L2-resident buffer (rbr_l2_read_bandwidth), "
                                           "measured in this run"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_key,
                         "peak_source": f"{peak_kind} HBM copy bandwidth",
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "per_ray": {"nodes": nodes / n, "leaf_records": recs / n,
                                     "bytes": alg_bytes / n},
                         "kernel": "k_trace_closest" if not tuned.get("trace.order") else
                         "k_trace_closest_perm (timed with its ray sort: the whole call)",
                         "avg_launch_ms": avg_launch_s * 1e3},
            "cpu_baseline": base,
            "clocks": clk,
            # the traversal, plus the sort's own kernels: keys, offsets and scatter of the
            # counting sort (orders 4, 5); the key kernel before CUB's radix sort (orders 1-3)
            "gpu_launches": args.steps * (1 + (0 if not tuned.get("trace.order") else
                                               3 if tuned.get("trace.order") >= 4 else 1)),
            "tuning": tuned,
            "bvh": {"wide_nodes": stats.num_wide_nodes, "leaf_records": stats.num_leaf_records,
                    "depth": stats.max_depth, "build_s": stats.build_seconds,
                    "device_mb": stats.device_bytes / 1e6, "wrapped_leaves": stats.wrapped_leaves},
        }
    if world == 1 and not args.no_sub:
        # the metric's other parts, after the headline's timed region: the plain path tracer on the
        # Cornell box and the GGX scene (Mpaths/s), and the radiance cache's RelMSE at equal time
        e2e_on = not args.no_e2e
        cpu_on = not args.no_cpu_baseline
        line["path_tracer"] = {
            "cornell": measure_render("cornell", ctx, local_rank, rank, world, 20, 3, 10 if e2e_on else 0,
                                      1.0 / 8 if cpu_on else 0),
            "ggx": measure_render("ggx", ctx, local_rank, rank, world, 5, 3, 3 if e2e_on else 0,
                                  1.0 / 32 if cpu_on else 0)}
        line["radiance_cache"] = measure_cache(ctx, local_rank, rank, 256, 3, 2048, {}, 8 if e2e_on else 0)
    if rank == 0:
        print(json.dumps(line))
    ctx.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
