#!/usr/bin/env python3
"""Benchmark of the path-tracing hot path (one JSON line on rank 0).

Workload ("large" configuration): ~1.15M triangles in 256 seeded instances,
DSPBR materials over the whole feature set, 2048x1024 log-normal HDR
environment with a 1e4 sun, 1920x1080, 12 bounces, MWC RNG of the reference.
A step is one progressive frame: one sample per pixel, all bounces, NEE,
accumulation.  Metric: Mrays/s (primary + extension + shadow rays).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

--impl reference times the reference's own CPU implementation (its fragment
shader compiled for the host, oracle/_ref) on a bounded pixel sample of the
same workload with all host threads.  Under torchrun (N>1) every rank renders
its own replica of the frame stream (weak scaling, no collective on the data
path); the reported value is the sum of rays over ranks / max device time.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "dspbr-pt_b200"))
sys.path.insert(0, ROOT)

METRIC = "Mrays/s"


def extend_traffic_rate():
    """DRAM bytes per millisecond of k_extend_dyn launches (ncu
    dram__bytes_read.sum + dram__bytes_write.sum over gpu__time_duration.sum
    of three launches of one capture, committed beside the ncu summaries
    under profiles/), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "k_extend_traffic.json")) as f:
            return float(json.load(f)["dram_bytes_per_ms"])
    except Exception:
        return None


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region:
    every 20 ms; the region starts after the first sample has arrived, and the
    samples taken before it are not counted."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "20"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return self
        self.skip = 0
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < 10.0 and self.proc.poll() is None:
            with open(self.path) as f:
                n = sum(1 for _ in f)
            if n:
                self.skip = n
                break
            time.sleep(0.01)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.out.close()

    def summary(self):
        if self.proc is None or not self.path:
            return None
        rows = []
        with open(self.path) as f:
            for k, line in enumerate(f):
                parts = [x.strip() for x in line.split(",")]
                if k >= getattr(self, "skip", 0) and len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
        return rank, ws, local, dist
    return 0, 1, 0, None


def reduce_max(dist, x: float) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(dist, x: float) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


# wide BVH of the path kernels in every GPU render of this run (--wide-bvh)
WIDE_BVH = 4


def make_workload():
    from dspbr import synth
    from dspbr.viewport import Bvh
    sc = synth.make_large(0)
    sc.bvh = Bvh.build(sc.vertices, sc.indices, 20)
    return sc


def write_workload_bvh(path):
    """Child-process entry (--write-bvh PATH): the workload's BVH, built by the
    library's host binned-SAH builder, saved as an .npz."""
    sc = make_workload()
    np.savez(path, nodes=sc.bvh.nodes, indices=sc.bvh.indices)
    return 0


def reference_workload():
    """The workload for the reference arm.  Its BVH (the reference's node
    layout) is built by a child process, so the process that times the
    reference's shader loads no library of this repository, only oracle/_ref."""
    from dspbr import synth
    from dspbr.viewport import Bvh  # a plain container: its constructor loads nothing
    fd, path = tempfile.mkstemp(suffix=".npz")
    os.close(fd)
    try:
        subprocess.run([sys.executable, os.path.abspath(__file__), "--write-bvh", path], check=True)
        with np.load(path) as z:
            nodes, indices = z["nodes"], z["indices"]
    finally:
        os.unlink(path)
    sc = synth.make_large(0)
    sc.bvh = Bvh(nodes, indices, 0, sc.num_triangles)
    return sc


def config_of(sc):
    return {"workload": "large: 256 seeded instances (displaced grids + icospheres), DSPBR feature-set materials, "
                        "2048x1024 log-normal HDR env + 1e4 sun", "triangles": int(sc.num_triangles),
            "bvh_nodes": int(sc.bvh.nodes.size // 16), "width": sc.width, "height": sc.height,
            "max_bounces": sc.max_bounces, "spp_per_step": 1, "rng": "mwc (reference rng.glsl)",
            "env_sampling": "alias", "l2": "inputs larger than L2 (BVH + triangles + vertices + env ~ 230 MB)",
            "seed": sc.seed}


def cpu_reference_sample(sc, seconds=12.0, steps=None, warmup=0, target_s=20.0):
    """Times oracle/_ref (the reference shader compiled for the host) on pixel
    samples of the workload; returns (Mrays/s, cores, sample description, per-step values).
    With `steps`, the warm-up steps (4096 pixels each, at least one) measure
    the rate and each timed step then takes enough pixels for the timed steps
    to last about `target_s` seconds together."""
    from oracle import ref_lib
    kind = "reference"
    if not ref_lib.available("f32"):
        return None
    ref = ref_lib.GlslReference("f32")
    ref.set_scene(sc.vertices, sc.indices, sc.materials, sc.bvh.nodes, sc.bvh.indices)
    ref.set_ibl(sc.env)
    cores = os.cpu_count() or 1
    rng = np.random.default_rng(7)
    npx = 4096
    vals = []
    tot_rays, tot_t = 0, 0.0
    step = 0
    t_start = time.perf_counter()
    while True:
        xy = np.stack([rng.integers(0, sc.width, npx), rng.integers(0, sc.height, npx)], 1).astype(np.int32)
        ref.set_uniforms(ref_lib.uniform_block(sc.camera.matrix_world, sc.camera.fov, sc.camera.near, sc.width,
                                               sc.height, step + 1, sc.max_bounces))
        t0 = time.perf_counter()
        _, rays = ref.render_pixels(xy, sc.width, sc.height, cores)
        dt = time.perf_counter() - t0
        if step >= warmup:
            vals.append(rays / dt / 1e6)
            tot_rays += rays
            tot_t += dt
        step += 1
        if steps is not None and step == max(warmup, 1) and step <= warmup + 1:
            # size the timed steps from the rate of the steps so far (pixels per second)
            px_rate = npx * step / max(time.perf_counter() - t_start, 1e-6)
            npx = int(min(max(4096, px_rate * target_s / max(steps, 1)), 1 << 20))
        if steps is not None and step >= steps + warmup:
            break
        if steps is None and time.perf_counter() - t_start > seconds:
            break
    sample = (f"{npx} random pixels x 1 sample per step, {len(vals)} steps ({tot_t:.2f} s of CPU time), "
              f"same scene/BVH/env")
    return tot_rays / tot_t / 1e6, cores, sample, vals, kind


def cpu_config_baseline(sc, bvh, full_image, seconds=10.0):
    """The reference shader compiled for the host (oracle/_ref, FP32, all host
    threads) on another scene configuration.  full_image: every pixel at the
    configuration's samples per pixel (its whole render); otherwise a fixed
    seeded subset of 16384 pixels, one sample per pixel and frame, frames
    until about `seconds` have passed, extrapolated to the full render.  The
    reference shader applies its own Russian roulette (after bounce 2,
    renderer.frag:119-123) whatever the configuration asks."""
    from oracle import ref_lib
    if not ref_lib.available("f32"):
        return None
    ref = ref_lib.GlslReference("f32")
    ref.set_scene(sc.vertices, sc.indices, sc.materials, bvh.nodes, bvh.indices)
    ref.set_ibl(sc.env)
    cores = os.cpu_count() or 1
    if full_image:
        ys, xs = np.mgrid[0:sc.height, 0:sc.width]
        xy = np.stack([xs.ravel(), ys.ravel()], 1).astype(np.int32)
    else:
        rng = np.random.default_rng(17)
        xy = np.stack([rng.integers(0, sc.width, 16384), rng.integers(0, sc.height, 16384)], 1).astype(np.int32)
    rays, frames, t = 0, 0, 0.0
    while (full_image and frames < sc.spp) or (not full_image and t < seconds):
        frames += 1
        ref.set_uniforms(ref_lib.uniform_block(sc.camera.matrix_world, sc.camera.fov, sc.camera.near, sc.width,
                                               sc.height, frames, sc.max_bounces))
        t0 = time.perf_counter()
        _, r = ref.render_pixels(xy, sc.width, sc.height, cores)
        t += time.perf_counter() - t0
        rays += r
    samples = xy.shape[0] * frames
    full_s = t * (sc.width * sc.height * sc.spp) / samples
    sample = (f"all {sc.width}x{sc.height} pixels x {frames} spp (the whole render)" if full_image else
              f"{xy.shape[0]} seeded pixels x {frames} spp; full render ({sc.width}x{sc.height} x {sc.spp} spp) "
              f"extrapolated by pixel samples")
    return {"value": rays / t / 1e6, "unit": "Mrays/s", "samples_per_s": samples / t, "cores": cores,
            "kind": "reference", "sample": sample, "cpu_s": t, "full_render_s": full_s}


# ---- batching / serving ---------------------------------------------------------------------
def _load_scene_set(ctx, scenes):
    from dspbr.viewport import Bvh, DeviceIbl, DeviceScene
    out = []
    for sc in scenes:
        sc.bvh = Bvh.build(sc.vertices, sc.indices, 20)
        out.append((DeviceScene(ctx, sc.vertices, sc.indices, sc.materials, sc.bvh), DeviceIbl(ctx, sc.env), sc))
    return out


def _submit(srv, dev, r, out=None):
    from dspbr.viewport import PathtracingCamera
    ds, di, _ = dev[r["scene"]]
    cam = PathtracingCamera(r["camera"].matrix_world, r["camera"].fov, r["camera"].near)
    return srv.submit(ds, di, cam, r["width"], r["height"], r["spp"], {"maxBounces": r["maxBounces"]}, out=out)


def _images(mix):
    """One output image per request, allocated and touched before any timing:
    both arms then time the library, not the host's page faults."""
    outs = []
    for r in mix:
        a = np.empty((r["height"], r["width"], 4), np.float32)
        a.fill(0.0)
        outs.append(a)
    return outs


def _one_at_a_time(ctx, dev, mix):
    """The same requests through the single-viewport API (dspbr_set_scene /
    set_camera / resize / render / read_accum), one after the other, scenes
    resident, each read into its own preallocated image.  Returns per-request
    service times (s) and the images.  The request with the most samples runs
    once untimed first, as the batched arm runs a warm-up request: the
    context's path pool reaches its size and its render graph is captured
    before the timed requests."""
    import ctypes as C
    from dspbr import _lib
    lib, h = ctx.lib, ctx.h
    times, imgs = [], []
    busy = {"device_ms": 0.0, "rays": 0}

    def diag():
        d = _lib.Diag()
        ctx.check(lib.dspbr_get_diagnostics(h, C.byref(d)))
        return d

    big = max(mix, key=lambda r: r["width"] * r["height"] * r["spp"])
    outs = _images([big] + list(mix))
    for k, r in enumerate([big] + list(mix)):
        t0 = time.perf_counter()
        ds, di, _ = dev[r["scene"]]
        p = _lib.default_params()
        p.max_bounces = r["maxBounces"]
        m = np.ascontiguousarray(r["camera"].matrix_world, np.float32).reshape(16)
        ctx.check(lib.dspbr_set_scene(h, ds.h))
        ctx.check(lib.dspbr_set_ibl(h, di.h))
        ctx.check(lib.dspbr_set_params(h, C.byref(p)))
        ctx.check(lib.dspbr_set_camera(h, _lib.fptr(m), float(r["camera"].fov), float(r["camera"].near)))
        ctx.check(lib.dspbr_resize(h, r["width"], r["height"]))
        d0 = diag()
        ctx.check(lib.dspbr_render(h, r["spp"]))
        out = outs[k]
        ctx.check(lib.dspbr_read_accum(h, _lib.fptr(out), out.size))
        if k == 0:
            continue
        times.append(time.perf_counter() - t0)
        imgs.append(out)
        d1 = diag()
        # device time of the render call (CUDA events around it on the context's stream)
        busy["device_ms"] += d1.last_render_ms
        busy["rays"] += sum(getattr(d1, f) - getattr(d0, f) for f in ("rays_primary", "rays_extension",
                                                                      "rays_shadow"))
    wall = sum(times)
    busy.update({"wall_ms": 1e3 * wall, "device_busy_fraction": busy["device_ms"] / (1e3 * wall),
                 "mrays_per_s_wall": busy["rays"] / wall / 1e6,
                 "mrays_per_s_device": busy["rays"] / (busy["device_ms"] * 1e-3) / 1e6})
    _one_at_a_time.busy = busy
    return times, imgs


def _rays(srv):
    st = srv.stats()
    return st["rays_closest"] + st["rays_shadow"]


def _pct(v, q):
    v = sorted(v)
    return float(v[min(len(v) - 1, int(round(q * (len(v) - 1))))]) if v else None


def server_stream(v, sc, steps, dist):
    """The e2e steps through the batch API (dspbr_server_submit / _wait): one
    request per step (its camera in; its 1-spp 1080p image out, into a
    page-locked host buffer), all submitted at once, so that a frame's
    latency-bound tail runs beside the next frames instead of alone.  Every
    step's image is on the host when the timed region ends."""
    from dspbr.server import Server
    from dspbr.viewport import PathtracingCamera
    cam = PathtracingCamera(sc.camera.matrix_world, sc.camera.fov, sc.camera.near)
    settings = {"maxBounces": sc.max_bounces}
    srv = Server(v.ctx)
    outs = [v.ctx.host_array((sc.height, sc.width, 4)) for _ in range(steps)]
    warm = [srv.submit(v._scene, v._ibl, cam, sc.width, sc.height, 1, settings, out=outs[k % steps])
            for k in range(min(3, steps))]
    for i in warm:
        srv.wait(i)
        srv.release(i)
    r0 = _rays(srv)
    barrier(dist)
    t0 = time.perf_counter()
    ids = [srv.submit(v._scene, v._ibl, cam, sc.width, sc.height, 1, settings, out=outs[k]) for k in range(steps)]
    for i in ids:
        srv.wait(i)
    t1 = time.perf_counter()
    rays = _rays(srv) - r0
    for i in ids:
        srv.release(i)
    srv.close()
    value = reduce_sum(dist, float(rays)) / reduce_max(dist, t1 - t0) / 1e6
    return {"value": value, "unit": "Mrays/s", "steps": steps, "h2d_bytes_per_step": 64 + 8 + 4 * 52,
            "d2h_bytes_per_step": int(outs[0].nbytes),
            "api": "dspbr_server_submit / dspbr_server_wait, one 1-spp request per step, submitted together"}


def scene_build_section(local, sc, args):
    """Scene creation (BVH build, 4-wide collapse, upload) of the workload with
    the host binned-SAH builder, the device binned-SAH builder and the device
    LBVH builder, and the render throughput over each tree."""
    from dspbr import synth
    from dspbr.viewport import Context, DeviceScene, PathtracingCamera, PathtracingViewport
    out = {}
    # process warm-up, untimed: each builder's first use loads its kernels
    small = synth.make_small(0)
    for builder in ("device", "device_lbvh"):
        wc = Context(local)
        wc.set_bvh_builder(builder)
        DeviceScene(wc, small.vertices, small.indices, small.materials).close()
        wc.close()
    for builder in ("host", "device", "device_lbvh"):
        v = PathtracingViewport(device=local, width=sc.width, height=sc.height,
                                settings={"maxBounces": sc.max_bounces, "bvhBuilder": builder})
        scene = type(sc)(sc.name, sc.vertices, sc.indices, sc.materials, sc.camera, sc.width, sc.height,
                         env=sc.env)  # no prebuilt BVH: the library builds it
        t0 = time.perf_counter()
        v.setScene(scene)
        t1 = time.perf_counter()
        v.setIBL(sc.env)
        v.setCamera(PathtracingCamera(sc.camera.matrix_world, sc.camera.fov, sc.camera.near))
        lib, h = v.ctx.lib, v.ctx.h
        v.ctx.check(lib.dspbr_render(h, 2))
        d0 = v.diagnostics
        v.ctx.check(lib.dspbr_render(h, max(2, min(args.steps, 10))))
        d1 = v.diagnostics
        rays = sum(d1[k] - d0[k] for k in ("rays_primary", "rays_extension", "rays_shadow"))
        out[builder] = {"scene_create_ms": 1e3 * (t1 - t0), "bvh_build_ms": d1["bvh_build_ms"],
                        "mrays_per_s": rays / (d1["last_render_ms"] * 1e-3) / 1e6, "bvh_nodes": d1["bvh_nodes"]}
        if builder == "device":
            # animated geometry: every vertex moved, the BVH refitted on the device
            moved = sc.vertices.copy()
            moved[:, 1] += (0.5 * np.sin(0.05 * moved[:, 0])).astype(np.float32)
            t2 = time.perf_counter()
            v._scene.update_vertices(moved)
            t3 = time.perf_counter()
            v.ctx.check(lib.dspbr_render(h, 2))
            d2 = v.diagnostics
            v.ctx.check(lib.dspbr_render(h, max(2, min(args.steps, 10))))
            d3 = v.diagnostics
            rays = sum(d3[k] - d2[k] for k in ("rays_primary", "rays_extension", "rays_shadow"))
            out["refit"] = {"update_vertices_ms": 1e3 * (t3 - t2), "vertices": int(moved.shape[0]),
                            "mrays_per_s_after": rays / (d3["last_render_ms"] * 1e-3) / 1e6}
        v.dispose()
    return out


def primary_hit_fraction(v):
    """Fraction of the viewport's camera rays (one per pixel, through the
    pixel's jitter centre) that hit geometry: dspbr_camera_rays, then
    dspbr_trace_closest over the viewport's scene."""
    from dspbr import _lib
    lib, h = v.ctx.lib, v.ctx.h
    ys, xs = np.mgrid[0:v.height, 0:v.width]
    xy = np.ascontiguousarray(np.stack([xs.ravel(), ys.ravel()], 1), np.int32)
    n = xy.shape[0]
    r2 = np.full((n, 2), 0.5, np.float32)
    rays6 = np.zeros((n, 6), np.float32)
    v.ctx.check(lib.dspbr_camera_rays(h, n, _lib.iptr(xy), _lib.fptr(r2), _lib.fptr(rays6)))
    rays8 = np.zeros((n, 8), np.float32)
    rays8[:, :6] = rays6
    rays8[:, 6] = 1e30
    tri, t, uv = np.zeros(n, np.int32), np.zeros(n, np.float32), np.zeros((n, 2), np.float32)
    v.ctx.check(lib.dspbr_trace_closest(h, v._scene.h, _lib.fptr(rays8), n, _lib.iptr(tri), _lib.fptr(t),
                                        _lib.fptr(uv)))
    return float((tri >= 0).mean())


def path_statistics(v, d0, d1):
    """What the frames between diagnostics d0 and d1 traced per path (one path
    per pixel sample): closest-hit segments (camera + extension rays) and
    shadow rays; and the camera rays' hit fraction."""
    prim = max(1, d1["rays_primary"] - d0["rays_primary"])
    return {"primary_hit_fraction": primary_hit_fraction(v),
            "closest_segments_per_path": (prim + d1["rays_extension"] - d0["rays_extension"]) / prim,
            "shadow_rays_per_path": (d1["rays_shadow"] - d0["rays_shadow"]) / prim}


CONFIG_CPU_WHOLE_RENDER = {"small": True, "large_framed": False, "divergence": False}  # True: the whole render


def configs_section(local, args):
    """The other scene configurations at one progressive frame (1 spp) per
    step: "small" (1,324 triangles, 512x512, 8 bounces: BVH and triangles sit
    in L2), "large_framed" (the headline scene and settings seen by a camera
    that frames the instance cloud: 72% of camera rays hit) and "divergence"
    (4M triangles, 60% transmissive / volume / dispersive and 20% iridescent
    materials, 4096x2048 env, 1280x720, 32 bounces, Russian roulette after
    bounce 4).  small and divergence use PCG32 per pixel sample, large_framed
    the headline's MWC; all use the alias-table environment sampling; the BVH
    is built by the library.  Device time of K frames in one render call, the
    k_extend time of the same frames, the reference traversal's node /
    triangle counts of one more frame for the traversal roofline, and the
    reference shader on the host cores (cpu_baseline)."""
    from dspbr import synth
    from dspbr.viewport import PathtracingCamera, PathtracingViewport
    out = {}
    peak, peak_kind = peaks()
    for name in ("small", "large_framed", "divergence"):
        t0 = time.perf_counter()
        sc = synth.WORKLOADS[name](0)
        t1 = time.perf_counter()
        v = PathtracingViewport(device=local, width=sc.width, height=sc.height,
                                settings={"maxBounces": sc.max_bounces,
                                          "russianRouletteStartDepth": sc.rr_start_depth,
                                          "rng": "mwc" if name == "large_framed" else "pcg",
                                          "envSampling": "alias", "wideBvh": WIDE_BVH})
        v.setScene(sc)
        v.setIBL(sc.env)
        v.setCamera(PathtracingCamera(sc.camera.matrix_world, sc.camera.fov, sc.camera.near))
        t2 = time.perf_counter()
        lib, h = v.ctx.lib, v.ctx.h
        k = max(2, min(args.steps, 10))
        v.ctx.check(lib.dspbr_render(h, max(3, args.warmup)))
        d0 = v.diagnostics
        v.ctx.check(lib.dspbr_render(h, k))
        d1 = v.diagnostics
        rays = sum(d1[f] - d0[f] for f in ("rays_primary", "rays_extension", "rays_shadow"))
        ms = d1["last_render_ms"]
        v.ctx.check(lib.dspbr_set_profiling(h, 1))
        v.ctx.check(lib.dspbr_render(h, k))
        dp = v.diagnostics
        v.ctx.check(lib.dspbr_set_profiling(h, 0))
        v.ctx.check(lib.dspbr_set_counting(h, 1))
        dc0 = v.diagnostics
        v.ctx.check(lib.dspbr_render(h, 1))
        dc1 = v.diagnostics
        v.ctx.check(lib.dspbr_set_counting(h, 0))
        alg = 64.0 * dc1["nodes_closest"] + 40.0 * dc1["tris_closest"]
        closest = (dc1["rays_primary"] + dc1["rays_extension"]) - (dc0["rays_primary"] + dc0["rays_extension"])
        ext_ms = dp["extend_ms"] / k
        achieved = alg / (ext_ms * 1e-3) / 1e9 if ext_ms > 0 else None
        out[name] = {
            "triangles": int(sc.num_triangles), "width": sc.width, "height": sc.height,
            "max_bounces": sc.max_bounces, "rr_start_depth": sc.rr_start_depth, "frames": k,
            "mrays_per_s": rays / (ms * 1e-3) / 1e6, "ms_per_frame": ms / k,
            "samples_per_s": sc.width * sc.height * k / (ms * 1e-3),
            "rays_per_frame": rays / k, "traversal_aborted": d1["traversal_aborted"] - d0["traversal_aborted"],
            "paths": path_statistics(v, d0, d1),
            "extend_roofline": {"achieved": achieved, "peak": peak, "unit": "GB/s", "peak_kind": peak_kind,
                                "frac": achieved / peak if achieved else None, "bytes_per_frame": alg,
                                "nodes_per_ray": dc1["nodes_closest"] / max(1, closest),
                                "tris_per_ray": dc1["tris_closest"] / max(1, closest),
                                "extend_ms_per_frame": ext_ms},
            "connect_ms_per_frame": dp["connect_ms"] / k, "shade_ms_per_frame": dp["shade_ms"] / k,
            "scene_gen_s": t1 - t0, "scene_load_s": t2 - t1,
            "full_config_estimate_s": ms / k * sc.spp / 1e3,
        }
        if name == "large_framed":
            out[name]["camera"] = "look_at((-48, 28, -33), (0, 5, -14)), fov 46"
        bvh = v._scene.bvh() if not args.no_cpu_baseline else None
        v.dispose()
        if bvh is not None:
            cpu = cpu_config_baseline(sc, bvh, CONFIG_CPU_WHOLE_RENDER[name])
            if cpu is not None:
                cpu["gpu_ratio"] = out[name]["mrays_per_s"] / cpu["value"]
            out[name]["cpu_baseline"] = cpu
    return out


def gltf_section(local, args):
    """glTF asset to first frame: a ~1.9M-triangle .glb (256 instancing nodes,
    four materials, four 1024x1024 PNG textures) packed by dspbr.gltf
    (scene_loader.ts), then setScene (binned-SAH BVH, 4-wide collapse,
    upload, textures) and setIBL, then frames at 1280x720.  The BVH is built
    by the default builder (the binned SAH on the device); `host_bvh`
    repeats the load with the host builder, which builds the same tree."""
    res = _gltf_first_frame(local, args, "device")
    res["host_bvh"] = {k: x for k, x in _gltf_first_frame(local, args, "host").items()
                       if k in ("load_gltf_ms", "set_scene_ms", "to_first_frame_ms", "mrays_per_s")}
    return res


def _gltf_first_frame(local, args, builder):
    from dspbr import gltf, synth
    from dspbr.viewport import PathtracingCamera, PathtracingViewport
    from dspbr.gltf_writer import large_asset
    glb = large_asset().glb_bytes()
    t0 = time.perf_counter()
    sc = gltf.load_gltf(glb)
    t1 = time.perf_counter()
    v = PathtracingViewport(device=local, width=1280, height=720, settings={"maxBounces": 8, "bvhBuilder": builder})
    v.setScene(sc)
    t2 = time.perf_counter()
    env = synth.make_small(0).env
    v.setIBL(env)
    cam = synth.Camera.look_at((0, 20, 120), (0, 0, 0), fov=45.0, near=0.1)
    v.setCamera(PathtracingCamera(cam.matrix_world, cam.fov, cam.near))
    lib, h = v.ctx.lib, v.ctx.h
    v.ctx.check(lib.dspbr_render(h, 1))
    t3 = time.perf_counter()
    d0 = v.diagnostics
    k = max(2, min(args.steps, 10))
    v.ctx.check(lib.dspbr_render(h, k))
    d1 = v.diagnostics
    v.dispose()
    rays = sum(d1[f] - d0[f] for f in ("rays_primary", "rays_extension", "rays_shadow"))
    return {"file_mb": len(glb) / 1e6, "triangles": int(sc.num_triangles), "materials": int(sc.materials.shape[0]),
            "texture_layers": int(sum(a.shape[0] for a in sc.tex_arrays)),
            "load_gltf_ms": 1e3 * (t1 - t0), "set_scene_ms": 1e3 * (t2 - t1),
            "to_first_frame_ms": 1e3 * (t3 - t0), "mrays_per_s": rays / (d1["last_render_ms"] * 1e-3) / 1e6,
            "ms_per_frame": d1["last_render_ms"] / k}


def serving_section(local, quick=False):
    """Batching (64 viewports over 8 scenes of 10k-2M triangles, 128^2-1024^2,
    1-64 spp) and serving (Poisson arrivals over 16 scenes of 50k-4M
    triangles, 256^2-1920x1080, 16-256 spp, 12 bounces, 120 GB budget) against
    the same requests rendered one at a time."""
    import threading
    from dspbr import synth
    from dspbr.server import Server
    from dspbr.viewport import Context, PathtracingCamera
    ctx = Context(local)
    res = {}
    # ---- batching ----
    t0 = time.perf_counter()
    nb = 8 if not quick else 3
    bdev = _load_scene_set(ctx, synth.scene_set(11, nb, 10_000, 2_000_000 if not quick else 100_000, (1024, 512)))
    mix = synth.request_mix(12, 64 if not quick else 8, nb, 128 * 128, 1024 * 1024, 1, 64, 30.0, 90.0, 12)
    gen_s = time.perf_counter() - t0
    srv = Server(ctx, hbm_budget_bytes=120 << 30)
    samples = []
    for k in range(min(4, len(mix))):
        c = mix[k]["camera"]
        samples.append(srv.request(bdev[mix[k]["scene"]][0], bdev[mix[k]["scene"]][1],
                                   PathtracingCamera(c.matrix_world, c.fov, c.near), 512, 512, 64,
                                   {"maxBounces": 12})[0])
    tuned = srv.autotune(samples, seconds=8.0 if not quick else 2.0)
    # warm-up request (graph capture, memory pool)
    srv.wait(_submit(srv, bdev, dict(mix[0], spp=1)))
    r0 = _rays(srv)
    outs_b = _images(mix)
    t0 = time.perf_counter()
    ids = [_submit(srv, bdev, r, out=outs_b[k]) for k, r in enumerate(mix)]
    done = [srv.wait(i) for i in ids]
    t_batch = time.perf_counter() - t0
    rays_b = _rays(srv) - r0
    lat = [d["done_ms"] - d["submit_ms"] for _, d in done]
    t_single, imgs1 = _one_at_a_time(ctx, bdev, mix)
    diff = max(float(np.max(np.abs(done[k][0] - imgs1[k]))) for k in range(len(mix)))
    spp_total = sum(r["spp"] for r in mix)
    res["batching"] = {
        "requests": len(mix), "scenes": nb, "scene_triangles": [int(d[2].num_triangles) for d in bdev],
        "batched_s": t_batch, "one_at_a_time_s": float(sum(t_single)),
        "requests_per_s": len(mix) / t_batch, "one_at_a_time_requests_per_s": len(mix) / sum(t_single),
        "speedup": float(sum(t_single)) / t_batch,
        "sample_frames_per_s": spp_total / t_batch, "mrays_per_s": rays_b / t_batch / 1e6,
        "p50_ms": _pct(lat, 0.5), "p99_ms": _pct(lat, 0.99),
        "max_abs_diff_vs_one_at_a_time": diff, "scene_gen_s": gen_s,
        "autotuned": {k: tuned[k] for k in ("path_pool", "trace_threads", "trace_blocks", "connect_blocks",
                                            "shade_threads", "shade_blocks", "autotune_source")},
        "one_at_a_time_busy": dict(_one_at_a_time.busy),
        # speedup = (1 / busy fraction of the one-at-a-time arm) x (batched ray
        # rate / the one-at-a-time arm's ray rate while its GPU is busy)
        "speedup_decomposition": {
            "idle_removed": 1.0 / _one_at_a_time.busy["device_busy_fraction"],
            "ray_rate_gain": (rays_b / t_batch / 1e6) / _one_at_a_time.busy["mrays_per_s_device"]}}
    for i in ids:
        srv.release(i)
    for d in bdev:
        d[0].close()
        d[1].close()
    # ---- serving ----
    t0 = time.perf_counter()
    ns = 16 if not quick else 3
    sdev = _load_scene_set(ctx, synth.scene_set(21, ns, 50_000, 4_000_000 if not quick else 100_000, (1024, 512)))
    n = 32 if not quick else 6
    smix = synth.request_mix(22, n, ns, 256 * 256, 1920 * 1080, 16, 256, 30.0, 90.0, 12, aspect_hi=16 / 9)
    gen_s = time.perf_counter() - t0
    t_single, imgs1 = _one_at_a_time(ctx, sdev, smix)
    busy_serving = dict(_one_at_a_time.busy)
    rates = []
    for rate in ((10.0, 50.0, 200.0, 500.0) if not quick else (50.0,)):
        arr = np.cumsum(np.random.default_rng(int(rate)).exponential(1.0 / rate, n))
        outs = _images(smix)
        ids = [None] * n
        r0 = _rays(srv)
        start = time.perf_counter()

        def feeder():
            for k, r in enumerate(smix):
                dt = start + arr[k] - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
                ids[k] = _submit(srv, sdev, r, out=outs[k])

        th = threading.Thread(target=feeder)
        th.start()
        th.join()
        infos = [srv.wait(i)[1] for i in ids]
        span = (max(d["done_ms"] for d in infos) - min(d["submit_ms"] for d in infos)) / 1e3
        lat = [d["done_ms"] - d["submit_ms"] for d in infos]
        # the same arrivals served one at a time (FIFO, measured service times)
        fin, lat1 = 0.0, []
        for a, sv in zip(arr, t_single):
            fin = max(fin, a) + sv
            lat1.append(1e3 * (fin - a))
        span1 = fin - arr[0]
        diff = max(float(np.max(np.abs(outs[k] - imgs1[k]))) for k in range(n))
        rates.append({"rate_req_s": rate, "requests": n, "frames_per_s": n / span,
                      "sample_frames_per_s": sum(r["spp"] for r in smix) / span,
                      "mrays_per_s": (_rays(srv) - r0) / span / 1e6,
                      "p50_ms": _pct(lat, 0.5), "p99_ms": _pct(lat, 0.99),
                      "one_at_a_time": {"frames_per_s": n / span1, "p50_ms": _pct(lat1, 0.5),
                                        "p99_ms": _pct(lat1, 0.99)},
                      "frames_per_s_ratio": (n / span) / (n / span1),
                      "max_abs_diff_vs_one_at_a_time": diff})
        for i in ids:
            srv.release(i)
    st = srv.stats()
    res["serving"] = {"scenes": ns, "scene_triangles": [int(d[2].num_triangles) for d in sdev],
                      "hbm_budget_gb": 120, "bytes_peak": st["bytes_peak"], "scene_gen_s": gen_s,
                      "one_at_a_time_service_s": {"p50": _pct(t_single, 0.5), "max": max(t_single)},
                      "one_at_a_time_busy": busy_serving,
                      "rates": rates}
    srv.close()
    for d in sdev:
        d[0].close()
        d[1].close()
    ctx.close()
    return res


def run_reference_arm(args):
    rank, ws, local, dist = dist_setup()
    if rank != 0:
        return 0
    sc = reference_workload()
    res = cpu_reference_sample(sc, steps=args.steps, warmup=args.warmup)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (reference shaders compiled for the host) "
                                                              "was not built"}))
        return 0
    value, cores, sample, vals, kind = res
    line = {"metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config_of(sc), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_gpu_arm(args):
    rank, ws, local, dist = dist_setup()
    from dspbr import _lib
    from dspbr.viewport import PathtracingViewport, PathtracingCamera

    sc = make_workload()
    v = PathtracingViewport(device=local, width=sc.width, height=sc.height,
                            settings={"maxBounces": sc.max_bounces, "wideBvh": WIDE_BVH})
    v.setScene(sc)
    wide_info = v._scene.wide_bvh()
    v.setIBL(sc.env)
    v.setCamera(PathtracingCamera(sc.camera.matrix_world, sc.camera.fov, sc.camera.near))
    lib, h = v.ctx.lib, v.ctx.h
    # warm-up frames (untimed)
    v.ctx.check(lib.dspbr_render(h, args.warmup))
    # ---- device-timed region: K frames in one render call, events on the
    #      render stream (no per-launch profiling inside it) ----
    v.ctx.check(lib.dspbr_set_profiling(h, 0))  # also zeroes the launch counters
    d0 = v.diagnostics
    barrier(dist)
    with ClockSampler(local) as clocks:
        v.ctx.check(lib.dspbr_render(h, args.steps))
    barrier(dist)
    d1 = v.diagnostics
    dev_ms = d1["last_render_ms"]
    rays = (d1["rays_primary"] + d1["rays_extension"] + d1["rays_shadow"]) - \
           (d0["rays_primary"] + d0["rays_extension"] + d0["rays_shadow"])
    t_max = reduce_max(dist, dev_ms)
    rays_all = reduce_sum(dist, float(rays))
    value = rays_all / (t_max * 1e-3) / 1e6
    gpu_launches = int(d1["extend_launches"] + d1["connect_launches"] + d1["shade_launches"] + d1["other_launches"])

    # ---- per-kernel device time of the same K frames (untimed, events around
    #      every launch), for the roofline of k_extend ----
    v.ctx.check(lib.dspbr_set_profiling(h, 1))
    v.ctx.check(lib.dspbr_render(h, args.steps))
    dp = v.diagnostics
    v.ctx.check(lib.dspbr_set_profiling(h, 0))
    extend_ms = dp["extend_ms"]

    # ---- traversal work of one more frame (untimed), for the roofline ----
    v.ctx.check(lib.dspbr_set_counting(h, 1))
    d1c = v.diagnostics
    v.ctx.check(lib.dspbr_render(h, 1))
    d2 = v.diagnostics
    v.ctx.check(lib.dspbr_set_counting(h, 0))
    alg_bytes_frame = 64.0 * d2["nodes_closest"] + 40.0 * d2["tris_closest"]
    rays_closest_frame = (d2["rays_primary"] + d2["rays_extension"]) - (d1c["rays_primary"] + d1c["rays_extension"])
    peak, peak_kind = peaks()
    ext_ms_frame = extend_ms / max(1, args.steps)
    achieved = alg_bytes_frame / (ext_ms_frame * 1e-3) / 1e9 if ext_ms_frame > 0 else None

    # ---- end to end through the public API: per step camera upload (H2D),
    #      one frame, read back of the accumulation buffer (D2H) ----
    cam = PathtracingCamera(sc.camera.matrix_world, sc.camera.fov, sc.camera.near)
    # the render-ahead loop (the headline) runs every step of the bench; the
    # other forms, measured beside it, 10 steps each
    e2e_steps = max(1, args.steps)
    part_steps = max(1, min(args.steps, 10))
    AHEAD = 16  # accumulations in flight (viewport setting pipelinedFrames)
    # the caller's page-locked frame buffers, reused in turn: step k's image
    # is copied while later steps render, and its buffer is taken again
    # AHEAD + 4 steps later, after readWaitReady() has seen the copy done
    ring = AHEAD + 4
    bufs = [v.allocReadbackBuffer() for _ in range(ring)]
    img = bufs[0]

    def e2e_run(pipelined, ahead=False, steps=part_steps):
        v.resetAccumulation()
        d3 = v.diagnostics
        parts = np.zeros(3)
        barrier(dist)
        t0 = time.perf_counter()
        for k in range(steps):
            ta = time.perf_counter()
            v.setCamera(cam)
            tb = time.perf_counter()
            v.start(1)
            tc = time.perf_counter()
            if ahead:
                # the copies of the frames that have finished are on the
                # host; this frame's copy is enqueued and starts when its
                # last paths have finished, during the next renders
                v.readWaitReady()
                v.readAccumulationAsync(out=bufs[k % ring])
            elif pipelined:
                v.readWait()  # step k-1's image is on the host
                v.readAccumulationAsync(out=bufs[k % 2])
            else:
                v.readAccumulation(out=img)
            td = time.perf_counter()
            parts += (tb - ta, tc - tb, td - tc)
        v.readWait()  # the last steps' images
        t1 = time.perf_counter()
        d4 = v.diagnostics
        rays = (d4["rays_primary"] + d4["rays_extension"] + d4["rays_shadow"]) - \
               (d3["rays_primary"] + d3["rays_extension"] + d3["rays_shadow"])
        value = reduce_sum(dist, float(rays)) / reduce_max(dist, t1 - t0) / 1e6
        iters = (d4["extend_launches"] - d3["extend_launches"]) / steps  # render-loop iterations per step
        return value, parts / steps, iters

    e2e_run(True)  # untimed: the second buffer's first use
    e2e_serial, parts_serial, _ = e2e_run(False)
    e2e_copy, parts_copy, _ = e2e_run(True)
    # pipelined frames: step k+1's samples start while step k's last paths
    # finish; step k's image is copied as soon as they have
    v.setSettings({"pipelinedFrames": True})
    e2e_run(True)  # untimed: the second sum buffer's first use
    e2e_two, parts_two, _ = e2e_run(True)
    v.setSettings({"pipelinedFrames": 3})
    e2e_run(True, ahead=True)  # untimed: the third sum buffer's first use
    e2e_three, parts_three, iters_three = e2e_run(True, ahead=True)
    # the headline: AHEAD accumulations in flight; each render call runs one
    # iteration over the new frame's camera rays and the earlier frames' last
    # paths, and returns while it runs
    v.setSettings({"pipelinedFrames": AHEAD})
    e2e_run(True, ahead=True, steps=2 * AHEAD)  # untimed: every sum buffer's first use
    e2e_value, parts, iters_ahead = e2e_run(True, ahead=True, steps=e2e_steps)
    # device clock between the commits of the loop's last iterations (the
    # steady state: each holds a new frame and the earlier frames' last paths)
    tla = v.timeline(64)
    full = tla[1:, 2] >= 0.5 * tla[:, 2].max() if len(tla) > 1 else np.zeros(0, bool)
    iter_ms = float(np.median(np.diff(tla[:, 1])[full])) if full.any() else None
    v.setSettings({"pipelinedFrames": False})
    e2e_parts = {"set_camera_ms": 1e3 * parts[0], "render_1_frame_ms": 1e3 * parts[1],
                 "read_wait_ready_and_enqueue_ms": 1e3 * parts[2],
                 "loop_iterations_per_step": iters_ahead,
                 "loop_iteration_ms_median": iter_ms,
                 "frames": f"pipelined, {AHEAD} accumulations in flight (viewport setting pipelinedFrames: "
                           f"{AHEAD}): a step's render enqueues one render-loop launch that runs until its "
                           "samples have started and returns without waiting for it; the next step's render "
                           f"waits for it, and for the frame that started {AHEAD - 1} steps earlier",
                 "readback": f"every step enqueues the device-to-host copy of its image into one of {ring} "
                             "page-locked buffers taken in turn; the copy starts when the frame's paths have "
                             "finished and runs beside later renders; each step first waits for the copies "
                             "of the frames that have finished (readWaitReady), the last step for every image",
                 "frames_three_in_flight": {"value": e2e_three, "steps": part_steps,
                                            "render_1_frame_ms": 1e3 * parts_three[1],
                                            "loop_iterations_per_step": iters_three},
                 "frames_two_in_flight": {"value": e2e_two, "steps": part_steps,
                                          "render_1_frame_ms": 1e3 * parts_two[1],
                                          "read_wait_and_enqueue_ms": 1e3 * parts_two[2],
                                          "readback": "step k waits for step k-1's image"},
                 "frames_not_pipelined": {"value": e2e_copy, "steps": part_steps,
                                          "render_1_frame_ms": 1e3 * parts_copy[1],
                                          "read_wait_and_enqueue_ms": 1e3 * parts_copy[2]},
                 "serial": {"value": e2e_serial, "steps": part_steps, "render_1_frame_ms": 1e3 * parts_serial[1],
                            "read_accumulation_ms": 1e3 * parts_serial[2]}}
    # the iterations of one more single-frame call (untimed): device clock at
    # the end of each iteration from the first one's end, and the paths left
    last = v.timeline(1)
    v.setCamera(cam)
    v.start(1)
    tl = v.timeline(256)
    tl = tl[tl[:, 0] > (last[-1, 0] if len(last) else -1)]
    if len(tl):
        e2e_parts["one_frame_iterations"] = [[round(float(r[1] - tl[0, 1]), 4), int(r[2])] for r in tl]
    e2e_parts["server_stream"] = server_stream(v, sc, part_steps, dist)
    cs = clocks.summary()
    paths = path_statistics(v, d0, d1)
    v.dispose()
    build = scene_build_section(local, sc, args) if ws == 1 and not args.no_serving else None
    other = configs_section(local, args) if ws == 1 and not args.no_serving else None
    gltf_load = gltf_section(local, args) if ws == 1 and not args.no_serving else None
    serving = None
    if ws == 1 and not args.no_serving:
        serving = serving_section(local, quick=args.quick_serving)

    if rank == 0:
        cpu = None
        if ws == 1 and not args.no_cpu_baseline:
            # steps sized like the reference arm's (about a second of CPU work
            # each), so that thread start-up is amortised the same way
            r = cpu_reference_sample(sc, steps=4, warmup=1, target_s=12.0)
            if r is not None:
                cpu = {"value": r[0], "unit": "Mrays/s", "cores": r[1], "kind": r[4], "sample": r[2]}
        line = {
            "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene + env map, no assets)",
            "config": config_of(sc),
            "e2e": {"value": e2e_value, "unit": "Mrays/s", "h2d_bytes_per_step": 64 + 8 + 4 * 52,
                    "d2h_bytes_per_step": int(img.nbytes), "steps": e2e_steps,
                    "per_step": e2e_parts},
            "gpu_launches": gpu_launches,
            "wide_bvh": wide_info,
            "roofline": {"bound": "hbm", "kernel": "k_extend (closest-hit traversal)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "peak_kind": peak_kind,
                         "traffic": (extend_traffic_rate() * ext_ms_frame)
                         if extend_traffic_rate() and WIDE_BVH == 4 else None,
                         "traffic_basis": "DRAM bytes per frame of k_extend_dyn: the DRAM bytes per ms of three "
                                          "launches of one ncu capture (profiles/) times this run's k_extend "
                                          "ms per frame; achieved and bytes_per_frame use the reference "
                                          "traversal's node/triangle counts",
                         "bytes_per_frame": alg_bytes_frame, "closest_rays_per_frame": rays_closest_frame,
                         "nodes_per_ray": d2["nodes_closest"] / max(1, rays_closest_frame),
                         "tris_per_ray": d2["tris_closest"] / max(1, rays_closest_frame),
                         "extend_ms_per_frame": ext_ms_frame,
                         "connect_ms_per_frame": dp["connect_ms"] / max(1, args.steps),
                         "shade_ms_per_frame": dp["shade_ms"] / max(1, args.steps),
                         "iterations": int(d1["extend_launches"])},
            "cpu_baseline": cpu,
            "clocks": cs,
            "rays_per_step": rays / max(1, args.steps),
            "paths": paths,
            "traversal_aborted": d1["traversal_aborted"],
        }
        if build is not None:
            line["scene_build"] = build
        if other is not None:
            line["configs"] = other
        if gltf_load is not None:
            line["gltf"] = gltf_load
        if serving is not None:
            line.update(serving)
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="skip the batching / serving sections")
    ap.add_argument("--quick-serving", action="store_true", help="small batching / serving mixes (smoke runs)")
    ap.add_argument("--write-bvh", metavar="PATH", help=argparse.SUPPRESS)
    ap.add_argument("--wide-bvh", type=int, default=4, choices=[4, 8],
                    help="wide BVH of the path kernels: 4 (float boxes, default) or 8 (compressed)")
    args = ap.parse_args()
    global WIDE_BVH
    WIDE_BVH = args.wide_bvh
    if args.write_bvh:
        return write_workload_bvh(args.write_bvh)
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
