"""Throughput of the B200 render path on the mesh workload at 1080p.

Workload (one step = one render of one frame): the noisy-icosphere mesh
scene (level-6 icosphere, 81,920 triangles, f32 vertices displaced +-5% by
seeded value noise; reflective grid plane; one disk light of diameter 2,
16 samples per shading point; fog start 5 / end 50 / density 0.05; outline
on; 50-degree perspective camera) at 1920x1080, max depth 10, seed 0.  The
scene enables outlines, so anti-aliasing is no-jitter, which is the mode the
reference CLI switches to for outlined scenes (cli/src/main.rs:364-376).

Metric: Mrays/s, counting every ray the reference would cast (primary +
reflection + shadow), and ms per frame.  `value` is the device-timed
pipeline with the scene resident; `e2e` is the same metric through the
public API with host buffers: each step uploads the host-side scene, renders
into pinned host memory and frees the device scene.

N > 1 GPUs: one process per GPU, each rendering its own copy of the frame
(replicas, weak scaling); no collective touches the data path.

--impl reference times the CPU restatement of the reference (oracle/,
std::thread over pixels like the reference's rayon loop) on this host's
cores, on bounded row bands of the same frame.
"""
import argparse
import ctypes
import datetime
import json
import math
import os
import signal
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mrays/s & ms/frame at 1080p, learned vs plain shadows at ≥40 dB PSNR, 1 B200"
W, H = 1920, 1080
WORKLOAD = "noisy_icosphere_l6_1080p"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "k_shadow_noisy_icosphere_1080p.md")

# Algorithmic bytes per unit of work of the any-hit (shadow) kernel: every
# shadow ray reads its direction and distance (32 B) and its hit's origin
# (24 B) and writes one visibility byte; each BVH node visit reads one
# single-precision node (64 B: two child boxes and their references), each
# triangle test one triangle record (80 B), each sphere test one sphere
# (40 B), each verification unit one 16-byte k-d record.
B_RAY, B_NODE, B_TRI, B_SPH, B_VERIFY = 57, 64, 80, 40, 16
# FP64 operations per unit (adds, multiplies, divisions and square roots of
# the restated reference formulas): Moller-Trumbore 40, sphere test 22,
# verification unit 2.  Node visits test their boxes in single precision
# (24 FP32 operations for the pair) and count no FP64 operations.
F_NODE, F_TRI, F_SPH, F_VERIFY = 0, 40, 22, 2


def frame_config(world, split):
    """The workload, identical in both arms' JSON lines (the reference arm
    renders the same frame on the CPU)."""
    return {"workload": WORKLOAD, "width": W, "height": H, "anti_aliasing": "no-jitter", "outline": True,
            "samples": 1, "max_depth": 10, "seed": 0, "triangles": 81920, "disk_samples": 16,
            "l2": "GPU arm: 512 MB written before each step (L2 flush)",
            "parallelism": "single" if world == 1 else ("row bands of one frame" if split else "replicas")}


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def make_workload(directory):
    from rtrace_b200 import workloads
    return workloads.make_noisy_icosphere(directory, level=6, seed=7, outline=True)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 20 ms, with
    timestamps.  Started well before the timed region (nvidia-smi takes a
    moment to start); mark() brackets the region, and stop() keeps the
    samples taken inside it."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.path = tempfile.mktemp(prefix="rtb_clocks_", suffix=".csv")
        self.proc = None
        self.window = [None, None]
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(gpu_index), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def mark(self):
        """Call at the start and at the end of the timed region."""
        self.window[0 if self.window[0] is None else 1] = datetime.datetime.now()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.send_signal(signal.SIGTERM)
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        t0, t1 = self.window
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f")
                if t0 is not None and t1 is not None and not (t0 <= ts <= t1):
                    continue
                sm.append(float(parts[2]))
                smax = float(parts[3])
            except ValueError:
                continue
            for n, v in zip(names, parts[6:10]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "interval_ms": 20}


PLAIN_RAYS = 64        # the configuration's plain arm: two area lights sampled 8x8
NOISE_CAP_RAYS = 1024  # a near-noise-free reference, reported beside the 64-ray one


def denoiser_roofline(rt, torch, ctx, feat, hbm, tflops):
    """The network alone on the frame's feature image: CUDA-event time of
    rt_denoiser_run, algorithmic bytes (every op's FP16 input and output
    once, FP32 outputs of the last op; a pooling that the library fuses into
    the convolution before it reads nothing) and FLOPs (2 x 9 x cin x cout
    per output pixel of each convolution), against HBM and the FP16/BF16
    tensor peak."""
    from rtrace_b200 import denoiser
    net = denoiser.unpack_net(denoiser.read_blob())
    P, H, W, _ = feat.shape
    dims = lambda lv: (-(-H // (1 << lv)), -(-W // (1 << lv)))
    ch, lv = [16], [0]
    nbytes, flops = 0.0, 0.0
    fused = 0
    for i, (kind, cin, cout, dil, src, src2) in enumerate(net.ops):
        level = lv[src] + 1 if kind == "pool" else (lv[src2] if kind == "upadd" else lv[src])
        h, w = dims(level)
        hs, ws = dims(lv[src])
        last = i + 1 == len(net.ops)
        prev = net.ops[i - 1] if i > 0 else None
        # the library's rule (denoise_run): a pooling right after the
        # dilation-1 32 -> 32 or 64 -> 64 layer it reads runs in its epilogue
        pooled_in_epilogue = (kind == "pool" and src == i and prev is not None and prev[0] == "conv" and
                              prev[3] == 1 and prev[1] == prev[2] and prev[1] in (32, 64))
        fused += pooled_in_epilogue
        if not pooled_in_epilogue:
            nbytes += P * hs * ws * ch[src] * 2
        nbytes += P * h * w * 16 if last else P * h * w * cout * 2
        if kind == "upadd":
            nbytes += P * h * w * ch[src2] * 2
        if kind == "conv":
            flops += 2.0 * 9 * cin * cout * P * h * w
        ch.append(cout)
        lv.append(level)
    vis = torch.empty((P, 2, H, W), dtype=torch.float32, device=feat.device)
    conf = torch.empty_like(vis)
    L = rt._capi.lib()
    ms = []
    for _ in range(8):
        d = ctypes.c_double()
        st = L.rt_denoiser_run(ctx.handle, feat.data_ptr(), P, H, W, vis.data_ptr(), conf.data_ptr(), ctypes.byref(d))
        if st != 0:
            raise RuntimeError(L.rt_last_error(ctx.handle))
        ms.append(d.value)
    t = sorted(ms[2:])[len(ms[2:]) // 2] * 1e-3
    n_conv = sum(o[0] == "conv" for o in net.ops)
    n_pool = sum(o[0] == "pool" for o in net.ops) - fused
    n_up = sum(o[0] == "upadd" for o in net.ops)
    name = "denoiser network (k_conv3x3_tc x %d, %d of them pooling in the epilogue; k_pool2 x %d, k_upadd x %d)" % (
        n_conv, fused, n_pool, n_up)
    return {"kernel": name,
            "bound": "hbm", "achieved": nbytes / t / 1e9, "peak": hbm, "unit": "GB/s", "frac": nbytes / t / 1e9 / hbm,
            "algorithmic_bytes": nbytes, "ms": t * 1e3, "params": net.param_count,
            "tensor": {"achieved_tflops": flops / t / 1e12, "peak_tflops": tflops,
                       "frac": flops / t / 1e12 / tflops if tflops else None}}


def learned_vs_plain(rt, torch, ctx, directory, steps, hbm=6650.0, tflops=1590.0):
    """The metric's second half, on the 1,000-sphere ring scene (two disk
    lights) at 1920x1080, stochastic, 4 samples per pixel:
      plain_64  every shading point casts 64 rays per disk light (the
                configuration's 8x8 plain arm);
      plain_16  the reference's 16 rays per disk light;
      learned   primary hits cast 1 ray per disk light and the denoiser
                estimates the visibility; hits whose estimated error exceeds
                the network's threshold fall back to the plain path with 64
                rays; reflection hits cast the reference's 16;
      learned_refl64  the same with 64 rays at the reflection hits too.
    Visibility of the primary samples (every hit sample x present light)
    against the plain 64-ray render of the same frame (PSNR and max abs
    error), and against a 1,024-ray render beside it; the network's raw
    input (its 1 ray) and the network without the fallback are scored too.
    Frames are timed with device events, L2 flushed before each."""
    from rtrace_b200 import denoiser, workloads
    if not os.path.exists(denoiser.DEFAULT_WEIGHTS):
        return {"unavailable": "no trained denoiser weights in the package"}
    path = workloads.write_scene(directory, "ring_spheres.json", workloads.ring_spheres_scene(seed=0))
    scene = rt.Scene.from_json_file(path, ctx)
    dev = torch.device("cuda", ctx.device)
    spp = 4
    ctx.load_denoiser()

    def renderer(mode):
        r = rt.Renderer(W, H)
        r.anti_aliasing_mode = rt.AntiAliasingMode.Stochastic
        r.samples = spp
        r.disk_samples = {"plain_64": PLAIN_RAYS, "learned_refl64": PLAIN_RAYS}.get(mode, 16)
        if mode.startswith("learned"):
            r.learned_shadows = True
            r.fallback_samples = PLAIN_RAYS
        if mode == "network_only":
            r.learned_shadows = True
            r.confidence_threshold = -1.0
        return r

    vis = {k: torch.zeros((spp, 2, H, W), dtype=torch.float32, device=dev)
           for k in ("t64", "t1024", "plain_16", "learned", "network_only")}
    feat = torch.zeros((spp, H, W, 16), dtype=torch.float16, device=dev)
    lfeat = torch.zeros((spp, H, W, 16), dtype=torch.float16, device=dev)
    torch.cuda.synchronize(dev)
    # visibility of the primary hits only: depth 1 is enough for the AOVs
    for key, mode, rays, fp in (("t64", "plain_64", PLAIN_RAYS, feat), ("t1024", "plain_64", NOISE_CAP_RAYS, None),
                                ("plain_16", "plain_16", 16, None), ("learned", "learned", None, lfeat),
                                ("network_only", "network_only", None, None)):
        r = renderer(mode)
        r.max_depth = 1
        if rays:
            r.disk_samples = rays
        r.render_shadow_aov(scene, vis[key].data_ptr(), None if fp is None else fp.data_ptr())
        if key == "learned":
            fb_hits, fb_lights, hits = r.last_stats.fallback_hits, r.last_stats.fallback_lights, r.last_stats.hits
    mask = denoiser.masks(feat)
    raw = torch.stack([lfeat[..., 5], lfeat[..., 9]], 1).float()

    def score(v):
        out = {}
        for tk, name in (("t64", "vs_64"), ("t1024", "vs_1024")):
            d = (v[mask] - vis[tk][mask]).abs()
            out[name] = {"psnr_db": denoiser.psnr(v, vis[tk], mask), "max_abs_err": float(d.max().item()),
                         "mean_abs_err": float(d.mean().item())}
        return out

    out = {"workload": "ring_spheres_1000_1080p_4spp", "network": denoiser.unpack_net(denoiser.read_blob()).param_count,
           "target": "visibility of the plain path with %d rays per disk light, same frame and samples" % PLAIN_RAYS,
           "scored_over": "primary-hit samples x present disk lights (%d)" % int(mask.sum().item()),
           "visibility": {"plain_16": score(vis["plain_16"]), "learned": score(vis["learned"]),
                          "network_only": score(vis["network_only"]), "raw_1_ray": score(raw),
                          "plain_64_vs_1024": score(vis["t64"])["vs_1024"]},
           "fallback_share": {"hit_samples": fb_hits / max(1, hits),
                              "sample_lights": fb_lights / max(1, int(mask.sum().item()))},
           "fallback_rays_per_light": PLAIN_RAYS}
    img = torch.empty(W * H * 3, dtype=torch.uint8, device=dev)
    flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device=dev)
    for mode in ("plain_64", "plain_16", "learned", "learned_refl64"):
        r = renderer(mode)
        for _ in range(3):
            r.render(scene, device_ptr=img.data_ptr())
        ms, rays = [], 0
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize(dev)
            r.render(scene, device_ptr=img.data_ptr())
            ms.append(r.last_stats.device_ms)
            rays += r.last_stats.rays
        m = sum(ms) / steps
        out[mode] = {"ms_per_frame": m, "mrays_per_s": rays / (sum(ms) * 1e-3) / 1e6, "rays_per_frame": rays // steps}
        r.flags = 1  # stage times of one more frame
        r.render(scene, device_ptr=img.data_ptr())
        out[mode]["stage_ms"] = {k: round(v, 3) for k, v in r.last_stats.stage_ms.items() if v}
    out["speedup_vs_plain_64"] = out["plain_64"]["ms_per_frame"] / out["learned"]["ms_per_frame"]
    out["speedup_vs_plain_16"] = out["plain_16"]["ms_per_frame"] / out["learned"]["ms_per_frame"]
    out["speedup_refl64_vs_plain_64"] = out["plain_64"]["ms_per_frame"] / out["learned_refl64"]["ms_per_frame"]
    try:
        out["roofline"] = denoiser_roofline(rt, torch, ctx, lfeat, hbm, tflops)
    except Exception as e:
        out["roofline"] = {"unavailable": str(e)}
    scene.close()
    return out


def ring_parity(rt, directory, rows=4):
    """RGB8 agreement of the 1080p ring-scene frame (plain path, 16 rays,
    stochastic 4 spp) with the oracle's render of a band of its rows."""
    import numpy as np
    from rtrace_b200 import workloads
    from tests import oracle_lib
    path = workloads.write_scene(directory, "ring_spheres.json", workloads.ring_spheres_scene(seed=0))
    scene = rt.Scene.from_json_file(path)
    r = rt.Renderer(W, H)
    r.anti_aliasing_mode = rt.AntiAliasingMode.Stochastic
    r.samples = 4
    frame = r.render(scene)
    st_rays, st_ms = r.last_stats.rays, r.last_stats.device_ms
    scene.close()
    y0 = H // 2 - rows // 2
    L = oracle_lib.load()
    band = np.zeros((H, W, 3), np.uint8)
    cnt = np.zeros(6, np.uint64)
    err = ctypes.create_string_buffer(512)
    t = time.perf_counter()
    if L.oracle_render_rows(path.encode(), None, W, H, 2, 4, 10, 0, 1, 0, os.cpu_count() or 1, y0, y0 + rows,
                            band.ctypes.data, None, cnt.ctypes.data, err, 512):
        raise RuntimeError(err.value.decode())
    dt = time.perf_counter() - t
    p = band_parity(frame, band, (y0, y0 + rows), halo=0)
    p["workload"] = "ring_spheres_1000_1080p_4spp (plain, 16 rays)"
    rays = int(cnt[0] + cnt[1] + cnt[2])
    p["cpu_port"] = {"mrays_per_s": rays / dt / 1e6, "rays": rays, "seconds": dt, "cores": os.cpu_count() or 1,
                     "gpu_rays_per_frame": st_rays, "gpu_ms_per_frame": st_ms}
    return p


def batch_run(rt, ctx, directory, steps):
    """The batch configuration: 64 seeded scenes (1-4 point or disk lights,
    0-3 noisy-icosphere meshes of 1,280-81,920 triangles, 0-200 spheres, a
    grid plane) x their 4 auto-camera views = 256 jobs at resolutions drawn
    from 128x128 .. 1920x1080, quincunx (the CLI's default), depth 10.
    The autotuner picks the lane count, the fused group's size limit and the
    fused kernels' grid budgets; the batch is then timed as tuned, without
    the fused group, and on one lane without it (the per-job pipelines run
    one after another); rays counted as the reference casts them."""
    from rtrace_b200 import workloads
    wl = workloads.batch_workload(os.path.join(directory, "batch"), n_scenes=64, seed=0)
    jobs = []
    for path, views in wl:
        scene = rt.Scene.from_json_file(path, ctx)
        for _, cam, (w, h) in views:
            jobs.append(rt.Job(scene, rt.Renderer(w, h), cam))
    tuned = rt.batch_autotune_ex(jobs, ctx=ctx)
    out = {"workload": "batch_64_scenes_x_4_auto_views", "jobs": len(jobs),
           "pixels": int(sum(j.renderer.width * j.renderer.height for j in jobs)), "tuning": tuned,
           "fused_jobs": sum(1 for j in jobs if j.renderer.width * j.renderer.height <= tuned["fuse_pixels"])}
    variants = (("tuned", 0, tuned["fuse_pixels"]), ("unfused", 0, 0), ("one_lane_unfused", 1, 0))
    for name, lanes, fuse in variants:
        rt.batch_tuning(ctx, fuse_pixels=fuse)
        rt.render_batch(jobs, lanes=lanes, ctx=ctx)  # captures the fused group's graph
        ms, rays = [], 0
        for _ in range(steps):
            _, st = rt.render_batch(jobs, lanes=lanes, ctx=ctx)
            ms.append(st.wall_ms)
            rays = st.rays
        ms.sort()
        med = ms[len(ms) // 2]
        out[name] = {"lanes": st.lanes, "fuse_pixels": fuse, "ms_per_batch": med,
                     "mrays_per_s": rays / (med * 1e-3) / 1e6, "rays_per_batch": rays}
    rt.batch_tuning(ctx, fuse_pixels=tuned["fuse_pixels"])
    out["speedup_vs_one_lane_unfused"] = out["one_lane_unfused"]["ms_per_batch"] / out["tuned"]["ms_per_batch"]
    out["timing"] = "host wall time of rt_render_batch (median of %d), scenes resident" % steps
    return out


def small_scene_run(rt, ctx, directory, reps, with_cpu):
    """The small configuration: one sphere over a grid-textured reflective
    plane, one point light, orthographic camera, 400x300 quincunx (the
    library call; the CLI's diagonal rule would give a square image), depth
    10, seed 0.  Device time per frame on the GPU and, when asked, the
    whole frame on the CPU restatement (oracle, all host threads)."""
    from rtrace_b200 import _capi, workloads
    path = workloads.write_scene(directory, "sphere_grid.json", workloads.sphere_grid_scene())
    scene = rt.Scene.from_json_file(path, ctx)
    r = rt.Renderer(400, 300)
    out = {"workload": "sphere_grid_400x300_quincunx"}
    # launched directly, then as a replayed CUDA graph (RT_FLAG_CUDA_GRAPH):
    # the frame is ~50 short launches, so submission cost shows
    for mode, flags in (("direct", 0), ("graph", _capi.RT_FLAG_CUDA_GRAPH)):
        r.flags = flags
        for _ in range(3):
            r.render(scene)
        ms, rays, call_ms = 0.0, 0, 0.0
        for _ in range(reps):
            r.render(scene)
            ms += r.last_stats.device_ms
            call_ms += r.last_stats.total_ms
            rays += r.last_stats.rays
        res = {"ms_per_frame": ms / reps, "mrays_per_s": rays / (ms * 1e-3) / 1e6, "call_ms": call_ms / reps,
               "kernel_launches": r.last_stats.kernel_launches}
        if mode == "direct":
            out.update(res)
            out["rays_per_frame"] = rays // reps
        else:
            res["replayed"] = r.last_stats.graph == 2
            out["graph"] = res
    if with_cpu:
        from tests import oracle_lib
        t = time.perf_counter()
        oracle_lib.render(path, width=400, height=300, aa="quincunx", threads=os.cpu_count() or 1)
        out["cpu_port_ms_per_frame"] = 1e3 * (time.perf_counter() - t)
        out["cpu_port_cores"] = os.cpu_count() or 1
    scene.close()
    return out


def large_mesh_run(rt, ctx, directory, reps):
    """The large-mesh configuration: a 1024x1024 fractal-noise heightfield
    (2,093,058 triangles, f32 STL), a mirror sphere (r 20, reflectivity
    0.9), one disk light (16 rays), fog density 0.02, outline on, rendered
    from its four auto-camera views at 3840x2160, no-jitter (outlines),
    depth 10.  Reports the scene load (JSON + STL + the reference's k-d
    build) with the k-d tree built on the host and on the device, the first
    upload (mesh search data prepared on the device), the wall time from
    load to the first 4K frame, and the device time per frame."""
    from rtrace_b200 import workloads
    path = workloads.make_terrain(os.path.join(directory, "terrain"), n=1024, seed=11)
    t0 = time.perf_counter()
    host_only = rt.HostScene.from_json_file(path)  # k-d tree built on the host threads
    t_host = time.perf_counter() - t0
    host_only.close()
    # time to first frame: load with the k-d tree built on the device, the
    # first upload (mesh search data prepared on the device), one 4K view
    t0 = time.perf_counter()
    host = rt.HostScene.from_json_file(path, ctx=ctx)
    t1 = time.perf_counter()
    scene = rt.Scene.upload(host, ctx)
    t2 = time.perf_counter()
    first = rt.Renderer(3840, 2160)
    first.anti_aliasing_mode = rt.AntiAliasingMode.NoJitter
    first.outline_config = scene.get_outline_config()
    img = first.render(scene)
    t3 = time.perf_counter()
    t_dev = t1 - t0
    png_ms = []
    for _ in range(3):  # Renderer::render_to_file's encode (rt_png_write's level)
        t = time.perf_counter()
        rt.encode_png(img, 1)
        png_ms.append((time.perf_counter() - t) * 1e3)
    cams = rt.auto_cameras(path=path)
    jobs = []
    for view in ("left", "front", "top", "perspective"):
        r = rt.Renderer(3840, 2160)
        r.anti_aliasing_mode = rt.AntiAliasingMode.NoJitter
        r.outline_config = scene.get_outline_config()
        jobs.append(rt.Job(scene, r, cams[view]))
    rt.render_batch(jobs, lanes=1, ctx=ctx)  # warm-up (scratch for 4K)
    ms, rays, frames = 0.0, 0, 0
    for _ in range(reps):
        rt.render_batch(jobs, lanes=1, ctx=ctx)
        for j in jobs:
            ms += j.renderer.last_stats.device_ms
            rays += j.renderer.last_stats.rays
            frames += 1
    learned = None
    try:
        learned = terrain_learned(rt, ctx, scene, cams, reps)
    except Exception as e:  # report, do not lose the rest
        learned = {"unavailable": "failed: %s" % e}
    out = {"workload": "terrain_1024_4k_4_auto_views", "triangles": 2 * 1023 * 1023, "learned_vs_plain": learned,
           "host_load_s": t_host, "load_with_device_kd_s": t_dev, "first_upload_s": t2 - t1,
           "time_to_first_frame_s": t3 - t0, "png_encode_ms": min(png_ms), "png_threads": os.cpu_count(),
           "device_bytes": scene.device_bytes,
           "ms_per_frame": ms / frames, "mrays_per_s": rays / (ms * 1e-3) / 1e6, "rays_per_frame": rays // frames,
           "timing": "CUDA events per render, 4 views x %d" % reps}
    scene.close()
    host.close()
    return out


def terrain_learned(rt, ctx, scene, cams, reps):
    """The large-mesh configuration's learned arm: the four 4K views with
    the plain path at 64 rays per disk light (8x8) and 16 (the reference's),
    and learned shadows (1 ray per disk light at primary hits, the
    denoiser, the plain 64-ray fallback where it is not confident, 16 rays
    at reflection hits); device time per frame.  Visibility of the primary
    hits from the scene's own camera against its plain 64-ray render."""
    import torch
    from rtrace_b200 import denoiser
    if not os.path.exists(denoiser.DEFAULT_WEIGHTS):
        return {"unavailable": "no trained denoiser weights in the package"}
    ctx.load_denoiser()
    dev = torch.device("cuda", ctx.device)
    Wt, Ht = 3840, 2160
    img = torch.empty(Wt * Ht * 3, dtype=torch.uint8, device=dev)

    def renderer(mode, cam_view):
        r = rt.Renderer(Wt, Ht)
        r.anti_aliasing_mode = rt.AntiAliasingMode.NoJitter
        r.outline_config = scene.get_outline_config()
        r.disk_samples = 64 if mode == "plain_64" else 16
        if mode == "learned":
            r.learned_shadows = True
            r.fallback_samples = 64
        return r

    out = {"views": ["left", "front", "top", "perspective"]}
    for mode in ("plain_64", "plain_16", "learned"):
        ms, rays, fb, hits = 0.0, 0, 0, 0
        for view in out["views"]:
            job = rt.Job(scene, renderer(mode, view), cams[view])
            rt.render_batch([job], lanes=1, ctx=ctx)  # warm-up (scratch, weights)
            for _ in range(reps):
                rt.render_batch([job], lanes=1, ctx=ctx)
                st = job.renderer.last_stats
                ms += st.device_ms
                rays += st.rays
                fb += st.fallback_hits
        frames = reps * 4
        out[mode] = {"ms_per_frame": ms / frames, "mrays_per_s": rays / (ms * 1e-3) / 1e6}
        if mode == "learned":
            out[mode]["fallback_hits_per_frame"] = fb / frames
    out["speedup_vs_plain_64"] = out["plain_64"]["ms_per_frame"] / out["learned"]["ms_per_frame"]
    out["speedup_vs_plain_16"] = out["plain_16"]["ms_per_frame"] / out["learned"]["ms_per_frame"]
    # visibility from the scene's own camera, at 4K
    vis = {}
    feat = torch.zeros((1, Ht, Wt, 16), dtype=torch.float16, device=dev)
    for key, mode in (("t64", "plain_64"), ("learned", "learned")):
        r = renderer(mode, None)
        r.max_depth = 1
        vis[key] = torch.zeros((1, 2, Ht, Wt), device=dev)
        torch.cuda.synchronize(dev)
        r.render_shadow_aov(scene, vis[key].data_ptr(), feat.data_ptr() if key == "t64" else None)
        if key == "learned":
            out["fallback_share"] = {"hit_samples": r.last_stats.fallback_hits / max(1, r.last_stats.hits),
                                     "fallback_lights": r.last_stats.fallback_lights}
    m = denoiser.masks(feat)
    out["vis_psnr_db_vs_64"] = denoiser.psnr(vis["learned"], vis["t64"], m)
    out["vis_max_abs_err_vs_64"] = float((vis["learned"][m] - vis["t64"][m]).abs().max().item())
    out["note"] = "the network is trained on the ring-sphere generator; the terrain is outside its training set"
    return out


def read_profile(path):
    """The `name: value` figure lines of a committed ncu summary (DRAM
    traffic per frame, issue-slot and cache hit rates of the kernel)."""
    out = {}
    try:
        for line in open(path):
            name, sep, val = line.partition(":")
            if sep and name.strip() in ("traffic_bytes_per_frame", "issue_slots_busy", "l2_hit_rate",
                                        "l1_hit_rate", "tensor_pipe_active", "dram_throughput"):
                try:
                    out[name.strip()] = float(val)
                except ValueError:
                    pass
    except OSError:
        pass
    return out


def cpu_baseline(scene_path, budget_s, threads, centre=None):
    """Mrays/s of the CPU restatement of the reference on a band of rows
    centred on row `centre` (default: the middle) and sized to take about
    budget_s seconds.  Also returns the band's pixels ("img": the full
    frame's array with only those rows rendered, "rows": (y0, y1)) for the
    parity check against the GPU frame."""
    from tests import oracle_lib
    import numpy as np
    L = oracle_lib.load()
    err = ctypes.create_string_buffer(512)

    def band(y0, y1, out):
        cnt = np.zeros(6, np.uint64)
        t = time.perf_counter()
        rc = L.oracle_render_rows(scene_path.encode(), None, W, H, 0, 1, 10, 0, 1, 1, threads, y0, y1,
                                  out.ctypes.data, None, cnt.ctypes.data, err, 512)
        if rc:
            raise RuntimeError(err.value.decode())
        return time.perf_counter() - t, int(cnt[0] + cnt[1] + cnt[2])

    mid = H // 2 if centre is None else min(max(int(centre), 1), H - 1)
    out = np.zeros((H, W, 3), np.uint8)
    dt, rays = band(mid - 1, mid + 1, out)  # calibration
    per_row = max(dt / 2.0, 1e-4)
    rows = int(max(4, min(H, budget_s / per_row)))
    y0 = min(max(0, mid - rows // 2), H - rows)
    dt, rays = band(y0, y0 + rows, out)
    return {"value": rays / dt / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "port",
            "sample": "rows %d-%d of the %dx%d frame (%d rays, %.1f s), CPU restatement of the reference, "
                      "%d threads" % (y0, y0 + rows, W, H, rays, dt, threads),
            "rays": rays, "seconds": dt, "img": out, "rows": (y0, y0 + rows)}


def band_parity(frame, band, rows, halo=1):
    """RGB8 agreement of the GPU frame with the oracle's band of the same
    frame.  The oracle renders only the band, so the outline stencil at its
    first and last `halo` rows lacks the neighbours' G-buffer: those rows
    are left out."""
    import numpy as np
    y0, y1 = rows[0] + halo, rows[1] - halo
    diff = np.abs(frame[y0:y1].astype(np.int16) - band[y0:y1].astype(np.int16)).max(2)
    n, bad = int(diff.size), int((diff > 0).sum())
    return {"rows": "%d-%d" % (y0, y1), "pixels": n, "identical_px_frac": (n - bad) / n if n else None,
            "max_lsb": int(diff.max()) if n else None, "checker": "oracle (CPU restatement of the reference)"}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    d = tempfile.mkdtemp(prefix="rtb_ref_")
    path = make_workload(d)
    threads = os.cpu_count() or 1
    # each step: a row band sized so that warm-up + steps take ~2 minutes;
    # step k's band is centred at row (k + 0.5) H / steps, so that the
    # steps together sample the whole frame, top to bottom
    per_step = max(2.0, 120.0 / max(1, args.steps + args.warmup))
    for _ in range(args.warmup):
        cpu_baseline(path, min(per_step, 5.0), threads)
    tot_rays, tot_s, samples = 0, 0.0, []
    for k in range(args.steps):
        r = cpu_baseline(path, per_step, threads, centre=(k + 0.5) * H / args.steps)
        tot_rays += r["rays"]
        tot_s += r["seconds"]
        samples.append("%d-%d" % r["rows"])
    value = tot_rays / tot_s / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": frame_config(world, args.split == "rows"),
        "step": "a band of rows of the frame on the CPU (%.0f s each), bands spread over the frame" % per_step,
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": threads, "kind": "port",
                         "sample": "rows %s of the %dx%d frame (%d rays, %.1f s), CPU restatement of the "
                                   "reference, %d threads" % (", ".join(samples), W, H, tot_rays, tot_s, threads)},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-vs-plain shadow comparison")
    ap.add_argument("--no-batch", action="store_true", help="skip the 256-job batch measurement")
    ap.add_argument("--no-large", action="store_true", help="skip the 2-million-triangle terrain measurement")
    ap.add_argument("--split", default="replicas", choices=["replicas", "rows"],
                    help="N > 1: every rank renders its own frame (replicas, weak scaling) or one frame is "
                         "split into row bands gathered to rank 0 (rows, strong scaling)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank, world, local = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import numpy as np
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    import rtrace_b200 as rt
    from rtrace_b200 import _capi
    from rtrace_b200.distributed import reduce_timings

    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = torch.device("cuda", local)
    d = tempfile.mkdtemp(prefix="rtb_bench_%d_" % rank)
    path = make_workload(d)

    ctx = rt.Context(local)
    scene = rt.Scene.from_json_file(path, ctx)
    r = rt.Renderer(W, H)
    r.anti_aliasing_mode = rt.AntiAliasingMode.NoJitter
    r.outline_config = scene.get_outline_config()
    out = torch.empty(W * H * 3, dtype=torch.uint8, device=dev)
    flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device=dev)  # > L2 (126 MB)

    clocks = ClockSampler(local)  # running well before the timed region
    for _ in range(args.warmup):
        r.render(scene, device_ptr=out.data_ptr())
    # profiling renders (not timed): the work counters come from a render
    # with the counting kernels, the stage times from plain kernels (mean
    # of three renders, L2 flushed before each), so the roofline divides
    # the counted work by the time of the kernels the timed frames run
    r.flags = _capi.RT_FLAG_COUNT_WORK
    r.render(scene, device_ptr=out.data_ptr())
    prof = r.last_stats
    r.flags = _capi.RT_FLAG_STAGE_TIMES
    stage_sum = {}
    for _ in range(3):
        flush.zero_()
        torch.cuda.synchronize(dev)
        r.render(scene, device_ptr=out.data_ptr())
        for k, v in r.last_stats.stage_ms.items():
            stage_sum[k] = stage_sum.get(k, 0.0) + v / 3
    # timed frames replay the frame's launch sequence as a CUDA graph
    # (RT_FLAG_CUDA_GRAPH; the same kernels, one submission); captured here
    r.flags = _capi.RT_FLAG_CUDA_GRAPH
    r.render(scene, device_ptr=out.data_ptr())

    split = world > 1 and args.split == "rows"
    if split:
        from rtrace_b200.distributed import render_frame
        for _ in range(2):  # warm-up of the band render and the gather
            render_frame(r, scene)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    dev_ms, rays, launches = 0.0, 0, 0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks.mark()
    wall0 = time.perf_counter()
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        if split:
            # this rank's band (rendered on the context's stream, which the
            # call waits for) and the gather to rank 0, between two events
            # on the current stream
            ev0.record()
            render_frame(r, scene)
            ev1.record()
            ev1.synchronize()
            dev_ms += ev0.elapsed_time(ev1)
        else:
            r.render(scene, device_ptr=out.data_ptr())
            dev_ms += r.last_stats.device_ms
        st = r.last_stats
        rays += st.rays
        launches += st.kernel_launches
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    wall_s = time.perf_counter() - wall0
    clocks.mark()
    clk = clocks.stop()
    frame = out.cpu().numpy().reshape(H, W, 3) if not split else None

    # end to end through the public API: upload the host scene, render into
    # pinned host memory, free
    host = rt.HostScene.from_json_file(path)
    pinned = torch.empty((H, W, 3), dtype=torch.uint8, pin_memory=True)
    pin_np = pinned.numpy()

    def e2e_step():
        sc = rt.Scene.upload(host, ctx)
        if split:
            img = render_frame(r, sc)  # this rank's band, gathered to rank 0 (host array there)
            if rank == 0:
                pin_np[...] = img
        else:
            r.render(sc, out=pin_np)
        nbytes = sc.device_bytes
        sc.close()
        return nbytes

    for _ in range(2):
        e2e_step()
    e2e_s, e2e_rays, h2d = 0.0, 0, 0
    if world > 1:
        dist.barrier()
    for _ in range(args.steps):
        t = time.perf_counter()
        h2d = e2e_step()
        e2e_s += time.perf_counter() - t
        e2e_rays += r.last_stats.rays

    # max over ranks of the device time, sum of the work
    (dev_ms_max, e2e_s_max), (rays_all, e2e_rays_all) = reduce_timings([dev_ms, e2e_s], [rays, e2e_rays],
                                                                        device=dev)
    value = rays_all / (dev_ms_max * 1e-3) / 1e6
    e2e_value = e2e_rays_all / e2e_s_max / 1e6

    if rank == 0:
        # roofline of the dominant kernel (the shadow any-hit kernel)
        stages = stage_sum
        dom = max(stages, key=lambda k: stages[k])
        w = prof.work
        sh_bytes = (prof.shadow_rays * B_RAY + w["shadow_nodes"] * B_NODE + w["shadow_triangles"] * B_TRI +
                    w["shadow_spheres"] * B_SPH + w["shadow_verifications"] * B_VERIFY)
        sh_flops = (w["shadow_nodes"] * F_NODE + w["shadow_triangles"] * F_TRI + w["shadow_spheres"] * F_SPH +
                    w["shadow_verifications"] * F_VERIFY)
        sh_s = stages["shadow"] * 1e-3
        try:
            peaks = json.load(open(PEAKS))
            hbm, peak_src = float(peaks["hbm_gbs"]), "measured"
        except (OSError, KeyError, ValueError):
            hbm, peak_src = 6650.0, "fallback"
        fp64 = rt.fp64_rate(ctx)
        l2 = max(rt.l2_read_bandwidth(ctx, mb, 40) for mb in (24, 48))
        achieved = sh_bytes / sh_s / 1e9 if sh_s > 0 else None
        pf = read_profile(TRAFFIC_FILE)
        traffic = pf.get("traffic_bytes_per_frame")
        roofline = {"kernel": "k_shadow", "bound": "l2", "achieved": achieved, "peak": l2, "unit": "GB/s",
                    "frac": achieved / l2 if achieved else None,
                    "peak_source": "measured in this run: L2-resident read bandwidth (rt_debug_l2_read_bandwidth, "
                                   "24 and 48 MB buffers, the larger figure)",
                    "frac_l2": achieved / l2 if achieved else None,
                    "peak_hbm": hbm, "peak_hbm_source": peak_src,
                    "frac_hbm": achieved / hbm if achieved else None,
                    "dram_frac_hbm": traffic / sh_s / 1e9 / hbm if traffic and sh_s > 0 else None,
                    "issue_busy": pf.get("issue_slots_busy"), "l2_hit_rate": pf.get("l2_hit_rate"),
                    "l1_hit_rate": pf.get("l1_hit_rate"),
                    "limiter": "latency of the chained BVH node loads (ncu: issue slots about half busy, "
                               "long-scoreboard stalls dominate); the working set is L2-resident",
                    "traffic": traffic, "traffic_unit": "DRAM bytes per frame (all k_shadow launches)",
                    "algorithmic_bytes_per_frame": sh_bytes, "kernel_ms_per_frame": stages["shadow"],
                    "dominant_stage": dom,
                    "fp64": {"achieved_gops": sh_flops / sh_s / 1e9 if sh_s > 0 else None,
                             "peak_gops": fp64, "peak_source": "measured FP64 add/mul issue rate (k_fp64_rate)",
                             "frac": (sh_flops / sh_s / 1e9) / fp64 if sh_s > 0 and fp64 else None}}
        cpu, parity = None, None
        if world == 1 and not args.no_cpu_baseline:
            try:
                cpu = cpu_baseline(path, args.cpu_seconds, os.cpu_count() or 1)
                cpu.pop("rays", None)
                cpu.pop("seconds", None)
                parity = band_parity(frame, cpu.pop("img"), cpu.pop("rows"))
            except Exception as e:  # the oracle is test infrastructure; report, do not fail
                cpu = {"value": None, "unit": "Mrays/s", "cores": os.cpu_count(), "kind": "port",
                       "sample": "failed: %s" % e}
        learned = None
        if world == 1 and not args.no_learned:
            try:
                tf = None
                try:
                    tf = float(json.load(open(PEAKS)).get("bf16_tflops"))
                except (OSError, TypeError, ValueError):
                    tf = 1590.0
                learned = learned_vs_plain(rt, torch, ctx, d, min(args.steps, 10), hbm, tf)
            except Exception as e:  # report, do not lose the headline line
                learned = {"unavailable": "failed: %s" % e}
        if isinstance(learned, dict) and isinstance(learned.get("roofline"), dict):
            roofline["conv"] = learned["roofline"]  # the learned form's tensor-core network
        if world == 1 and not args.no_cpu_baseline and parity is not None:
            try:
                parity = {"headline_frame": parity, "ring_scene": ring_parity(rt, d)}
            except Exception as e:
                parity = {"headline_frame": parity, "ring_scene": {"unavailable": "failed: %s" % e}}
        small = None
        if world == 1:
            try:
                small = small_scene_run(rt, ctx, d, 20, not args.no_cpu_baseline)
            except Exception as e:
                small = {"unavailable": "failed: %s" % e}
        large = None
        if world == 1 and not args.no_large:
            try:
                large = large_mesh_run(rt, ctx, d, 2)
            except Exception as e:
                large = {"unavailable": "failed: %s" % e}
        batch = None
        if world == 1 and not args.no_batch:
            try:
                batch = batch_run(rt, ctx, d, 3)
            except Exception as e:
                batch = {"unavailable": "failed: %s" % e}
        line = {
            "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
            "scaling": "strong" if split else "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": frame_config(world, split),
            "rays_per_frame": rays_all / (1 if split else world) / args.steps,
            "launch": ("each rank's band of the frame, then a gather to rank 0 (NCCL)" if split else
                       "CUDA graph replay of the frame's kernels (RT_FLAG_CUDA_GRAPH)"),
            "ms_per_frame": dev_ms_max / args.steps,
            "parity": parity,
            "wall_ms_per_step": 1e3 * wall_s / args.steps,
            "gpu_launches": launches,
            "e2e": {"value": e2e_value, "unit": "Mrays/s", "ms_per_frame": 1e3 * e2e_s_max / args.steps,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": W * H * 3},
            "roofline": roofline,
            "stage_ms": {k: round(v, 4) for k, v in stages.items()},
            "work_per_frame": w,
            "shadow_rays_untraced_per_frame": prof.shadow_rays_untraced,
            "cpu_baseline": cpu,
            "learned_vs_plain": learned,
            "batch": batch,
            "large_mesh": large,
            "small_scene": small,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
