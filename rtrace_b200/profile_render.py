"""Renders one of the benchmark workloads a few times, for profiler captures.

    python -m rtrace_b200.profile_render --workload noisy_icosphere --width 960 --height 540 --reps 1
    python -m rtrace_b200.profile_render --workload ring_spheres --width 1920 --height 1080 --learned --fallback-samples 64
    python -m rtrace_b200.profile_render --kd-build terrain --reps 2
    python -m rtrace_b200.profile_render --train-steps 3
    python -m rtrace_b200.profile_render --denoiser-net 3 --width 1920 --height 1080

Workloads (see rtrace_b200.workloads): sphere_grid (quincunx), noisy_icosphere
(no-jitter + outline, the bench.py scene), ring_spheres (stochastic, 4 spp).
Scene files are written to --dir (default: a temporary directory).
--kd-build builds the k-d tree of a workload's mesh (terrain: the 1024x1024
heightfield, 2,093,058 triangles; icosphere: the level-6 noisy icosphere)
on the device --reps times after one warm-up build of 1,000 of its
triangles, checks it against the host build, then uploads the scene once
(the mesh's search data prepared on the device).
--denoiser-net runs the shipped denoiser network on seeded features of
4 sample planes at --width x --height (what a learned render's network pass
reads), printing its CUDA-event times.
--train-steps runs that many steps of the denoiser's training on the
library's kernels, on a batch of 16 seeded random 256x256 feature crops.
"""
import argparse
import json
import os
import sys
import tempfile


def main(argv=None):
    import rtrace_b200 as rt
    from rtrace_b200 import workloads
    ap = argparse.ArgumentParser(description="render a benchmark workload for profiling")
    ap.add_argument("--workload", default="noisy_icosphere", choices=["sphere_grid", "noisy_icosphere", "ring_spheres"])
    ap.add_argument("--width", type=int, default=960)
    ap.add_argument("--height", type=int, default=540)
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--dir", default=None)
    ap.add_argument("--disk-samples", type=int, default=16, help="shadow rays per disk light (16: the reference)")
    ap.add_argument("--learned", action="store_true", help="learned soft shadows with the shipped denoiser weights")
    ap.add_argument("--fallback-samples", type=int, default=0,
                    help="rays per disk light where a learned render falls back (0: --disk-samples)")
    ap.add_argument("--kd-build", default=None, choices=["terrain", "icosphere"])
    ap.add_argument("--train-steps", type=int, default=0)
    ap.add_argument("--denoiser-net", type=int, default=0, metavar="REPS",
                    help="run the shipped denoiser network REPS times on 4 planes of seeded "
                         "--width x --height features (rt_denoiser_run)")
    a = ap.parse_args(argv)
    d = a.dir or tempfile.mkdtemp(prefix="rtb_prof_")
    if a.kd_build:
        return kd_build(rt, workloads, a.kd_build, d, a.reps)
    if a.train_steps:
        return train_steps(rt, a.train_steps)
    if a.denoiser_net:
        return denoiser_net(rt, a.width, a.height, a.denoiser_net)
    if a.workload == "sphere_grid":
        path, aa, spp = workloads.write_scene(d, "sphere_grid.json", workloads.sphere_grid_scene()), 1, 1
    elif a.workload == "noisy_icosphere":
        path, aa, spp = workloads.make_noisy_icosphere(d, level=6, seed=7), 0, 1
    else:
        path, aa, spp = workloads.write_scene(d, "ring_spheres.json", workloads.ring_spheres_scene(seed=0)), 2, 4
    scene = rt.Scene.from_json_file(path)
    r = rt.Renderer(a.width, a.height)
    r.anti_aliasing_mode = rt.AntiAliasingMode(aa)
    r.samples = spp
    if aa != 1:
        r.outline_config = scene.get_outline_config()
    r.disk_samples = a.disk_samples
    if a.learned:
        scene._ctx.load_denoiser()
        r.learned_shadows = True
        r.fallback_samples = a.fallback_samples
    for _ in range(a.reps):
        r.render(scene)
    st = r.last_stats
    print(json.dumps({"workload": a.workload, "width": a.width, "height": a.height, "rays": st.rays,
                      "device_ms": st.device_ms}))
    return 0


def denoiser_net(rt, W, H, reps, planes=4):
    import ctypes
    import torch
    ctx = rt.default_context(0)
    ctx.load_denoiser()
    g = torch.Generator(device="cpu").manual_seed(0)
    f = torch.rand((planes, H, W, 16), generator=g) * 2 - 0.5
    f[..., 0] = 1.0
    feat = f.half().cuda()
    vis = torch.empty((planes, 2, H, W), device="cuda")
    conf = torch.empty_like(vis)
    torch.cuda.synchronize()
    L = rt._capi.lib()
    ms = []
    for _ in range(reps):
        d = ctypes.c_double()
        st = L.rt_denoiser_run(ctx.handle, feat.data_ptr(), planes, H, W, vis.data_ptr(), conf.data_ptr(),
                               ctypes.byref(d))
        if st != 0:
            msg = L.rt_last_error(ctx.handle)
            raise RuntimeError("rt_denoiser_run failed: %s" % (msg.decode() if msg else st))
        ms.append(d.value)
    torch.cuda.synchronize()
    # checksums of the outputs: equal across builds that compute the same bytes
    print(json.dumps({"denoiser_net": reps, "planes": planes, "width": W, "height": H,
                      "ms_min": min(ms), "ms_median": sorted(ms)[len(ms) // 2],
                      "vis_sum": float(vis.double().sum()), "conf_sum": float(conf.double().sum())}))
    return 0


def train_steps(rt, steps):
    import time
    import torch
    from rtrace_b200 import denoiser
    from rtrace_b200.dn_train import Trainer
    ctx = rt.default_context(0)
    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(0)
    f = torch.rand((16, 256, 256, 16), generator=g) * 2 - 0.5
    f[..., 0] = 1.0
    f[..., 8] = 1.0
    f[..., 12] = 1.0
    feats = f.half().to(dev)
    targs = torch.rand((16, 2, 256, 256), generator=g).half().to(dev)
    tr = Trainer(ctx, denoiser.random_net(0), 16, 256, 256)
    tr.step(feats, targs, 1e-3, want_loss=True)
    t = time.perf_counter()
    for _ in range(steps):
        loss = tr.step(feats, targs, 1e-3, want_loss=True)
    print(json.dumps({"train_steps": steps, "ms_per_step": (time.perf_counter() - t) * 1e3 / steps,
                      "loss": list(loss)}))
    tr.close()
    return 0


def kd_build(rt, workloads, which, d, reps):
    import time
    import numpy as np
    if which == "terrain":
        path = workloads.make_terrain(d, n=1024, seed=11)
    else:
        path = workloads.make_noisy_icosphere(d, level=6, seed=7)
    host = rt.HostScene.from_json_file(path)
    (v, nodes, idx), = host.meshes()
    ctx = rt.default_context(0)
    rt.kd_build(v[:1000], ctx=ctx)
    times = []
    for _ in range(reps):
        t = time.perf_counter()
        n2, i2 = rt.kd_build(v, ctx=ctx)
        times.append((time.perf_counter() - t) * 1e3)
    same = n2.tobytes() == nodes.tobytes() and np.array_equal(i2, idx)
    t = time.perf_counter()
    scene = rt.Scene.upload(host, ctx)
    upload_ms = (time.perf_counter() - t) * 1e3
    scene.close()
    print(json.dumps({"kd_build": which, "triangles": len(v), "nodes": len(nodes), "leaf_entries": len(idx),
                      "device_ms": times, "same_as_host": same, "first_upload_ms": upload_ms}))
    return 0 if same else 1


if __name__ == "__main__":
    sys.exit(main())
