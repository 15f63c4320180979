"""CUDA graph replay (RT_FLAG_CUDA_GRAPH): a render captured once and then
replayed writes the image a directly launched render writes, and a change of
any launch argument (seed, camera, image size, output pointer) captures anew
instead of replaying a stale sequence."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_header_flags_and_stats_layout_match_the_binding(tmp_path):
    from rtrace_b200 import _capi
    text = open(os.path.join(ROOT, "include", "rtrace_gpu.h")).read()
    flags = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define (RT_FLAG_\w+) (\d+)u", text)}
    assert flags == {k: getattr(_capi, k) for k in flags} and "RT_FLAG_CUDA_GRAPH" in flags
    # rt_stats offsets as the C compiler lays them out
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "rtrace_gpu.h"\n'
                   'int main(void) { printf("%zu %zu %zu %zu\\n", sizeof(rt_stats), offsetof(rt_stats, graph),'
                   ' offsetof(rt_stats, device_ms), sizeof(rt_render_params)); return 0; }\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert got == [ctypes.sizeof(_capi.rt_stats), _capi.rt_stats.graph.offset, _capi.rt_stats.device_ms.offset,
                   ctypes.sizeof(_capi.rt_render_params)]


# --------------------------------------------------------------------------
# GPU
# --------------------------------------------------------------------------
def _scene(case, ctx, tmp_path):
    import json
    import rtrace_b200 as rt
    from rtrace_b200 import workloads
    if case == "sphere_grid_quincunx":
        return rt.Scene.from_json_str(json.dumps(workloads.sphere_grid_scene()), ctx), rt.AntiAliasingMode.Quincunx
    if case == "ring_disk_stochastic":
        js = workloads.ring_spheres_scene(seed=3, n_rings=2, per_ring=6)
        return rt.Scene.from_json_str(json.dumps(js), ctx), rt.AntiAliasingMode.Stochastic
    path = workloads.make_noisy_icosphere(str(tmp_path), level=3)
    return rt.Scene.from_json_file(path, ctx), rt.AntiAliasingMode.NoJitter


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["sphere_grid_quincunx", "ring_disk_stochastic", "icosphere_outline"])
def test_replay_equals_direct_launch(gpu_ctx, tmp_path, case):
    import rtrace_b200 as rt
    from rtrace_b200 import _capi
    scene, aa = _scene(case, gpu_ctx, tmp_path)
    r = rt.Renderer(120, 80)
    r.anti_aliasing_mode = aa
    r.samples = 3
    if case == "icosphere_outline":
        r.outline_config = rt.OutlineConfig(line_thickness=2.5)
    want = r.render(scene)
    direct = r.last_stats
    assert direct.graph == 0
    r.flags = _capi.RT_FLAG_CUDA_GRAPH
    a = r.render(scene)
    assert r.last_stats.graph == 1
    b = r.render(scene)
    replay = r.last_stats
    assert replay.graph == 2
    assert np.array_equal(a, want) and np.array_equal(b, want)
    # the replay's queues and counters are this frame's, reset on the device
    assert (replay.primary_rays, replay.reflection_rays, replay.shadow_rays, replay.hits) == \
        (direct.primary_rays, direct.reflection_rays, direct.shadow_rays, direct.hits)
    assert replay.kernel_launches == direct.kernel_launches
    # another seed and another size are other launch sequences
    for change in ("seed", "size"):
        if change == "seed":
            r.seed = 12345
        else:
            r.width, r.height = 64, 48
        r.flags = _capi.RT_FLAG_CUDA_GRAPH
        c = r.render(scene)
        assert r.last_stats.graph == 1, change
        r.flags = 0
        assert np.array_equal(c, r.render(scene)), change
    # profiling flags launch directly
    r.flags = _capi.RT_FLAG_CUDA_GRAPH | _capi.RT_FLAG_STAGE_TIMES
    r.render(scene)
    assert r.last_stats.graph == 0 and r.last_stats.stage_ms["trace"] > 0
    scene.close()


@pytest.mark.gpu
def test_replay_matches_the_oracle(gpu_ctx, oracle):
    import json
    import rtrace_b200 as rt
    from rtrace_b200 import _capi, workloads
    from tests import oracle_lib
    js = json.dumps(workloads.sphere_grid_scene())
    scene = rt.Scene.from_json_str(js, gpu_ctx)
    r = rt.Renderer(96, 64)
    r.flags = _capi.RT_FLAG_CUDA_GRAPH
    want = oracle_lib.render(json_text=js, width=96, height=64, aa="quincunx")
    for k in range(3):
        assert np.array_equal(r.render(scene), want), k
    assert r.last_stats.graph == 2


@pytest.mark.gpu
def test_replay_to_device_output_and_in_batches(gpu_ctx):
    import json
    import torch
    import rtrace_b200 as rt
    from rtrace_b200 import _capi, workloads
    js = workloads.ring_spheres_scene(seed=3, n_rings=2, per_ring=6)
    scene = rt.Scene.from_json_str(json.dumps(js), gpu_ctx)
    r = rt.Renderer(100, 60)
    r.anti_aliasing_mode = rt.AntiAliasingMode.Stochastic
    r.samples = 2
    want = r.render(scene)
    r.flags = _capi.RT_FLAG_CUDA_GRAPH
    dev = torch.device("cuda", gpu_ctx.device)
    bufs = [torch.zeros((60, 100, 3), dtype=torch.uint8, device=dev) for _ in range(2)]
    torch.cuda.synchronize()  # torch's stream is not the render's
    states = []
    for buf in (bufs[0], bufs[0], bufs[1]):
        r.render(scene, device_ptr=buf.data_ptr())
        states.append(r.last_stats.graph)
    torch.cuda.synchronize()
    assert states == [1, 2, 1]  # a new output pointer is a new sequence
    for buf in bufs:
        assert np.array_equal(buf.cpu().numpy(), want)
    # batch jobs with the flag, outside a fused group (a fused group is always
    # one captured sequence, tests/test_batch.py): each lane captures its
    # jobs, a second batch replays them (every job shares `r`, whose stats
    # are the last job's)
    cams = list(rt.auto_cameras(json_text=json.dumps(js)).values())[:3]
    saved = rt.batch_tuning(gpu_ctx)["fuse_pixels"]
    rt.batch_tuning(gpu_ctx, fuse_pixels=0)
    try:
        r.flags = 0
        plain, _ = rt.render_batch([rt.Job(scene, r, cam) for cam in cams], lanes=2, ctx=gpu_ctx)
        r.flags = _capi.RT_FLAG_CUDA_GRAPH
        jobs = [rt.Job(scene, r, cam) for cam in cams]
        for k in range(2):
            imgs, _ = rt.render_batch(jobs, lanes=2, ctx=gpu_ctx)
            assert r.last_stats.graph == k + 1
            assert all(np.array_equal(a, b) for a, b in zip(imgs, plain))
    finally:
        rt.batch_tuning(gpu_ctx, fuse_pixels=saved)
    scene.close()


@pytest.mark.gpu
def test_replay_of_learned_shadows_and_reload(gpu_ctx):
    import json
    import torch
    import rtrace_b200 as rt
    from rtrace_b200 import _capi, denoiser, workloads
    js = json.dumps(workloads.ring_spheres_scene(seed=3, n_rings=2, per_ring=6))
    scene = rt.Scene.from_json_str(js, gpu_ctx)
    r = rt.Renderer(128, 72)
    r.anti_aliasing_mode = rt.AntiAliasingMode.Stochastic
    r.samples = 2
    r.learned_shadows = True
    out = []
    for seed in (7, 8):
        gpu_ctx.load_denoiser(denoiser.pack(denoiser.random_layers(seed)))
        r.flags = 0
        want = r.render(scene)
        r.flags = _capi.RT_FLAG_CUDA_GRAPH
        a = r.render(scene)
        assert r.last_stats.graph == 1  # loading weights drops captured renders
        b = r.render(scene)
        assert r.last_stats.graph == 2
        assert np.array_equal(a, want) and np.array_equal(b, want)
        out.append(want)
    assert not np.array_equal(out[0], out[1])
    # the AOV outputs of a replay are the direct render's
    dev = torch.device("cuda", gpu_ctx.device)
    r.flags = 0
    v0 = torch.zeros((2, 2, 72, 128), device=dev)
    torch.cuda.synchronize()
    r.render_shadow_aov(scene, v0.data_ptr())
    r.flags = _capi.RT_FLAG_CUDA_GRAPH
    v1 = torch.full((2, 2, 72, 128), -3.0, device=dev)
    for _ in range(2):
        v1.fill_(-3.0)
        torch.cuda.synchronize()
        r.render_shadow_aov(scene, v1.data_ptr())
    assert r.last_stats.graph == 2
    assert torch.equal(v0, v1)
    scene.close()
