"""Learned soft shadows (extension): the tensor-core denoiser against a plain
PyTorch fp32 forward pass of the same network, the disk_samples extension of
the plain path against the oracle, and the learned render's plumbing."""
import ctypes
import json

import numpy as np
import pytest

from rtrace_b200 import denoiser


def test_blob_roundtrip():
    layers = denoiser.random_layers(3)
    blob = denoiser.pack(layers)
    back = denoiser.unpack(blob)
    assert len(back) == len(layers)
    for (w0, b0, d0), (w1, b1, d1) in zip(layers, back):
        assert np.array_equal(np.asarray(w0, np.float16), w1) and np.array_equal(np.float32(b0), b1) and d0 == d1
    with pytest.raises(ValueError):
        denoiser.unpack(b"XXXX" + blob[4:])
    with pytest.raises(ValueError):
        denoiser.unpack(blob + b"\0")


def test_training_scenes_are_seeded():
    a, b, c = denoiser.training_scene(5), denoiser.training_scene(5), denoiser.training_scene(6)
    assert json.dumps(a) == json.dumps(b) and json.dumps(a) != json.dumps(c)
    assert all("diameter" in L for L in a["lights"]) and len(a["lights"]) == 2


# --------------------------------------------------------------------------
# GPU
# --------------------------------------------------------------------------
def _run_net(ctx, layers, feat):
    import torch
    import rtrace_b200 as rt
    ctx.load_denoiser(denoiser.pack(layers))
    planes, H, W, _ = feat.shape
    vis = torch.full((planes, 2, H, W), -7.0, dtype=torch.float32, device=feat.device)
    torch.cuda.synchronize()  # torch's fills run on torch's stream, the network on the context's
    L = rt._capi.lib()
    st = L.rt_denoiser_run(ctx.handle, feat.data_ptr(), planes, H, W, vis.data_ptr(), None, None)
    assert st == 0, L.rt_last_error(ctx.handle)
    torch.cuda.synchronize()
    return vis


@pytest.mark.gpu
@pytest.mark.parametrize("arch", [
    [(16, 16, 1)],
    [(16, 32, 1), (32, 16, 2)],
    [(16, 16, 3), (16, 32, 1), (32, 32, 5), (32, 16, 1)],
    denoiser.ARCH,
])
def test_tensor_core_network_matches_torch_fp32(gpu_ctx, arch):
    import torch
    torch.manual_seed(0)
    dev = torch.device("cuda", gpu_ctx.device)
    layers = denoiser.random_layers(1, arch, scale=1.0)
    # 300 = two full 128-pixel tiles and a ragged one; 2 planes keep the
    # planes' borders apart
    feat = (torch.rand((2, 37, 300, 16), device=dev) * 2 - 0.5).half()
    got = _run_net(gpu_ctx, layers, feat)
    ref = denoiser.torch_forward(layers, feat, round_fp16=True)
    # FP16 operands, FP32 accumulation in either order; hidden activations
    # rounded to FP16 on both sides.  Tolerance on the sigmoid outputs:
    err = (got - ref).abs().max().item()
    assert err < 2e-3, err


@pytest.mark.gpu
def test_tensor_core_conv_edges_are_zero_padded(gpu_ctx):
    import torch
    dev = torch.device("cuda", gpu_ctx.device)
    # one layer summing channel 0 over the 3x3 neighbourhood, dilation 4:
    # out = sigmoid(sum of in-image taps)
    w = np.zeros((16, 3, 3, 16), np.float16)
    w[0, :, :, 0] = 1.0
    layers = [(w, np.zeros(16, np.float32), 4)]
    H, W = 9, 130
    feat = torch.zeros((1, H, W, 16), dtype=torch.float16, device=dev)
    feat[..., 0] = 0.25
    got = _run_net(gpu_ctx, layers, feat)[0, 0].cpu().numpy()
    ys, xs = np.mgrid[0:H, 0:W]
    n = np.zeros((H, W))
    for dy in (-4, 0, 4):
        for dx in (-4, 0, 4):
            n += ((ys + dy >= 0) & (ys + dy < H) & (xs + dx >= 0) & (xs + dx < W))
    want = 1.0 / (1.0 + np.exp(-0.25 * n))
    assert np.abs(got - want).max() < 1e-6


def _disk_scene_json(n_rings=2, per_ring=6, seed=3):
    from rtrace_b200 import workloads
    return json.dumps(workloads.ring_spheres_scene(seed=seed, n_rings=n_rings, per_ring=per_ring))


@pytest.mark.gpu
@pytest.mark.parametrize("samples,aa", [(1, "no-jitter"), (5, "stochastic"), (64, "no-jitter")])
def test_disk_samples_match_the_oracle(gpu_ctx, oracle, samples, aa):
    import rtrace_b200 as rt
    from tests import oracle_lib
    js = _disk_scene_json()
    scene = rt.Scene.from_json_str(js, gpu_ctx)
    r = rt.Renderer(96, 64)
    r.anti_aliasing_mode = rt.AntiAliasingMode.NoJitter if aa == "no-jitter" else rt.AntiAliasingMode.Stochastic
    r.samples = 2 if aa == "stochastic" else 1
    r.disk_samples = samples
    got = r.render(scene)
    want = oracle_lib.render(json_text=js, width=96, height=64, aa=aa, samples=r.samples, disk_samples=samples)
    assert np.array_equal(got, want), int((got != want).any(2).sum())
    # 16 is the reference's count: the default
    r.disk_samples = 16
    a = r.render(scene)
    r.disk_samples = 0
    assert np.array_equal(a, r.render(scene))


@pytest.mark.gpu
def test_shadow_aov_is_visible_fraction(gpu_ctx):
    import torch
    import rtrace_b200 as rt
    js = _disk_scene_json()
    scene = rt.Scene.from_json_str(js, gpu_ctx)
    dev = torch.device("cuda", gpu_ctx.device)
    r = rt.Renderer(96, 64)
    r.anti_aliasing_mode = rt.AntiAliasingMode.NoJitter
    r.disk_samples = 16
    vis = torch.full((1, 2, 64, 96), -1.0, device=dev)
    feat = torch.zeros((1, 64, 96, 16), dtype=torch.float16, device=dev)
    torch.cuda.synchronize()
    img = r.render_shadow_aov(scene, vis.data_ptr(), feat.data_ptr())
    assert np.array_equal(img, r.render(scene))  # the AOVs do not change the image
    valid = feat[..., 0] == 1
    assert valid.any()
    v = vis[:, :, :, :][valid.unsqueeze(1).expand_as(vis)].cpu().numpy()
    assert np.allclose(v * 16, np.round(v * 16)) and v.min() >= 0 and v.max() <= 1
    # feature slot visibility equals the AOV (FP16 holds k/16 exactly)
    f0 = feat[..., 5].float()
    assert torch.equal(f0[valid], vis[:, 0][valid])


@pytest.mark.gpu
def test_learned_render_shades_with_the_network_output(gpu_ctx):
    import torch
    import rtrace_b200 as rt
    js = _disk_scene_json()
    scene = rt.Scene.from_json_str(js, gpu_ctx)
    dev = torch.device("cuda", gpu_ctx.device)
    layers = denoiser.random_layers(7)
    gpu_ctx.load_denoiser(denoiser.pack(layers))
    r = rt.Renderer(128, 72)
    r.anti_aliasing_mode = rt.AntiAliasingMode.Stochastic
    r.samples = 2
    r.learned_shadows = True
    vis = torch.zeros((2, 2, 72, 128), device=dev)
    feat = torch.zeros((2, 72, 128, 16), dtype=torch.float16, device=dev)
    torch.cuda.synchronize()
    img = r.render_shadow_aov(scene, vis.data_ptr(), feat.data_ptr())
    st = r.last_stats
    # level 0 casts one ray per disk light
    r2 = rt.Renderer(128, 72)
    r2.anti_aliasing_mode = rt.AntiAliasingMode.Stochastic
    r2.samples = 2
    r2.render(scene)
    assert st.primary_rays == r2.last_stats.primary_rays
    assert st.shadow_rays < r2.last_stats.shadow_rays
    # the visibility the render used is the network's output on its features
    again = _run_net(gpu_ctx, layers, feat)
    assert torch.equal(vis, again)
    # deterministic, and the image without AOVs is the same
    assert np.array_equal(img, r.render(scene))
    assert img.max() > 0
    # learned shadows need whole frames, at most two disk lights, weights
    with pytest.raises(ValueError):
        r.render_rows(scene, 0, 10)
    r.anti_aliasing_mode = rt.AntiAliasingMode.Quincunx
    with pytest.raises(ValueError):
        r.render(scene)
