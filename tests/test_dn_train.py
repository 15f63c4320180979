"""The denoiser's 3-level network (blob version 3), its confidence-gated
fallback to the plain path, and its training on the library's own kernels,
against PyTorch fp32 references: the forward pass against a PyTorch forward
of the same FP16 weights, weight gradients against torch's convolution
weight gradient, and a whole network's gradients against autograd."""
import json

import numpy as np
import pytest

from rtrace_b200 import denoiser


def test_net_blob_roundtrip_and_size():
    net = denoiser.random_net(4)
    assert net.param_count == 212_432
    back = denoiser.unpack_net(denoiser.pack_net(net))
    assert back.ops == net.ops and back.rays == net.rays and abs(back.threshold - net.threshold) < 1e-7
    for (w0, b0), (w1, b1) in zip(net.params, back.params):
        assert np.array_equal(w0, w1) and np.array_equal(b0, b1)
    old = denoiser.unpack_net(denoiser.pack(denoiser.random_layers(2)))
    assert not old.conf and len(old.ops) == len(denoiser.ARCH)


def test_reference_forward_shapes_on_cpu():
    import torch
    net = denoiser.random_net(5)
    f = (torch.rand((2, 19, 45, 16)) * 2 - 0.5).half()  # odd sizes: ragged pooling blocks
    vis, conf = denoiser.net_forward(net, f)
    assert vis.shape == (2, 2, 19, 45) and conf.shape == (2, 2, 19, 45)
    assert float(vis.min()) >= 0 and float(vis.max()) <= 1


def _feats(torch, dev, P, H, W, seed):
    g = torch.Generator(device="cpu").manual_seed(seed)
    f = torch.rand((P, H, W, 16), generator=g) * 2 - 0.5
    f[..., 0] = (torch.rand((P, H, W), generator=g) < 0.8).float()  # hit
    f[..., 8] = 1.0  # slot 0 present
    f[..., 12] = (torch.rand((P, H, W), generator=g) < 0.7).float()
    t = torch.rand((P, 2, H, W), generator=g)
    return f.half().to(dev), t.half().to(dev)


# --------------------------------------------------------------------------
# GPU
# --------------------------------------------------------------------------
@pytest.mark.gpu
def test_unet_forward_matches_torch_fp32(gpu_ctx):
    import torch
    import rtrace_b200 as rt
    dev = torch.device("cuda", gpu_ctx.device)
    net = denoiser.random_net(1, scale=1.0)
    gpu_ctx.load_denoiser(denoiser.pack_net(net))
    L = rt._capi.lib()
    # 300 wide: two full 128-pixel tiles and a ragged one; odd heights pool
    # raggedly.  301 wide: odd widths at both poolings (301, 151)
    for H, W in ((37, 300), (35, 301)):
        feat = (torch.rand((2, H, W, 16), device=dev) * 2 - 0.5).half()
        vis = torch.full((2, 2, H, W), -7.0, device=dev)
        conf = torch.full((2, 2, H, W), -7.0, device=dev)
        torch.cuda.synchronize()
        st = L.rt_denoiser_run(gpu_ctx.handle, feat.data_ptr(), 2, H, W, vis.data_ptr(), conf.data_ptr(), None)
        assert st == 0, L.rt_last_error(gpu_ctx.handle)
        torch.cuda.synchronize()
        rv, rc = denoiser.net_forward(net, feat, round_fp16=True)
        assert (vis - rv).abs().max().item() < 3e-3, (H, W)
        assert (conf - rc).abs().max().item() < 3e-3, (H, W)


@pytest.mark.gpu
@pytest.mark.parametrize("cin,cout,dil", [(16, 32, 1), (32, 32, 2), (32, 64, 1), (64, 64, 4), (64, 32, 1),
                                          (32, 16, 1), (16, 16, 3)])
def test_weight_gradient_matches_torch(gpu_ctx, cin, cout, dil):
    import torch
    import rtrace_b200 as rt
    dev = torch.device("cuda", gpu_ctx.device)
    P, H, W = 2, 7, 200  # a full 128-pixel run and a ragged one
    g = torch.Generator(device="cpu").manual_seed(cin * 100 + cout + dil)
    x = (torch.rand((P, H, W, cin), generator=g) * 2 - 1).half().to(dev)
    dz = (torch.rand((P, H, W, cout), generator=g) * 2 - 1).half().to(dev)
    dw = torch.zeros((cout, 3, 3, cin), device=dev)
    db = torch.zeros(cout, device=dev)
    torch.cuda.synchronize()
    L = rt._capi.lib()
    st = L.rt_debug_conv_wgrad(gpu_ctx.handle, x.data_ptr(), dz.data_ptr(), P, H, W, cin, cout, dil,
                               dw.data_ptr(), db.data_ptr())
    assert st == 0, L.rt_last_error(gpu_ctx.handle)
    xr = x.float().permute(0, 3, 1, 2)
    gr = dz.float().permute(0, 3, 1, 2)
    ref = torch.nn.grad.conv2d_weight(xr, (cout, cin, 3, 3), gr, padding=dil, dilation=dil).permute(0, 2, 3, 1)
    # FP16 products are exact in FP32; only the summation order differs
    scale = ref.abs().max().item()
    assert (dw - ref).abs().max().item() < 1e-4 * scale
    assert (db - gr.sum((0, 2, 3))).abs().max().item() < 1e-4 * max(1.0, gr.sum((0, 2, 3)).abs().max().item())


@pytest.mark.gpu
def test_network_gradients_match_autograd(gpu_ctx):
    import torch
    from rtrace_b200.dn_train import Trainer
    dev = torch.device("cuda", gpu_ctx.device)
    net = denoiser.random_net(3, scale=1.0)
    P, H, W = 2, 37, 150
    feats, targs = _feats(torch, dev, P, H, W, 8)
    tr = Trainer(gpu_ctx, net, P, H, W)
    got, (cnt, lv, lc) = tr.grads(feats, targs)
    tr.close()
    # autograd of the same summed loss on the FP16-rounded forward pass
    params = denoiser.torch_params(net, dev)
    vis, conf = denoiser.net_forward(net, feats, round_fp16=True, weights=params)
    m = denoiser.masks(feats).float()
    t = targs.float()
    err = (vis - t).abs()
    loss_v = ((vis - t) ** 2 * m).sum()
    loss_c = ((conf - err.detach()) ** 2 * m).sum()
    (loss_v + loss_c).backward()
    assert abs(cnt - m.sum().item()) < 0.5
    assert abs(lv - loss_v.item()) < 1e-2 * loss_v.item() and abs(lc - loss_c.item()) < 1e-2 * loss_c.item()
    # FP16 activation gradients on the library's side: relative L2 error per tensor
    for k, ((dw, db), (w, b)) in enumerate(zip(got, params)):
        rw = w.grad.permute(0, 2, 3, 1).cpu().numpy()
        rb = b.grad.cpu().numpy()
        ew = np.linalg.norm(dw - rw) / max(np.linalg.norm(rw), 1e-12)
        eb = np.linalg.norm(db - rb) / max(np.linalg.norm(rb), 1e-12)
        assert ew < 2e-2 and eb < 2e-2, (k, ew, eb)


@pytest.mark.gpu
def test_native_training_reduces_the_loss(gpu_ctx):
    import torch
    from rtrace_b200.dn_train import Trainer
    dev = torch.device("cuda", gpu_ctx.device)
    net = denoiser.random_net(6)
    P, H, W = 4, 64, 128
    feats, _ = _feats(torch, dev, P, H, W, 2)
    # a learnable target: the cast ray's visibility channel smoothed
    t = feats[..., 5].float().clamp(0, 1).unsqueeze(1).repeat(1, 2, 1, 1)
    targs = torch.nn.functional.avg_pool2d(t, 5, 1, 2).half().contiguous()
    tr = Trainer(gpu_ctx, net, P, H, W)
    first = tr.step(feats, targs, 1e-3, want_loss=True)
    for _ in range(60):
        tr.step(feats, targs, 1e-3)
    last = tr.step(feats, targs, 1e-3, want_loss=True)
    assert (last[1] + last[2]) < 0.5 * (first[1] + first[2]), (first, last)
    out = tr.export(threshold=0.05)
    tr.close()
    assert abs(out.threshold - 0.05) < 1e-7 and out.ops == net.ops
    assert any(not np.array_equal(a[0], b[0]) for a, b in zip(out.params, net.params))


def _disk_scene_json(n_rings=2, per_ring=6, seed=3):
    from rtrace_b200 import workloads
    return json.dumps(workloads.ring_spheres_scene(seed=seed, n_rings=n_rings, per_ring=per_ring))


@pytest.mark.gpu
def test_confidence_fallback_uses_the_plain_path(gpu_ctx):
    """With every light of every hit falling back, a learned render is the
    plain render; with none, it shades with the network; in between, each
    hit's visibility of each light is the plain path's where the error
    estimate exceeds the threshold and the network's elsewhere."""
    import torch
    import rtrace_b200 as rt
    js = _disk_scene_json()
    scene = rt.Scene.from_json_str(js, gpu_ctx)
    dev = torch.device("cuda", gpu_ctx.device)
    net = denoiser.random_net(9, threshold=0.5)
    gpu_ctx.load_denoiser(denoiser.pack_net(net))
    W, H, S = 128, 72, 2
    plain = rt.Renderer(W, H)
    plain.anti_aliasing_mode = rt.AntiAliasingMode.Stochastic
    plain.samples = S
    pv = torch.zeros((S, 2, H, W), device=dev)
    feat = torch.zeros((S, H, W, 16), dtype=torch.float16, device=dev)
    torch.cuda.synchronize()
    want = plain.render_shadow_aov(scene, pv.data_ptr(), feat.data_ptr())
    r = rt.Renderer(W, H)
    r.anti_aliasing_mode = rt.AntiAliasingMode.Stochastic
    r.samples = S
    r.learned_shadows = True
    r.confidence_threshold = 1e-30  # every estimate exceeds it
    vis = torch.zeros((S, 2, H, W), device=dev)
    img = r.render_shadow_aov(scene, vis.data_ptr(), None)
    assert np.array_equal(img, want)
    hits = int((feat[..., 0] > 0).sum().item())
    assert r.last_stats.fallback_hits == hits
    m = denoiser.masks(feat)
    assert torch.equal(vis[m], pv[m])
    # none: the network alone
    r.confidence_threshold = -1.0
    r.render_shadow_aov(scene, vis.data_ptr(), None)
    assert r.last_stats.fallback_hits == 0
    lfeat = torch.zeros((S, H, W, 16), dtype=torch.float16, device=dev)
    r.confidence_threshold = 2.0  # above every sigmoid
    r.render_shadow_aov(scene, vis.data_ptr(), lfeat.data_ptr())
    assert r.last_stats.fallback_hits == 0
    nv, _ = denoiser.net_forward(net, lfeat, round_fp16=True)
    assert (vis[m] - nv[m]).abs().max().item() < 3e-3
    # the same kernels on the same features give the render's estimates exactly
    gv = torch.zeros_like(vis)
    gc = torch.zeros_like(vis)
    torch.cuda.synchronize()
    L = rt._capi.lib()
    assert L.rt_denoiser_run(gpu_ctx.handle, lfeat.data_ptr(), S, H, W, gv.data_ptr(), gc.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert torch.equal(vis[m], gv[m])
    # the threshold stored with the weights (0.5): per light, the plain
    # path's visibility where the estimate exceeds it, the network's elsewhere
    r.confidence_threshold = 0.0
    r.render_shadow_aov(scene, vis.data_ptr(), None)
    fb = (gc > 0.5) & m
    assert r.last_stats.fallback_hits == int(fb.any(1).sum().item())
    assert 0 < int(fb.sum().item()) < int(m.sum().item())
    assert torch.equal(vis[fb], pv[fb])
    keep = m & ~fb
    assert torch.equal(vis[keep], gv[keep])


@pytest.mark.gpu
def test_confidence_fallback_with_point_lights(gpu_ctx):
    """A point light before and one between the disk lights: each hit's
    shadow rays are then point, disk (n rays), point, disk (n rays), so the
    rays of a falling slot start at an offset that is not a multiple of the
    warp width.  Every light falling back gives the plain render's bytes and
    visibility; at the stored threshold each slot's visibility is the plain
    path's where its error estimate exceeds the threshold, the network's
    elsewhere, in both halves of the bucketed fallback list."""
    import torch
    import rtrace_b200 as rt
    from rtrace_b200 import workloads
    sc = workloads.ring_spheres_scene(seed=5, n_rings=2, per_ring=6)
    disks = sc["lights"]
    sc["lights"] = [{"position": [2.0, -3.0, 7.0], "color": "#FFE0C0", "intensity": 0.4}, disks[0],
                    {"position": [-4.0, 2.0, 6.0], "color": "#C0E0FF", "intensity": 0.3}, disks[1]]
    scene = rt.Scene.from_json_str(json.dumps(sc), gpu_ctx)
    dev = torch.device("cuda", gpu_ctx.device)
    net = denoiser.random_net(11, threshold=0.5)
    gpu_ctx.load_denoiser(denoiser.pack_net(net))
    W, H, S = 120, 64, 2
    for fb_rays in (5, 16):
        plain = rt.Renderer(W, H)
        plain.anti_aliasing_mode = rt.AntiAliasingMode.Stochastic
        plain.samples = S
        plain.disk_samples = fb_rays
        pv = torch.zeros((S, 2, H, W), device=dev)
        feat = torch.zeros((S, H, W, 16), dtype=torch.float16, device=dev)
        torch.cuda.synchronize()
        want = plain.render_shadow_aov(scene, pv.data_ptr(), feat.data_ptr())
        m = denoiser.masks(feat)
        r = rt.Renderer(W, H)
        r.anti_aliasing_mode = rt.AntiAliasingMode.Stochastic
        r.samples = S
        r.disk_samples = fb_rays
        r.learned_shadows = True
        r.fallback_samples = fb_rays
        r.confidence_threshold = 1e-30  # every slot of every hit falls back
        vis = torch.zeros((S, 2, H, W), device=dev)
        img = r.render_shadow_aov(scene, vis.data_ptr(), None)
        assert np.array_equal(img, want), fb_rays
        assert torch.equal(vis[m], pv[m]), fb_rays
        # the stored threshold: some hits with one falling slot, some with two
        r.confidence_threshold = 0.0
        lfeat = torch.zeros((S, H, W, 16), dtype=torch.float16, device=dev)
        r.render_shadow_aov(scene, vis.data_ptr(), lfeat.data_ptr())
        gv = torch.zeros_like(vis)
        gc = torch.zeros_like(vis)
        torch.cuda.synchronize()
        L = rt._capi.lib()
        assert L.rt_denoiser_run(gpu_ctx.handle, lfeat.data_ptr(), S, H, W, gv.data_ptr(), gc.data_ptr(), None) == 0
        torch.cuda.synchronize()
        fb = (gc > 0.5) & m
        both = fb.all(1)
        one = fb.any(1) & ~both
        assert int(both.sum().item()) > 0 and int(one.sum().item()) > 0
        assert r.last_stats.fallback_hits == int(fb.any(1).sum().item())
        assert r.last_stats.fallback_lights == int(fb.sum().item())
        assert torch.equal(vis[fb], pv[fb])
        keep = m & ~fb
        assert torch.equal(vis[keep], gv[keep])


@pytest.mark.gpu
def test_pixel_mean_visibility_feature(gpu_ctx):
    """Channels 13 and 14 of each hit sample hold the mean cast-ray
    visibility of slots 0 and 1 over the pixel's samples that hit."""
    import torch
    import rtrace_b200 as rt
    scene = rt.Scene.from_json_str(_disk_scene_json(), gpu_ctx)
    dev = torch.device("cuda", gpu_ctx.device)
    S, H, W = 3, 40, 64
    r = rt.Renderer(W, H)
    r.anti_aliasing_mode = rt.AntiAliasingMode.Stochastic
    r.samples = S
    r.disk_samples = 2
    feat = torch.zeros((S, H, W, 16), dtype=torch.float16, device=dev)
    torch.cuda.synchronize()
    r.render_shadow_aov(scene, None, feat.data_ptr())
    f = feat.float()
    valid = f[..., 0] > 0
    n = valid.sum(0)
    for j, ch in ((0, 5), (1, 9)):
        mean = torch.where(n > 0, (f[..., ch] * valid).sum(0) / n.clamp_min(1), torch.zeros_like(n, dtype=f.dtype))
        want = mean.unsqueeze(0).expand_as(valid)[valid].half().float()
        assert torch.equal(f[..., 13 + j][valid], want)
    assert (f[..., 13:15][~valid] == 0).all()
