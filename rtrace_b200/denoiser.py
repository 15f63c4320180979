"""Learned soft-shadow denoiser: weight blobs, the network's definition, its
training data and its training.

This is an extension with no counterpart in the reference, which always
casts 16 shadow rays per disk light (src/lighting.rs:145-217).  In learned
mode the renderer casts one ray per disk light at each primary hit, writes a
16-channel feature image (visibility of that ray, depth, normal, and per
light the cosine and angular radius towards its centre), runs the network
below on the tensor cores (rtrace_b200/csrc/denoise.cu) and shades with the
estimated visibility.

The network is a stack of dilated 3x3 convolutions (zero padding, ReLU),
the last one with a sigmoid; its first two output channels are the
visibility of disk-light slots 0 and 1.  Training (``python -m
rtrace_b200.denoiser train``) renders seeded variations of the 1,000-sphere
ring scene on the GPU, pairs the 1-ray feature image with the 64-ray
visibility, fits the network with PyTorch, and writes the FP16 blob that
``Context.load_denoiser`` loads.  PyTorch is used only for this offline fit;
rendering and inference run the library's own kernels.
"""
import argparse
import json
import math
import os
import struct
import sys
import time

import numpy as np

FEAT_CHANNELS = 16
SLOTS = 2
MAGIC = b"RTDN"
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "denoiser_weights.bin")

# (cin, cout, dilation); ReLU after every layer but the last (sigmoid)
ARCH = [(16, 32, 1), (32, 32, 2), (32, 32, 4), (32, 32, 8), (32, 32, 16), (32, 32, 32), (32, 32, 1), (32, 16, 1)]


# --------------------------------------------------------------------------
# Blobs
# --------------------------------------------------------------------------
def pack(layers, rays=1):
    """layers: [(weight [cout][3][3][cin] array, bias [cout] array, dilation)]
    -> bytes in the rt_denoiser_load format (version 2: FP16 weights, FP32
    bias, and the rays per disk light the network expects)."""
    n = len(layers)
    out = [MAGIC, struct.pack("<III", 2, n, int(rays))]
    for i, (w, b, dil) in enumerate(layers):
        cout, kh, kw, cin = np.asarray(w).shape
        assert (kh, kw) == (3, 3) and np.asarray(b).shape == (cout,)
        out.append(struct.pack("<IIII", cin, cout, int(dil), 2 if i == n - 1 else 0))
    for w, b, _ in layers:
        out.append(np.ascontiguousarray(np.asarray(w, dtype=np.float16)).tobytes())
        out.append(np.ascontiguousarray(np.asarray(b, dtype=np.float32)).tobytes())
    return b"".join(out)


def unpack(blob, with_rays=False):
    """bytes -> [(weight float16 [cout][3][3][cin], bias float32 [cout],
    dilation)] (and the rays per disk light, with_rays=True)."""
    if blob[:4] != MAGIC:
        raise ValueError("not a denoiser weight blob")
    ver, n = struct.unpack_from("<II", blob, 4)
    if ver not in (1, 2):
        raise ValueError("unsupported blob version")
    head = 12 if ver == 1 else 16
    rays = 1 if ver == 1 else struct.unpack_from("<I", blob, 12)[0]
    heads = [struct.unpack_from("<IIII", blob, head + 16 * i) for i in range(n)]
    off = head + 16 * n
    layers = []
    for cin, cout, dil, _act in heads:
        nw = cout * 9 * cin
        w = np.frombuffer(blob, np.float16, nw, off).reshape(cout, 3, 3, cin)
        off += 2 * nw
        b = np.frombuffer(blob, np.float32, cout, off)
        off += 4 * cout
        layers.append((w, b, dil))
    if off != len(blob):
        raise ValueError("trailing bytes in denoiser blob")
    return (layers, rays) if with_rays else layers


def read_blob(weights=None):
    """bytes of a blob given as bytes, a path, or None (the shipped weights)."""
    if isinstance(weights, (bytes, bytearray)):
        return bytes(weights)
    path = weights or DEFAULT_WEIGHTS
    with open(path, "rb") as f:
        return f.read()


def random_layers(seed=0, arch=ARCH, scale=1.0):
    """Seeded He-initialised layers (tests and training start point)."""
    rng = np.random.default_rng(seed)
    layers = []
    for cin, cout, dil in arch:
        std = scale * math.sqrt(2.0 / (9 * cin))
        layers.append((rng.normal(0, std, (cout, 3, 3, cin)).astype(np.float16),
                       rng.normal(0, 0.05, cout).astype(np.float32), dil))
    return layers


# --------------------------------------------------------------------------
# The network in PyTorch (fp32 reference and training)
# --------------------------------------------------------------------------
def torch_forward(layers, feat, round_fp16=True):
    """Reference forward pass.  feat: [planes, H, W, 16] tensor; returns the
    visibility [planes, 2, H, W] (float32).  With round_fp16 the hidden
    activations are rounded to FP16 between layers, as the kernels store
    them."""
    import torch
    import torch.nn.functional as Fn
    x = feat.float().permute(0, 3, 1, 2)
    n = len(layers)
    for i, (w, b, dil) in enumerate(layers):
        wt = torch.as_tensor(np.asarray(w, np.float32), device=x.device).permute(0, 3, 1, 2).contiguous()
        bt = torch.as_tensor(np.asarray(b, np.float32), device=x.device)
        x = Fn.conv2d(x, wt, bt, padding=dil, dilation=dil)
        if i + 1 < n:
            x = torch.relu(x)
            if round_fp16:
                x = x.half().float()
        else:
            x = torch.sigmoid(x[:, :SLOTS])
    return x


def _torch_model(arch):
    import torch
    import torch.nn as nn

    class Net(nn.Module):
        def __init__(self):
            super().__init__()
            self.convs = nn.ModuleList(nn.Conv2d(ci, co, 3, padding=d, dilation=d) for ci, co, d in arch)

        def forward(self, x):
            for i, c in enumerate(self.convs):
                x = c(x)
                x = torch.relu(x) if i + 1 < len(self.convs) else torch.sigmoid(x[:, :SLOTS])
            return x

        def export(self):
            out = []
            for c, (_, _, d) in zip(self.convs, arch):
                w = c.weight.detach().float().permute(0, 2, 3, 1).cpu().numpy()  # [cout][3][3][cin]
                out.append((w.astype(np.float16), c.bias.detach().float().cpu().numpy(), d))
            return out

    return Net()


# --------------------------------------------------------------------------
# Training data
# --------------------------------------------------------------------------
def training_scene(seed):
    """A seeded variation of the 1,000-sphere ring scene: the sphere layout of
    ring_spheres_scene(seed) with the camera and both disk lights moved."""
    from .workloads import ring_spheres_scene
    sc = ring_spheres_scene(seed=seed)
    rng = np.random.default_rng(10_000 + seed)
    az = rng.uniform(0, 2 * math.pi)
    el = rng.uniform(0.35, 1.1)
    dist = rng.uniform(12, 22)
    sc["camera"]["position"] = [round(dist * math.cos(el) * math.cos(az), 4),
                                round(dist * math.cos(el) * math.sin(az), 4), round(dist * math.sin(el), 4)]
    sc["camera"]["target"] = [round(rng.uniform(-2, 2), 4), round(rng.uniform(-2, 2), 4), 0]
    for L in sc["lights"]:
        a = rng.uniform(0, 2 * math.pi)
        r = rng.uniform(3, 10)
        L["position"] = [round(r * math.cos(a), 4), round(r * math.sin(a), 4), round(rng.uniform(5, 12), 4)]
        L["diameter"] = round(float(rng.uniform(1.0, 3.0)), 4)
    return sc


def render_pair(ctx, scene_path, width, height, rays=1, target_samples=128, seed=0):
    """(features [1,H,W,16] half, target visibility [1,2,H,W] float) on the
    GPU: the feature image of `rays` rays per disk light (what learned mode
    casts at primary hits) and the target_samples-ray visibility."""
    import torch
    import rtrace_b200 as rt
    scene = rt.Scene.from_json_file(scene_path, ctx)
    dev = torch.device("cuda", ctx.device)
    r = rt.Renderer(width, height)
    r.anti_aliasing_mode = rt.AntiAliasingMode.NoJitter
    r.seed = seed
    r.max_depth = 1
    feat = torch.empty((1, height, width, FEAT_CHANNELS), dtype=torch.float16, device=dev)
    r.disk_samples = rays
    r.render_shadow_aov(scene, feat_ptr=feat.data_ptr())
    vis = torch.empty((1, SLOTS, height, width), dtype=torch.float32, device=dev)
    r.disk_samples = target_samples
    r.render_shadow_aov(scene, vis_ptr=vis.data_ptr())
    scene.close()
    return feat, vis


def psnr(est, ref, mask):
    """Visibility PSNR in dB over masked entries (peak 1)."""
    import torch
    m = mask.bool()
    if m.sum() == 0:
        return float("inf")
    mse = torch.mean((est[m].double() - ref[m].double()) ** 2).item()
    return float("inf") if mse == 0 else 10.0 * math.log10(1.0 / mse)


def train(out_path, n_scenes=160, width=1920, height=1080, iters=6000, batch=12, crop=192, seed=0, rays=1,
          target_samples=128, log=print):
    import tempfile
    import torch
    import rtrace_b200 as rt
    from .workloads import write_scene
    torch.manual_seed(seed)
    ctx = rt.default_context(0)
    dev = torch.device("cuda", 0)
    d = tempfile.mkdtemp(prefix="rtb_dn_")
    feats, targs = [], []
    t0 = time.time()
    for k in range(n_scenes):
        path = write_scene(d, "s%d.json" % k, training_scene(1 + k))
        f, v = render_pair(ctx, path, width, height, rays=rays, target_samples=target_samples, seed=k)
        feats.append(f)
        targs.append(v)
    log("rendered %d training scenes in %.1f s" % (n_scenes, time.time() - t0))
    feats = torch.cat(feats)  # [N,H,W,16] half
    targs = torch.cat(targs)  # [N,2,H,W]
    net = _torch_model(ARCH).to(dev)
    opt = torch.optim.Adam(net.parameters(), lr=2e-3)
    sched = torch.optim.lr_scheduler.OneCycleLR(opt, max_lr=2e-3, total_steps=iters, pct_start=0.05)
    g = torch.Generator(device="cpu").manual_seed(seed)
    t0 = time.time()
    for it in range(iters):
        idx = torch.randint(0, feats.shape[0], (batch,), generator=g)
        ys = torch.randint(0, height - crop + 1, (batch,), generator=g)
        xs = torch.randint(0, width - crop + 1, (batch,), generator=g)
        fb = torch.stack([feats[i, y:y + crop, x:x + crop] for i, y, x in zip(idx, ys, xs)])
        tb = torch.stack([targs[i, :, y:y + crop, x:x + crop] for i, y, x in zip(idx, ys, xs)])
        x = fb.float().permute(0, 3, 1, 2)
        pred = net(x)
        valid = x[:, 0:1]
        present = torch.stack([x[:, 5 + 3], x[:, 9 + 3]], 1)  # slot-present channels
        m = valid * present
        loss = ((pred - tb) ** 2 * m).sum() / m.sum().clamp_min(1.0)
        opt.zero_grad(set_to_none=True)
        loss.backward()
        opt.step()
        sched.step()
        if it % 500 == 0 or it == iters - 1:
            log("iter %d loss %.6f (%.1f s)" % (it, loss.item(), time.time() - t0))
    blob = pack(net.export(), rays=rays)
    with open(out_path, "wb") as f:
        f.write(blob)
    log("wrote %s (%d bytes, %d parameters)" % (out_path, len(blob),
                                                sum(p.numel() for p in net.parameters())))
    return out_path


def main(argv=None):
    ap = argparse.ArgumentParser(description="train the soft-shadow denoiser")
    ap.add_argument("command", choices=["train"])
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--scenes", type=int, default=160)
    ap.add_argument("--iters", type=int, default=6000)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--rays", type=int, default=1, help="rays per disk light at primary hits")
    ap.add_argument("--target-samples", type=int, default=128)
    ap.add_argument("--log", default=None)
    a = ap.parse_args(argv)
    logf = open(a.log, "w") if a.log else None

    def log(msg):
        print(msg, flush=True)
        if logf:
            logf.write(msg + "\n")
            logf.flush()

    train(a.out, n_scenes=a.scenes, width=a.width, height=a.height, iters=a.iters, rays=a.rays,
          target_samples=a.target_samples, log=log)
    return 0


if __name__ == "__main__":
    sys.exit(main())
