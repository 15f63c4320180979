"""Learned soft-shadow denoiser: weight blobs, the network's definition, its
training data and its training.

This is an extension with no counterpart in the reference, which always
casts 16 shadow rays per disk light (src/lighting.rs:145-217).  In learned
mode the renderer casts one ray per disk light at each primary hit, writes a
16-channel feature image (visibility of that ray, depth, normal, and per
light the cosine and angular radius towards its centre), runs the network
below on the tensor cores (rtrace_b200/csrc/denoise.cu) and shades with the
estimated visibility.  The network also estimates its own absolute error per
light; where that estimate exceeds a threshold the hit is shaded by the
plain path instead (the confidence-gated fallback).

The shipped network (UNET) is a 3-level encoder/decoder: 3x3 convolutions
at full, half and quarter resolution, 2x2 average pooling down, nearest
upsampling added to the skip connections up, ReLU, and a sigmoid on the
four output channels (visibility and estimated error of disk-light slots 0
and 1); 212,432 parameters.  Training (``python -m rtrace_b200.denoiser
train``) renders seeded variations of the 1,000-sphere ring scene on the GPU,
pairs the 1-ray feature image with the 64-ray visibility of the plain path,
fits the network and writes the blob ``Context.load_denoiser`` loads.
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

# (cin, cout, dilation); ReLU after every layer but the last (sigmoid).  A
# chain of dilated convolutions (blob versions 1 and 2).
ARCH = [(16, 32, 1), (32, 32, 2), (32, 32, 4), (32, 32, 8), (32, 32, 16), (32, 32, 32), (32, 32, 1), (32, 16, 1)]

# Blob version 3: ops (kind, cin, cout, dilation, src, src2).  Buffer 0 is the
# feature image and op i writes buffer i + 1; "pool" halves the resolution,
# "upadd" adds the nearest 2x upsampling of src to src2.  Every convolution
# but the last is followed by a ReLU; the last one's channels 0-3 go through
# a sigmoid (visibility of slots 0, 1; estimated error of slots 0, 1).
KINDS = {"conv": 0, "pool": 1, "upadd": 2}
UNET = [
    ("conv", 16, 32, 1, 0, None),    # 1  level 0
    ("conv", 32, 32, 1, 1, None),    # 2  level 0, skip
    ("pool", 32, 32, 1, 2, None),    # 3  level 1
    ("conv", 32, 64, 1, 3, None),    # 4
    ("conv", 64, 64, 1, 4, None),    # 5  level 1, skip
    ("pool", 64, 64, 1, 5, None),    # 6  level 2
    ("conv", 64, 64, 1, 6, None),    # 7
    ("conv", 64, 64, 2, 7, None),    # 8
    ("conv", 64, 64, 4, 8, None),    # 9
    ("upadd", 64, 64, 1, 9, 5),      # 10 level 1
    ("conv", 64, 32, 1, 10, None),   # 11
    ("upadd", 32, 32, 1, 11, 2),     # 12 level 0
    ("conv", 32, 32, 1, 12, None),   # 13
    ("conv", 32, 16, 1, 13, None),   # 14 output
]


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


class Net:
    """A network of any blob version: ops (as in UNET), per convolution
    (weight [cout][3][3][cin] float16, bias [cout] float32), the rays per
    disk light it expects, its default confidence threshold and whether its
    output carries error estimates (version 3)."""

    def __init__(self, ops, params, rays=1, threshold=1.0, conf=True):
        self.ops = [tuple(o) for o in ops]
        self.params = [(np.asarray(w, np.float16), np.asarray(b, np.float32)) for w, b in params]
        self.rays = int(rays)
        self.threshold = float(threshold)
        self.conf = bool(conf)
        if len(self.params) != sum(1 for o in self.ops if o[0] == "conv"):
            raise ValueError("one (weight, bias) pair per convolution expected")

    @property
    def param_count(self):
        return int(sum(w.size + b.size for w, b in self.params))

    @classmethod
    def from_layers(cls, layers, rays=1):
        ops = [("conv", np.asarray(w).shape[3], np.asarray(w).shape[0], d, i, None)
               for i, (w, _, d) in enumerate(layers)]
        return cls(ops, [(w, b) for w, b, _ in layers], rays=rays, conf=False)


def random_net(seed=0, ops=UNET, scale=1.0, rays=1, threshold=0.1):
    """Seeded He-initialised network of the given op list."""
    rng = np.random.default_rng(seed)
    params = []
    for kind, cin, cout, _, _, _ in ops:
        if kind == "conv":
            std = scale * math.sqrt(2.0 / (9 * cin))
            params.append((rng.normal(0, std, (cout, 3, 3, cin)).astype(np.float16),
                           rng.normal(0, 0.05, cout).astype(np.float32)))
    return Net(ops, params, rays=rays, threshold=threshold)


def pack_net(net):
    """Net -> bytes in the rt_denoiser_load format, version 3."""
    out = [MAGIC, struct.pack("<IIIf", 3, len(net.ops), net.rays, net.threshold)]
    n = len(net.ops)
    for i, (kind, cin, cout, dil, src, src2) in enumerate(net.ops):
        act = 2 if i == n - 1 else 0  # the last op's sigmoid outputs
        out.append(struct.pack("<7I", KINDS[kind], cin, cout, dil, act, src, 0xFFFFFFFF if src2 is None else src2))
    for w, b in net.params:
        out.append(np.ascontiguousarray(np.asarray(w, dtype=np.float16)).tobytes())
        out.append(np.ascontiguousarray(np.asarray(b, dtype=np.float32)).tobytes())
    return b"".join(out)


def unpack_net(blob):
    """bytes of any version -> Net."""
    if blob[:4] != MAGIC:
        raise ValueError("not a denoiser weight blob")
    ver = struct.unpack_from("<I", blob, 4)[0]
    if ver in (1, 2):
        layers, rays = unpack(blob, with_rays=True)
        return Net.from_layers(layers, rays)
    if ver != 3:
        raise ValueError("unsupported blob version")
    _, n, rays, thr = struct.unpack_from("<IIIf", blob, 4)
    ops = []
    off = 20
    names = {v: k for k, v in KINDS.items()}
    for _ in range(n):
        kind, cin, cout, dil, _act, src, src2 = struct.unpack_from("<7I", blob, off)
        ops.append((names[kind], cin, cout, dil, src, None if src2 == 0xFFFFFFFF else src2))
        off += 28
    params = []
    for kind, cin, cout, _, _, _ in ops:
        if kind != "conv":
            continue
        nw = cout * 9 * cin
        w = np.frombuffer(blob, np.float16, nw, off).reshape(cout, 3, 3, cin)
        off += 2 * nw
        b = np.frombuffer(blob, np.float32, cout, off)
        off += 4 * cout
        params.append((w, b))
    if off != len(blob):
        raise ValueError("trailing bytes in denoiser blob")
    return Net(ops, params, rays=rays, threshold=thr)


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
    """Reference forward pass of a chain of convolutions (or a Net: its
    visibility).  feat: [planes, H, W, 16] tensor; returns the visibility
    [planes, 2, H, W] (float32).  With round_fp16 the hidden activations are
    rounded to FP16 between layers, as the kernels store them."""
    if isinstance(layers, Net):
        return net_forward(layers, feat, round_fp16)[0]
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


def _pool2(x):
    """2x2 average pooling over the pixels of each block that exist (odd
    sizes round up), as the library's pooling kernel."""
    import torch.nn.functional as Fn
    H, W = x.shape[-2:]
    xp = Fn.pad(x, (0, W % 2, 0, H % 2))
    ones = Fn.pad(x.new_ones((1, 1, H, W)), (0, W % 2, 0, H % 2))
    return Fn.avg_pool2d(xp, 2) / Fn.avg_pool2d(ones, 2)


def _upadd(low, skip):
    import torch.nn.functional as Fn
    H, W = skip.shape[-2:]
    return Fn.interpolate(low, scale_factor=2, mode="nearest")[..., :H, :W] + skip


def net_forward(net, feat, round_fp16=True, weights=None):
    """Reference forward pass of a Net in PyTorch.  feat: [planes, H, W, 16]
    tensor; returns (visibility [planes, 2, H, W], error estimate [planes, 2,
    H, W] or None), float32.  With round_fp16 every stored activation is
    rounded to FP16, as the kernels store them.  weights: optional list of
    (weight [cout][cin][3][3], bias) tensors replacing net.params (training)."""
    import torch
    import torch.nn.functional as Fn
    bufs = [feat.float().permute(0, 3, 1, 2)]
    rnd = (lambda t: t.half().float()) if round_fp16 else (lambda t: t)
    k = 0
    n = len(net.ops)
    out = None
    for i, (kind, cin, cout, dil, src, src2) in enumerate(net.ops):
        x = bufs[src]
        if kind == "conv":
            if weights is not None:
                wt, bt = weights[k]
            else:
                w, b = net.params[k]
                wt = torch.as_tensor(np.array(w, np.float32), device=x.device).permute(0, 3, 1, 2).contiguous()
                bt = torch.as_tensor(np.array(b, np.float32), device=x.device)
            k += 1
            y = Fn.conv2d(x, wt, bt, padding=dil, dilation=dil)
            if i + 1 < n:
                y = rnd(torch.relu(y))
            else:
                out = torch.sigmoid(y[:, :2 * SLOTS])
        elif kind == "pool":
            y = rnd(_pool2(x))
        else:
            y = rnd(_upadd(x, bufs[src2]))
        bufs.append(y)
    vis = out[:, :SLOTS]
    conf = out[:, SLOTS:2 * SLOTS] if net.conf else None
    return vis, conf


def torch_params(net, device):
    """Trainable float32 copies of a Net's convolutions: [(weight [cout][cin]
    [3][3], bias [cout])] tensors with requires_grad."""
    import torch
    out = []
    for w, b in net.params:
        wt = torch.tensor(np.asarray(w, np.float32), device=device).permute(0, 3, 1, 2).contiguous()
        bt = torch.tensor(np.asarray(b, np.float32), device=device)
        out.append((wt.requires_grad_(True), bt.requires_grad_(True)))
    return out


def net_with_params(net, params):
    """A copy of net whose convolutions are the given float32 tensors
    ([cout][cin][3][3] weights), rounded to FP16."""
    conv = [(w.detach().permute(0, 2, 3, 1).cpu().numpy().astype(np.float16), b.detach().cpu().numpy())
            for w, b in params]
    return Net(net.ops, conv, rays=net.rays, threshold=net.threshold, conf=net.conf)


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


def render_pair(ctx, scene_path, width, height, rays=1, target_samples=64, seed=0, spp=4):
    """(features [spp,H,W,16] half, target visibility [spp,2,H,W] float) on
    the GPU for spp stochastic samples per pixel (the learned render's
    sample planes): the feature image of `rays` rays per disk light (what
    learned mode casts at primary hits) and the plain path's visibility
    with target_samples rays per disk light (the first samples of the same
    StdRng streams)."""
    import torch
    import rtrace_b200 as rt
    scene = rt.Scene.from_json_file(scene_path, ctx)
    dev = torch.device("cuda", ctx.device)
    r = rt.Renderer(width, height)
    r.anti_aliasing_mode = rt.AntiAliasingMode.Stochastic
    r.samples = spp
    r.seed = seed
    r.max_depth = 1
    feat = torch.empty((spp, height, width, FEAT_CHANNELS), dtype=torch.float16, device=dev)
    r.disk_samples = rays
    r.render_shadow_aov(scene, feat_ptr=feat.data_ptr())
    vis = torch.empty((spp, SLOTS, height, width), dtype=torch.float32, device=dev)
    r.disk_samples = target_samples
    r.render_shadow_aov(scene, vis_ptr=vis.data_ptr())
    scene.close()
    return feat, vis


def masks(feat):
    """[planes, 2, H, W] bool: the primary sample hit, and the slot's disk
    light exists (feature channels FEAT_VALID and slot-present)."""
    import torch
    valid = feat[..., 0] > 0
    present = torch.stack([feat[..., 8] > 0, feat[..., 12] > 0], 1)
    return valid.unsqueeze(1) & present


def psnr(est, ref, mask):
    """Visibility PSNR in dB over masked entries (peak 1)."""
    import torch
    m = mask.bool()
    if m.sum() == 0:
        return float("inf")
    mse = torch.mean((est[m].double() - ref[m].double()) ** 2).item()
    return float("inf") if mse == 0 else 10.0 * math.log10(1.0 / mse)


def gated(vis, conf, target, mask, threshold):
    """The visibility a render with the confidence-gated fallback uses: per
    sample and present light, the network's estimate, or where its estimated
    error exceeds the threshold the plain path's (= target: the same
    samples).  Returns (visibility, fraction of the sample-light pairs that
    fall back)."""
    import torch
    fb = (conf > threshold) & mask
    share = fb.sum().item() / max(1, mask.sum().item())
    return torch.where(fb, target, vis), share


def choose_threshold(vis, conf, target, mask, target_db=40.5, max_share=0.35):
    """The largest threshold whose gated visibility reaches target_db PSNR
    against the target on these (validation) samples, among the error
    estimates' quantiles; if none does within max_share fallback, the
    threshold at that share.  Returns (threshold, psnr, share)."""
    import torch
    c = conf[mask].float()
    qs = torch.quantile(c[torch.randperm(len(c), device=c.device)[:1_000_000]],
                        torch.linspace(0.5, 0.999, 60, device=c.device))
    best = None
    for t in sorted(qs.tolist(), reverse=True):
        g, share = gated(vis, conf, target, mask, t)
        p = psnr(g, target, mask)
        if share > max_share:
            break
        best = (t, p, share)
        if p >= target_db:
            return best
    return best if best else (float(qs[-1]), psnr(vis, target, mask), 0.0)


def make_dataset(ctx, n_scenes, first_seed, width=1920, height=1080, rays=1, target_samples=64, crops=6, crop=256,
                 log=print):
    """Renders n_scenes training scenes (training_scene(first_seed + k)) and
    keeps `crops` random crop x crop windows of each: (features [N, crop,
    crop, 16] half, target visibility [N, 2, crop, crop] half), on the GPU."""
    import tempfile
    import torch
    from .workloads import write_scene
    d = tempfile.mkdtemp(prefix="rtb_dn_")
    g = torch.Generator(device="cpu").manual_seed(first_seed)
    feats, targs = [], []
    t0 = time.time()
    for k in range(n_scenes):
        path = write_scene(d, "s.json", training_scene(first_seed + k))
        f, v = render_pair(ctx, path, width, height, rays=rays, target_samples=target_samples, seed=first_seed + k)
        ys = torch.randint(0, height - crop + 1, (crops,), generator=g).tolist()
        xs = torch.randint(0, width - crop + 1, (crops,), generator=g).tolist()
        ps = torch.randint(0, f.shape[0], (crops,), generator=g).tolist()  # one sample plane per crop
        for y, x, q in zip(ys, xs, ps):
            feats.append(f[q, y:y + crop, x:x + crop].clone())
            targs.append(v[q, :, y:y + crop, x:x + crop].half())
        if (k + 1) % 250 == 0:
            log("rendered %d/%d scenes (%.0f s)" % (k + 1, n_scenes, time.time() - t0))
    return torch.stack(feats), torch.stack(targs)


def loss_fn(vis, conf, target, mask, conf_weight=1.0):
    """Masked MSE of the visibility, plus the error head's MSE against the
    visibility's absolute error (not propagated into the visibility)."""
    m = mask.float()
    n = m.sum().clamp_min(1.0)
    err = (vis - target).abs()
    lv = ((vis - target) ** 2 * m).sum() / n
    if conf is None:
        return lv, lv
    lc = ((conf - err.detach()) ** 2 * m).sum() / n
    return lv + conf_weight * lc, lv


def fit_torch(net, feats, targs, iters=8000, batch=16, lr=2e-3, seed=0, log=print):
    """Adam on float32 copies of the convolutions (PyTorch autograd); returns
    the fitted Net (FP16 weights)."""
    import torch
    dev = feats.device
    params = torch_params(net, dev)
    flat = [t for p in params for t in p]
    opt = torch.optim.Adam(flat, lr=lr)
    sched = torch.optim.lr_scheduler.OneCycleLR(opt, max_lr=lr, total_steps=iters, pct_start=0.05)
    g = torch.Generator(device="cpu").manual_seed(seed)
    t0 = time.time()
    for it in range(iters):
        idx = torch.randint(0, feats.shape[0], (batch,), generator=g).to(dev)
        fb, tb = feats[idx], targs[idx].float()
        vis, conf = net_forward(net, fb, round_fp16=False, weights=params)
        loss, lv = loss_fn(vis, conf, tb, masks(fb))
        opt.zero_grad(set_to_none=True)
        loss.backward()
        opt.step()
        sched.step()
        if it % 500 == 0 or it == iters - 1:
            log("iter %d loss %.6f vis-mse %.6f (%.1f s)" % (it, loss.item(), lv.item(), time.time() - t0))
    return net_with_params(net, params)


def evaluate(net, feats, targs, batch=32):
    """(visibility, error estimate) of the FP16 network on the samples."""
    import torch
    vs, cs = [], []
    with torch.no_grad():
        for i in range(0, feats.shape[0], batch):
            v, c = net_forward(net, feats[i:i + batch], round_fp16=True)
            vs.append(v)
            cs.append(c)
    return torch.cat(vs), torch.cat(cs)


def train(out_path, n_scenes=2000, n_val=60, width=1920, height=1080, iters=8000, batch=16, crop=256, seed=0, rays=1,
          target_samples=64, engine="native", target_db=40.5, lr=None, log=print):
    """Renders the training set (n_scenes scenes) and a validation set
    (n_val other scenes), fits UNET (engine "native": the library's own
    tensor-core training kernels; "torch": PyTorch autograd), picks the
    confidence threshold on the validation set and writes the blob."""
    import torch
    import rtrace_b200 as rt
    torch.manual_seed(seed)
    ctx = rt.default_context(0)
    t0 = time.time()
    feats, targs = make_dataset(ctx, n_scenes, 1, width, height, rays, target_samples, 6, crop, log)
    vf, vt = make_dataset(ctx, n_val, 100_001, width, height, rays, target_samples, 6, crop, log)
    log("rendered %d training and %d validation crops in %.1f s" % (len(feats), len(vf), time.time() - t0))
    net = random_net(seed, UNET, rays=rays)
    if engine == "torch":
        net = fit_torch(net, feats, targs, iters, batch, lr=lr or 2e-3, seed=seed, log=log)
    else:
        from . import dn_train
        net = dn_train.fit_native(ctx, net, feats, targs, iters, batch, lr=lr or 1e-3, seed=seed, log=log)
    vis, conf = evaluate(net, vf, vt)
    vt = vt.float()
    m = masks(vf)
    thr, p, share = choose_threshold(vis, conf, vt, m, target_db)
    net.threshold = thr
    log("validation: visibility PSNR %.2f dB without fallback; threshold %.4f -> %.2f dB with %.1f%% of the "
        "hit-sample lights falling back" % (psnr(vis, vt, m), thr, p, 100 * share))
    blob = pack_net(net)
    with open(out_path, "wb") as f:
        f.write(blob)
    log("wrote %s (%d bytes, %d parameters)" % (out_path, len(blob), net.param_count))
    return out_path


def main(argv=None):
    ap = argparse.ArgumentParser(description="train the soft-shadow denoiser")
    ap.add_argument("command", choices=["train"])
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--scenes", type=int, default=2000)
    ap.add_argument("--val-scenes", type=int, default=60)
    ap.add_argument("--iters", type=int, default=8000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--rays", type=int, default=1, help="rays per disk light at primary hits")
    ap.add_argument("--target-samples", type=int, default=64)
    ap.add_argument("--engine", choices=["native", "torch"], default="native",
                    help="native: the library's tcgen05 training kernels; torch: PyTorch autograd")
    ap.add_argument("--target-db", type=float, default=40.5)
    ap.add_argument("--lr", type=float, default=None, help="peak learning rate (native: 1e-3, torch: 2e-3)")
    ap.add_argument("--log", default=None)
    a = ap.parse_args(argv)
    logf = open(a.log, "w") if a.log else None

    def log(msg):
        print(msg, flush=True)
        if logf:
            logf.write(msg + "\n")
            logf.flush()

    train(a.out, n_scenes=a.scenes, n_val=a.val_scenes, width=a.width, height=a.height, iters=a.iters,
          batch=a.batch, rays=a.rays, target_samples=a.target_samples, engine=a.engine, target_db=a.target_db,
          lr=a.lr, log=log)
    return 0


if __name__ == "__main__":
    sys.exit(main())
