"""Shared helpers for the outline post-process tests: seeded G-buffers and
a ctypes call of the outline entry points with torch-held device buffers."""
import ctypes

import numpy as np


def gbuffers(w, h, seed):
    """Colours, validity, depths and normals with foreground blobs, depth
    steps and normal discontinuities."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w]
    valid = np.zeros((h, w), np.uint8)
    depth = np.zeros((h, w))
    normal = np.zeros((h, w, 3))
    for _ in range(6):
        cx, cy, rad = rng.uniform(0, w), rng.uniform(0, h), rng.uniform(3, max(4, w / 4))
        m = (xx - cx) ** 2 + (yy - cy) ** 2 < rad * rad
        valid[m] = 1
        depth[m] = rng.uniform(1, 20) + 0.01 * xx[m]
        nrm = rng.normal(size=3)
        normal[m] = nrm / np.linalg.norm(nrm)
    color = rng.uniform(-0.1, 1.2, size=(h, w, 3))
    return color, valid, depth, normal


def device_outline(ctx, entry, color, valid, depth, normal, cfg):
    """Runs rt_outline_apply-like `entry` (a ctypes function) on device
    copies of the buffers; returns (status, (H, W, 3) uint8)."""
    import torch
    from rtrace_b200 import _capi
    h, w = valid.shape
    dev = torch.device("cuda", ctx.device)
    planes = [torch.tensor(np.ascontiguousarray(color[..., k]), dtype=torch.float64, device=dev) for k in range(3)]
    nplanes = [torch.tensor(np.ascontiguousarray(normal[..., k]), dtype=torch.float64, device=dev) for k in range(3)]
    v = torch.tensor(valid, dtype=torch.uint8, device=dev)
    d = torch.tensor(depth, dtype=torch.float64, device=dev)
    out = torch.zeros(h * w * 3, dtype=torch.uint8, device=dev)
    oc = _capi.rt_outline_config()
    oc.enabled = 1
    oc.use_8_neighbors = 1 if cfg.get("use_8_neighbors") else 0
    oc.depth_weight = cfg.get("depth_weight", 1.0)
    oc.normal_weight = cfg.get("normal_weight", 1.0)
    oc.threshold = cfg.get("threshold", 0.1)
    for k, c in enumerate(cfg.get("edge_color", (0.0, 0.0, 0.0))):
        oc.edge_color[k] = c
    oc.line_thickness = cfg.get("thickness", 1.0)
    torch.cuda.synchronize(dev)
    st = entry(ctx.handle, w, h, planes[0].data_ptr(), planes[1].data_ptr(), planes[2].data_ptr(), v.data_ptr(),
               d.data_ptr(), nplanes[0].data_ptr(), nplanes[1].data_ptr(), nplanes[2].data_ptr(), ctypes.byref(oc),
               out.data_ptr())
    return st, out.cpu().numpy().reshape(h, w, 3)
