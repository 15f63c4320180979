"""The k-d traversal ray set of tools/test_kdtree_consistency.rs:102-187
(144 axis-aligned and near-axis rays, 20 ring rays through the centre and
50 deterministic rays aimed at the centre), restated for any STL, plus an
optional block of seeded random rays."""
import math
import struct

import numpy as np


def stl_bounds(path):
    data = open(path, "rb").read()
    if data[:80].lstrip().startswith(b"solid") and b"facet normal" in data[:2000]:
        vs = [list(map(float, l.split()[1:4])) for l in data.decode().splitlines() if l.strip().startswith("vertex")]
        v = np.array(vs, np.float64)
    else:
        n = struct.unpack("<I", data[80:84])[0]
        rec = np.frombuffer(data[84:84 + 50 * n], dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", (3, 3)), ("a", "<u2")]))
        v = rec["v"].reshape(-1, 3).astype(np.float64)
    return v.min(0), v.max(0)


def plus_rays(path, extra_random=0, seed=1):
    bmin, bmax = stl_bounds(path)
    center = (bmin + bmax) / 2.0
    size = bmax - bmin
    me = max(size[0], size[1], size[2])
    cx, cy, cz = center
    pos = [
        (bmin[0] - me, cy, cz), (bmax[0] + me, cy, cz), (cx, bmin[1] - me, cz), (cx, bmax[1] + me, cz),
        (cx, cy, bmin[2] - me), (cx, cy, bmax[2] + me),
        (bmin[0] - me, cy + 0.1, cz + 0.1), (bmax[0] + me, cy - 0.1, cz - 0.1),
        (cx + 0.1, bmin[1] - me, cz + 0.1), (cx - 0.1, bmax[1] + me, cz - 0.1),
        (cx + 0.1, cy + 0.1, bmin[2] - me), (cx - 0.1, cy - 0.1, bmax[2] + me),
    ]
    dirs = [
        (1.0, 0.0, 0.0), (-1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, -1.0, 0.0), (0.0, 0.0, 1.0), (0.0, 0.0, -1.0),
        (1.0, 1e-9, 1e-9), (-1.0, 1e-9, -1e-9), (1e-9, 1.0, 1e-9), (-1e-9, -1.0, 1e-9), (1e-9, 1e-9, 1.0),
        (-1e-9, -1e-9, -1.0),
    ]
    rays = [p + d for p in pos for d in dirs]
    for i in range(20):
        theta = 2.0 * math.pi * i / 20
        phi = math.pi * 0.5
        d = (math.sin(theta) * math.cos(phi), math.cos(theta) * math.cos(phi), math.sin(phi))
        o = tuple(center[k] - d[k] * me * 2.0 for k in range(3))
        rays.append(o + d)
    for i in range(50):
        a1 = 2.0 * math.pi * (i / 50.0)
        a2 = math.pi * ((i * 3) % 50) / 50.0
        o = (cx + math.sin(a1) * me * 1.5, cy + math.cos(a2) * me * 1.5, cz + math.sin(a1 + a2) * me * 1.5)
        d = np.array(center) - np.array(o)
        d = d / math.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
        rays.append(o + tuple(d))
    if extra_random:
        rng = np.random.default_rng(seed)
        o = center + (rng.random((extra_random, 3)) - 0.5) * 3 * me
        tgt = center + (rng.random((extra_random, 3)) - 0.5) * me
        d = tgt - o
        rays.extend(np.concatenate([o, d], 1).tolist())
    return np.array(rays, np.float64)
