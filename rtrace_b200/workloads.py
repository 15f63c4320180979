"""Seeded synthetic scenes for the benchmark configurations.

Every scene is written as the reference's own input format (scene JSON +
binary STL with f32 vertices) so that the same files drive this renderer
and the CPU oracle.  No public dataset is involved; the seeds and
parameters below are the whole definition of each workload.

  sphere_grid   small scene: ortho camera at (0,-10,5), 6x6 view, sphere
                r=1.5, grid plane at z=-1.5 (reflectivity 0.2), point
                light (3,-3,5); rendered at 400x300 quincunx, depth 10.
  noisy_icosphere  mesh path: level-6 icosphere (81,920 triangles)
                radially displaced by seeded value noise (+-5%), reflective
                ground plane (0.3), one disk light of diameter 2 (the
                reference samples 16 points per shading point), fog start 5
                end 50 density 0.05, outline on, perspective FOV 50, 16:9.
  ring_spheres  1,000 spheres on 10 rings (radius 1..10), radii U(0.05,
                0.3), HSV colours, reflectivity 0.5, two disk lights.
  terrain       fractal value-noise heightfield (2 * (n-1)^2 triangles),
                mirror sphere r=20 (reflectivity 0.9), one disk light,
                fog density 0.02, outline on.
"""
import colorsys
import json
import math
import os
import struct

import numpy as np


# ----------------------------------------------------------------- meshes --
def icosphere(level):
    """Vertices (V, 3) and faces (F, 3) of a unit icosphere."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        cache = {}

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts), np.array(faces, np.int64)


def _hash3(ix, iy, iz, seed):
    h = (ix * 73856093) ^ (iy * 19349663) ^ (iz * 83492791) ^ (seed * 2654435761)
    h = (h ^ (h >> 13)) * 1274126177
    h = h ^ (h >> 16)
    return (h & 0xFFFFFF).astype(np.float64) / float(0xFFFFFF) * 2.0 - 1.0


def value_noise3(p, seed, freq=4.0):
    """Trilinear value noise on an integer hash lattice, in [-1, 1]."""
    q = p * freq
    i0 = np.floor(q).astype(np.int64)
    f = q - i0
    s = f * f * (3 - 2 * f)
    out = np.zeros(len(p))
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                w = (s[:, 0] if dx else 1 - s[:, 0]) * (s[:, 1] if dy else 1 - s[:, 1]) * (s[:, 2] if dz else 1 - s[:, 2])
                out += w * _hash3(i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz, seed)
    return out


def value_noise2(x, y, seed):
    xi, yi = np.floor(x).astype(np.int64), np.floor(y).astype(np.int64)
    fx, fy = x - xi, y - yi
    sx, sy = fx * fx * (3 - 2 * fx), fy * fy * (3 - 2 * fy)
    z = np.zeros_like(xi)
    n00 = _hash3(xi, yi, z, seed)
    n10 = _hash3(xi + 1, yi, z, seed)
    n01 = _hash3(xi, yi + 1, z, seed)
    n11 = _hash3(xi + 1, yi + 1, z, seed)
    return (n00 * (1 - sx) + n10 * sx) * (1 - sy) + (n01 * (1 - sx) + n11 * sx) * sy


def write_binary_stl(path, verts, faces):
    """Binary STL, f32 vertices (the reference widens them to f64)."""
    tri = verts[faces].astype(np.float32)
    n = len(faces)
    rec = np.zeros(n, dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", (3, 3)), ("a", "<u2")]))
    e1 = tri[:, 1] - tri[:, 0]
    e2 = tri[:, 2] - tri[:, 0]
    nn = np.cross(e1, e2)
    nn /= np.maximum(np.linalg.norm(nn, axis=1, keepdims=True), 1e-30)
    rec["n"] = nn
    rec["v"] = tri
    with open(path, "wb") as f:
        f.write(b"binary STL written by rtrace_b200.workloads".ljust(80, b" "))
        f.write(struct.pack("<I", n))
        f.write(rec.tobytes())


def noisy_icosphere(level, seed, amplitude=0.05):
    v, f = icosphere(level)
    v = v * (1.0 + amplitude * value_noise3(v, seed))[:, None]
    return v, f


def heightfield(n, seed, scale=1.0, height=40.0, octaves=5):
    """n x n grid heightfield of fractal value noise: 2 (n-1)^2 triangles."""
    xs = np.arange(n, dtype=np.float64)
    X, Y = np.meshgrid(xs, xs, indexing="xy")
    z = np.zeros_like(X)
    amp, freq = 1.0, 1.0 / 128.0
    for o in range(octaves):
        z += amp * value_noise2(X * freq, Y * freq, seed + o)
        amp *= 0.5
        freq *= 2.0
    verts = np.stack([(X - (n - 1) / 2) * scale, (Y - (n - 1) / 2) * scale, z * height], -1).reshape(-1, 3)
    idx = np.arange(n * n).reshape(n, n)
    a, b, c, d = idx[:-1, :-1].ravel(), idx[:-1, 1:].ravel(), idx[1:, :-1].ravel(), idx[1:, 1:].ravel()
    faces = np.concatenate([np.stack([a, b, d], 1), np.stack([a, d, c], 1)])
    return verts, faces


# ----------------------------------------------------------------- scenes --
def _mat(color, ambient=0.1, diffuse=0.8, specular=0.4, shininess=32, reflectivity=None, texture=None):
    m = {"color": color, "ambient": ambient, "diffuse": diffuse, "specular": specular, "shininess": shininess}
    if reflectivity is not None:
        m["reflectivity"] = reflectivity
    if texture is not None:
        m["texture"] = texture
    return m


def _hex(rgb):
    return "#%02X%02X%02X" % tuple(int(round(255 * c)) for c in rgb)


def sphere_grid_scene():
    """The small CPU-runnable configuration (400x300 quincunx)."""
    return {
        "camera": {"kind": "ortho", "position": [0, -10, 5], "target": [0, 0, 0], "up": [0, 0, 1],
                   "width": 6, "height": 6},
        "objects": [
            {"kind": "sphere", "center": [0, 0, 0], "radius": 1.5, "material": _mat("#FF4444")},
            {"kind": "plane", "point": [0, 0, -1.5], "normal": [0, 0, 1],
             "material": _mat("#CCCCCC", 0.1, 0.7, 0.2, 16, reflectivity=0.2,
                              texture={"type": "grid", "line_color": "#333333", "line_width": 0.05,
                                       "cell_size": 1.0})},
        ],
        "lights": [{"position": [3, -3, 5], "color": "#FFFFFF", "intensity": 1.0}],
        "scene_settings": {"ambient_illumination": {"color": "#FFFFFF", "intensity": 0.1},
                           "background_color": "#000000"},
    }


def noisy_icosphere_scene(mesh_file, outline=True):
    """Mesh configuration; mesh_file is a path relative to the scene file."""
    return {
        "camera": {"kind": "perspective", "position": [3.2, -4.2, 2.1], "target": [0, 0, 0.1], "up": [0, 0, 1],
                   "fov": 50, "width": 16, "height": 9},
        "objects": [
            {"kind": "mesh", "filename": mesh_file, "material": _mat("#4A90D9", 0.1, 0.75, 0.5, 48)},
            {"kind": "plane", "point": [0, 0, -1.1], "normal": [0, 0, 1],
             "material": _mat("#D8D8D8", 0.12, 0.7, 0.2, 16, reflectivity=0.3,
                              texture={"type": "grid", "line_color": "#555555", "line_width": 0.04,
                                       "cell_size": 1.0})},
        ],
        "lights": [{"position": [2.5, -2.0, 5.0], "color": "#FFFFFF", "intensity": 1.2, "diameter": 2.0}],
        "scene_settings": {
            "ambient_illumination": {"color": "#FFFFFF", "intensity": 0.12},
            "background_color": "#0B1020",
            "fog": {"color": "#8090A0", "density": 0.05, "start": 5.0, "end": 50.0},
            "outline": {"enabled": bool(outline), "depth_weight": 1.0, "normal_weight": 1.0, "threshold": 0.1,
                        "color": "#101010", "thickness": 1.0, "use_8_neighbors": False},
        },
    }


def ring_spheres_scene(seed=0, n_rings=10, per_ring=100):
    rng = np.random.default_rng(seed)
    objs = []
    for ring in range(n_rings):
        R = 1.0 + 9.0 * ring / max(1, n_rings - 1)
        for _ in range(per_ring):
            a = rng.uniform(0, 2 * math.pi)
            r = rng.uniform(0.05, 0.3)
            z = rng.uniform(-0.2, 0.6)
            col = colorsys.hsv_to_rgb(rng.uniform(0, 1), rng.uniform(0.5, 1.0), rng.uniform(0.6, 1.0))
            objs.append({"kind": "sphere", "center": [round(R * math.cos(a), 6), round(R * math.sin(a), 6),
                                                      round(z, 6)],
                         "radius": round(r, 6), "material": _mat(_hex(col), 0.1, 0.7, 0.5, 64, reflectivity=0.5)})
    objs.append({"kind": "plane", "point": [0, 0, -0.5], "normal": [0, 0, 1],
                 "material": _mat("#C8C8C8", 0.1, 0.8, 0.1, 8)})
    return {
        "camera": {"kind": "perspective", "position": [0, -16, 11], "target": [0, 0, 0], "up": [0, 0, 1],
                   "fov": 50, "width": 16, "height": 9},
        "objects": objs,
        "lights": [{"position": [-6, -6, 9], "color": "#FFF4E0", "intensity": 0.8, "diameter": 2.0},
                   {"position": [7, 3, 8], "color": "#E0F0FF", "intensity": 0.6, "diameter": 2.0}],
        "scene_settings": {"ambient_illumination": {"color": "#FFFFFF", "intensity": 0.1},
                           "background_color": "#101418"},
    }


def terrain_scene(mesh_file, n):
    half = (n - 1) / 2.0
    return {
        "camera": {"kind": "perspective", "position": [half * 0.9, -half * 0.9, half * 0.7],
                   "target": [0, 0, 0], "up": [0, 0, 1], "fov": 50, "width": 16, "height": 9},
        "objects": [
            {"kind": "mesh", "filename": mesh_file, "material": _mat("#7A8F5A", 0.1, 0.8, 0.1, 8)},
            {"kind": "sphere", "center": [0, 0, 60], "radius": 20,
             "material": _mat("#E0E0E0", 0.05, 0.2, 0.9, 128, reflectivity=0.9)},
        ],
        "lights": [{"position": [half * 0.5, -half * 0.2, 400], "color": "#FFFFFF", "intensity": 1.1,
                    "diameter": 2.0}],
        "scene_settings": {
            "ambient_illumination": {"color": "#FFFFFF", "intensity": 0.15},
            "background_color": "#7FA6D0",
            "fog": {"color": "#B0C4DE", "density": 0.02, "start": 0.0, "end": 1000.0},
            "outline": {"enabled": True, "color": "#202020"},
        },
    }


def write_scene(directory, name, scene):
    os.makedirs(directory, exist_ok=True)
    path = os.path.join(directory, name)
    with open(path, "w") as f:
        json.dump(scene, f, indent=1)
    return path


def make_noisy_icosphere(directory, level=6, seed=7, outline=True):
    """Writes the mesh-path scene; returns the scene path."""
    os.makedirs(directory, exist_ok=True)
    stl = "icosphere_l%d_s%d.stl" % (level, seed)
    sp = os.path.join(directory, stl)
    if not os.path.exists(sp):
        v, f = noisy_icosphere(level, seed)
        write_binary_stl(sp, v, f)
    return write_scene(directory, "noisy_icosphere_l%d.json" % level, noisy_icosphere_scene(stl, outline))


def make_terrain(directory, n=1024, seed=11):
    os.makedirs(directory, exist_ok=True)
    stl = "terrain_%d_s%d.stl" % (n, seed)
    sp = os.path.join(directory, stl)
    if not os.path.exists(sp):
        v, f = heightfield(n, seed)
        write_binary_stl(sp, v, f)
    return write_scene(directory, "terrain_%d.json" % n, terrain_scene(stl, n))


def cli_size(aspect, diagonal):
    """Image size from a diagonal (cli/src/main.rs:339-350)."""
    from rtrace_b200.cli import image_size
    return image_size(aspect, diagonal)


# ------------------------------------------------------------ batch (C4) --
BATCH_RESOLUTIONS = [(128, 128), (256, 256), (640, 480), (1280, 720), (1920, 1080)]
BATCH_MESH_LEVELS = [3, 4, 5, 6]  # noisy icospheres of 1,280 .. 81,920 triangles


def batch_scene(seed, mesh_dir_rel="meshes"):
    """One scene of the batch workload: 1-4 lights (point or disk), 0-3
    noisy-icosphere meshes placed by transforms, 0-200 spheres and one grid
    plane.  Mesh files are referenced as mesh_dir_rel/ico_l<level>_s<k>.stl
    (batch_meshes writes them)."""
    rng = np.random.default_rng(50_000 + seed)
    objs = []
    n_mesh = int(rng.integers(0, 4))
    for _ in range(n_mesh):
        level = int(rng.choice(BATCH_MESH_LEVELS))
        k = int(rng.integers(0, 2))
        s = float(rng.uniform(0.8, 2.5))
        tx, ty = (float(v) for v in rng.uniform(-6, 6, 2))
        col = colorsys.hsv_to_rgb(rng.uniform(0, 1), rng.uniform(0.3, 0.9), rng.uniform(0.6, 1.0))
        objs.append({"kind": "mesh", "filename": "%s/ico_l%d_s%d.stl" % (mesh_dir_rel, level, k),
                     "transform": ["scale(%.4f, %.4f, %.4f)" % (s, s, s), "translate(%.4f, %.4f, %.4f)" % (tx, ty, s)],
                     "material": _mat(_hex(col), 0.1, 0.7, 0.4, 32,
                                      reflectivity=round(float(rng.uniform(0, 0.5)), 3))})
    n_sph = int(rng.integers(0, 201))
    for _ in range(n_sph):
        r = float(rng.uniform(0.1, 0.6))
        c = [round(float(v), 4) for v in (rng.uniform(-9, 9), rng.uniform(-9, 9), r + rng.uniform(0, 2))]
        col = colorsys.hsv_to_rgb(rng.uniform(0, 1), rng.uniform(0.4, 1.0), rng.uniform(0.6, 1.0))
        m = _mat(_hex(col), 0.1, 0.7, 0.5, 64)
        if rng.uniform() < 0.3:
            m["reflectivity"] = round(float(rng.uniform(0.2, 0.8)), 3)
        objs.append({"kind": "sphere", "center": c, "radius": round(r, 4), "material": m})
    objs.append({"kind": "plane", "point": [0, 0, 0], "normal": [0, 0, 1],
                 "material": _mat("#B4B4B4", 0.1, 0.8, 0.1, 8, reflectivity=0.2,
                                  texture={"type": "grid", "line_color": "#404040", "line_width": 0.04,
                                           "cell_size": 1.0})})
    lights = []
    for _ in range(int(rng.integers(1, 5))):
        L = {"position": [round(float(v), 3) for v in (rng.uniform(-10, 10), rng.uniform(-10, 10),
                                                        rng.uniform(6, 14))],
             "color": _hex(colorsys.hsv_to_rgb(rng.uniform(0, 1), 0.15, 1.0)),
             "intensity": round(float(rng.uniform(0.3, 0.8)), 3)}
        if rng.uniform() < 0.5:
            L["diameter"] = round(float(rng.uniform(0.5, 2.5)), 3)
        lights.append(L)
    if not n_mesh and not n_sph:  # keep a finite object for the auto cameras
        objs.insert(0, {"kind": "sphere", "center": [0, 0, 1], "radius": 1.0, "material": _mat("#E0C080")})
    return {
        "camera": {"kind": "perspective", "position": [12, -12, 9], "target": [0, 0, 0], "up": [0, 0, 1],
                   "fov": 50, "width": 16, "height": 9},
        "objects": objs,
        "lights": lights,
        "scene_settings": {"ambient_illumination": {"color": "#FFFFFF", "intensity": 0.1},
                           "background_color": "#1A2030"},
    }


def batch_meshes(directory):
    """Writes the batch workload's mesh files (two noise seeds per level)."""
    d = os.path.join(directory, "meshes")
    os.makedirs(d, exist_ok=True)
    for level in BATCH_MESH_LEVELS:
        for k in range(2):
            p = os.path.join(d, "ico_l%d_s%d.stl" % (level, k))
            if not os.path.exists(p):
                v, f = noisy_icosphere(level, 300 + 10 * level + k)
                write_binary_stl(p, v, f)


def batch_workload(directory, n_scenes=64, seed=0):
    """The batch configuration: n_scenes seeded scenes, each rendered from
    its four auto-camera views (left, front, top, perspective) at a
    resolution drawn uniformly from BATCH_RESOLUTIONS.  Returns
    [(scene_path, [(view, camera_dict, (width, height)), ...]), ...]."""
    import rtrace_b200 as rt
    batch_meshes(directory)
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_scenes):
        path = write_scene(directory, "batch_%03d.json" % k, batch_scene(seed * 1000 + k))
        cams = rt.auto_cameras(path=path)
        views = []
        for name in ("left", "front", "top", "perspective"):
            w, h = BATCH_RESOLUTIONS[int(rng.integers(0, len(BATCH_RESOLUTIONS)))]
            views.append((name, cams[name], (w, h)))
        out.append((path, views))
    return out
