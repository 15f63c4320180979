"""Parity of the CUDA render path with the reference (golden renders) and
with the CPU oracle, through the C ABI.  Integer/byte outputs (RNG words,
RGB8 pixels) must be bit-exact, and so must the traversal's t / point /
normal (pure + - * / sqrt, which the device rounds exactly like the
reference's CPU code).  The double-precision colours before quantisation
may differ in the last bits where the reference calls a transcendental
function: CUDA's pow/exp/sin/cos are within 2 ulp of glibc's, so those are
compared with a relative tolerance of LINEAR_RTOL."""
import hashlib
import json
import os

import numpy as np
import pytest

import rtrace_b200 as rt
from rtrace_b200 import workloads
from tests import oracle_lib

pytestmark = pytest.mark.gpu

LINEAR_RTOL = 1e-13  # a few ulp of a colour channel in [0, 1]

GOLD = json.load(open(os.path.join(oracle_lib.GOLDEN, "images.json")))
AA = {"no-jitter": rt.AntiAliasingMode.NoJitter, "quincunx": rt.AntiAliasingMode.Quincunx,
      "stochastic": rt.AntiAliasingMode.Stochastic}


def gpu_render(scene_path, w, h, aa="quincunx", samples=1, outline=False, max_depth=10, seed=0, use_kdtree=True,
               linear=False):
    sc = rt.Scene.from_json_file(scene_path)
    r = rt.Renderer(w, h)
    r.anti_aliasing_mode = AA[aa]
    r.samples = samples
    r.max_depth = max_depth
    r.seed = seed
    r.use_kdtree = use_kdtree
    if outline:
        r.outline_config = sc.get_outline_config()
    out = r.render(sc, linear=linear)
    return out, r.last_stats


@pytest.mark.parametrize("case", GOLD, ids=[c["image"] for c in GOLD])
def test_gpu_matches_reference_render(gpu_ctx, case):
    img, _ = gpu_render(os.path.join(oracle_lib.SCENES, case["scene"]), case["width"], case["height"],
                        case["anti_aliasing"], case["samples"], case["outline"])
    if hashlib.sha256(img.tobytes()).hexdigest() != case["sha256_rgb"]:
        ref = oracle_lib.render(os.path.join(oracle_lib.SCENES, case["scene"]), width=case["width"],
                                height=case["height"], aa=case["anti_aliasing"], samples=case["samples"],
                                outline=case["outline"])
        d = np.abs(img.astype(int) - ref.astype(int)).max(2)
        pytest.fail("differs from the reference render: %d pixels, max %d" % ((d > 0).sum(), d.max()))


def test_device_stdrng_words(gpu_ctx):
    import ctypes
    rng = np.random.default_rng(3)
    seeds = np.concatenate([np.array([0, 1, 42, 2 ** 64 - 1], np.uint64),
                            rng.integers(0, 2 ** 63, 500, dtype=np.uint64)])
    out = np.zeros((len(seeds), 150), np.uint32)
    st = rt._capi.lib().rt_debug_stdrng_u32(gpu_ctx.handle, seeds.ctypes.data, len(seeds), 150, out.ctypes.data)
    assert st == 0
    for i, s in enumerate(seeds):
        assert np.array_equal(out[i], oracle_lib.stdrng_u32(int(s), 150)), int(s)


@pytest.mark.parametrize("radius", [1.0, 0.37, 12.5])
def test_device_disk_samples(gpu_ctx, radius):
    rng = np.random.default_rng(5)
    seeds = rng.integers(0, 2 ** 63, 400, dtype=np.uint64)
    out = np.zeros((len(seeds), 32), np.float64)
    st = rt._capi.lib().rt_debug_disk_offsets(gpu_ctx.handle, seeds.ctypes.data, len(seeds), radius, out.ctypes.data)
    assert st == 0
    for i, s in enumerate(seeds):
        assert np.array_equal(out[i], oracle_lib.disk_offsets(int(s), radius))


def _mesh_scene(stl):
    return json.dumps({
        "camera": {"kind": "ortho", "position": [0, -5, 0], "target": [0, 0, 0], "up": [0, 0, 1], "width": 1,
                   "height": 1},
        "objects": [{"kind": "mesh", "filename": stl, "material": {"color": "#FFFFFF", "ambient": 0.1,
                                                                  "diffuse": 0.7, "specular": 0.3,
                                                                  "shininess": 32}}],
        "lights": [], "scene_settings": {"ambient_illumination": {"color": "#FFFFFF", "intensity": 0.1}}})


def _surface_rays(stl, n, seed):
    """Rays starting on (or 0.001 above) triangles, in random directions:
    the shape of shadow and reflection rays."""
    from tests.kd_rays import stl_bounds
    import struct
    data = open(stl, "rb").read()
    nt = struct.unpack("<I", data[80:84])[0]
    rec = np.frombuffer(data[84:84 + 50 * nt], dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", (3, 3)),
                                                               ("a", "<u2")]))
    v = rec["v"].astype(np.float64)
    rng = np.random.default_rng(seed)
    t = rng.integers(0, nt, n)
    a, b = rng.random(n), rng.random(n)
    flip = a + b > 1
    a[flip], b[flip] = 1 - a[flip], 1 - b[flip]
    p = v[t, 0] + a[:, None] * (v[t, 1] - v[t, 0]) + b[:, None] * (v[t, 2] - v[t, 0])
    d = rng.normal(size=(n, 3))
    return np.concatenate([p, d], 1)


def _gpu_mesh(ctx, sc, rays, use_kd, mode, tmax=float("inf")):
    out = np.zeros((len(rays), 8))
    st = rt._capi.lib().rt_debug_mesh_hit(ctx.handle, sc._handle, 0, (1 if use_kd else 0) | (mode << 1),
                                          np.ascontiguousarray(rays).ctypes.data, len(rays), 0.001, tmax,
                                          out.ctypes.data)
    assert st == 0, rt._capi.lib().rt_last_error(ctx.handle)
    return out


@pytest.mark.parametrize("stl_name", ["plus.stl", "icosphere", "heightfield"])
@pytest.mark.parametrize("use_kd", [True, False])
def test_mesh_queries_match_oracle(gpu_ctx, tmp_path, use_kd, stl_name):
    from tests.kd_rays import plus_rays
    if stl_name == "plus.stl":
        stl = os.path.join(oracle_lib.SCENES, "plus.stl")
    elif stl_name == "icosphere":
        stl = os.path.join(str(tmp_path), "ico.stl")
        v, f = workloads.noisy_icosphere(4, 3)
        workloads.write_binary_stl(stl, v, f)
    else:
        # grid-aligned triangles: many edges lie exactly on k-d split planes
        stl = os.path.join(str(tmp_path), "hf.stl")
        v, f = workloads.heightfield(41, 5, height=4.0)
        workloads.write_binary_stl(stl, v, f)
    sc = rt.Scene.from_json_str(_mesh_scene(stl))
    rays = np.concatenate([plus_rays(stl, extra_random=3000), _surface_rays(stl, 3000, 9)])
    ref = oracle_lib.mesh_hit(stl, rays, use_kdtree=use_kd)
    # closest hit: BVH candidates + reference-leaf verification, and the plain k-d walk
    for mode in ((0, 1) if use_kd else (0,)):
        out = _gpu_mesh(gpu_ctx, sc, rays, use_kd, mode)
        bad = np.nonzero((out != ref).any(1))[0]
        assert len(bad) == 0, (mode, len(bad), rays[bad[:3]].tolist(), out[bad[:3]].tolist(), ref[bad[:3]].tolist())
    # any hit below a finite t_max == the reference's closest hit below it exists
    tmax = 0.7
    refa = oracle_lib.mesh_hit(stl, rays, use_kdtree=use_kd, tmax=tmax)
    outa = _gpu_mesh(gpu_ctx, sc, rays, use_kd, 2, tmax)
    assert np.array_equal(outa[:, 0], refa[:, 0])


def _culling_rays(centre, radius, rng):
    """Rays aimed at the margins of single-precision box culling: exactly
    axis-parallel rays and rays with one zero component through the mesh,
    origins a million units away aimed at it, and direction components
    below 1e-30."""
    rays = []
    for axis in range(3):
        for sign in (1.0, -1.0):
            o = centre + rng.uniform(-radius, radius, (150, 3))
            o[:, axis] = centre[axis] - sign * 3 * radius
            d = np.zeros((150, 3))
            d[:, axis] = sign
            rays.append(np.concatenate([o, d], 1))
        o = centre + rng.uniform(-1.5 * radius, 1.5 * radius, (150, 3))
        d = rng.normal(size=(150, 3))
        d[:, axis] = 0.0
        rays.append(np.concatenate([o, d], 1))
    u = rng.normal(size=(300, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    o = centre + 1e6 * u
    aim = centre + rng.uniform(-radius, radius, (300, 3))
    rays.append(np.concatenate([o, aim - o], 1))
    o = centre + rng.uniform(-radius, radius, (150, 3))
    o[:, 0] = centre[0] - 3 * radius
    d = np.stack([np.ones(150), rng.normal(size=150) * 1e-35, rng.normal(size=150) * 0.3], 1)
    rays.append(np.concatenate([o, d], 1))
    return np.concatenate(rays)


@pytest.mark.parametrize("use_kd", [True, False])
def test_shadow_box_culling_margins(gpu_ctx, tmp_path, use_kd):
    """Shadow rays cull mesh boxes in single precision, with margins taken
    from the ray origin and the mesh's coordinate scale.  The any-hit answer
    must stay the reference's on a mesh 25,000 units from the origin (float
    spacing there is 2e-3 against triangles of 0.15) and on rays that put
    those margins to the test."""
    stl = os.path.join(str(tmp_path), "far.stl")
    v, f = workloads.noisy_icosphere(3, 5)
    v = v + np.array([1.0e4, -2.5e4, 3.0e3])
    workloads.write_binary_stl(stl, v, f)
    sc = rt.Scene.from_json_str(_mesh_scene(stl))
    rng = np.random.default_rng(21)
    centre = v.mean(0)
    rays = np.concatenate([_surface_rays(stl, 2000, 13), _culling_rays(centre, 1.0, rng)])
    for tmax in (0.7, 4.0, float("inf")):
        refa = oracle_lib.mesh_hit(stl, rays, use_kdtree=use_kd, tmax=tmax)
        outa = _gpu_mesh(gpu_ctx, sc, rays, use_kd, 2, tmax)
        bad = np.nonzero(outa[:, 0] != refa[:, 0])[0]
        assert len(bad) == 0, (tmax, len(bad), rays[bad[:3]].tolist())
        assert 0 < refa[:, 0].sum() < len(rays)
    # the same rays around the origin, where the margins are tightest
    stl0 = os.path.join(str(tmp_path), "near.stl")
    v0 = v - v.mean(0)
    workloads.write_binary_stl(stl0, v0, f)
    sc0 = rt.Scene.from_json_str(_mesh_scene(stl0))
    rays0 = np.concatenate([_surface_rays(stl0, 2000, 14), _culling_rays(v0.mean(0), 1.0, rng)])
    refa = oracle_lib.mesh_hit(stl0, rays0, use_kdtree=use_kd, tmax=4.0)
    outa = _gpu_mesh(gpu_ctx, sc0, rays0, use_kd, 2, 4.0)
    assert np.array_equal(outa[:, 0], refa[:, 0])


def _synthetic_scenes(tmp):
    d = str(tmp)
    paths = {"sphere_grid": workloads.write_scene(d, "sphere_grid.json", workloads.sphere_grid_scene()),
             "icosphere": workloads.make_noisy_icosphere(d, level=3, seed=5),
             "rings": workloads.write_scene(d, "rings.json", workloads.ring_spheres_scene(seed=1, n_rings=3,
                                                                                         per_ring=15))}
    # area light + reflections + cube + checkerboard + transforms
    s = json.load(open(os.path.join(oracle_lib.SCENES, "checkerboard-advanced.json")))
    s["lights"].append({"position": [1, -2, 4], "color": "#FFEEDD", "intensity": 0.7, "diameter": 1.5})
    s["objects"].append({"kind": "cube", "center": [1, 1, 0.5], "size": [1, 2, 0.5],
                         "transform": ["rotate(10, 20, 30)", "scale(1, 2, 1)", "translate(0.5, 0, 0)"],
                         "material": {"color": "#33AA77", "ambient": 0.1, "diffuse": 0.7, "specular": 0.3,
                                      "shininess": 16, "reflectivity": 0.4}})
    paths["mixed"] = workloads.write_scene(d, "mixed.json", s)
    # the large-mesh configuration's scene at a small size
    hv, hf = workloads.heightfield(25, 11)
    workloads.write_binary_stl(os.path.join(d, "terrain.stl"), hv, hf)
    t = workloads.terrain_scene("terrain.stl", 25)
    t["objects"][1]["center"] = [0, 0, 12]
    t["objects"][1]["radius"] = 4
    paths["terrain"] = workloads.write_scene(d, "terrain.json", t)
    return paths


@pytest.mark.parametrize("aa,samples", [("quincunx", 1), ("no-jitter", 1), ("no-jitter", 3), ("stochastic", 1),
                                        ("stochastic", 4)])
def test_modes_match_oracle(gpu_ctx, tmp_path, aa, samples):
    for name, path in _synthetic_scenes(tmp_path).items():
        outline = name in ("icosphere", "terrain") and aa != "quincunx"
        (img, lin), st = gpu_render(path, 71, 43, aa, samples, outline=outline, linear=True)
        ref, rlin, cnt = oracle_lib.render(path, width=71, height=43, aa=aa, samples=samples, outline=outline,
                                           linear=True, counts=True)
        assert np.array_equal(img, ref), (name, int((img != ref).any(2).sum()))
        assert np.allclose(lin, rlin, rtol=LINEAR_RTOL, atol=1e-15), (name, float(np.abs(lin - rlin).max()))
        assert (st.primary_rays, st.reflection_rays, st.shadow_rays) == (int(cnt[0]), int(cnt[1]), int(cnt[2])), name


def test_facing_away_lights_are_not_traced(gpu_ctx, tmp_path):
    """Shadow rays toward a light the surface faces away from are not traced
    (the reference's light term is exactly zero there); the image stays the
    reference's and the rays are still counted as the reference casts them."""
    paths = _synthetic_scenes(tmp_path)
    for name in ("icosphere", "rings", "mixed"):
        img, st = gpu_render(paths[name], 80, 50, "no-jitter")
        ref, cnt = oracle_lib.render(paths[name], width=80, height=50, aa="no-jitter", counts=True)
        assert np.array_equal(img, ref), name
        assert st.shadow_rays == int(cnt[2]) and 0 < st.shadow_rays_untraced < st.shadow_rays, name


def test_brute_force_and_seed(gpu_ctx, tmp_path):
    path = _synthetic_scenes(tmp_path)["icosphere"]
    for kd in (True, False):
        img, _ = gpu_render(path, 40, 30, "stochastic", 2, seed=12345, use_kdtree=kd)
        ref = oracle_lib.render(path, width=40, height=30, aa="stochastic", samples=2, seed=12345, use_kdtree=kd)
        assert np.array_equal(img, ref)


def test_depth_limits(gpu_ctx, tmp_path):
    path = _synthetic_scenes(tmp_path)["mixed"]
    for depth in (0, 1, 2, 3):
        img, _ = gpu_render(path, 33, 21, "no-jitter", 1, max_depth=depth)
        ref = oracle_lib.render(path, width=33, height=21, aa="no-jitter", max_depth=depth)
        assert np.array_equal(img, ref), depth


def test_render_errors(gpu_ctx):
    scene = json.load(open(os.path.join(oracle_lib.SCENES, "object-sphere.json")))
    sc = rt.Scene.from_json_str(json.dumps(scene))
    r = rt.Renderer(10, 10)
    r.samples = 0
    with pytest.raises(rt.RenderError, match="Samples must be greater than 0"):
        r.render(sc)
    for mut, msg in [(lambda s: s["camera"].__setitem__("kind", "fisheye"), "Unsupported camera type: fisheye"),
                     (lambda s: s["camera"].update(kind="perspective", fov=0), "Field of view"),
                     (lambda s: s["objects"][0]["material"].__setitem__("color", "#12345"), "Invalid hex color"),
                     (lambda s: s["lights"][0].__setitem__("diameter", 0.0), "cannot sample empty range")]:
        s2 = json.loads(json.dumps(scene))
        mut(s2)
        with pytest.raises(rt.RenderError, match=msg):
            rt.Renderer(10, 10).render(rt.Scene.from_json_str(json.dumps(s2)))
    with pytest.raises(rt.SceneError):
        rt.Scene.from_json_str("{\"camera\": 3}")


OUTLINE_CFGS = [
    {},
    {"use_8_neighbors": True, "thickness": 2.0, "depth_weight": 0.8, "normal_weight": 2.0, "threshold": 0.06,
     "edge_color": (0.2, 0.3, 0.4)},
    {"thickness": 3.5, "threshold": 0.9, "edge_color": (1.0, 0.0, 0.5)},
]


@pytest.mark.parametrize("cfg", OUTLINE_CFGS)
def test_outline_entry_point_matches_oracle(gpu_ctx, cfg):
    from tests.gpu_outline import device_outline, gbuffers
    for (w, h, seed) in [(97, 61, 1), (320, 200, 2)]:
        color, valid, depth, normal = gbuffers(w, h, seed)
        st, img = device_outline(gpu_ctx, rt._capi.lib().rt_outline_apply, color, valid, depth, normal, cfg)
        assert st == 0
        ref = oracle_lib.outline(color, valid, depth, normal, cfg.get("depth_weight", 1.0),
                                 cfg.get("normal_weight", 1.0), cfg.get("threshold", 0.1),
                                 cfg.get("edge_color", (0.0, 0.0, 0.0)), cfg.get("use_8_neighbors", False),
                                 cfg.get("thickness", 1.0))
        assert np.array_equal(img, ref), (w, h, int((img != ref).any(2).sum()))


@pytest.mark.parametrize("thickness", [65.0, 80.0, 130.5])
def test_thick_outlines_match_oracle(gpu_ctx, tmp_path, thickness):
    """Dilation radii beyond the shared-memory tile (thickness above 65)
    take the global-memory path; the reference dilates at any thickness
    (src/outline.rs:227-268).  The outline entry point against the oracle's
    outline, and a whole render with such an outline against the oracle's
    render."""
    from tests.gpu_outline import device_outline, gbuffers
    cfg = {"thickness": thickness, "threshold": 0.3, "edge_color": (0.9, 0.1, 0.2), "use_8_neighbors": True}
    color, valid, depth, normal = gbuffers(97, 61, 7)
    st, img = device_outline(gpu_ctx, rt._capi.lib().rt_outline_apply, color, valid, depth, normal, cfg)
    assert st == 0
    ref = oracle_lib.outline(color, valid, depth, normal, 1.0, 1.0, 0.3, (0.9, 0.1, 0.2), True, thickness)
    assert np.array_equal(img, ref), int((img != ref).any(2).sum())
    path = workloads.make_noisy_icosphere(str(tmp_path), level=3, seed=5)
    s = json.load(open(path))
    s["scene_settings"]["outline"]["thickness"] = thickness
    p2 = workloads.write_scene(str(tmp_path), "thick.json", s)
    got, _ = gpu_render(p2, 64, 40, "no-jitter", 1, outline=True)
    want = oracle_lib.render(p2, width=64, height=40, aa="no-jitter", outline=True)
    assert np.array_equal(got, want), int((got != want).any(2).sum())


def test_object_id_outline_term(gpu_ctx):
    """Extension: with object_id_weight > 0 the outline also marks edges
    between different objects.  Two unit cubes touch along x = 0 with
    coplanar tops; seen from above, depth and normal are continuous across
    the seam, so the reference's outline (weight 0, the oracle's render)
    draws nothing there, and the object term draws the seam."""
    cube = lambda x: {"kind": "cube", "center": [x, 0, 0], "size": [1, 1, 1],
                      "material": {"color": "#D0D0D0", "ambient": 0.3, "diffuse": 0.7, "specular": 0.0,
                                   "shininess": 8}}
    scene = {"camera": {"kind": "ortho", "position": [0.013, 0.007, 10], "target": [0.013, 0.007, 0],
                        "up": [0, 1, 0], "width": 4, "height": 2},
             "objects": [cube(-0.5), cube(0.5)],
             "lights": [{"position": [2, 3, 8], "color": "#FFFFFF", "intensity": 1.0}],
             "scene_settings": {"ambient_illumination": {"color": "#FFFFFF", "intensity": 0.2},
                                "background_color": "#000000",
                                "outline": {"enabled": True, "color": "#FF00FF", "threshold": 0.1}}}
    js = json.dumps(scene)
    sc = rt.Scene.from_json_str(js)
    W, H = 80, 40
    r = rt.Renderer(W, H)
    r.anti_aliasing_mode = rt.AntiAliasingMode.NoJitter
    r.outline_config = sc.get_outline_config()
    assert r.outline_config.object_id_weight == 0.0
    base = r.render(sc)
    assert np.array_equal(base, oracle_lib.render(json_text=js, width=W, height=H, aa="no-jitter", outline=True))
    magenta = (base == [255, 0, 255]).all(2)
    r.outline_config.object_id_weight = 1.0
    ids = r.render(sc)
    changed = (ids != base).any(2)
    cols = np.nonzero(changed.any(0))[0]
    # only the two columns on either side of the seam change, to the edge colour
    assert changed.sum() > 10 and set(cols.tolist()) <= {W // 2 - 1, W // 2}
    assert (ids[changed] == [255, 0, 255]).all()
    assert not magenta[:, W // 2 - 1:W // 2 + 1][changed[:, W // 2 - 1:W // 2 + 1]].any()


@pytest.mark.gpu
def test_host_scene_uploads_render_the_same(gpu_ctx, tmp_path):
    """A host scene's first upload prepares its meshes and keeps them packed
    in pinned memory; later uploads copy that image.  Both, and the generic
    description path (rt_scene_upload), must give the same frame."""
    import ctypes
    import rtrace_b200 as rt
    from rtrace_b200 import _capi, workloads
    path = workloads.make_noisy_icosphere(str(tmp_path), level=4, seed=3)
    host = rt.HostScene.from_json_file(path)
    r = rt.Renderer(200, 120)
    r.anti_aliasing_mode = rt.AntiAliasingMode.NoJitter
    imgs = []
    for _ in range(3):
        sc = rt.Scene.upload(host, gpu_ctx)
        imgs.append(r.render(sc))
        assert sc.device_bytes > 0
        sc.close()
    L = _capi.lib()
    h = ctypes.c_void_p()
    st = L.rt_scene_upload(gpu_ctx.handle, L.rt_host_scene_desc(host.handle), ctypes.byref(h))
    assert st == 0, L.rt_last_error(gpu_ctx.handle)
    generic = rt.Scene(h, gpu_ctx)
    imgs.append(r.render(generic))
    generic.close()
    direct = r.render(rt.Scene.from_json_file(path, gpu_ctx))
    for img in imgs:
        assert np.array_equal(img, direct)


@pytest.mark.parametrize("stl_name", ["plus.stl", "heightfield", "far_icosphere"])
def test_leaf_visits_from_cells_match_root_walk(gpu_ctx, tmp_path, stl_name):
    """Verification decides whether the reference visits a k-d leaf from the
    leaf's cell (the splits on its root path) instead of walking from the
    root.  For every leaf and every ray the two must agree: rays from the
    k-d edge-case generator (axis-aligned, on split planes), surface rays,
    and the culling rays (zero and tiny direction components, far origins)."""
    from tests.kd_rays import plus_rays
    rng = np.random.default_rng(31)
    if stl_name == "plus.stl":
        stl = os.path.join(oracle_lib.SCENES, "plus.stl")
        centre, radius = np.zeros(3), 1.0
    elif stl_name == "heightfield":
        stl = os.path.join(str(tmp_path), "hf.stl")
        v, f = workloads.heightfield(17, 5, height=4.0)
        workloads.write_binary_stl(stl, v, f)
        centre, radius = v.mean(0), 2.0
    else:
        stl = os.path.join(str(tmp_path), "far.stl")
        v, f = workloads.noisy_icosphere(2, 5)
        v = v + np.array([1.0e4, -2.5e4, 3.0e3])
        workloads.write_binary_stl(stl, v, f)
        centre, radius = v.mean(0), 1.0
    sc = rt.Scene.from_json_str(_mesh_scene(stl))
    rays = np.concatenate([plus_rays(stl, extra_random=600), _surface_rays(stl, 600, 33),
                           _culling_rays(centre, radius, rng)])
    out = _gpu_mesh(gpu_ctx, sc, rays, True, 3)
    assert out[:, 0].sum() == 0, (int(out[:, 0].sum()), rays[np.nonzero(out[:, 0])[0][:3]].tolist())
    assert out[:, 1].min() > 0 and out[:, 2].sum() > 0
