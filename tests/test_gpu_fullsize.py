"""Parity at the benchmark configurations' own sizes.

The other parity tests render miniatures (at most 400x300).  Here each
benchmark scene is rendered whole on the GPU at its native resolution, the
way the benchmark renders it, and a band of its rows is compared with the
oracle's render of the same rows (the oracle's k-d walk has no t-pruning,
so whole frames would take it minutes to hours).  With the outline on, the
oracle's band lacks the neighbouring rows' depth and normals, so its first
and last 1 + ceil(thickness - 1) rows differ by construction; those halo
rows are rendered but not compared.

Tolerance (the renderer's stated bar): RGB8 identical on at least 99.9% of
the compared pixels and within 1 LSB elsewhere.  The count of differing
pixels is reported in the assertion message."""
import copy
import json
import math
import os

import numpy as np
import pytest

import rtrace_b200 as rt
from rtrace_b200 import workloads
from tests import oracle_lib

pytestmark = pytest.mark.gpu

AA_CODE = {rt.AntiAliasingMode.NoJitter: 0, rt.AntiAliasingMode.Quincunx: 1, rt.AntiAliasingMode.Stochastic: 2}
MIN_IDENTICAL = 0.999
MAX_LSB = 1


@pytest.fixture(scope="module")
def scenes(tmp_path_factory):
    return str(tmp_path_factory.mktemp("fullsize"))


def oracle_rows(path, w, h, renderer, y0, y1):
    """The oracle's rows [y0, y1) of the frame renderer would render."""
    import ctypes
    L = oracle_lib.load()
    out = np.zeros((h, w, 3), np.uint8)
    err = ctypes.create_string_buffer(1024)
    outline = 1 if renderer.outline_config is not None else 0
    rc = L.oracle_render_ex(path.encode(), None, w, h, AA_CODE[renderer.anti_aliasing_mode], renderer.samples,
                            renderer.max_depth, renderer.seed, 1, outline, os.cpu_count() or 1, y0, y1,
                            renderer.disk_samples, out.ctypes.data, None, None, err, 1024)
    assert rc == 0, err.value.decode()
    return out[y0:y1]


def halo(renderer):
    cfg = renderer.outline_config
    if cfg is None:
        return 0
    return 1 + max(0, math.ceil(cfg.line_thickness - 1.0))


def check_band(gpu_img, path, renderer, y0, y1):
    """Compares rows [y0, y1) of the GPU frame with the oracle, dropping the
    outline halo at both ends; returns (compared pixels, differing pixels)."""
    h, w = gpu_img.shape[:2]
    ref = oracle_rows(path, w, h, renderer, y0, y1)
    k = halo(renderer)
    got, want = gpu_img[y0 + k:y1 - k], ref[k:y1 - y0 - k]
    assert got.shape[0] > 0
    diff = np.abs(got.astype(np.int16) - want.astype(np.int16)).max(2)
    n, bad = diff.size, int((diff > 0).sum())
    assert (n - bad) / n >= MIN_IDENTICAL and diff.max() <= MAX_LSB, \
        "rows %d-%d: %d of %d pixels differ, max %d LSB" % (y0 + k, y1 - k, bad, n, int(diff.max()))
    return n, bad


def test_mesh_frame_1080p(gpu_ctx, scenes):
    """The headline frame: 81,920-triangle noisy icosphere, disk light,
    fog, outline on, no-jitter, 1920x1080, depth 10."""
    path = workloads.make_noisy_icosphere(scenes, level=6, seed=7, outline=True)
    sc = rt.Scene.from_json_file(path, gpu_ctx)
    r = rt.Renderer(1920, 1080)
    r.anti_aliasing_mode = rt.AntiAliasingMode.NoJitter
    r.outline_config = sc.get_outline_config()
    img = r.render(sc)
    for y0 in (530, 250):  # through the mesh and its reflection; the upper half
        check_band(img, path, r, y0, y0 + 12)
    sc.close()


def test_ring_spheres_1080p_stochastic_4spp(gpu_ctx, scenes):
    """1,000 spheres on 10 rings, two disk lights, reflectivity 0.5,
    stochastic anti-aliasing at 4 samples per pixel, 1920x1080 (plain
    path, the reference's 16 rays per disk light)."""
    path = workloads.write_scene(scenes, "ring_spheres.json", workloads.ring_spheres_scene(seed=0))
    sc = rt.Scene.from_json_file(path, gpu_ctx)
    r = rt.Renderer(1920, 1080)
    r.anti_aliasing_mode = rt.AntiAliasingMode.Stochastic
    r.samples = 4
    img = r.render(sc)
    for y0 in (536, 700):
        check_band(img, path, r, y0, y0 + 4)
    sc.close()


def test_batch_jobs_at_native_size(gpu_ctx, scenes):
    """Two jobs of the 256-job batch at their drawn sizes (scene 2 of the
    seed-0 workload: three meshes, 112 spheres, three lights, one of them a
    disk): its top view at 1280x720 and its perspective view at 1920x1080,
    quincunx, rendered as one batch."""
    wl = workloads.batch_workload(os.path.join(scenes, "batch"), n_scenes=3, seed=0)
    path, views = wl[2]
    sc = rt.Scene.from_json_file(path, gpu_ctx)
    jobs, files = [], []
    for name, cam, (w, h) in views:
        if name not in ("top", "perspective"):
            continue
        assert (w, h) == {"top": (1280, 720), "perspective": (1920, 1080)}[name]
        jobs.append(rt.Job(sc, rt.Renderer(w, h), cam))
        js = json.load(open(path))
        js["camera"] = copy.deepcopy(cam)
        p2 = os.path.join(os.path.dirname(path), "job_%s.json" % name)
        with open(p2, "w") as f:
            json.dump(js, f)
        files.append(p2)
    imgs, _ = rt.render_batch(jobs, lanes=2, ctx=gpu_ctx)
    for img, job, p2, rows in zip(imgs, jobs, files, (8, 4)):
        y0 = job.renderer.height // 2 - rows // 2
        check_band(img, p2, job.renderer, y0, y0 + rows)
    sc.close()


def test_terrain_4k_band(gpu_ctx, scenes):
    """The large-mesh configuration at 3840x2160: the 2,093,058-triangle
    fractal terrain, the mirror sphere, one disk light, fog, outline on
    (no-jitter), from the scene's own camera.  Two compared rows (plus the
    outline halo) through the terrain's middle."""
    path = workloads.make_terrain(os.path.join(scenes, "terrain"), n=1024, seed=11)
    sc = rt.Scene.from_json_file(path, gpu_ctx)
    r = rt.Renderer(3840, 2160)
    r.anti_aliasing_mode = rt.AntiAliasingMode.NoJitter
    r.outline_config = sc.get_outline_config()
    img = r.render(sc)
    check_band(img, path, r, 1079, 1083)
    sc.close()


def test_sphere_grid_400x300_whole_frame(gpu_ctx, scenes):
    """The small configuration, whole: sphere over a reflective grid plane,
    point light, orthographic, 400x300 quincunx."""
    path = workloads.write_scene(scenes, "sphere_grid.json", workloads.sphere_grid_scene())
    sc = rt.Scene.from_json_file(path, gpu_ctx)
    r = rt.Renderer(400, 300)
    img = r.render(sc)
    n, bad = check_band(img, path, r, 0, 300)
    assert n == 400 * 300 and bad == 0
    sc.close()
