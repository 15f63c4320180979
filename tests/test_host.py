"""Host-side logic that needs no GPU: CLI sizing rules, PNG writer, bench
and workload helpers."""
import json
import math
import os
import struct

import numpy as np
import pytest

from rtrace_b200 import cli, workloads
from tests import oracle_lib


def test_cli_image_size_matches_shipped_images():
    # cli/src/main.rs:339-350 with the doc images' -s 500
    for c in json.load(open(os.path.join(oracle_lib.GOLDEN, "images.json"))):
        scene = json.load(open(os.path.join(oracle_lib.SCENES, c["scene"])))
        aspect = scene["camera"]["width"] / scene["camera"]["height"]
        assert list(cli.image_size(aspect, 500.0)) == c["cli_size_500"]
    assert cli.image_size(16 / 9, 2203.0) == (1920, 1080)
    assert cli.round_u32(2.5) == 3 and cli.round_u32(0.49999999999999994) == 0 and cli.round_u32(float("nan")) == 0


def test_png_writer_roundtrip(tmp_path):
    from rtrace_b200 import write_png
    img = (np.arange(7 * 5 * 3) % 256).astype(np.uint8).reshape(5, 7, 3)
    p = tmp_path / "x.png"
    write_png(str(p), img)
    data = p.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    w, h = struct.unpack(">II", data[16:24])
    assert (w, h) == (7, 5)
    from tests.test_png import decode_png
    assert np.array_equal(decode_png(data), img)


def test_workload_scenes_parse_in_oracle(tmp_path):
    d = str(tmp_path)
    for path in [workloads.write_scene(d, "a.json", workloads.sphere_grid_scene()),
                 workloads.make_noisy_icosphere(d, level=2, seed=1),
                 workloads.write_scene(d, "r.json", workloads.ring_spheres_scene(seed=0, n_rings=2, per_ring=5))]:
        img = oracle_lib.render(path, width=16, height=9, aa="no-jitter")
        assert img.shape == (9, 16, 3)
    v, f = workloads.icosphere(2)
    assert len(f) == 20 * 16 and np.allclose(np.linalg.norm(v, axis=1), 1.0)
    hv, hf = workloads.heightfield(9, 3)
    assert len(hf) == 2 * 8 * 8


# AutoCamera::generate_cameras (src/auto_camera.rs): the reference's unit
# tests (src/auto_camera.rs:160-270) and the formulas they exercise.
def _scene(objects):
    mat = {"color": "#FF0000", "ambient": 0.1, "diffuse": 0.7, "specular": 0.3, "shininess": 10}
    for o in objects:
        o.setdefault("material", mat)
    return json.dumps({"camera": {"kind": "ortho", "position": [0, 0, 10], "target": [0, 0, 0], "up": [0, 1, 0],
                                  "width": 1, "height": 1},
                       "objects": objects, "lights": [{"position": [2, 2, 2], "color": "#FFFFFF", "intensity": 1.0}],
                       "scene_settings": {"ambient_illumination": {"color": "#FFFFFF", "intensity": 0.1}}})


def test_auto_camera_with_sphere():
    import rtrace_b200 as rt
    r = rt.auto_cameras(json_text=_scene([{"kind": "sphere", "center": [0, 0, 0], "radius": 1.0}]))
    for v in r.values():
        assert v["target"] == [0.0, 0.0, 0.0]
    assert r["left"]["position"][1] < 0 and r["front"]["position"][0] < 0 and r["top"]["position"][2] > 0
    assert all(c > 0 for c in r["perspective"]["position"])
    assert r["perspective"]["fov"] == 50.0 and r["perspective"]["kind"] == "perspective"
    # viewport = max extent * 1.15, distance = 2 * viewport
    w = 2.0 * 1.15
    assert r["left"]["width"] == w and r["left"]["height"] == w and r["left"]["kind"] == "ortho"
    assert r["left"]["position"] == [0.0, -2 * w, 0.0] and r["top"]["up"] == [0.0, 1.0, 0.0]
    d = w / math.tan(50.0 * (math.pi / 180.0) / 2.0)
    h = d * math.cos(35.0 * (math.pi / 180.0))
    assert r["perspective"]["position"] == [h * math.cos(45.0 * (math.pi / 180.0)),
                                            h * math.sin(45.0 * (math.pi / 180.0)),
                                            d * math.sin(35.0 * (math.pi / 180.0))]


def test_auto_camera_with_cube_and_transforms(tmp_path):
    import rtrace_b200 as rt
    from rtrace_b200 import workloads
    r = rt.auto_cameras(json_text=_scene([{"kind": "cube", "center": [1, 1, 1], "size": [2, 2, 2]}]))
    for v in r.values():
        assert v["target"] == [1.0, 1.0, 1.0]
    # a translated mesh: bounds are its transformed box corners
    verts, tris = workloads.icosphere(1)
    stl = tmp_path / "ico.stl"
    workloads.write_binary_stl(str(stl), verts, tris)
    js = _scene([{"kind": "mesh", "filename": "ico.stl", "transform": ["translate(10, 0, 0)"]}])
    (tmp_path / "s.json").write_text(js)
    r = rt.auto_cameras(path=str(tmp_path / "s.json"))
    assert abs(r["top"]["target"][0] - 10.0) < 1e-6 and abs(r["top"]["target"][1]) < 1e-6


@pytest.mark.parametrize("objects", [[], [{"kind": "plane", "point": [0, 0, 0], "normal": [0, 0, 1]}]])
def test_auto_camera_needs_finite_objects(objects):
    import rtrace_b200 as rt
    with pytest.raises(rt.SceneError, match="no finite objects"):
        rt.auto_cameras(json_text=_scene(objects))
