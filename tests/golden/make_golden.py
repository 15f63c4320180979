"""Regenerates the golden fixtures from a checkout of SeaRyanC/rtrace.

Usage: python tests/golden/make_golden.py /path/to/rtrace

Copies the reference's scene files that have shipped renders (doc/scenes,
examples) plus their STL meshes into tests/golden/scenes/, and records for
each shipped render the CLI settings that produced it (herebyfile.mjs
render:doc:* tasks: `rtrace -i <scene> -o <png> -s 500 [params]`) with the
SHA-256 of its decoded RGB8 pixels.  Only renders that the current
reference code reproduces are listed; renders produced by older versions
of the reference (the stochastic and area-light 800x600 images) are not.
"""
import hashlib
import json
import math
import os
import shutil
import sys

import numpy as np
from PIL import Image

HERE = os.path.dirname(os.path.abspath(__file__))

# (image, scene, anti-aliasing, samples) -- anti-aliasing as on the CLI;
# the CLI switches quincunx to no-jitter when the scene enables outlines.
CASES = [
    ("doc/images/camera-basic.png", "doc/scenes/camera-basic.json", "quincunx", 1),
    ("doc/images/camera-perspective.png", "doc/scenes/camera-perspective.json", "quincunx", 1),
    ("doc/images/object-sphere.png", "doc/scenes/object-sphere.json", "quincunx", 1),
    ("doc/images/object-plane-grid.png", "doc/scenes/object-plane-grid.json", "quincunx", 1),
    ("doc/images/object-cube.png", "doc/scenes/object-cube.json", "quincunx", 1),
    ("doc/images/object-mesh.png", "doc/scenes/object-mesh.json", "quincunx", 1),
    ("doc/images/material-properties.png", "doc/scenes/material-properties.json", "quincunx", 1),
    ("doc/images/material-reflectivity.png", "doc/scenes/material-reflectivity.json", "quincunx", 1),
    ("doc/images/texture-grid-variations.png", "doc/scenes/texture-grid-variations.json", "quincunx", 1),
    ("doc/images/checkerboard-basic.png", "doc/scenes/checkerboard-basic.json", "quincunx", 1),
    ("doc/images/checkerboard-advanced.png", "doc/scenes/checkerboard-advanced.json", "quincunx", 1),
    ("doc/images/lighting-multiple.png", "doc/scenes/lighting-multiple.json", "quincunx", 1),
    ("doc/images/sampling-antialiasing.png", "doc/scenes/sampling-antialiasing.json", "quincunx", 4),
    ("doc/images/sampling-antialiasing-nosamples.png", "doc/scenes/sampling-antialiasing.json", "no-jitter", 1),
    ("doc/images/example-complete.png", "doc/scenes/example-complete.json", "quincunx", 1),
    ("doc/images/outline_complex.png", "doc/scenes/outline_complex.json", "quincunx", 1),
    ("doc/images/outline-demo-complex.png", "doc/scenes/outline_complex.json", "no-jitter", 1),
    ("doc/images/outline-demo-basic.png", "examples/outline_demo.json", "no-jitter", 1),
    ("doc/images/scene-backgrounds-1.png", "doc/scenes/scene-backgrounds-1.json", "quincunx", 1),
    ("doc/images/scene-backgrounds-2.png", "doc/scenes/scene-backgrounds-2.json", "quincunx", 1),
    ("doc/images/scene-fog-light.png", "doc/scenes/scene-fog-light.json", "quincunx", 1),
    ("doc/images/scene-fog-heavy.png", "doc/scenes/scene-fog-heavy.json", "quincunx", 1),
    ("doc/images/quincunx-demo.png", "doc/scenes/quincunx-demo.json", "quincunx", 1),
    ("doc/images/fog-demonstration.png", "doc/scenes/fog-demonstration.json", "quincunx", 1),
    ("doc/images/sampling-comparison-quincunx.png", "doc/scenes/sampling-comparison.json", "quincunx", 1),
    ("doc/images/sampling-comparison-no-jitter.png", "doc/scenes/sampling-comparison.json", "no-jitter", 1),
]
# outline-demo-no-outline.png: the same scene with the outline settings removed
EXTRA = [("doc/images/outline-demo-no-outline.png", "examples/outline_demo.json", "no-jitter", 1, "drop_outline")]
MESHES = ["doc/scenes/sphere.stl", "examples/plus.stl"]


def cli_size(scene, diag):
    """cli/src/main.rs:339-350 (f64::round is half away from zero)."""
    r = scene["camera"]["width"] / scene["camera"]["height"]
    h = diag / math.sqrt(r * r + 1.0)
    w = r * h
    rnd = lambda v: int(math.floor(v + 0.5))
    return rnd(w), rnd(h)


def main(ref):
    out_scenes = os.path.join(HERE, "scenes")
    os.makedirs(out_scenes, exist_ok=True)
    entries = []
    for case in CASES + EXTRA:
        img_rel, scene_rel, aa, samples = case[:4]
        mod = case[4] if len(case) > 4 else None
        scene = json.load(open(os.path.join(ref, scene_rel)))
        name = os.path.basename(scene_rel)
        if mod == "drop_outline":
            scene["scene_settings"].pop("outline", None)
            name = name.replace(".json", "_no_outline.json")
            with open(os.path.join(out_scenes, name), "w") as f:
                json.dump(scene, f, indent=2)
        else:
            shutil.copyfile(os.path.join(ref, scene_rel), os.path.join(out_scenes, name))
        img = np.asarray(Image.open(os.path.join(ref, img_rel)).convert("RGB"))
        h, w = img.shape[:2]
        ol = scene.get("scene_settings", {}).get("outline") or {}
        outline = bool(ol.get("enabled"))
        if outline and aa == "quincunx":
            aa = "no-jitter"
        entries.append({
            "image": os.path.basename(img_rel), "scene": name, "width": w, "height": h,
            "cli_size_500": list(cli_size(scene, 500)), "anti_aliasing": aa, "samples": samples,
            "outline": outline, "sha256_rgb": hashlib.sha256(img.tobytes()).hexdigest(),
        })
    for m in MESHES:
        shutil.copyfile(os.path.join(ref, m), os.path.join(out_scenes, os.path.basename(m)))
    with open(os.path.join(HERE, "images.json"), "w") as f:
        json.dump(entries, f, indent=1)
    print("wrote %d golden cases" % len(entries))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
