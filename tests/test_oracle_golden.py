"""The oracle reproduces the reference's shipped renders byte for byte.

Each case is a PNG the reference renderer produced (doc/images, rendered by
`rtrace -i <scene> -o <png> -s 500`, herebyfile.mjs render:doc:* tasks);
the fixture holds the SHA-256 of its decoded RGB8 pixels.  This pins the
oracle's double-precision path (cameras, primitives, k-d meshes, textures,
Phong, fog, reflections, quincunx and no-jitter sampling, outlines)."""
import hashlib
import json
import os

import pytest

from tests import oracle_lib

CASES = json.load(open(os.path.join(oracle_lib.GOLDEN, "images.json")))


@pytest.mark.parametrize("case", CASES, ids=[c["image"] for c in CASES])
def test_oracle_matches_reference_render(case):
    img = oracle_lib.render(os.path.join(oracle_lib.SCENES, case["scene"]), width=case["width"],
                            height=case["height"], aa=case["anti_aliasing"], samples=case["samples"],
                            outline=case["outline"])
    assert hashlib.sha256(img.tobytes()).hexdigest() == case["sha256_rgb"]


def test_cli_sizes_match_shipped_images():
    # cli/src/main.rs:339-350 sizes most doc images from -s 500
    for c in CASES:
        if c["image"].startswith(("sampling-comparison", "fog-demonstration")):
            continue  # 800x600 renders of the earlier --width/--height CLI
        assert [c["width"], c["height"]] == c["cli_size_500"], c["image"]
