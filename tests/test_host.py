"""Host-side logic that needs no GPU: CLI sizing rules, PNG writer, bench
and workload helpers."""
import json
import os
import struct
import zlib

import numpy as np

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
    i = data.index(b"IDAT")
    n = struct.unpack(">I", data[i - 4:i])[0]
    raw = np.frombuffer(zlib.decompress(data[i + 4:i + 4 + n]), np.uint8).reshape(5, 1 + 21)
    assert (raw[:, 0] == 0).all() and np.array_equal(raw[:, 1:].reshape(5, 7, 3), img)


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
