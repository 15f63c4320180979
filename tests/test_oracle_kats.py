"""Known-answer checks of the oracle against the reference's own unit tests
and published algorithm test vectors."""
import ctypes
import math

import numpy as np
import pytest

from tests import oracle_lib


def test_transform_composition_kat():
    # src/scene.rs:275-308: rotate(0,0,180), translate(15,0,0), scale(8,8,8)
    L = oracle_lib.load()
    ts = (ctypes.c_char_p * 3)(b"rotate(0, 0, 180)", b"translate(15, 0, 0)", b"scale(8, 8, 8)")
    p = np.array([1.0, 0.0, 0.0])
    out = np.zeros(3)
    assert L.oracle_transform_point(ts, 3, p.ctypes.data, out.ctypes.data) == 0
    assert abs(out[0] - 112.0) < 1e-10 and abs(out[1]) < 1e-10 and abs(out[2]) < 1e-10


@pytest.mark.parametrize("bad", [b"invalid(1, 2, 3)", b"rotate(1, 2, 3", b"rotate(a, b, c)", b"rotate(1, 2)"])
def test_transform_errors(bad):
    # src/scene.rs:260-272
    L = oracle_lib.load()
    ts = (ctypes.c_char_p * 1)(bad)
    out = np.zeros(3)
    assert L.oracle_transform_point(ts, 1, np.zeros(3).ctypes.data, out.ctypes.data) == 1


def test_hex_to_color():
    # src/lighting.rs:513-519 and src/scene.rs:15-30
    L = oracle_lib.load()
    out = np.zeros(3)
    assert L.oracle_hex_to_color(b"#FF0000", out.ctypes.data) == 0
    assert tuple(out) == (1.0, 0.0, 0.0)
    assert L.oracle_hex_to_color(b"##00FF00", out.ctypes.data) == 0  # trim_start_matches strips every '#'
    assert tuple(out) == (0.0, 1.0, 0.0)
    assert L.oracle_hex_to_color(b"#+F+F+F", out.ctypes.data) == 0  # from_str_radix accepts '+'
    assert tuple(out) == (15 / 255, 15 / 255, 15 / 255)
    for bad in (b"#FFF", b"#GG0000", b"#-10000", b"#FF00000"):
        assert L.oracle_hex_to_color(bad, out.ctypes.data) == 1


def test_chacha20_block_vectors():
    # ChaCha20 (10 double rounds) with an all-zero key, counter and stream:
    # the published first keystream block.
    z = oracle_lib.chacha_block([0] * 8, 0, [0, 0], 10)
    assert list(z) == [0xade0b876, 0x903df1a0, 0xe56a5d40, 0x28bd8653, 0xb819d2bd, 0x1aed8da0, 0xccef36a8,
                       0xc70d778b, 0x7c5941da, 0x8d485751, 0x3fe02477, 0x374ad8b8, 0xf4b8436a, 0x1ca11815,
                       0x69b687c3, 0x8665eeb2]
    # RFC 7539 section 2.3.2 block (key 00..1f, block count 1, nonce
    # 00:00:00:09:00:00:00:4a:00:00:00:00) in the 64-bit-counter layout.
    key = [int.from_bytes(bytes(range(4 * i, 4 * i + 4)), "little") for i in range(8)]
    out = oracle_lib.chacha_block(key, 1 | (0x09000000 << 32), [0x4a000000, 0], 10)
    assert list(out) == [0xe4e7f110, 0x15593bd1, 0x1fdd0f50, 0xc47120a3, 0xc7f4d1c7, 0x0368c033, 0x9aaa2204,
                         0x4e6cd4c3, 0x466482d2, 0x09aa9f07, 0x05d7c214, 0xa2028bd9, 0xd19c12b5, 0xb94e16de,
                         0xe883d0cb, 0x4e3c50a2]


def test_stdrng_is_chacha12_over_pcg32_key():
    # StdRng::seed_from_u64: PCG32 expands the u64 into the 8 key words,
    # then the stream is ChaCha12 blocks 0, 1, 2, ... with stream id 0.
    seed = 0x0123456789ABCDEF
    st = seed
    key = []
    for _ in range(8):
        st = (st * 6364136223846793005 + 11634580027462260723) & (2 ** 64 - 1)
        xs = (((st >> 18) ^ st) >> 27) & 0xFFFFFFFF
        rot = st >> 59
        key.append(((xs >> rot) | (xs << ((32 - rot) & 31))) & 0xFFFFFFFF)
    words = oracle_lib.stdrng_u32(seed, 80)
    expect = np.concatenate([oracle_lib.chacha_block(key, b, [0, 0], 6) for b in range(5)])
    assert np.array_equal(words, expect)


def test_gen_f64_and_disk_sampling_bounds():
    # src/lighting.rs:538-555 (100 draws of radius 2 stay inside the disk)
    f = oracle_lib.stdrng_f64(42, 1000)
    assert (f >= 0).all() and (f < 1).all()
    for s in range(20):
        off = oracle_lib.disk_offsets(s, 1.0).reshape(16, 2)
        assert ((off ** 2).sum(1) <= 1.0).all()
    with pytest.raises(oracle_lib.OracleError):
        oracle_lib.disk_offsets(1, 0.0)  # gen_range(-0.0..0.0): "cannot sample empty range"


@pytest.mark.parametrize("text,value", [("0.1", 0.1), ("1.5", 1.5), ("-0", -0.0), ("1e-3", 1e-3), ("32", 32.0),
                                        ("12345678901234567890", 12345678901234567890.0),
                                        ("0.30000000000000004441", 0.30000000000000004)])
def test_json_number_semantics(text, value):
    out = np.zeros(1)
    assert oracle_lib.load().oracle_json_f64(text.encode(), out.ctypes.data) == 0
    assert out[0] == value and math.copysign(1, out[0]) == math.copysign(1, value)


def test_scaled_mesh_hit_kat(tmp_path):
    # src/renderer.rs:1258-1344: one triangle scaled 8x is hit at z = 0
    stl = tmp_path / "tri.stl"
    stl.write_text("solid test\nfacet normal 0 0 1\n  outer loop\n    vertex -8 -8 0\n    vertex 8 -8 0\n"
                   "    vertex 0 8 0\n  endloop\nendfacet\nendsolid test")
    out = oracle_lib.mesh_hit(str(stl), np.array([[4.0, 0.0, 1.0, 0.0, 0.0, -1.0]]), tmax=1000.0)
    assert out[0, 0] == 1 and abs(out[0, 4]) < 1e-10 and -8 <= out[0, 2] <= 8


def test_kd_tree_matches_brute_force_on_plus_stl():
    # tools/test_kdtree_consistency.rs: k-d and brute force agree (1e-6)
    from tests.kd_rays import plus_rays
    stl = oracle_lib.SCENES + "/plus.stl"
    rays = plus_rays(stl)
    a = oracle_lib.mesh_hit(stl, rays, use_kdtree=True)
    b = oracle_lib.mesh_hit(stl, rays, use_kdtree=False)
    assert (a[:, 0] == b[:, 0]).all()
    hit = a[:, 0] == 1
    assert hit.sum() > 50
    assert np.abs(a[hit, 1:] - b[hit, 1:]).max() <= 1e-6


def test_render_errors():
    import json
    scene = json.load(open(oracle_lib.SCENES + "/object-sphere.json"))
    with pytest.raises(oracle_lib.OracleError, match="Samples must be greater than 0"):
        oracle_lib.render(json_text=json.dumps(scene), width=10, height=10, samples=0)
    s2 = json.loads(json.dumps(scene))
    s2["camera"]["kind"] = "fisheye"
    with pytest.raises(oracle_lib.OracleError, match="Unsupported camera type: fisheye"):
        oracle_lib.render(json_text=json.dumps(s2), width=10, height=10)
    s3 = json.loads(json.dumps(scene))
    s3["camera"]["kind"] = "perspective"
    s3["camera"]["fov"] = 180
    with pytest.raises(oracle_lib.OracleError, match="Field of view must be between 0 and 180 degrees"):
        oracle_lib.render(json_text=json.dumps(s3), width=10, height=10)
    s4 = json.loads(json.dumps(scene))
    s4["objects"][0]["material"]["color"] = "#12345"
    with pytest.raises(oracle_lib.OracleError, match="Invalid hex color"):
        oracle_lib.render(json_text=json.dumps(s4), width=10, height=10)
