"""PNG output (Renderer::render_to_file, src/renderer.rs:914-920): the
library's encoder, checked by decoding its files with an independent
decoder (zlib inflate and the five PNG filters in numpy) back to the
image's bytes.  The reference is compared on decoded pixels: file bytes
depend on the encoder."""
import struct
import zlib

import numpy as np
import pytest


def decode_png(data):
    """A PNG decoder for 8-bit RGB, non-interlaced images."""
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, ihdr = 8, b"", None
    while pos < len(data):
        n, = struct.unpack(">I", data[pos:pos + 4])
        tag, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        crc, = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert crc == zlib.crc32(tag + body) & 0xFFFFFFFF, tag
        if tag == b"IHDR":
            ihdr = struct.unpack(">IIBBBBB", body)
        elif tag == b"IDAT":
            idat += body
        pos += 12 + n
    w, h, depth, ctype, comp, filt, inter = ihdr
    assert (depth, ctype, comp, filt, inter) == (8, 2, 0, 0, 0)
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, 1 + 3 * w)  # checks the Adler-32 too
    out = np.zeros((h, 3 * w), np.int32)
    for y in range(h):
        f, line = raw[y, 0], raw[y, 1:].astype(np.int32)
        up = out[y - 1] if y else np.zeros(3 * w, np.int32)
        row = np.zeros(3 * w, np.int32)
        for i in range(3 * w):
            a = row[i - 3] if i >= 3 else 0
            b = up[i]
            c = up[i - 3] if i >= 3 else 0
            if f == 0:
                p = 0
            elif f == 1:
                p = a
            elif f == 2:
                p = b
            elif f == 3:
                p = (a + b) >> 1
            else:
                pp = a + b - c
                pa, pb, pc = abs(pp - a), abs(pp - b), abs(pp - c)
                p = a if pa <= pb and pa <= pc else (b if pb <= pc else c)
            row[i] = (line[i] + p) & 255
        out[y] = row
    return out.reshape(h, w, 3).astype(np.uint8)


def _images():
    rng = np.random.default_rng(4)
    noise = rng.integers(0, 256, (37, 53, 3), dtype=np.uint8)
    grad = np.zeros((64, 48, 3), np.uint8)
    grad[..., 0] = np.arange(48)[None, :] * 5
    grad[..., 1] = np.arange(64)[:, None] * 3
    grad[..., 2] = 7
    flat = np.full((5, 7, 3), 200, np.uint8)
    one = np.array([[[1, 2, 3]]], np.uint8)
    tall = rng.integers(0, 4, (700, 9, 3), dtype=np.uint8)  # many bands of few bytes
    return {"noise": noise, "gradient": grad, "flat": flat, "one_pixel": one, "tall": tall}


@pytest.mark.parametrize("name", list(_images()))
@pytest.mark.parametrize("level", [-1, 0, 1, 9])
def test_encoded_png_decodes_to_the_image(name, level):
    import rtrace_b200 as rt
    img = _images()[name]
    assert np.array_equal(decode_png(rt.encode_png(img, level)), img)


def test_write_png_and_errors(tmp_path):
    import rtrace_b200 as rt
    img = _images()["gradient"]
    p = tmp_path / "g.png"
    rt.write_png(p, img)
    assert np.array_equal(decode_png(p.read_bytes()), img)
    with pytest.raises(OSError):
        rt.write_png(tmp_path / "missing_dir" / "x.png", img)
    with pytest.raises(ValueError):
        rt.encode_png(img, level=12)


def test_large_image_uses_many_bands():
    """A 4K-sized image: decoded with zlib in one piece (the bands form one
    deflate stream with one Adler-32)."""
    import rtrace_b200 as rt
    rng = np.random.default_rng(1)
    img = (rng.random((2160, 3840, 3)) * 30).astype(np.uint8)
    img[:, :1000] = 9
    data = rt.encode_png(img)
    n, = struct.unpack(">I", data[33:37])
    raw = np.frombuffer(zlib.decompress(data[41:41 + n]), np.uint8).reshape(2160, 1 + 3 * 3840)
    assert set(np.unique(raw[:, 0])) <= {0, 1, 2, 3, 4}
    # rows filtered "none" hold the pixels themselves
    none = raw[:, 0] == 0
    assert np.array_equal(raw[none, 1:], img.reshape(2160, -1)[none])
