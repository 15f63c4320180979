"""ctypes access to the CPU oracle (oracle/rtrace_oracle.cpp).

Test infrastructure: the oracle is the checker the CUDA path is compared
against; the library under test never loads it."""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB = os.path.join(ORACLE_DIR, "_build", "liboracle.so")
GOLDEN = os.path.join(ROOT, "tests", "golden")
SCENES = os.path.join(GOLDEN, "scenes")

AA = {"no-jitter": 0, "quincunx": 1, "stochastic": 2}

_lib = None


def build():
    src = os.path.join(ORACLE_DIR, "rtrace_oracle.cpp")
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    build()
    L = ctypes.CDLL(LIB)
    vp = ctypes.c_void_p
    L.oracle_render.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int,
                                ctypes.c_uint32, ctypes.c_int, ctypes.c_uint64, ctypes.c_int, ctypes.c_int,
                                ctypes.c_int, vp, vp, vp, ctypes.c_char_p, ctypes.c_int]
    L.oracle_render.restype = ctypes.c_int
    L.oracle_render_rows.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32,
                                     ctypes.c_int, ctypes.c_uint32, ctypes.c_int, ctypes.c_uint64, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, vp, vp, vp,
                                     ctypes.c_char_p, ctypes.c_int]
    L.oracle_render_rows.restype = ctypes.c_int
    L.oracle_render_ex.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int,
                                   ctypes.c_uint32, ctypes.c_int, ctypes.c_uint64, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, vp, vp, vp,
                                   ctypes.c_char_p, ctypes.c_int]
    L.oracle_render_ex.restype = ctypes.c_int
    L.oracle_stdrng_u32.argtypes = [ctypes.c_uint64, ctypes.c_int, vp]
    L.oracle_stdrng_f64.argtypes = [ctypes.c_uint64, ctypes.c_int, vp]
    L.oracle_stdrng_range.argtypes = [ctypes.c_uint64, ctypes.c_double, ctypes.c_double, ctypes.c_int, vp]
    L.oracle_stdrng_range.restype = ctypes.c_int
    L.oracle_disk_offsets.argtypes = [ctypes.c_uint64, ctypes.c_double, vp]
    L.oracle_disk_offsets.restype = ctypes.c_int
    L.oracle_mesh_hit.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_long, vp, ctypes.c_double,
                                  ctypes.c_double, vp, ctypes.c_char_p, ctypes.c_int]
    L.oracle_mesh_hit.restype = ctypes.c_long
    L.oracle_transform_point.argtypes = [ctypes.POINTER(ctypes.c_char_p), ctypes.c_int, vp, vp]
    L.oracle_transform_point.restype = ctypes.c_int
    L.oracle_hex_to_color.argtypes = [ctypes.c_char_p, vp]
    L.oracle_hex_to_color.restype = ctypes.c_int
    L.oracle_json_f64.argtypes = [ctypes.c_char_p, vp]
    L.oracle_json_f64.restype = ctypes.c_int
    L.oracle_chacha_block.argtypes = [vp, ctypes.c_uint64, vp, ctypes.c_int, vp]
    L.oracle_outline.argtypes = [ctypes.c_uint32, ctypes.c_uint32] + [vp] * 8 + [ctypes.c_double] * 3 + \
        [vp, ctypes.c_int, ctypes.c_double, vp]
    L.oracle_kd_build.argtypes = [vp, ctypes.c_int64, vp, vp, vp, vp, ctypes.c_char_p, ctypes.c_int]
    L.oracle_kd_build.restype = ctypes.c_int
    _lib = L
    return L


def kd_build(vertices):
    """The oracle's KdTree::new(triangles, 16, 10) of an (n, 9) float64
    array: (nodes as raw 72-byte preorder records, leaf index list)."""
    import numpy as np
    v = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 9)
    L = load()
    nn, ni = ctypes.c_int64(), ctypes.c_int64()
    err = ctypes.create_string_buffer(512)
    args = (v.ctypes.data if len(v) else None, len(v))
    if L.oracle_kd_build(*args, None, None, ctypes.byref(nn), ctypes.byref(ni), err, 512):
        raise OracleError(err.value.decode())
    nodes = np.zeros(nn.value * 72, np.uint8)
    idx = np.zeros(ni.value, np.int32)
    L.oracle_kd_build(*args, nodes.ctypes.data, idx.ctypes.data, ctypes.byref(nn), ctypes.byref(ni), err, 512)
    return nodes, idx


class OracleError(Exception):
    pass


def render(path=None, json_text=None, width=100, height=100, aa="quincunx", samples=1, max_depth=10, seed=0,
           use_kdtree=True, outline=False, threads=None, linear=False, counts=False, disk_samples=16):
    """Renders like Renderer::render; returns uint8 (H, W, 3) [, linear] [, counts].
    disk_samples: shadow rays per disk light (16 is the reference)."""
    L = load()
    out = np.zeros((height, width, 3), np.uint8)
    lin = np.zeros((height, width, 3), np.float64) if linear else None
    cnt = np.zeros(6, np.uint64) if counts else None
    err = ctypes.create_string_buffer(1024)
    threads = threads or os.cpu_count() or 1
    rc = L.oracle_render_ex(path.encode() if path else None, json_text.encode() if json_text else None, width, height,
                            AA[aa] if isinstance(aa, str) else int(aa), samples, max_depth, seed,
                            1 if use_kdtree else 0, 1 if outline else 0,
                            1 if (counts and aa in ("quincunx", 1)) else threads, 0, 0xFFFFFFFF, disk_samples,
                            out.ctypes.data, lin.ctypes.data if linear else None,
                            cnt.ctypes.data if counts else None, err, 1024)
    if rc != 0:
        raise OracleError(err.value.decode())
    res = [out]
    if linear:
        res.append(lin)
    if counts:
        res.append(cnt)
    return res[0] if len(res) == 1 else tuple(res)


def stdrng_u32(seed, n):
    out = np.zeros(n, np.uint32)
    load().oracle_stdrng_u32(seed, n, out.ctypes.data)
    return out


def stdrng_f64(seed, n):
    out = np.zeros(n, np.float64)
    load().oracle_stdrng_f64(seed, n, out.ctypes.data)
    return out


def disk_offsets(light_seed, radius):
    out = np.zeros(32, np.float64)
    if load().oracle_disk_offsets(light_seed, radius, out.ctypes.data):
        raise OracleError("cannot sample empty range")
    return out


def chacha_block(key_words, counter, nonce_words, double_rounds):
    key = np.asarray(key_words, np.uint32)
    nonce = np.asarray(nonce_words, np.uint32)
    out = np.zeros(16, np.uint32)
    load().oracle_chacha_block(key.ctypes.data, counter, nonce.ctypes.data, double_rounds, out.ctypes.data)
    return out


def mesh_hit(stl_path, rays, use_kdtree=True, tmin=0.001, tmax=float("inf")):
    rays = np.ascontiguousarray(rays, np.float64)
    n = rays.shape[0]
    out = np.zeros((n, 8), np.float64)
    err = ctypes.create_string_buffer(512)
    r = load().oracle_mesh_hit(stl_path.encode(), 1 if use_kdtree else 0, n, rays.ctypes.data, tmin, tmax,
                               out.ctypes.data, err, 512)
    if r < 0:
        raise OracleError(err.value.decode())
    return out


def outline(color, valid, depth, normal, depth_weight=1.0, normal_weight=1.0, threshold=0.1,
            edge_color=(0.0, 0.0, 0.0), use_8_neighbors=False, thickness=1.0):
    """apply_outline_detection + quantisation on (H, W, 3) colours,
    (H, W) valid/depth and (H, W, 3) normals; returns (H, W, 3) uint8."""
    H, W = valid.shape
    c = [np.ascontiguousarray(color[..., k], np.float64) for k in range(3)]
    n = [np.ascontiguousarray(normal[..., k], np.float64) for k in range(3)]
    v = np.ascontiguousarray(valid, np.uint8)
    d = np.ascontiguousarray(depth, np.float64)
    ec = np.asarray(edge_color, np.float64)
    out = np.zeros((H, W, 3), np.uint8)
    load().oracle_outline(W, H, c[0].ctypes.data, c[1].ctypes.data, c[2].ctypes.data, v.ctypes.data, d.ctypes.data,
                          n[0].ctypes.data, n[1].ctypes.data, n[2].ctypes.data, depth_weight, normal_weight,
                          threshold, ec.ctypes.data, 1 if use_8_neighbors else 0, thickness, out.ctypes.data)
    return out
