"""Device preparation of large meshes' search data (triangle records and
normals, the triangle BVH, the k-d occurrence lists): byte-identical to the
host preparation, and scenes uploaded through it render the same image in
each of the upload paths (prepared on the device; prepared on the device
and kept on the host; copied from the host's pinned image)."""
import ctypes

import numpy as np
import pytest

from rtrace_b200 import workloads


def _desc(v, nodes, idx):
    from rtrace_b200 import _capi
    d = _capi.rt_mesh_desc()
    d.vertices = v.ctypes.data
    d.n_triangles = len(v)
    d.nodes = nodes.ctypes.data if len(nodes) else None
    d.n_nodes = len(nodes)
    d.tri_index = idx.ctypes.data if len(idx) else None
    d.n_tri_index = len(idx)
    return d


def _mesh(name):
    import rtrace_b200 as rt
    rng = np.random.default_rng(5)
    if name == "terrain":
        v, f = workloads.heightfield(200, 3, height=6.0)
        v = v[f].reshape(-1, 9)
    elif name == "icosphere":
        v, f = workloads.noisy_icosphere(6, 7)
        v = v[f].reshape(-1, 9)
    else:  # soup with repeated and degenerate triangles and signed zeros
        c = rng.random((30000, 1, 3)) * 20
        v = (c + rng.normal(0, 0.1, (30000, 3, 3))).reshape(-1, 9)
        v[100:400] = v[100]            # repeats: equal centroids, ties by id
        v[500:700, 3:9] = np.tile(v[500:700, 0:3], 2)  # points: degenerate
        v[800:900, 2::3] = -0.0
    v = np.ascontiguousarray(v, dtype=np.float64)
    nodes, idx = rt.kd_build(v)
    return v, nodes, idx


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["terrain", "icosphere", "soup"])
def test_device_preparation_equals_host(gpu_ctx, name):
    from rtrace_b200 import _capi
    v, nodes, idx = _mesh(name)
    assert len(v) >= 16384
    mask = ctypes.c_uint32(99)
    L = _capi.lib()
    st = L.rt_debug_mesh_prep(gpu_ctx.handle, ctypes.byref(_desc(v, nodes, idx)), ctypes.byref(mask))
    assert st == 0, L.rt_last_error(gpu_ctx.handle)
    assert mask.value == 0, bin(mask.value)


@pytest.mark.gpu
def test_upload_paths_render_the_same(gpu_ctx, oracle, tmp_path):
    import rtrace_b200 as rt
    from tests import oracle_lib
    # 2 x 399^2 = 318,402 triangles: above the size from which uploads
    # prepare meshes on the device
    path = workloads.make_terrain(str(tmp_path), n=400, seed=4)
    host = rt.HostScene.from_json_file(path)
    r = rt.Renderer(96, 54)
    r.anti_aliasing_mode = rt.AntiAliasingMode.NoJitter
    r.disk_samples = 4
    imgs, sizes = [], []
    for _ in range(3):  # device; device kept on the host; pinned image
        s = rt.Scene.upload(host, gpu_ctx)
        imgs.append(r.render(s))
        sizes.append(s.device_bytes)
        s.close()
    want = r.render(rt.Scene.from_json_file(path, gpu_ctx))
    assert all(np.array_equal(i, want) for i in imgs)
    assert imgs[0].any()
    assert np.array_equal(want, oracle_lib.render(path=path, width=96, height=54, aa="no-jitter", disk_samples=4))
    # the first two uploads copy the mesh's inputs, the third its prepared arrays
    assert sizes[0] == sizes[1] and sizes[2] > sizes[0]


@pytest.mark.gpu
def test_invalid_leaf_lists_are_rejected(gpu_ctx):
    import rtrace_b200 as rt
    from rtrace_b200 import _capi
    v, nodes, idx = _mesh("icosphere")
    L = _capi.lib()
    mask = ctypes.c_uint32()
    bad = nodes.copy()
    leaf = np.nonzero(bad["axis"] < 0)[0][3]
    bad["first"][leaf] = bad["first"][leaf - 1] if bad["axis"][leaf - 1] < 0 else 0  # overlaps another leaf
    st = L.rt_debug_mesh_prep(gpu_ctx.handle, ctypes.byref(_desc(v, bad, idx)), ctypes.byref(mask))
    assert st == _capi.RT_ERR_INVALID_ARGUMENT
    assert b"k-d leaves" in L.rt_last_error(gpu_ctx.handle)
    assert len(rt.kd_build(v[:100], ctx=gpu_ctx)[0]) > 0  # the context stays usable
