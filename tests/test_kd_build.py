"""The k-d tree build (KdTree::new(triangles, 16, 10), src/mesh.rs:75-197):
the library's host builder and its device builder against the oracle's
recursive build, byte for byte, on meshes that reach every rule of the
reference's build: stable-sort ties, signed zeros in centres and bounds,
straddlers, both empty-side moves, the depth limit, a NaN centre, tiny and
empty meshes."""
import json
import zlib

import numpy as np
import pytest

from rtrace_b200 import workloads

# A coordinate whose Triangle::center ((a + a + a) / 3) rounds below a: a
# node of triangles collapsed to this point finds every box above the split
# and moves one triangle left (the empty-left rule).
BELOW = 0.8158535541215322


def _grid(n, seed):
    v, f = workloads.heightfield(n, seed, height=4.0)
    return v[f].reshape(-1, 9)


def _case(name):
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    if name == "soup":
        c = rng.random((4000, 1, 3)) * 10
        return (c + rng.normal(0, 0.05, (4000, 3, 3))).reshape(-1, 9)
    if name == "grid_ties":  # x/y centres repeat along every row and column
        return _grid(40, 3)
    if name == "signed_zeros":
        v = _grid(24, 5)
        v[:, 2::3] = 0.0  # flat: every z is zero, half of them negative zero
        v[::2, 2::3] = -0.0
        v[:, 0:9:3][np.abs(v[:, 0:9:3]) < 1e-12] = -0.0
        return v
    if name == "empty_sides":
        pts = np.concatenate([np.full((30, 9), BELOW), np.full((30, 9), 2.0)])
        rest = rng.random((300, 1, 3)) * 4 + rng.normal(0, 0.02, (300, 3, 3))
        return np.concatenate([pts, rest.reshape(-1, 9)])
    if name == "straddlers":
        small = rng.random((1500, 1, 3)) * 8 + rng.normal(0, 0.03, (1500, 3, 3))
        big = rng.random((6, 3, 3)) * 8
        return np.concatenate([small.reshape(-1, 9), big.reshape(-1, 9)])
    if name == "icosphere":
        v, f = workloads.noisy_icosphere(4, 9)
        return v[f].reshape(-1, 9)
    if name == "tiny":
        return rng.random((7, 9))
    if name == "empty":
        return np.zeros((0, 9))
    raise KeyError(name)


CASES = ["soup", "grid_ties", "signed_zeros", "empty_sides", "straddlers", "icosphere", "tiny", "empty"]


def _same_tree(nodes, want_raw):
    """Node records equal field by field; bounds compared as numbers.  The
    reference folds bounds with f64::min/max (llvm.minnum/maxnum, which may
    return either operand when they compare equal), so the sign of a zero
    bound is not defined by it; the oracle's compiled fmin keeps the last
    zero in one place and the first in another.  Bounds only enter
    subtractions and comparisons, whose outcomes do not depend on that
    sign."""
    import rtrace_b200 as rt
    want = np.frombuffer(want_raw.tobytes(), rt.KD_NODE_DTYPE)
    assert len(nodes) == len(want)
    for f in ("axis", "right", "first", "count"):
        assert np.array_equal(nodes[f], want[f]), f
    assert nodes["split"].tobytes() == want["split"].tobytes()
    for f in ("bounds_min", "bounds_max"):
        assert np.array_equal(nodes[f], want[f], equal_nan=True), f


def _check(v, ctx):
    import rtrace_b200 as rt
    from tests import oracle_lib
    nodes, idx = rt.kd_build(v, ctx=ctx)
    want_nodes, want_idx = oracle_lib.kd_build(v)
    _same_tree(nodes, want_nodes)
    assert np.array_equal(idx, want_idx)
    if ctx is not None:  # the device build is the library's host build, bit for bit
        host_nodes, host_idx = rt.kd_build(v)
        assert nodes.tobytes() == host_nodes.tobytes() and np.array_equal(idx, host_idx)
    return nodes, idx


@pytest.mark.parametrize("name", CASES)
def test_host_builder_matches_the_oracle(name, oracle):
    nodes, idx = _check(_case(name), None)
    if name == "empty":
        assert len(nodes) == 0
    elif name == "tiny":
        assert len(nodes) == 1 and nodes[0]["axis"] == -1 and nodes[0]["count"] == 7
    else:
        assert (nodes["axis"] >= 0).any()


def _centres(v):
    return (v[:, 0:3] + v[:, 3:6] + v[:, 6:9]) / 3.0


def test_cases_reach_the_rules():
    """The inputs do what their names say, so that the parity tests cover
    those rules."""
    z = _case("signed_zeros")[:, 2::3]
    assert (np.signbit(z) & (z == 0)).any() and (~np.signbit(z) & (z == 0)).any()
    g = _case("grid_ties")
    assert len(np.unique(_centres(g)[:, 0])) < len(g) // 10  # centre ties on x
    assert (BELOW + BELOW + BELOW) / 3.0 < BELOW  # empty-left move
    e = _case("empty_sides")
    assert (e[30:60] == 2.0).all()  # coincident points: empty-right moves
    assert len(_case("straddlers")) == 1506


def test_nan_centre_panics_like_the_reference(oracle):
    import rtrace_b200 as rt
    from tests import oracle_lib
    v = _case("soup")
    v[17, 4] = np.nan
    with pytest.raises(rt.SceneError, match="called `Option::unwrap\\(\\)` on a `None` value"):
        rt.kd_build(v)
    with pytest.raises(oracle_lib.OracleError, match="None"):
        oracle_lib.kd_build(v)
    # a root leaf is never sorted, so a NaN there does not panic
    t = _case("tiny")
    t[2, 0] = np.nan
    _check(t, None)


# --------------------------------------------------------------------------
# GPU
# --------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_device_builder_matches_the_oracle(gpu_ctx, oracle, name):
    _check(_case(name), gpu_ctx)


@pytest.mark.gpu
def test_device_builder_on_a_terrain_and_nan(gpu_ctx, oracle):
    import rtrace_b200 as rt
    # 2 * 255^2 = 130,050 grid triangles, depth-16 tree
    nodes, _ = _check(_grid(256, 11), gpu_ctx)
    assert len(nodes) > 10000
    v = _case("soup")
    v[17, 4] = np.nan
    with pytest.raises(rt.SceneError, match="called `Option::unwrap\\(\\)` on a `None` value"):
        rt.kd_build(v, ctx=gpu_ctx)
    # the context stays usable after the failed build
    _check(_case("icosphere"), gpu_ctx)


@pytest.mark.gpu
def test_scene_loaded_with_device_trees_is_identical(gpu_ctx, tmp_path):
    """A scene whose mesh is above the device-build threshold: the host
    scene loaded with a context holds the same vertices, nodes and leaf
    lists as the one loaded on the host, and renders the same image."""
    import rtrace_b200 as rt
    path = workloads.make_noisy_icosphere(str(tmp_path), level=6)  # 81,920 triangles
    a = rt.HostScene.from_json_file(path)
    b = rt.HostScene.from_json_file(path, ctx=gpu_ctx)
    (va, na, ia), = a.meshes()
    (vb, nb, ib), = b.meshes()
    assert len(va) == 81920
    assert np.array_equal(va, vb) and na.tobytes() == nb.tobytes() and np.array_equal(ia, ib)
    r = rt.Renderer(160, 90)
    r.anti_aliasing_mode = rt.AntiAliasingMode.NoJitter
    sa, sb = rt.Scene.upload(a, gpu_ctx), rt.Scene.upload(b, gpu_ctx)
    assert np.array_equal(r.render(sa), r.render(sb))
    s3 = rt.Scene.from_json_file(path, gpu_ctx)  # rt_scene_load_json_file builds on the device too
    assert np.array_equal(r.render(s3), r.render(sa))
