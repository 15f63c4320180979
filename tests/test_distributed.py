"""Row-band sharding of one frame across ranks: partition, gather and the
whole-job timing reduction, run as two gloo ranks on the CPU; and (gpu) the
band render itself against the whole-frame render."""
import os
import socket
import types

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from rtrace_b200.distributed import gather_bands, reduce_timings, render_frame, row_bands


def _pattern(width, height):
    y, x = np.mgrid[0:height, 0:width]
    img = np.stack([(x * 7 + y) % 256, (y * 13 + 3 * x) % 256, (x ^ y) % 256], axis=-1)
    return img.astype(np.uint8)


@pytest.mark.parametrize("height,world", [(0, 2), (1, 2), (7, 2), (1080, 2), (1080, 8), (5, 8), (300, 3)])
def test_row_bands_cover_in_order(height, world):
    bands = row_bands(height, world)
    assert len(bands) == world
    assert bands[0][0] == 0 and bands[-1][1] == height
    for (b0, e0), (b1, e1) in zip(bands, bands[1:]):
        assert e0 == b1
    sizes = [e - b for b, e in bands]
    assert min(sizes) >= 0 and max(sizes) - min(sizes) <= 1


def test_row_bands_follow_costs():
    costs = np.ones(100)
    costs[:10] = 50.0  # the top rows are expensive
    bands = row_bands(100, 2, costs)
    assert bands[0][0] == 0 and bands[1][1] == 100 and bands[0][1] == bands[1][0]
    load = [costs[b:e].sum() for b, e in bands]
    assert abs(load[0] - load[1]) <= costs.max()
    assert bands[0][1] < 50
    with pytest.raises(ValueError):
        row_bands(10, 2, np.ones(9))
    with pytest.raises(ValueError):
        row_bands(10, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, width, height, costs, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        full = _pattern(width, height)
        seen = []

        def band_renderer(b, e):
            seen.append((b, e))
            return torch.from_numpy(full[b:e].copy())

        r = types.SimpleNamespace(width=width, height=height)
        img = render_frame(r, None, row_costs=costs, band_renderer=band_renderer)
        # timing: rank-dependent values, max of times and sum of counts
        times, counts = reduce_timings([1.0 + rank, 10.0 - rank], [100 + rank, 1])
        q.put((rank, seen, None if img is None else img.tobytes(), times, counts))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("width,height,costs", [(64, 48, None), (33, 7, None), (16, 9, "skewed")])
def test_two_gloo_ranks_assemble_the_frame(width, height, costs):
    if costs == "skewed":
        costs = [100.0] * 2 + [1.0] * (height - 2)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, width, height, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort(key=lambda t: t[0])
    bands = row_bands(height, 2, costs)
    for rank, seen, img, times, counts in res:
        assert seen == [bands[rank]]
        assert times == [2.0, 10.0]
        assert counts == [201.0, 2.0]
    assert res[1][2] is None
    got = np.frombuffer(res[0][2], np.uint8).reshape(height, width, 3)
    assert np.array_equal(got, _pattern(width, height))


def test_single_process_reduction_is_identity():
    assert reduce_timings([3.0], [4]) == ([3.0], [4.0])


def test_gather_rejects_a_band_of_the_wrong_shape():
    port = _free_port()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        with pytest.raises(ValueError):
            gather_bands(torch.zeros((3, 4, 3), dtype=torch.uint8), [(0, 2)], 4)
        img = gather_bands(torch.ones((2, 4, 3), dtype=torch.uint8), [(0, 2)], 4)
        assert img.shape == (2, 4, 3) and (img == 1).all()
    finally:
        dist.destroy_process_group()


# --------------------------------------------------------------------------
# GPU: bands are the whole frame's rows
# --------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("aa,outline,thickness", [("no_jitter", True, 1.0), ("no_jitter", True, 2.5),
                                                  ("stochastic", True, 2.0), ("quincunx", False, 1.0),
                                                  ("stochastic", False, 1.0)])
def test_row_bands_equal_the_whole_frame(gpu_ctx, tmp_path, aa, outline, thickness):
    import rtrace_b200 as rt
    from rtrace_b200 import workloads
    path = workloads.make_noisy_icosphere(str(tmp_path), level=3)
    scene = rt.Scene.from_json_file(path, gpu_ctx)
    r = rt.Renderer(160, 97)
    r.anti_aliasing_mode = {"no_jitter": rt.AntiAliasingMode.NoJitter, "quincunx": rt.AntiAliasingMode.Quincunx,
                            "stochastic": rt.AntiAliasingMode.Stochastic}[aa]
    if aa == "stochastic":
        r.samples = 2
    if outline:
        oc = scene.get_outline_config() or rt.OutlineConfig()
        oc.line_thickness = thickness
        r.outline_config = oc
    full = r.render(scene)
    for world in (2, 3, 5):
        parts = [r.render_rows(scene, b, e) for b, e in row_bands(r.height, world) if e > b]
        assert np.array_equal(np.concatenate(parts, 0), full), world
    one = r.render_rows(scene, 40, 41)
    assert np.array_equal(one, full[40:41])
    with pytest.raises(ValueError):
        r.render_rows(scene, 5, 5)
    with pytest.raises(ValueError):
        r.render_rows(scene, 0, r.height + 1)
