"""Batched rendering (extension): the lane planner and the batch workload on
the CPU; on the GPU, every job of a batch against the same render done on
its own (camera override = the view written into the scene) and against the
oracle."""
import copy
import json

import numpy as np
import pytest

import rtrace_b200 as rt
from rtrace_b200 import workloads


def test_longest_first_assignment():
    costs = [5, 1, 4, 2, 3, 9]
    assert list(rt.batch_assign(costs, 2)) == [1, 1, 1, 1, 0, 0]
    assert list(rt.batch_assign(costs, 1)) == [0] * 6
    lanes = rt.batch_assign(costs, 6)
    assert sorted(lanes) == list(range(6))
    rng = np.random.default_rng(0)
    c = rng.uniform(1, 100, 257)
    for k in (2, 3, 8):
        lane = rt.batch_assign(c, k)
        loads = np.bincount(lane, weights=c, minlength=k)
        # LPT bound: max load <= mean load + largest job
        assert loads.max() <= c.sum() / k + c.max() + 1e-9
    assert len(rt.batch_assign([], 4)) == 0
    with pytest.raises(ValueError):
        rt.batch_assign([1.0], 0)


def test_batch_workload_is_seeded(tmp_path):
    a = workloads.batch_workload(str(tmp_path / "a"), n_scenes=3, seed=1)
    b = workloads.batch_workload(str(tmp_path / "b"), n_scenes=3, seed=1)
    assert len(a) == 3 and all(len(v) == 4 for _, v in a)
    for (pa, va), (pb, vb) in zip(a, b):
        assert open(pa).read() == open(pb).read()
        assert va == vb
        for name, cam, (w, h) in va:
            assert (w, h) in workloads.BATCH_RESOLUTIONS
            assert cam["kind"] == ("perspective" if name == "perspective" else "ortho")


def _with_camera(path, cam):
    sc = json.load(open(path))
    sc["camera"] = copy.deepcopy(cam)
    return sc


@pytest.mark.gpu
def test_batch_jobs_equal_single_renders(gpu_ctx, tmp_path, oracle):
    from tests import oracle_lib
    wl = workloads.batch_workload(str(tmp_path), n_scenes=3, seed=4)
    jobs, singles = [], []
    for k, (path, views) in enumerate(wl):
        scene = rt.Scene.from_json_file(path, gpu_ctx)
        for name, cam, _ in views:
            r = rt.Renderer(96 + 16 * k, 64)
            r.anti_aliasing_mode = rt.AntiAliasingMode.Stochastic if k == 1 else rt.AntiAliasingMode.Quincunx
            r.samples = 2
            jobs.append(rt.Job(scene, r, cam))
            singles.append((path, cam, r))
    imgs, st = rt.render_batch(jobs, lanes=3, ctx=gpu_ctx)
    assert st.jobs == len(jobs) and st.lanes == 3 and st.rays > 0
    for img, (path, cam, r) in zip(imgs, singles):
        js = _with_camera(path, cam)
        p2 = tmp_path / "single.json"
        p2.write_text(json.dumps(js))
        s2 = rt.Scene.from_json_file(str(p2), gpu_ctx)
        want = r.render(s2)
        s2.close()
        assert np.array_equal(img, want)
    # two jobs against the oracle (meshes resolve against the scene's directory)
    for idx in (0, 5):
        path, cam, r = singles[idx]
        p2 = tmp_path / "oracle_job.json"
        p2.write_text(json.dumps(_with_camera(path, cam)))
        aa = {0: "no-jitter", 1: "quincunx", 2: "stochastic"}[int(r.anti_aliasing_mode)]
        want = oracle_lib.render(path=str(p2), width=r.width, height=r.height, aa=aa, samples=r.samples)
        assert np.array_equal(imgs[idx], want), idx
    # autotune picks one of its candidates and keeps it for lanes=0
    best = rt.batch_autotune(jobs, ctx=gpu_ctx)
    assert best in (1, 2, 4, 8)
    imgs2, st2 = rt.render_batch(jobs, ctx=gpu_ctx)
    assert st2.lanes == min(best, len(jobs))
    assert all(np.array_equal(a, b) for a, b in zip(imgs, imgs2))


@pytest.mark.gpu
def test_batch_reports_the_failing_job(gpu_ctx, tmp_path):
    wl = workloads.batch_workload(str(tmp_path), n_scenes=1, seed=2)
    path, views = wl[0]
    scene = rt.Scene.from_json_file(path, gpu_ctx)
    good = rt.Renderer(32, 32)
    bad = rt.Renderer(32, 32)
    bad.samples = 0  # "Samples must be greater than 0"
    jobs = [rt.Job(scene, good, views[0][1]), rt.Job(scene, bad, views[1][1]), rt.Job(scene, good, views[2][1])]
    with pytest.raises(rt.RenderError, match="job 1: Samples must be greater than 0"):
        rt.render_batch(jobs, lanes=2, ctx=gpu_ctx)


@pytest.mark.gpu
def test_fused_group_equals_separate_renders(gpu_ctx, tmp_path):
    """Small frames of a batch render as one fused launch sequence over a
    table of frames (then replayed as a graph); every image must equal the
    unfused batch's and rt_render's, and a frame with the outline on (not
    fusable) renders beside the group."""
    wl = workloads.batch_workload(str(tmp_path), n_scenes=4, seed=7)
    jobs = []
    sizes = [(64, 48), (96, 64), (40, 40), (128, 72)]
    for k, (path, views) in enumerate(wl):
        scene = rt.Scene.from_json_file(path, gpu_ctx)
        for v, (name, cam, _) in enumerate(views):
            w, h = sizes[(k + v) % 4]
            r = rt.Renderer(w, h)
            if v == 1:
                r.anti_aliasing_mode = rt.AntiAliasingMode.Stochastic
                r.samples = 3
            if v == 2:
                r.anti_aliasing_mode = rt.AntiAliasingMode.NoJitter
                r.max_depth = 2 + k
            if k == 3 and v == 3:
                r.anti_aliasing_mode = rt.AntiAliasingMode.NoJitter
                r.outline_config = rt.OutlineConfig()
            jobs.append(rt.Job(scene, r, cam))
    saved = rt.batch_tuning(gpu_ctx)
    try:
        rt.batch_tuning(gpu_ctx, fuse_pixels=0)
        want, _ = rt.render_batch(jobs, lanes=2, ctx=gpu_ctx)
        rt.batch_tuning(gpu_ctx, fuse_pixels=1 << 20, blocks_per_sm={"trace": 8, "shadow": 16})
        for rep in range(2):  # capture, then replay
            got, st = rt.render_batch(jobs, lanes=2, ctx=gpu_ctx)
            assert st.jobs == len(jobs)
            for a, b in zip(got, want):
                assert np.array_equal(a, b), rep
        fused = [j for j in jobs if j.renderer.outline_config is None]
        assert all(j.renderer.last_stats.graph == 2 for j in fused)
        assert jobs[-1].renderer.last_stats.graph == 0
        # against rt_render of the same camera written into the scene
        for idx in (0, 5, 10):
            path, cam, r = wl[idx // 4][0], jobs[idx].camera, jobs[idx].renderer
            p2 = tmp_path / "single.json"
            p2.write_text(json.dumps(_with_camera(path, cam)))
            s2 = rt.Scene.from_json_file(str(p2), gpu_ctx)
            assert np.array_equal(got[idx], r.render(s2))
            s2.close()
        # a scratch budget no frame fits: no group, the same images
        rt.batch_tuning(gpu_ctx, fuse_bytes=1)
        got, _ = rt.render_batch(jobs, lanes=2, ctx=gpu_ctx)
        assert all(j.renderer.last_stats.graph == 0 for j in jobs)
        assert all(np.array_equal(a, b) for a, b in zip(got, want))
    finally:
        rt.batch_tuning(gpu_ctx, lanes=saved["lanes"], fuse_pixels=saved["fuse_pixels"],
                        fuse_bytes=saved["fuse_bytes"], blocks_per_sm=saved["blocks_per_sm"])


@pytest.mark.gpu
def test_autotuner_reports_its_choice(gpu_ctx, tmp_path):
    wl = workloads.batch_workload(str(tmp_path), n_scenes=2, seed=9)
    jobs = []
    for path, views in wl:
        scene = rt.Scene.from_json_file(path, gpu_ctx)
        for _, cam, _ in views:
            jobs.append(rt.Job(scene, rt.Renderer(80, 60), cam))
    t = rt.batch_autotune_ex(jobs, ctx=gpu_ctx)
    assert t["lanes"] in (1, 2, 4, 8) and t["fuse_pixels"] in (0, 256 * 256, 640 * 480, 1280 * 720)
    assert t["trials"] >= 5 and t["best_ms"] > 0
    assert rt.batch_tuning(gpu_ctx)["lanes"] == t["lanes"]
    with pytest.raises(ValueError):
        rt.batch_tuning(gpu_ctx, lanes=0)
