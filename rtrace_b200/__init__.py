"""B200 render path for SeaRyanC/rtrace scenes.

The Python surface mirrors the reference crate's public API
(src/lib.rs re-exports): ``Scene.from_json_file`` / ``Scene.from_json_str``
(src/scene.rs:462-480), ``Renderer`` with its fields and constructors
(src/renderer.rs:37-118), ``AntiAliasingMode`` (src/renderer.rs:16-24),
``OutlineConfig`` (src/outline.rs:5-31) and ``Renderer.render`` /
``Renderer.render_to_file`` (src/renderer.rs:120, 914).  Rendering runs on
the GPU through the C ABI in include/rtrace_gpu.h; there is no CPU path.
Errors the reference returns as ``Err(String)`` raise ``RenderError`` /
``SceneError`` with the reference's message.
"""
import ctypes
import enum
import threading
from dataclasses import dataclass, field

import numpy as np

from . import _capi

__all__ = [
    "AntiAliasingMode", "OutlineConfig", "Scene", "Renderer", "RtraceError", "SceneError",
    "RenderError", "DeviceError", "Context", "RenderStats", "default_context", "write_png", "HostScene",
    "fp64_rate", "l2_read_bandwidth", "batch_autotune_ex", "batch_tuning", "auto_cameras", "Job", "BatchStats", "render_batch", "batch_autotune", "batch_assign",
    "camera_config",
]


class RtraceError(Exception):
    """Base class; ``status`` is the rt_status code."""

    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


class SceneError(RtraceError):
    """Scene::from_json_* failures (JSON, STL, I/O)."""


class RenderError(RtraceError):
    """Errors Renderer::render returns (samples, camera, colours, ranges)."""


class DeviceError(RtraceError):
    """CUDA, memory or device-watchdog failures."""


def _raise(status, ctx_handle):
    msg = _capi.lib().rt_last_error(ctx_handle)
    msg = msg.decode("utf-8", "replace") if msg else _capi.STATUS_NAMES.get(status, str(status))
    if status in (_capi.RT_ERR_SCENE, _capi.RT_ERR_IO):
        raise SceneError(status, msg)
    if status == _capi.RT_ERR_RENDER:
        raise RenderError(status, msg)
    if status == _capi.RT_ERR_INVALID_ARGUMENT:
        raise ValueError(msg)
    raise DeviceError(status, msg)


class AntiAliasingMode(enum.IntEnum):
    """src/renderer.rs:16-24"""
    NoJitter = 0
    Quincunx = 1
    Stochastic = 2


@dataclass
class OutlineConfig:
    """src/outline.rs:5-31 (defaults from OutlineConfig::default)."""
    depth_weight: float = 1.0
    normal_weight: float = 1.0
    threshold: float = 0.1
    edge_color: tuple = (0.0, 0.0, 0.0)
    use_8_neighbors: bool = False
    line_thickness: float = 1.0
    # extension: edges between different objects (0 keeps the reference's outline)
    object_id_weight: float = 0.0


@dataclass
class RenderStats:
    primary_rays: int = 0
    reflection_rays: int = 0
    shadow_rays: int = 0
    device_ms: float = 0.0
    total_ms: float = 0.0
    hits: int = 0
    kernel_launches: int = 0
    stage_ms: dict = field(default_factory=dict)
    work: dict = field(default_factory=dict)
    graph: int = 0  # RT_FLAG_CUDA_GRAPH: 1 captured by this render, 2 replayed
    fallback_hits: int = 0  # learned shadows: primary hits with a light shaded by the plain fallback
    fallback_lights: int = 0  # learned shadows: (primary hit, disk light) pairs shaded by it
    shadow_rays_untraced: int = 0  # counted shadow rays not traced: the surface faces away from the light

    @property
    def rays(self):
        return self.primary_rays + self.reflection_rays + self.shadow_rays

    @classmethod
    def from_c(cls, st):
        work = {k: int(getattr(st, k)) for k in (
            "trace_nodes", "trace_triangles", "trace_spheres", "trace_verifications", "shadow_nodes",
            "shadow_triangles", "shadow_spheres", "shadow_verifications")}
        stages = {name: float(st.stage_ms[i]) for i, name in enumerate(_capi.STAGES)}
        return cls(int(st.primary_rays), int(st.reflection_rays), int(st.shadow_rays), float(st.device_ms),
                   float(st.total_ms), int(st.hits), int(st.kernel_launches), stages, work, int(st.graph),
                   int(st.fallback_hits), int(st.fallback_lights), int(st.shadow_rays_untraced))


class Context:
    """One CUDA device and stream (rt_ctx).  Not shared between threads."""

    def __init__(self, device=0):
        L = _capi.lib()
        h = ctypes.c_void_p()
        st = L.rt_ctx_create(int(device), ctypes.byref(h))
        if st != _capi.RT_OK:
            _raise(st, None)
        self.handle = h
        self.device = device

    def load_denoiser(self, weights=None):
        """Loads the learned soft-shadow denoiser: a weight blob (bytes) or a
        path; None loads the weights shipped with the package."""
        from . import denoiser
        blob = denoiser.read_blob(weights)
        buf = ctypes.create_string_buffer(blob, len(blob))
        st = _capi.lib().rt_denoiser_load(self.handle, buf, len(blob))
        if st != _capi.RT_OK:
            _raise(st, self.handle)

    def close(self):
        if self.handle:
            _capi.lib().rt_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_tls = threading.local()


def default_context(device=0):
    """The calling thread's context for `device` (created on first use)."""
    ctxs = getattr(_tls, "ctxs", None)
    if ctxs is None:
        ctxs = _tls.ctxs = {}
    if device not in ctxs:
        ctxs[device] = Context(device)
    return ctxs[device]


class Scene:
    """A scene uploaded to the device (rt_scene)."""

    def __init__(self, handle, ctx):
        self._handle = handle
        self._ctx = ctx

    @classmethod
    def from_json_file(cls, path, ctx=None):
        """Scene::from_json_file: meshes resolve against the file's directory."""
        ctx = ctx or default_context()
        h = ctypes.c_void_p()
        st = _capi.lib().rt_scene_load_json_file(ctx.handle, str(path).encode(), ctypes.byref(h))
        if st != _capi.RT_OK:
            _raise(st, ctx.handle)
        return cls(h, ctx)

    @classmethod
    def from_json_str(cls, text, ctx=None):
        """Scene::from_json_str: meshes resolve against the current directory."""
        ctx = ctx or default_context()
        h = ctypes.c_void_p()
        st = _capi.lib().rt_scene_load_json_str(ctx.handle, text.encode(), ctypes.byref(h))
        if st != _capi.RT_OK:
            _raise(st, ctx.handle)
        return cls(h, ctx)

    def get_outline_config(self):
        """Scene::get_outline_config (src/scene.rs:515-534): None or OutlineConfig."""
        oc = _capi.rt_outline_config()
        st = _capi.lib().rt_scene_outline_config(self._ctx.handle, self._handle, ctypes.byref(oc))
        if st != _capi.RT_OK:
            _raise(st, self._ctx.handle)
        if not oc.enabled:
            return None
        return OutlineConfig(oc.depth_weight, oc.normal_weight, oc.threshold, tuple(oc.edge_color),
                             bool(oc.use_8_neighbors), oc.line_thickness, oc.object_id_weight)

    @classmethod
    def upload(cls, host_scene, ctx=None):
        """Uploads a HostScene (rt_host_scene_upload: its meshes' device data
        is prepared on the first upload and copied on later ones)."""
        ctx = ctx or default_context()
        h = ctypes.c_void_p()
        L = _capi.lib()
        st = L.rt_host_scene_upload(ctx.handle, host_scene.handle, ctypes.byref(h))
        if st != _capi.RT_OK:
            _raise(st, ctx.handle)
        return cls(h, ctx)

    @property
    def device_bytes(self):
        v = ctypes.c_uint64()
        st = _capi.lib().rt_scene_device_bytes(self._ctx.handle, self._handle, ctypes.byref(v))
        if st != _capi.RT_OK:
            _raise(st, self._ctx.handle)
        return int(v.value)

    @property
    def camera_aspect(self):
        v = ctypes.c_double()
        st = _capi.lib().rt_scene_camera_aspect(self._ctx.handle, self._handle, ctypes.byref(v))
        if st != _capi.RT_OK:
            _raise(st, self._ctx.handle)
        return v.value

    def close(self):
        if self._handle:
            _capi.lib().rt_scene_free(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HostScene:
    """A parsed scene held in host memory only (rt_host_scene): JSON and STL
    parsed, primitives transformed, k-d trees built.  Scene.upload() puts it
    on a device."""

    def __init__(self, handle):
        self.handle = handle

    @classmethod
    def from_json_file(cls, path, ctx=None):
        """ctx: build the k-d trees of large meshes on that context's device
        (the same trees as the host build)."""
        h = ctypes.c_void_p()
        L = _capi.lib()
        if ctx is None:
            st = L.rt_host_scene_load_json_file(str(path).encode(), ctypes.byref(h))
        else:
            st = L.rt_host_scene_load_json_file_on(ctx.handle, str(path).encode(), ctypes.byref(h))
        if st != _capi.RT_OK:
            _raise(st, None if ctx is None else ctx.handle)
        return cls(h)

    @classmethod
    def from_json_str(cls, text, ctx=None):
        h = ctypes.c_void_p()
        L = _capi.lib()
        if ctx is None:
            st = L.rt_host_scene_load_json_str(text.encode(), ctypes.byref(h))
        else:
            st = L.rt_host_scene_load_json_str_on(ctx.handle, text.encode(), ctypes.byref(h))
        if st != _capi.RT_OK:
            _raise(st, None if ctx is None else ctx.handle)
        return cls(h)

    def meshes(self):
        """Copies of each mesh's (vertices (n, 9) float64, k-d nodes, leaf
        index list) as the flattened description holds them."""
        d = _capi.lib().rt_host_scene_desc(self.handle).contents
        out = []
        for i in range(d.n_meshes):
            m = d.meshes[i]
            out.append((_array(m.vertices, np.float64, 9 * m.n_triangles).reshape(-1, 9),
                        _array(m.nodes, KD_NODE_DTYPE, m.n_nodes), _array(m.tri_index, np.int32, m.n_tri_index)))
        return out

    def close(self):
        if self.handle:
            _capi.lib().rt_host_scene_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


KD_NODE_DTYPE = np.dtype(_capi.KD_NODE_FIELDS)


def _array(ptr, dtype, n):
    dtype = np.dtype(dtype)
    if not n:
        return np.zeros(0, dtype)
    return np.frombuffer((ctypes.c_char * (int(n) * dtype.itemsize)).from_address(ptr), dtype).copy()


def kd_build(vertices, ctx=None):
    """rt_kd_build: KdTree::new(triangles, 16, 10) (src/mesh.rs:75-197) of
    an (n, 9) float64 triangle array, on ctx's device or (ctx None) on the
    host.  Returns (nodes, leaf index list): the nodes in preorder as a
    KD_NODE_DTYPE array, the index list as int32."""
    v = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 9)
    L = _capi.lib()
    t = ctypes.c_void_p()
    h = None if ctx is None else ctx.handle
    st = L.rt_kd_build(h, v.ctypes.data if len(v) else None, len(v), ctypes.byref(t))
    if st != _capi.RT_OK:
        _raise(st, h)
    try:
        nn, ni = ctypes.c_int64(), ctypes.c_int64()
        pn = L.rt_kd_tree_nodes(t, ctypes.byref(nn))
        pi = L.rt_kd_tree_index(t, ctypes.byref(ni))
        return _array(pn, KD_NODE_DTYPE, nn.value), _array(pi, np.int32, ni.value)
    finally:
        L.rt_kd_tree_free(t)


def fp64_rate(ctx=None):
    """Measured FP64 add/multiply issue rate of the device, Gop/s."""
    ctx = ctx or default_context()
    v = ctypes.c_double()
    st = _capi.lib().rt_debug_fp64_rate(ctx.handle, ctypes.byref(v))
    if st != _capi.RT_OK:
        _raise(st, ctx.handle)
    return v.value


def l2_read_bandwidth(ctx=None, mbytes=32, reps=50):
    """Measured read bandwidth (GB/s) of an L2-resident buffer of about
    mbytes MB: the ceiling of kernels whose working set stays in L2."""
    ctx = ctx or default_context()
    v = ctypes.c_double()
    st = _capi.lib().rt_debug_l2_read_bandwidth(ctx.handle, int(mbytes * 1e6), int(reps), ctypes.byref(v))
    if st != _capi.RT_OK:
        _raise(st, ctx.handle)
    return v.value


class Renderer:
    """src/renderer.rs:37-118.  thread_count is accepted and ignored."""

    def __init__(self, width, height):
        self.width = int(width)
        self.height = int(height)
        self.max_depth = 10
        self.use_kdtree = True
        self.thread_count = None
        self.samples = 1
        self.anti_aliasing_mode = AntiAliasingMode.Quincunx
        self.seed = 0
        self.outline_config = None
        self.flags = 0  # rtrace_b200._capi.RT_FLAG_* (profiling, CUDA graph replay)
        # extensions (the reference always casts 16 rays per disk light)
        self.disk_samples = 16
        self.learned_shadows = False  # needs Context.load_denoiser first
        self.learned_rays = 0  # rays per disk light at primary hits; 0: what the network was trained on
        # learned shadows: a primary hit whose estimated visibility error
        # exceeds confidence_threshold falls back to the plain path with
        # fallback_samples rays per disk light (0: disk_samples); threshold 0
        # takes the one stored with the weights, a negative one disables it
        self.confidence_threshold = 0.0
        self.fallback_samples = 0
        self.last_stats = RenderStats()

    @classmethod
    def new(cls, width, height):
        return cls(width, height)

    @classmethod
    def new_brute_force(cls, width, height):
        r = cls(width, height)
        r.use_kdtree = False
        return r

    @classmethod
    def new_with_threads(cls, width, height, thread_count):
        r = cls(width, height)
        r.thread_count = thread_count
        return r

    @classmethod
    def new_with_options(cls, width, height, use_kdtree, thread_count):
        r = cls(width, height)
        r.use_kdtree = bool(use_kdtree)
        r.thread_count = thread_count
        return r

    def with_outline_detection(self, config):
        self.outline_config = config
        return self

    def _params(self):
        p = _capi.rt_render_params()
        p.width = self.width
        p.height = self.height
        p.max_depth = int(self.max_depth)
        p.use_kdtree = 1 if self.use_kdtree else 0
        p.samples = int(self.samples)
        p.anti_aliasing_mode = int(self.anti_aliasing_mode)
        p.seed = int(self.seed or 0) & 0xFFFFFFFFFFFFFFFF
        p.flags = int(self.flags)
        p.disk_samples = int(self.disk_samples)
        p.learned_shadows = 1 if self.learned_shadows else 0
        p.learned_rays = int(self.learned_rays)
        p.confidence_threshold = float(self.confidence_threshold)
        p.fallback_samples = int(self.fallback_samples)
        oc = self.outline_config
        if oc is not None:
            p.outline.enabled = 1
            p.outline.use_8_neighbors = 1 if oc.use_8_neighbors else 0
            p.outline.depth_weight = oc.depth_weight
            p.outline.normal_weight = oc.normal_weight
            p.outline.threshold = oc.threshold
            for k in range(3):
                p.outline.edge_color[k] = oc.edge_color[k]
            p.outline.line_thickness = oc.line_thickness
            p.outline.object_id_weight = oc.object_id_weight
        return p

    def render(self, scene, out=None, linear=False, device_ptr=None):
        """Renderer::render: returns an (height, width, 3) uint8 array.

        out: a C-contiguous host uint8 array to fill.  device_ptr: write the
        image to this device address instead (width*height*3 bytes on the
        scene's device); returns None.  linear=True also returns the float64
        colours before quantisation (parity tests)."""
        p = self._params()
        st = _capi.rt_stats()
        L = _capi.lib()
        ctxh = scene._ctx.handle
        if device_ptr is not None:
            code = L.rt_render(ctxh, scene._handle, ctypes.byref(p), int(device_ptr), 1, ctypes.byref(st))
            if code != _capi.RT_OK:
                _raise(code, ctxh)
            self.last_stats = RenderStats.from_c(st)
            return None
        img = _check_out(out, (self.height, self.width, 3))
        if linear:
            lin = np.empty((self.height, self.width, 3), np.float64)
            code = L.rt_render_linear(ctxh, scene._handle, ctypes.byref(p), img.ctypes.data, lin.ctypes.data,
                                      ctypes.byref(st))
        else:
            code = L.rt_render(ctxh, scene._handle, ctypes.byref(p), img.ctypes.data, 0, ctypes.byref(st))
        if code != _capi.RT_OK:
            _raise(code, ctxh)
        self.last_stats = RenderStats.from_c(st)
        return (img, lin) if linear else img

    def render_rows(self, scene, row_begin, row_end, out=None, device_ptr=None):
        """Rows [row_begin, row_end) of the image render() returns, as a
        (row_end - row_begin, width, 3) uint8 array (or written to device_ptr,
        returning None).  The unit of work of a frame split across GPUs."""
        p = self._params()
        st = _capi.rt_stats()
        L = _capi.lib()
        ctxh = scene._ctx.handle
        if device_ptr is not None:
            img, ptr, on_dev = None, int(device_ptr), 1
        else:
            img = _check_out(out, (max(0, int(row_end) - int(row_begin)), self.width, 3))
            ptr, on_dev = img.ctypes.data, 0
        code = L.rt_render_rows(ctxh, scene._handle, ctypes.byref(p), int(row_begin), int(row_end), ptr, on_dev,
                                ctypes.byref(st))
        if code != _capi.RT_OK:
            _raise(code, ctxh)
        self.last_stats = RenderStats.from_c(st)
        return img

    def render_shadow_aov(self, scene, vis_ptr=None, feat_ptr=None, out=None):
        """Renders and also writes the primary samples' disk-light visibility
        ([samples][2][H][W] float) and the denoiser feature image
        ([samples][H][W][16] half) to the given device pointers (either may
        be None).  Returns the (H, W, 3) uint8 image."""
        p = self._params()
        st = _capi.rt_stats()
        ctxh = scene._ctx.handle
        img = _check_out(out, (self.height, self.width, 3))
        code = _capi.lib().rt_render_shadow_aov(ctxh, scene._handle, ctypes.byref(p), img.ctypes.data,
                                                 None if vis_ptr is None else int(vis_ptr),
                                                 None if feat_ptr is None else int(feat_ptr), ctypes.byref(st))
        if code != _capi.RT_OK:
            _raise(code, ctxh)
        self.last_stats = RenderStats.from_c(st)
        return img

    def render_to_file(self, scene, output_path):
        """Renderer::render_to_file: renders and writes a PNG."""
        write_png(output_path, self.render(scene))


def _check_out(out, shape):
    if out is None:
        return np.empty(shape, np.uint8)
    if out.dtype != np.uint8 or tuple(out.shape) != tuple(shape) or not out.flags.c_contiguous:
        raise ValueError(f"out must be a C-contiguous uint8 array of shape {tuple(shape)}")
    return out


def camera_config(cam):
    """A scene-JSON camera dict as an rt_camera_config."""
    c = _capi.rt_camera_config()
    c.kind = cam["kind"].encode()[:31]
    for k in range(3):
        c.position[k] = cam["position"][k]
        c.target[k] = cam["target"][k]
        c.up[k] = cam["up"][k]
    c.width = cam.get("width", 1.0)
    c.height = cam.get("height", 1.0)
    if cam.get("fov") is not None:
        c.has_fov = 1
        c.fov = cam["fov"]
    return c


@dataclass
class Job:
    """One render of a batch: a scene, the Renderer settings, optionally a
    camera dict that replaces the scene's (an auto-camera view)."""
    scene: "Scene"
    renderer: "Renderer"
    camera: dict = None


@dataclass
class BatchStats:
    jobs: int
    lanes: int
    rays: int
    wall_ms: float
    device_ms: float
    busiest_lane_ms: float


def _jobs_array(jobs, outs):
    arr = (_capi.rt_job * len(jobs))()
    keep = []
    for i, j in enumerate(jobs):
        a = arr[i]
        a.scene = j.scene._handle.value if isinstance(j.scene._handle, ctypes.c_void_p) else j.scene._handle
        if j.camera is not None:
            c = camera_config(j.camera)
            keep.append(c)
            a.camera = ctypes.pointer(c)
        a.params = j.renderer._params()
        a.rgb_out = outs[i].ctypes.data
        a.out_on_device = 0
    return arr, keep


def render_batch(jobs, lanes=0, ctx=None):
    """rt_render_batch: renders every job (longest first over `lanes`
    concurrent streams; 0 = the autotuned count) and returns their (H, W, 3)
    uint8 images and the BatchStats.  Each image equals
    job.renderer.render(job.scene) with the job's camera."""
    if not jobs:
        return [], BatchStats(0, 0, 0, 0.0, 0.0, 0.0)
    ctx = ctx or jobs[0].scene._ctx
    outs = [np.empty((j.renderer.height, j.renderer.width, 3), np.uint8) for j in jobs]
    arr, keep = _jobs_array(jobs, outs)
    bs = _capi.rt_batch_stats()
    st = _capi.lib().rt_render_batch(ctx.handle, arr, len(jobs), int(lanes), ctypes.byref(bs))
    if st != _capi.RT_OK:
        _raise(st, ctx.handle)
    for j, a in zip(jobs, arr):
        j.renderer.last_stats = RenderStats.from_c(a.stats)
    return outs, BatchStats(bs.jobs, bs.lanes, bs.rays, bs.wall_ms, bs.device_ms, bs.busiest_lane_ms)


def batch_autotune(jobs, ctx=None):
    """rt_batch_autotune: the fastest lane count for this batch (the context
    keeps every tuned parameter for render_batch(lanes=0))."""
    return batch_autotune_ex(jobs, ctx)["lanes"]


_KINDS = ("raygen", "trace", "emit", "shadow", "resolve", "fold", "pixels")


def _tuning_dict(t):
    return {"lanes": int(t.lanes), "fuse_pixels": int(t.fuse_pixels), "fuse_bytes": int(t.fuse_bytes),
            "blocks_per_sm": {k: int(t.blocks_per_sm[i]) for i, k in enumerate(_KINDS)},
            "trials": int(t.trials), "best_ms": float(t.best_ms)}


def batch_autotune_ex(jobs, ctx=None):
    """rt_batch_autotune_ex: searches lanes, the fused group's size limit and
    its kernels' grid budgets on this batch; returns the chosen parameters."""
    ctx = ctx or jobs[0].scene._ctx
    outs = [np.empty((j.renderer.height, j.renderer.width, 3), np.uint8) for j in jobs]
    arr, keep = _jobs_array(jobs, outs)
    t = _capi.rt_batch_tuning()
    st = _capi.lib().rt_batch_autotune_ex(ctx.handle, arr, len(jobs), ctypes.byref(t))
    if st != _capi.RT_OK:
        _raise(st, ctx.handle)
    return _tuning_dict(t)


def batch_tuning(ctx=None, **changes):
    """The context's batch parameters (rt_batch_get_tuning); keyword
    arguments (lanes, fuse_pixels, fuse_bytes, blocks_per_sm={kind: n})
    change them."""
    ctx = ctx or default_context()
    t = _capi.rt_batch_tuning()
    L = _capi.lib()
    st = L.rt_batch_get_tuning(ctx.handle, ctypes.byref(t))
    if st != _capi.RT_OK:
        _raise(st, ctx.handle)
    if changes:
        if "lanes" in changes:
            t.lanes = int(changes["lanes"])
        if "fuse_pixels" in changes:
            t.fuse_pixels = int(changes["fuse_pixels"])
        if "fuse_bytes" in changes:
            t.fuse_bytes = int(changes["fuse_bytes"])
        for k, v in changes.get("blocks_per_sm", {}).items():
            t.blocks_per_sm[_KINDS.index(k)] = int(v)
        st = L.rt_batch_set_tuning(ctx.handle, ctypes.byref(t))
        if st != _capi.RT_OK:
            _raise(st, ctx.handle)
    return _tuning_dict(t)


def batch_assign(costs, lanes):
    """rt_batch_assign: the lane of each job for the given cost estimates."""
    c = np.ascontiguousarray(costs, dtype=np.float64)
    out = np.zeros(len(c), np.uint32)
    st = _capi.lib().rt_batch_assign(c.ctypes.data if len(c) else None, len(c), int(lanes),
                                     out.ctypes.data if len(c) else None)
    if st != _capi.RT_OK:
        _raise(st, None)
    return out


def auto_cameras(path=None, json_text=None):
    """AutoCamera::generate_cameras (src/auto_camera.rs:9-130): the left,
    front, top and perspective cameras framing the scene's finite objects,
    as scene-JSON camera dicts keyed like AutoCameraResult::to_cameras_json."""
    L = _capi.lib()
    out = (_capi.rt_camera_config * 4)()
    if path is not None:
        st = L.rt_auto_cameras_json_file(str(path).encode(), out)
    else:
        st = L.rt_auto_cameras_json_str(json_text.encode(), out)
    if st != _capi.RT_OK:
        _raise(st, None)
    res = {}
    for name, c in zip(("left", "front", "top", "perspective"), out):
        cam = {"kind": c.kind.decode(), "position": list(c.position), "target": list(c.target), "up": list(c.up),
               "width": c.width, "height": c.height}
        if c.has_fov:
            cam["fov"] = c.fov
        res[name] = cam
    return res


def write_png(path, img):
    """Writes an (H, W, 3) uint8 array as an 8-bit RGB PNG (rt_png_write:
    encoded on the host's threads)."""
    img = np.ascontiguousarray(img, dtype=np.uint8)
    h, w, _ = img.shape
    st = _capi.lib().rt_png_write(str(path).encode(), img.ctypes.data, w, h)
    if st != _capi.RT_OK:
        raise OSError("cannot write %s (%s)" % (path, _capi.STATUS_NAMES.get(st, st)))


def encode_png(img, level=-1):
    """rt_png_encode: the PNG file bytes of an (H, W, 3) uint8 array."""
    img = np.ascontiguousarray(img, dtype=np.uint8)
    h, w, _ = img.shape
    L = _capi.lib()
    buf, n = ctypes.c_void_p(), ctypes.c_size_t()
    st = L.rt_png_encode(img.ctypes.data, w, h, int(level), ctypes.byref(buf), ctypes.byref(n))
    if st != _capi.RT_OK:
        raise ValueError("PNG encoding failed (%s)" % _capi.STATUS_NAMES.get(st, st))
    try:
        return ctypes.string_at(buf, n.value)
    finally:
        L.rt_png_free(buf)
