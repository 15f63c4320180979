"""ctypes bindings of include/rtrace_gpu.h.

The library is the in-tree ``rtrace_b200/_lib/librtrace_b200.so``; importing
this module fails loudly when it is missing (there is no CPU fallback).
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "librtrace_b200.so")

RT_OK = 0
RT_ERR_INVALID_ARGUMENT = 1
RT_ERR_SCENE = 2
RT_ERR_RENDER = 3
RT_ERR_CUDA = 4
RT_ERR_OUT_OF_MEMORY = 5
RT_ERR_DEVICE_WATCHDOG = 6
RT_ERR_IO = 7

STATUS_NAMES = {
    RT_OK: "RT_OK",
    RT_ERR_INVALID_ARGUMENT: "RT_ERR_INVALID_ARGUMENT",
    RT_ERR_SCENE: "RT_ERR_SCENE",
    RT_ERR_RENDER: "RT_ERR_RENDER",
    RT_ERR_CUDA: "RT_ERR_CUDA",
    RT_ERR_OUT_OF_MEMORY: "RT_ERR_OUT_OF_MEMORY",
    RT_ERR_DEVICE_WATCHDOG: "RT_ERR_DEVICE_WATCHDOG",
    RT_ERR_IO: "RT_ERR_IO",
}


class rt_outline_config(ctypes.Structure):
    _fields_ = [
        ("enabled", ctypes.c_int32),
        ("use_8_neighbors", ctypes.c_int32),
        ("depth_weight", ctypes.c_double),
        ("normal_weight", ctypes.c_double),
        ("threshold", ctypes.c_double),
        ("edge_color", ctypes.c_double * 3),
        ("line_thickness", ctypes.c_double),
        ("object_id_weight", ctypes.c_double),
    ]


class rt_camera_config(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_char * 32),
        ("position", ctypes.c_double * 3),
        ("target", ctypes.c_double * 3),
        ("up", ctypes.c_double * 3),
        ("width", ctypes.c_double),
        ("height", ctypes.c_double),
        ("has_fov", ctypes.c_int32),
        ("has_grid_pitch", ctypes.c_int32),
        ("has_grid_thickness", ctypes.c_int32),
        ("grid_color_state", ctypes.c_int32),
        ("fov", ctypes.c_double),
        ("grid_pitch", ctypes.c_double),
        ("grid_thickness", ctypes.c_double),
        ("grid_color", ctypes.c_double * 3),
    ]


class rt_render_params(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("max_depth", ctypes.c_int32),
        ("use_kdtree", ctypes.c_int32),
        ("samples", ctypes.c_uint32),
        ("anti_aliasing_mode", ctypes.c_int32),
        ("seed", ctypes.c_uint64),
        ("outline", rt_outline_config),
        ("flags", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
        ("disk_samples", ctypes.c_uint32),
        ("learned_shadows", ctypes.c_int32),
        ("learned_rays", ctypes.c_uint32),
        ("fallback_samples", ctypes.c_uint32),
        ("confidence_threshold", ctypes.c_float),
        ("reserved3", ctypes.c_uint32),
    ]


RT_OUTLINE_NOALLOC_MAX_PIXELS = 2048 * 2048
RT_FLAG_STAGE_TIMES = 1
RT_FLAG_COUNT_WORK = 2
RT_FLAG_CUDA_GRAPH = 4
STAGES = ["raygen", "trace", "emit", "shadow", "resolve", "fold", "post", "denoise"]


class rt_stats(ctypes.Structure):
    _fields_ = [
        ("primary_rays", ctypes.c_uint64),
        ("reflection_rays", ctypes.c_uint64),
        ("shadow_rays", ctypes.c_uint64),
        ("hits", ctypes.c_uint64),
        ("trace_nodes", ctypes.c_uint64),
        ("trace_triangles", ctypes.c_uint64),
        ("trace_spheres", ctypes.c_uint64),
        ("trace_verifications", ctypes.c_uint64),
        ("shadow_nodes", ctypes.c_uint64),
        ("shadow_triangles", ctypes.c_uint64),
        ("shadow_spheres", ctypes.c_uint64),
        ("shadow_verifications", ctypes.c_uint64),
        ("kernel_launches", ctypes.c_uint32),
        ("graph", ctypes.c_uint32),
        ("device_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double),
        ("stage_ms", ctypes.c_double * 8),
        ("fallback_hits", ctypes.c_uint64),
        ("fallback_lights", ctypes.c_uint64),
        ("shadow_rays_untraced", ctypes.c_uint64),
    ]


class rt_batch_tuning(ctypes.Structure):
    _fields_ = [
        ("lanes", ctypes.c_uint32),
        ("fuse_pixels", ctypes.c_uint32),
        ("fuse_bytes", ctypes.c_uint64),
        ("blocks_per_sm", ctypes.c_int32 * 7),
        ("trials", ctypes.c_uint32),
        ("best_ms", ctypes.c_double),
    ]


class rt_job(ctypes.Structure):
    _fields_ = [
        ("scene", ctypes.c_void_p),
        ("camera", ctypes.POINTER(rt_camera_config)),
        ("params", rt_render_params),
        ("rgb_out", ctypes.c_void_p),
        ("out_on_device", ctypes.c_int32),
        ("status", ctypes.c_int32),
        ("stats", rt_stats),
    ]


class rt_batch_stats(ctypes.Structure):
    _fields_ = [
        ("jobs", ctypes.c_uint32),
        ("lanes", ctypes.c_uint32),
        ("rays", ctypes.c_uint64),
        ("wall_ms", ctypes.c_double),
        ("device_ms", ctypes.c_double),
        ("busiest_lane_ms", ctypes.c_double),
    ]


_vp = ctypes.c_void_p
_lib = None


class rt_mesh_desc(ctypes.Structure):
    _fields_ = [
        ("vertices", ctypes.c_void_p),
        ("n_triangles", ctypes.c_int64),
        ("bounds_min", ctypes.c_double * 3),
        ("bounds_max", ctypes.c_double * 3),
        ("nodes", ctypes.c_void_p),
        ("n_nodes", ctypes.c_int64),
        ("tri_index", ctypes.c_void_p),
        ("n_tri_index", ctypes.c_int64),
    ]


class rt_scene_desc(ctypes.Structure):
    """The leading fields of rt_scene_desc, up to the meshes."""
    _fields_ = [
        ("camera", rt_camera_config),
        ("objects", ctypes.c_void_p),
        ("n_objects", ctypes.c_int32),
        ("n_materials", ctypes.c_int32),
        ("materials", ctypes.c_void_p),
        ("lights", ctypes.c_void_p),
        ("n_lights", ctypes.c_int32),
        ("n_meshes", ctypes.c_int32),
        ("meshes", ctypes.POINTER(rt_mesh_desc)),
    ]


# rt_kd_node_desc (72 bytes, no padding)
KD_NODE_FIELDS = [("axis", "<i4"), ("right", "<i4"), ("first", "<i4"), ("count", "<i4"), ("split", "<f8"),
                  ("bounds_min", "<f8", (3,)), ("bounds_max", "<f8", (3,))]


def lib():
    """Loads the CUDA library (once); raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "rtrace_b200 CUDA library not found at %s; build it with "
            "`python -m rtrace_b200.build` (nvcc, sm_100a)" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    sig = {
        "rt_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp)]),
        "rt_ctx_destroy": (None, [_vp]),
        "rt_last_error": (ctypes.c_char_p, [_vp]),
        "rt_scene_load_json_file": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.POINTER(_vp)]),
        "rt_scene_load_json_str": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.POINTER(_vp)]),
        "rt_scene_upload": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(_vp)]),
        "rt_scene_outline_config": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(rt_outline_config)]),
        "rt_scene_camera_aspect": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(ctypes.c_double)]),
        "rt_scene_free": (None, [_vp]),
        "rt_render": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(rt_render_params), _vp, ctypes.c_int,
                                     ctypes.POINTER(rt_stats)]),
        "rt_render_rows": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(rt_render_params), ctypes.c_uint32,
                                          ctypes.c_uint32, _vp, ctypes.c_int, ctypes.POINTER(rt_stats)]),
        "rt_host_scene_upload": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(_vp)]),
        "rt_auto_cameras_json_file": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(rt_camera_config)]),
        "rt_auto_cameras_json_str": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(rt_camera_config)]),
        "rt_render_batch": (ctypes.c_int, [_vp, ctypes.POINTER(rt_job), ctypes.c_uint32, ctypes.c_uint32,
                                           ctypes.POINTER(rt_batch_stats)]),
        "rt_batch_autotune": (ctypes.c_int, [_vp, ctypes.POINTER(rt_job), ctypes.c_uint32,
                                             ctypes.POINTER(ctypes.c_uint32)]),
        "rt_batch_assign": (ctypes.c_int, [_vp, ctypes.c_uint32, ctypes.c_uint32, _vp]),
        "rt_batch_autotune_ex": (ctypes.c_int, [_vp, ctypes.POINTER(rt_job), ctypes.c_uint32,
                                                ctypes.POINTER(rt_batch_tuning)]),
        "rt_batch_get_tuning": (ctypes.c_int, [_vp, ctypes.POINTER(rt_batch_tuning)]),
        "rt_batch_set_tuning": (ctypes.c_int, [_vp, ctypes.POINTER(rt_batch_tuning)]),
        "rt_denoiser_load": (ctypes.c_int, [_vp, _vp, ctypes.c_size_t]),
        "rt_denoiser_run": (ctypes.c_int, [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _vp, _vp,
                                           _vp]),
        "rt_dn_train_create": (ctypes.c_int, [_vp, _vp, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint32,
                                              ctypes.c_uint32, _vp]),
        "rt_dn_train_step": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                            ctypes.c_float, _vp]),
        "rt_dn_train_grads": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp]),
        "rt_dn_train_export": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(ctypes.c_size_t)]),
        "rt_dn_train_set_threshold": (ctypes.c_int, [_vp, ctypes.c_float]),
        "rt_dn_train_free": (None, [_vp]),
        "rt_debug_conv_wgrad": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                               ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _vp, _vp]),
        "rt_render_shadow_aov": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(rt_render_params), _vp, _vp, _vp,
                                                ctypes.POINTER(rt_stats)]),
        "rt_render_linear": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(rt_render_params), _vp, _vp,
                                            ctypes.POINTER(rt_stats)]),
        "rt_host_scene_load_json_file": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_vp)]),
        "rt_host_scene_load_json_str": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_vp)]),
        "rt_host_scene_load_json_file_on": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.POINTER(_vp)]),
        "rt_host_scene_load_json_str_on": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.POINTER(_vp)]),
        "rt_kd_build": (ctypes.c_int, [_vp, _vp, ctypes.c_int64, ctypes.POINTER(_vp)]),
        "rt_kd_tree_nodes": (_vp, [_vp, ctypes.POINTER(ctypes.c_int64)]),
        "rt_kd_tree_index": (_vp, [_vp, ctypes.POINTER(ctypes.c_int64)]),
        "rt_kd_tree_free": (None, [_vp]),
        "rt_host_scene_desc": (ctypes.POINTER(rt_scene_desc), [_vp]),
        "rt_host_scene_free": (None, [_vp]),
        "rt_scene_device_bytes": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(ctypes.c_uint64)]),
        "rt_debug_fp64_rate": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_double)]),
        "rt_debug_l2_read_bandwidth": (ctypes.c_int, [_vp, ctypes.c_uint64, ctypes.c_int32,
                                                      ctypes.POINTER(ctypes.c_double)]),
        "rt_outline_apply": (ctypes.c_int, [_vp, ctypes.c_uint32, ctypes.c_uint32, _vp, _vp, _vp, _vp, _vp, _vp,
                                            _vp, _vp, ctypes.POINTER(rt_outline_config), _vp]),
        "rt_outline_apply_noalloc": (ctypes.c_int, [_vp, ctypes.c_uint32, ctypes.c_uint32, _vp, _vp, _vp, _vp,
                                                    _vp, _vp, _vp, _vp, ctypes.POINTER(rt_outline_config), _vp]),
        "rt_debug_stdrng_u32": (ctypes.c_int, [_vp, _vp, ctypes.c_int64, ctypes.c_int32, _vp]),
        "rt_debug_disk_offsets": (ctypes.c_int, [_vp, _vp, ctypes.c_int64, ctypes.c_double, _vp]),
        "rt_png_encode": (ctypes.c_int, [_vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int32,
                                         ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_size_t)]),
        "rt_png_free": (None, [_vp]),
        "rt_png_write": (ctypes.c_int, [ctypes.c_char_p, _vp, ctypes.c_uint32, ctypes.c_uint32]),
        "rt_debug_mesh_prep": (ctypes.c_int, [_vp, ctypes.POINTER(rt_mesh_desc), ctypes.POINTER(ctypes.c_uint32)]),
        "rt_debug_mesh_hit": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, ctypes.c_int32, _vp, ctypes.c_int64,
                                             ctypes.c_double, ctypes.c_double, _vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L
