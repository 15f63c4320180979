"""rt_outline_apply_noalloc: the outline post-process for callers that must
not allocate device memory (their device memory belongs to another
allocator, they cannot afford cudaMalloc's synchronisation in a frame loop,
or they must not meet out-of-memory mid-frame).  Its scratch is a static device
array shared by all calls, so two calls in a row must each give exactly what
the allocating rt_outline_apply gives for the same inputs, and an image
beyond the array's size must be refused.

The file name sorts last so that a run stopping at the first failure has
run every other test before this one."""
import numpy as np
import pytest

import rtrace_b200 as rt
from tests.gpu_outline import device_outline, gbuffers

pytestmark = pytest.mark.gpu

CFG = {"use_8_neighbors": True, "thickness": 2.5, "depth_weight": 0.8, "normal_weight": 2.0, "threshold": 0.06,
       "edge_color": (0.1, 0.2, 0.3)}


def test_noalloc_outline_matches_allocating_entry_point(gpu_ctx):
    L = rt._capi.lib()
    # two calls in a row with different images: the second must not see the
    # first call's scratch contents
    for (w, h, seed, cfg) in [(640, 360, 11, CFG), (257, 129, 12, {})]:
        color, valid, depth, normal = gbuffers(w, h, seed)
        st_ref, ref = device_outline(gpu_ctx, L.rt_outline_apply, color, valid, depth, normal, cfg)
        st, got = device_outline(gpu_ctx, L.rt_outline_apply_noalloc, color, valid, depth, normal, cfg)
        assert st_ref == 0 and st == 0, L.rt_last_error(gpu_ctx.handle)
        assert np.array_equal(got, ref), (w, h, int((got != ref).any(2).sum()))


def test_noalloc_outline_rejects_images_beyond_its_scratch(gpu_ctx):
    L = rt._capi.lib()
    w = 4096
    h = rt._capi.RT_OUTLINE_NOALLOC_MAX_PIXELS // w + 1
    import ctypes
    import torch
    dev = torch.device("cuda", gpu_ctx.device)
    small = torch.zeros(16, dtype=torch.float64, device=dev)  # never read: the size check comes first
    flags = torch.zeros(16, dtype=torch.uint8, device=dev)
    oc = rt._capi.rt_outline_config()
    p = small.data_ptr()
    st = L.rt_outline_apply_noalloc(gpu_ctx.handle, w, h, p, p, p, flags.data_ptr(), p, p, p, p, ctypes.byref(oc),
                                    flags.data_ptr())
    assert st == rt._capi.RT_ERR_INVALID_ARGUMENT
    assert b"RT_OUTLINE_NOALLOC_MAX_PIXELS" in L.rt_last_error(gpu_ctx.handle)
