// KdTree::new(triangles, 16, 10) (src/mesh.rs:75-197) built on the device.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/rtrace_gpu.h"
#include "build_arena.hpp"

namespace rtb {

// Device memory a context keeps for its builds (freed with it).
KdArena* kd_arena_new();
void kd_arena_free(KdArena* arena);

// Builds the k-d tree of n triangles (9 doubles each: v0, v1, v2) on the
// current device, on stream s, in arena (null: memory of this build only).
// The nodes (preorder, left child next) and the leaf lists are those of
// the host builder, byte for byte.  Returns "" on success; the reference's
// panic message for a NaN centre in a node it sorts; otherwise a
// description of the CUDA failure (*cuda_err set).
std::string kd_build_device(const double* h_vertices, int64_t n, cudaStream_t s, KdArena* arena,
                            std::vector<rt_kd_node_desc>* nodes, std::vector<int32_t>* idx, cudaError_t* cuda_err);

}  // namespace rtb
