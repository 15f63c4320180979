// A large mesh's device search data, computed on the device: the work the
// host preparation does (triangle records and normals, the triangle BVH,
// the k-d occurrence lists), with the same results, byte for byte.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "build_arena.hpp"

namespace rtb {

// Device destinations: bvh 7 x bvh_internal_nodes(n, leaf) double2, fbvh
// (the BVH in single precision, dscene.cuh's FNode layout) 1 + 4 x
// bvh_internal_nodes(n, leaf) float4, cells (each k-d leaf's cell, DMesh's
// layout) 3 x n_kd_nodes double2, btris and brute 5n double2, normals n
// double4, occ n_index int2, occ_off n + 1 int.
struct MeshPrepOut {
  double2* bvh;
  float4* fbvh;
  double2* cells;
  double2* btris;
  double2* brute;
  double4* normals;
  int2* occ;
  int* occ_off;
};

// Internal nodes of the median-split BVH over n primitives with leaves of
// at most `leaf` (a function of n alone; at least 1 when n > 0).
int bvh_internal_nodes(int n, int leaf);

// h_vertices: 9n doubles (host); d_kd_nodes: the packed reference k-d
// nodes on the device (4 double2 each, leaves {first, -1 - count} in the
// last word); d_leaf_tris: the leaf lists on the device (n_index entries,
// validated: every entry in [0, n), the leaves cover each entry once);
// d_leaf_path: each node's root path {bits, depth} on the device.
// n > leaf.  Runs on stream s and returns when the results are written;
// scratch (the vertices included) from arena.  Returns "" or the CUDA
// failure (*cuda_err set).
std::string prep_mesh_device(const double* h_vertices, int n, const double2* d_kd_nodes, int n_kd_nodes,
                             const int* d_leaf_tris, const int2* d_leaf_path, int n_index, int leaf, cudaStream_t s,
                             KdArena* arena, const MeshPrepOut& out, cudaError_t* cuda_err);

// The arrays of a host-prepared mesh that follow from its BVH (nb nodes),
// its records in BVH order and its k-d tree: the single-precision BVH, the
// k-d leaf cells, and with the host preparation's bytes the records in mesh
// order, the normals and the k-d occurrence lists.  d_btris: 5n double2
// (each record's triangle id in [0, n)); d_kd_nodes, d_leaf_tris,
// d_leaf_path as for prep_mesh_device.  Destinations as in MeshPrepOut
// (fbvh 1 + 4 nb float4; with d_bvh or fbvh null the single-precision BVH
// is not made).  Queues the work on stream s (scratch from arena) and
// returns without waiting.
std::string derive_mesh_device(const double2* d_bvh, int nb, const double2* d_btris, int n,
                               const double2* d_kd_nodes, int n_kd_nodes, const int* d_leaf_tris,
                               const int2* d_leaf_path, int n_index, cudaStream_t s, KdArena* arena, float4* fbvh,
                               double2* cells, double2* brute, double4* normals, int2* occ, int* occ_off,
                               cudaError_t* cuda_err);

}  // namespace rtb
