// Host-side builders of the device acceleration data.
//
// The reference intersects meshes by walking its k-d tree (src/mesh.rs:
// 399-465) and tests every sphere of the World in scene order
// (src/ray.rs:699-711).  The device answers the same queries with two
// structures built here:
//   * a binary BVH over each mesh's triangles (every triangle stored once),
//     whose hits are then checked against the reference's k-d leaves
//     (kd_leaf_paths gives each leaf's root path for that check), and
//   * a binary BVH over each run of consecutive spheres in the World.
// Node boxes are padded so that a box never rejects a ray that the exact
// primitive test would accept.
#pragma once

#include <cstdint>
#include <vector>

namespace rtb {

// One BVH node: the boxes of both children and how to reach them.
// child count > 0: leaf holding primitives [index, index + count) of the
// node-ordered primitive list; count == 0: internal node `index`;
// count < 0: empty.
struct BvhNode {
  double lmin[3], lmax[3], rmin[3], rmax[3];
  int32_t lidx, lcnt, ridx, rcnt;
};

// Builds a BVH over n primitive boxes; returns nodes (root = 0, preorder,
// left subtree first) and the primitive order (order[k] = primitive id
// stored at position k, ids ascending within a leaf).  A node splits its
// primitives at the median centroid (ties by id) of the axis with the
// widest centroid extent; node boxes are padded by `pad`.
void build_bvh(const std::vector<double>& bmin, const std::vector<double>& bmax, int leaf_size, double pad,
               std::vector<BvhNode>* nodes, std::vector<int32_t>* order);

// The same interface, layout and leaf order, with each node split at the
// boundary of 16 centroid bins (per axis) that minimises the children's
// surface area times primitive count: fewer node visits per ray than the
// median split, at a build cost that keeps it on the host.
void build_bvh_sah(const std::vector<double>& bmin, const std::vector<double>& bmax, int leaf_size, double pad,
                   std::vector<BvhNode>* nodes, std::vector<int32_t>* order);

}  // namespace rtb
