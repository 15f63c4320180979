// Device-resident scene layout and the intersection routines of the render
// path.  Each primitive test restates one reference function in the same
// IEEE operation order; see the comments for the reference lines.
//
// Acceleration.  The reference tests objects in scene order
// (World::hit, src/ray.rs:699-711) and walks each mesh's k-d tree without
// t-interval pruning (src/mesh.rs:399-465).  The device reaches the same
// answers faster:
//   * Meshes: a BVH over the mesh's triangles proposes candidates; a
//     candidate counts only if the reference's traversal would have tested
//     it, i.e. if one of the k-d leaves holding it is visited by the
//     reference's rules (near child always, far child iff t_split >= 0,
//     one side for axis-parallel rays, then the leaf's slab test).  Among
//     equal-t candidates the one the reference's depth-first walk meets
//     first wins (the strict `t < closest` test keeps the first).  When
//     verification cannot settle a closest-hit query (more ties than the
//     buffer holds, or no minimal candidate is visited), the exact k-d walk
//     runs instead.
//   * Runs of consecutive spheres: a BVH over the run.  Spheres accept
//     `root <= closest`, so the sequential scan's result is the minimal
//     accepted t with ties resolved to the latest sphere; the group search
//     returns exactly that.
//   * Shadow rays only ask `world.hit(..).is_some()`; every per-object
//     test is monotone in t_max, so any accepting object suffices.
// Boxes are padded and pruning uses a relative margin, so a box never
// rejects a primitive the exact test would accept.  Mesh BVH boxes are
// tested in single precision with margins that keep this (RayF).
#pragma once

#include "dmath.cuh"

namespace rtb {

#ifndef RTB_INF
#define RTB_INF __longlong_as_double(0x7ff0000000000000LL)
#endif

enum { OBJ_SPHERE = 0, OBJ_PLANE = 1, OBJ_CUBE = 2, OBJ_MESH = 3, OBJ_SPHERE_GROUP = 4 };

// Device error flags (bitmask in DFrame::err)
enum { ERR_WATCHDOG = 1, ERR_EMPTY_RANGE = 2, ERR_STACK = 4, ERR_RANGE_OVERFLOW = 8 };

// Pruning: a box is skipped only when its entry exceeds t * REL + ABS.
#define RTB_PRUNE_REL 1.000001
#define RTB_PRUNE_ABS 1e-9
#define RTB_STACK 64
#define RTB_TIES 8

struct DCube {
  double c[3], half[3];
  double w2l[12];  // rows 0..2 of the world-to-local matrix
  double l2w[12];  // rows 0..2 of the local-to-world matrix
  double ntr[9];   // inverse-transpose of w2l's rotation part
  int identity;
  int pad;
};

// BVH node: 7 double2 = lmin, lmax, rmin, rmax (12 doubles) + int4
// {lidx, lcnt, ridx, rcnt} (cnt > 0 leaf range, 0 internal node, < 0 empty).
// Triangle records: 5 double2 = v0, e1 = v1 - v0, e2 = v2 - v0,
// meta = int2{triangle index, degenerate}.
// k-d nodes: 4 double2 = (bmin.x, bmin.y) (bmin.z, bmax.x) (bmax.y, bmax.z)
// (split, int2 meta): internal {right child, axis}, leaf {first, -1-count}.
struct DMesh {
  double bmin[3], bmax[3];
  // triangle BVH nodes in double precision: set only for meshes prepared on
  // the device (null for host-prepared ones) and read by no walk; the
  // walks test fbvh
  const double2* bvh;
  const float4* fbvh;      // the BVH in single precision (FNode), which the walks test
  const double2* btris;    // triangle records in BVH leaf order
  const double2* brute;    // triangle records in original order
  const double4* normals;  // normalize(e1 x e2) per triangle
  const double2* nodes;    // reference k-d tree, preorder
  const int* leaf_tris;    // k-d leaf triangle lists, leaf order (KdNode::Leaf.triangles)
  const int2* leaf_path;   // per k-d node: {path bits (bit k: right at depth k), depth}
  const double2* cells;    // per k-d leaf: its cell lo < p <= hi (3 double2: lo.xyz, hi.xyz)
  const int* occ_off;      // per triangle: occurrences [occ_off[t], occ_off[t+1])
  const int2* occ;         // {k-d leaf node, position in the leaf}
  int n_nodes;
  int n_tris;
};

// A run of consecutive spheres [first_obj, first_obj + count) in the World.
struct DSphGroup {
  const float4* fbvh;  // BVH over the run in single precision (FNode); leaves index `order`
  const int* order;    // BVH position -> position in the run
  int first_sphere;    // index of the run's first sphere in DScene::sph
  int first_obj;       // World index of the run's first sphere
  int count;
  int pad;
};

struct DMat {
  double color[3];
  double ambient, diffuse, specular, shininess;
  double refl;
  int has_refl;
  int texture;
  double grid_color[3];  // the grid colour after its #RRGGBB round trip
  double half_width, cell_size;
  double cb_color[3];
  double cb_ambient, cb_diffuse, cb_specular, cb_shininess;
};

struct DLight {
  double pos[3];
  double color[3];
  double intensity;
  double diameter;
  int disk;
  int pad;
};

struct DScene {
  int n_obj;  // entries of `obj` (a sphere group is one entry)
  int n_lights;
  const int4* obj;     // {kind, index in its kind array, material, World index}
  const double* sph;   // 5 per sphere: cx cy cz r r*r
  const int* sph_mat;  // per sphere: material index
  const double* pln;   // 12 per plane: p, n, u axis, v axis
  const DCube* cub;
  const DMesh* mesh;
  const DSphGroup* grp;
  const DMat* mat;
  const DLight* lights;
  double amb_color[3];
  double amb_int;
  double fog_color[3];
  double fog_density, fog_start, fog_end;
  double bg[3];
  int has_fog;
  int shadow_per_hit;
};

struct DCam {
  double origin[3], hor[3], ver[3], llc[3], vdir[3];
  double campos[3];
  double pitch, half_th, gcolor[3];
  int persp;
  int grid;
};

// Work counters (profiling renders only).
struct Work {
  unsigned long long nodes, tris, spheres, verify;
};

// Per-ray constants shared by all object tests.
struct RayC {
  V3 o, d;
  double dd;  // d.d (sphere `a`)
  V3 inv;     // 1/d per axis
  int par;    // bit a: |d[a]| < 1e-9 (k-d slabs treat the axis as parallel)
};
__device__ __forceinline__ RayC make_rayc(V3 o, V3 d) {
  RayC r;
  r.o = o;
  r.d = d;
  r.dd = dot(d, d);
  r.inv = mk(1.0 / d.x, 1.0 / d.y, 1.0 / d.z);
  r.par = (fabs(d.x) < 1e-9 ? 1 : 0) | (fabs(d.y) < 1e-9 ? 2 : 0) | (fabs(d.z) < 1e-9 ? 4 : 0);
  return r;
}

// Sphere::hit (src/ray.rs:89-120): returns the accepted root
__device__ __forceinline__ bool sphere_t(const double* s, const RayC& r, double tmin, double tmax, double* t) {
  V3 oc = r.o - mk(s[0], s[1], s[2]);
  double a = r.dd;
  double hb = dot(oc, r.d);
  double c = dot(oc, oc) - s[4];
  double disc = hb * hb - a * c;
  if (disc < 0.0) return false;
  double sq = sqrt(disc);
  double root = (-hb - sq) / a;
  if (root < tmin || tmax < root) {
    root = (-hb + sq) / a;
    if (root < tmin || tmax < root) return false;
  }
  *t = root;
  return true;
}

// Plane::hit (src/ray.rs:136-148)
__device__ __forceinline__ bool plane_t(const double* p, const RayC& r, double tmin, double tmax, double* t) {
  V3 n = mk(p[3], p[4], p[5]);
  double denom = dot(n, r.d);
  if (fabs(denom) < 1e-8) return false;
  double tt = dot(mk(p[0], p[1], p[2]) - r.o, n) / denom;
  if (tt < tmin || tt > tmax) return false;
  *t = tt;
  return true;
}

// Cube::hit (src/ray.rs:411-465).  axis receives the index whose slab set
// the entry (the local normal is -e_axis), or 3 when none did.
__device__ __forceinline__ bool cube_t(const DCube& C, const RayC& r, double tmin, double tmax, double* t,
                                       int* axis) {
  V3 lo = gemv34(C.w2l, r.o - ld3(C.c), 0.0);
  V3 ld = gemv34(C.w2l, r.d, 0.0);
  if (norm(ld) < 1e-8) return false;
  V3 dn = normalize(ld);
  double tl = tmin, th = tmax;
  int ax = 3;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    double inv = 1.0 / dn[a];
    double t0 = (-C.half[a] - lo[a]) * inv;
    double t1 = (C.half[a] - lo[a]) * inv;
    if (inv < 0.0) {
      double tmp = t0;
      t0 = t1;
      t1 = tmp;
    }
    if (t0 > tl) {
      tl = t0;
      ax = a;
    }
    if (t1 < th) th = t1;
    if (tl > th) return false;
  }
  double tt = tl > tmin ? tl : th;
  if (tt < tmin || tt > tmax) return false;
  *t = tt;
  *axis = ax;
  return true;
}

// MeshObject::intersect_bounds (src/ray.rs:586-610)
__device__ __forceinline__ bool mesh_bounds(const DMesh& M, const RayC& r, double tmin, double tmax) {
  double tl = tmin, th = tmax;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    double inv = r.inv[a];
    double t0 = (M.bmin[a] - r.o[a]) * inv;
    double t1 = (M.bmax[a] - r.o[a]) * inv;
    if (inv < 0.0) {
      double tmp = t0;
      t0 = t1;
      t1 = tmp;
    }
    tl = rmax(tl, t0);
    th = rmin(th, t1);
    if (tl > th) return false;
  }
  return true;
}

// MeshObject::intersect_triangle (src/ray.rs:527-583) up to the acceptance
// test; the normal is looked up afterwards for the winning triangle.
__device__ __forceinline__ bool tri_t(const double2* E, const RayC& r, double tmin, double tmax, double* t) {
  double2 q0 = __ldg(E + 0), q1 = __ldg(E + 1), q2 = __ldg(E + 2), q3 = __ldg(E + 3), q4 = __ldg(E + 4);
  V3 v0 = mk(q0.x, q0.y, q1.x);
  V3 e1 = mk(q1.y, q2.x, q2.y);
  V3 e2 = mk(q3.x, q3.y, q4.x);
  V3 h = cross(r.d, e2);
  double a = dot(e1, h);
  if (a > -1e-8 && a < 1e-8) return false;
  double f = 1.0 / a;
  V3 s = r.o - v0;
  double u = f * dot(s, h);
  if (!(u >= 0.0 && u <= 1.0)) return false;
  V3 q = cross(s, e1);
  double v = f * dot(r.d, q);
  if (v < 0.0 || u + v > 1.0) return false;
  double tt = f * dot(e2, q);
  if (tt > tmin && tt < tmax) {
    if (hi32(q4.y)) return false;  // ||e1 x e2|| < 1e-8
    *t = tt;
    return true;
  }
  return false;
}

// KdTree::ray_intersects_bounds (src/mesh.rs:218-255); *te = slab entry
__device__ __forceinline__ bool kd_slab(const double2* N, const RayC& r, double* te) {
  double2 n0 = __ldg(N + 0), n1 = __ldg(N + 1), n2 = __ldg(N + 2);
  double bmin[3] = {n0.x, n0.y, n1.x}, bmax[3] = {n1.y, n2.x, n2.y};
  double tl = -RTB_INF, th = RTB_INF;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    double o = r.o[a];
    if (r.par & (1 << a)) {
      if (o < bmin[a] || o > bmax[a]) return false;
    } else {
      double inv = r.inv[a];
      double t0 = (bmin[a] - o) * inv;
      double t1 = (bmax[a] - o) * inv;
      if (t0 > t1) {
        double tmp = t0;
        t0 = t1;
        t1 = tmp;
      }
      tl = rmax(tl, t0);
      th = rmin(th, t1);
      if (tl > th) return false;
    }
  }
  *te = tl;
  return th >= 0.0;
}

// `(split - origin) / dir >= 0.0` without the division (src/mesh.rs:441,
// :448).  Here |dir| >= 1e-9 and |dir| <= 1 (a unit direction), so a
// non-zero numerator gives a quotient of magnitude at least the smallest
// subnormal: the quotient is non-negative exactly when the numerator is
// zero or both signs agree (and neither operand is NaN).
__device__ __forceinline__ bool split_ahead(double split, double origin, double dir) {
  double diff = split - origin;
  return (diff == 0.0 && dir == dir) || (diff > 0.0 && dir > 0.0) || (diff < 0.0 && dir < 0.0);
}

// Whether the reference's traversal tests k-d leaf `leaf` for this ray
// (src/mesh.rs:399-465, leaf test :411); *key orders visited leaves in the
// reference's depth-first visiting order (bit 31-k: far child at depth k).
__device__ __forceinline__ bool kd_leaf_visited(const DMesh& M, const RayC& r, int leaf, unsigned* key) {
  int2 lp = __ldg(M.leaf_path + leaf);
  unsigned path = (unsigned)lp.x;
  int depth = lp.y;
  int node = 0;
  unsigned k_out = 0;
  for (int k = 0; k < depth; k++) {
    double2 n3 = __ldg(M.nodes + 4 * (size_t)node + 3);
    int right = lo32(n3.y), axis = hi32(n3.y);
    double split = n3.x;
    bool go_right = (path >> k) & 1u;
    double op = r.o[axis];
    bool left_side = op <= split;
    if (r.par & (1 << axis)) {
      if (go_right == left_side) return false;  // only the origin's side
    } else if (go_right == left_side) {         // far child: needs t_split >= 0
      if (!split_ahead(split, op, r.d[axis])) return false;
      k_out |= 1u << (31 - k);
    }
    node = go_right ? right : node + 1;
  }
  double te;
  if (!kd_slab(M.nodes + 4 * (size_t)node, r, &te)) return false;
  *key = k_out;
  return true;
}

// kd_leaf_visited's answer without its root-to-leaf walk, from the leaf's
// cell: per axis, lo = the largest split the path turns right at and hi =
// the smallest it turns left at (k_prep_cells).  The walk fails at a
// right turn at split s only when o <= s and split_ahead(s, o, d) fails,
// and that happens at some right turn of an axis exactly when
// !(o > lo || d > 0 || (o == lo && d == d)); at a left turn only when
// o > s and d is not negative, i.e. when !(o <= hi || d < 0).  On an axis
// the reference treats as parallel, the origin must be on the leaf's side
// of every split: lo < o <= hi.  Then the leaf's slab test.  A cell that
// could not be built (NaN split on the path, marked by a NaN lo) or a
// non-finite origin takes the walk.
__device__ __forceinline__ bool kd_leaf_visited_cell(const DMesh& M, const RayC& r, int leaf, Work* w) {
  const double2* C = M.cells + 3 * (size_t)leaf;
  const double2 c0 = __ldg(C), c1 = __ldg(C + 1), c2 = __ldg(C + 2);
  const double lo[3] = {c0.x, c0.y, c1.x}, hi[3] = {c1.y, c2.x, c2.y};
  if (w) w->verify += 4;
  const bool finite_o = fabs(r.o.x) < RTB_INF && fabs(r.o.y) < RTB_INF && fabs(r.o.z) < RTB_INF;
  if (lo[0] != lo[0] || !finite_o) {
    if (w) w->verify += (unsigned)__ldg(M.leaf_path + leaf).y;
    unsigned key;
    return kd_leaf_visited(M, r, leaf, &key);
  }
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const double o = r.o[a], d = r.d[a];
    if (r.par & (1 << a)) {
      if (!(o > lo[a] && o <= hi[a])) return false;
    } else {
      if (!(o > lo[a] || d > 0.0 || (o == lo[a] && d == d))) return false;
      if (!(o <= hi[a] || d < 0.0)) return false;
    }
  }
  if (w) w->verify += 3;
  double te;
  return kd_slab(M.nodes + 4 * (size_t)leaf, r, &te);
}

// Whether the reference tests triangle `tri` for this ray: whether it
// visits some k-d leaf holding it.
__device__ __forceinline__ bool tri_visited(const DMesh& M, const RayC& r, int tri, Work* w) {
  const int b = __ldg(M.occ_off + tri), e = __ldg(M.occ_off + tri + 1);
  for (int k = b; k < e; k++)
    if (kd_leaf_visited_cell(M, r, __ldg(M.occ + k).x, w)) return true;
  return false;
}

// The reference's first test of triangle `tri` for this ray: the smallest
// (leaf key, position) over the visited leaves holding it.
__device__ __forceinline__ bool tri_first_visit(const DMesh& M, const RayC& r, int tri, unsigned long long* order,
                                                Work* w) {
  int b = __ldg(M.occ_off + tri), e = __ldg(M.occ_off + tri + 1);
  bool any = false;
  unsigned long long best = ~0ULL;
  for (int k = b; k < e; k++) {
    int2 oc = __ldg(M.occ + k);
    // work unit: one 16-byte read (occurrence, each ancestor's split record,
    // and three for the leaf box)
    if (w) w->verify += 4 + (unsigned)__ldg(M.leaf_path + oc.x).y;
    unsigned key;
    if (kd_leaf_visited(M, r, oc.x, &key)) {
      unsigned long long o = ((unsigned long long)key << 32) | (unsigned)oc.y;
      if (o < best) best = o;
      any = true;
    }
  }
  *order = best;
  return any;
}

// The exact reference k-d walk (MeshObject::hit with KdTree::traverse,
// src/ray.rs:614-649, src/mesh.rs:399-465) with exact subtree culling by
// node bounds and closest-t pruning.  Returns the winning triangle index.
template <bool ANY>
__device__ bool mesh_kd_walk(const DMesh& M, const RayC& r, double tmin, double& closest, int& best_tri, int* err,
                             Work* w) {
  if (M.n_nodes == 0) return false;
  bool found = false;
  int stack[RTB_STACK];
  int sp = 0;
  int node = 0;
  for (;;) {
    const double2* N = M.nodes + 4 * (size_t)node;
    double te;
    if (w) w->nodes++;
    bool visit = kd_slab(N, r, &te) && !(te > closest * RTB_PRUNE_REL + RTB_PRUNE_ABS);
    if (visit) {
      double2 n3 = __ldg(N + 3);
      int ma = lo32(n3.y), mb = hi32(n3.y);
      if (mb < 0) {
        int first = ma, cnt = -1 - mb;
        for (int k = 0; k < cnt; k++) {
          double t;
          int tri = __ldg(M.leaf_tris + first + k);
          const double2* E = M.brute + 5 * (size_t)tri;
          if (w) w->tris++;
          if (tri_t(E, r, tmin, closest, &t) && t < closest) {
            closest = t;
            best_tri = tri;
            found = true;
            if (ANY) return true;
          }
        }
      } else {
        int axis = mb;
        double split = n3.x;
        double op = r.o[axis];
        int near_c = op <= split ? node + 1 : ma;
        int far_c = op <= split ? ma : node + 1;
        if (r.par & (1 << axis)) {
          node = near_c;
          continue;
        }
        if (split_ahead(split, op, r.d[axis])) {
          if (sp >= RTB_STACK) {
            atomicOr(err, ERR_STACK);
            return found;
          }
          stack[sp++] = far_c;
        }
        node = near_c;
        continue;
      }
    }
    if (sp == 0) break;
    node = stack[--sp];
  }
  return found;
}

// A BVH node in single precision: the double node's child boxes rounded
// outwards to floats, the same child references.  Layout: fbvh[0].x is
// the largest |coordinate| of any child box (the scale the slab constants
// below need; elements 1-3 unused); node k is fbvh[H + 4k .. H + 3 + 4k]
// (H = RTB_FBVH_HEAD) = {lmn.xyz, lmx.x},
// {lmx.yz, rmn.xy}, {rmn.z, rmx.xyz}, {lidx, lcnt, ridx, rcnt as int bits}.
struct FNode {
  float lmn[3], lmx[3], rmn[3], rmx[3];
  int lidx, lcnt, ridx, rcnt;
};
__device__ __forceinline__ FNode load_fnode(const float4* fbvh, int node) {
  const float4* N = fbvh + RTB_FBVH_HEAD + 4 * (size_t)node;
  const float4 a = __ldg(N + 0), b = __ldg(N + 1), c = __ldg(N + 2), d = __ldg(N + 3);
  FNode n;
  n.lmn[0] = a.x; n.lmn[1] = a.y; n.lmn[2] = a.z;
  n.lmx[0] = a.w; n.lmx[1] = b.x; n.lmx[2] = b.y;
  n.rmn[0] = b.z; n.rmn[1] = b.w; n.rmn[2] = c.x;
  n.rmx[0] = c.y; n.rmx[1] = c.z; n.rmx[2] = c.w;
  n.lidx = __float_as_int(d.x);
  n.lcnt = __float_as_int(d.y);
  n.ridx = __float_as_int(d.z);
  n.rcnt = __float_as_int(d.w);
  return n;
}

// A ray's single-precision slab constants.  Entry distances are taken from
// hi = o + delta rounded up, exit distances from lo = o - delta rounded
// down: the distances of the box grown by delta on every side.  One float
// subtraction and one product with the rounded reciprocal move a computed
// slab plane by at most 3.0002 * 2^-24 * (|box coordinate| + |hi|), so
// delta = 3e-7 * (scale + max |o|) keeps every computed interval around
// the exact interval of the float box (which holds the double box): a box
// the exact ray meets is never rejected.  An axis with d = 0 has an
// infinite reciprocal: the slab is everything or nothing (0 * inf = NaN
// only when the origin lies outside the unpadded box, where either answer
// is right).  all: the constants cannot bound the rounding (NaN, an origin
// or scale beyond 1e30, a component of d nonzero but below 1e-30, whose
// reciprocal would overflow), so every box is accepted.
struct RayF {
  float lo[3], hi[3], inv[3];
  bool all;
};
__device__ __forceinline__ RayF make_rayf(const RayC& r, float scale) {
  RayF f;
  bool bad = !(scale < 1e30f);
  double om = 0.0;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const double o = r.o[a], d = r.d[a];
    bad = bad || !(fabs(o) < 1e30) || d != d || (d != 0.0 && fabs(d) < 1e-30);
    om = fmax(om, fabs(o));
  }
  const double delta = 3e-7 * ((double)scale + om) + 1e-30;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    f.lo[a] = __double2float_rd(r.o[a] - delta);
    f.hi[a] = __double2float_ru(r.o[a] + delta);
    f.inv[a] = __double2float_rn(r.inv[a]);
  }
  f.all = bad;
  return f;
}

// Ray/box entry for BVH culling (padded boxes; not a reference test), in
// single precision: never rejects a box that the exact ray meets within
// tmax (see RayF); tmax is the rounded-up pruning bound
// t * RTB_PRUNE_REL + RTB_PRUNE_ABS.
__device__ __forceinline__ bool box_hit_f(const float* mn, const float* mx, const RayF& f, float tmax, float* te) {
  float tl = -__int_as_float(0x7f800000), th = __int_as_float(0x7f800000);
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const float t0 = (mn[a] - f.hi[a]) * f.inv[a];
    const float t1 = (mx[a] - f.lo[a]) * f.inv[a];
    tl = fmaxf(tl, fminf(t0, t1));
    th = fminf(th, fmaxf(t0, t1));
  }
  *te = tl;
  return f.all || (tl <= th && th >= 0.0f && !(tl > tmax));
}

// Node source of the BVH walks (meshes and sphere runs): a BVH's FP32
// nodes and one ray's box test.  bound(t) turns a pruning distance into
// the form test() takes.
struct FNodes {
  typedef FNode Node;
  typedef float T;
  const float4* fbvh;
  RayF f;
  __device__ __forceinline__ Node load(int k) const { return load_fnode(fbvh, k); }
  // the pruning bound t * RTB_PRUNE_REL + RTB_PRUNE_ABS, rounded up
  __device__ __forceinline__ float bound(double t) const {
    return __double2float_ru(t * RTB_PRUNE_REL + RTB_PRUNE_ABS);
  }
  __device__ __forceinline__ bool test(const T* mn, const T* mx, float b, T* te) const {
    return box_hit_f(mn, mx, f, b, te);
  }
};
__device__ __forceinline__ FNodes mesh_nodes(const DMesh& M, const RayC& r) {
  return FNodes{M.fbvh, make_rayf(r, __ldg(M.fbvh).x)};
}
__device__ __forceinline__ FNodes group_nodes(const DSphGroup& G, const RayC& r) {
  return FNodes{G.fbvh, make_rayf(r, __ldg(G.fbvh).x)};
}

// Generic BVH walk.  visit_leaf(first, count) tests a leaf's primitives and
// returns true to stop; bound() is the current pruning t.  Children are
// visited nearest first.
template <class Nodes, class Leaf, class Bound>
__device__ __forceinline__ bool bvh_walk(const Nodes& src, Leaf visit_leaf, Bound bound, int* err, Work* w) {
  int stack[RTB_STACK];
  int sp = 0;
  int node = 0;
  for (;;) {
    const typename Nodes::Node n = src.load(node);
    if (w) w->nodes++;
    typename Nodes::T tl = 0, tr = 0;
    const auto b = src.bound(bound());
    bool hl = n.lcnt >= 0 && src.test(n.lmn, n.lmx, b, &tl);
    bool hr = n.rcnt >= 0 && src.test(n.rmn, n.rmx, b, &tr);
    bool swap = hl && hr && tr < tl;
    int aidx = swap ? n.ridx : n.lidx, acnt = swap ? n.rcnt : n.lcnt;
    int bidx = swap ? n.lidx : n.ridx, bcnt = swap ? n.lcnt : n.rcnt;
    bool ha = swap ? hr : hl, hb = swap ? hl : hr;
    int next = -1;
    if (ha) {
      if (acnt > 0) {
        if (visit_leaf(aidx, acnt)) return true;
      } else {
        next = aidx;
      }
    }
    if (hb) {
      if (bcnt > 0) {
        if (visit_leaf(bidx, bcnt)) return true;
      } else if (next < 0) {
        next = bidx;
      } else {
        if (sp >= RTB_STACK) {
          atomicOr(err, ERR_STACK);
          return false;
        }
        stack[sp++] = bidx;
      }
    }
    if (next >= 0) {
      node = next;
      continue;
    }
    if (sp == 0) return false;
    node = stack[--sp];
  }
}

// Closest hit on a mesh (MeshObject::hit, src/ray.rs:614-675).  On entry
// `closest` is the World's closest-so-far; on a hit it becomes the hit's t
// and best_tri the winning triangle (original index).
__device__ bool mesh_closest(const DMesh& M, const RayC& r, double tmin, double& closest, int& best_tri,
                             bool use_kd, int* err, Work* w) {
  if (!mesh_bounds(M, r, tmin, closest)) return false;
  const double cin = closest;
  double bt = closest;
  bool have = false;
  int ties[RTB_TIES];
  int nt = 0;
  bool overflow = false;
  bvh_walk(
      mesh_nodes(M, r),
      [&](int first, int cnt) {
        for (int k = 0; k < cnt; k++) {
          const double2* E = M.btris + 5 * (size_t)(first + k);
          double t;
          if (w) w->tris++;
          if (tri_t(E, r, tmin, cin, &t)) {
            int tri = lo32(__ldg(E + 4).y);
            if (!have || t < bt) {
              bt = t;
              have = true;
              nt = 0;
              ties[nt++] = tri;
              overflow = false;
            } else if (t == bt) {
              if (nt < RTB_TIES) ties[nt++] = tri;
              else overflow = true;
            }
          }
        }
        return false;
      },
      [&]() { return bt; }, err, w);
  // No triangle meets t in (tmin, closest): the reference finds none either.
  if (!have) return false;
  if (!use_kd) {
    // brute force tests in original order: lowest index among the minimal t
    int bi = ties[0];
    for (int k = 1; k < nt; k++) bi = min(bi, ties[k]);
    if (overflow) {
      for (int i = 0; i < M.n_tris; i++) {
        double t;
        if (tri_t(M.brute + 5 * (size_t)i, r, tmin, cin, &t) && t == bt) {
          bi = i;
          break;
        }
      }
    }
    closest = bt;
    best_tri = bi;
    return true;
  }
  if (nt == 1 && tri_visited(M, r, ties[0], w)) {
    closest = bt;
    best_tri = ties[0];
    return true;
  }
  if (!overflow) {
    unsigned long long bo = ~0ULL;
    int bi = -1;
    for (int k = 0; k < nt; k++) {
      unsigned long long o;
      if (tri_first_visit(M, r, ties[k], &o, w) && o < bo) {
        bo = o;
        bi = ties[k];
      }
    }
    if (bi >= 0) {
      closest = bt;
      best_tri = bi;
      return true;
    }
  }
  // The reference does not test the nearest triangle (or too many tie):
  // answer with the reference's own walk.
  return mesh_kd_walk<false>(M, r, tmin, closest, best_tri, err, w);
}

// world.hit(..).is_some() restricted to one mesh: a triangle accepted in
// (tmin, tmax) that the reference's traversal would test.
__device__ bool mesh_any(const DMesh& M, const RayC& r, double tmin, double tmax, bool use_kd, int* err, Work* w) {
  if (!mesh_bounds(M, r, tmin, tmax)) return false;
  return bvh_walk(
      mesh_nodes(M, r),
      [&](int first, int cnt) {
        for (int k = 0; k < cnt; k++) {
          const double2* E = M.btris + 5 * (size_t)(first + k);
          double t;
          if (w) w->tris++;
          if (tri_t(E, r, tmin, tmax, &t)) {
            if (!use_kd) return true;
            if (tri_visited(M, r, lo32(__ldg(E + 4).y), w)) return true;
          }
        }
        return false;
      },
      [&]() { return tmax; }, err, w);
}

// A run of spheres: minimal accepted root, ties to the latest sphere.  On
// entry `closest` is the World's closest-so-far (an inclusive bound, as
// Sphere::hit accepts root == t_max).
template <bool ANY>
__device__ bool group_hit(const DScene& S, const DSphGroup& G, const RayC& r, double tmin, double& closest,
                          int& best, int* err, Work* w) {
  bool have = false;
  double bt = closest;
  int bi = -1;
  bool stop = bvh_walk(
      group_nodes(G, r),
      [&](int first, int cnt) {
        for (int k = 0; k < cnt; k++) {
          int sidx = __ldg(G.order + first + k);  // position in the run
          double t;
          if (w) w->spheres++;
          if (sphere_t(S.sph + 5 * (size_t)(G.first_sphere + sidx), r, tmin, bt, &t)) {
            if (ANY) {
              bi = sidx;
              bt = t;
              return true;
            }
            if (!have || t < bt || sidx > bi) {
              bt = t;
              bi = sidx;
              have = true;
            }
          }
        }
        return false;
      },
      [&]() { return bt; }, err, w);
  if (ANY) {
    if (!stop) return false;
    best = bi;
    closest = bt;
    return true;
  }
  if (!have) return false;
  closest = bt;
  best = bi;
  return true;
}

struct WHit {
  int obj;  // World index of the winner, -1 = miss
  int aux;  // mesh triangle / cube axis
  double t;
  int ent;  // entry of DScene::obj that produced the hit
};

// World::hit (src/ray.rs:699-711): scene order, closest narrowing
__device__ __forceinline__ WHit world_closest(const DScene& S, const RayC& r, double tmin, bool use_kd, int* err,
                                             Work* w) {
  double closest = RTB_INF;
  WHit h{-1, 0, 0.0, -1};
  for (int i = 0; i < S.n_obj; i++) {
    int4 ob = __ldg(S.obj + i);
    double t;
    switch (ob.x) {
      case OBJ_SPHERE:
        if (w) w->spheres++;
        if (sphere_t(S.sph + 5 * (size_t)ob.y, r, tmin, closest, &t)) {
          closest = t;
          h = WHit{ob.w, 0, t, i};
        }
        break;
      case OBJ_PLANE:
        if (plane_t(S.pln + 12 * (size_t)ob.y, r, tmin, closest, &t)) {
          closest = t;
          h = WHit{ob.w, 0, t, i};
        }
        break;
      case OBJ_CUBE: {
        int ax;
        if (cube_t(S.cub[ob.y], r, tmin, closest, &t, &ax)) {
          closest = t;
          h = WHit{ob.w, ax, t, i};
        }
        break;
      }
      case OBJ_MESH: {
        int tri = -1;
        if (mesh_closest(S.mesh[ob.y], r, tmin, closest, tri, use_kd, err, w)) h = WHit{ob.w, tri, closest, i};
        break;
      }
      default: {
        int k = -1;
        if (group_hit<false>(S, S.grp[ob.y], r, tmin, closest, k, err, w)) h = WHit{ob.w + k, 0, closest, i};
        break;
      }
    }
  }
  return h;
}

// world.hit(ray, t_min, t_max).is_some()
__device__ __forceinline__ bool world_any(const DScene& S, const RayC& r, double tmin, double tmax, bool use_kd,
                                          int* err, Work* w) {
  for (int i = 0; i < S.n_obj; i++) {
    int4 ob = __ldg(S.obj + i);
    double t;
    switch (ob.x) {
      case OBJ_SPHERE:
        if (w) w->spheres++;
        if (sphere_t(S.sph + 5 * (size_t)ob.y, r, tmin, tmax, &t)) return true;
        break;
      case OBJ_PLANE:
        if (plane_t(S.pln + 12 * (size_t)ob.y, r, tmin, tmax, &t)) return true;
        break;
      case OBJ_CUBE: {
        int ax;
        if (cube_t(S.cub[ob.y], r, tmin, tmax, &t, &ax)) return true;
        break;
      }
      case OBJ_MESH:
        if (mesh_any(S.mesh[ob.y], r, tmin, tmax, use_kd, err, w)) return true;
        break;
      default: {
        double c = tmax;
        int k;
        if (group_hit<true>(S, S.grp[ob.y], r, tmin, c, k, err, w)) return true;
        break;
      }
    }
  }
  return false;
}

// ---------------------------------------------------------------------------
// Warp-packet any-hit (shadow rays).  All 32 lanes of a warp call these
// together, each with its own ray (or none: active = false).  The warp walks
// one BVH with one stack: every lane loads the same node (a broadcast load),
// tests its own ray against both child boxes, and the warp descends into a
// child when any still-searching lane's ray hits its box.  A lane tests a
// leaf's primitives only when its own ray hits the leaf's box, and stops
// searching at its first accepted primitive.  Every leaf the lane's own
// walk would test is tested (the packet visits a superset of its nodes and
// the boxes are conservative), and extra box tests never accept anything, so
// each lane's answer is that of world_any: the packet only changes how the
// work is shared out.  The stack and the control flow are warp-uniform.
// ---------------------------------------------------------------------------
//
// `stack` is the warp's RTB_STACK-entry traversal stack in shared memory:
// every lane writes the same value to the same entry and reads back only
// values it wrote itself, so it needs no synchronisation.
template <class Nodes, class Leaf>
__device__ __forceinline__ bool bvh_any_warp(const Nodes& src, double tmax, bool active, Leaf visit_leaf,
                                             volatile int* stack, int* err, Work* w) {
  const unsigned FULL = 0xffffffffu;
  bool found = false;
  if (!__any_sync(FULL, active)) return false;
  int sp = 0;
  int node = 0;
  // work counting only: whether this lane's own walk reaches the node (its
  // ray hit the node's box), one bit per stack entry, so that the counters
  // hold the single-ray work rather than the packet's shared visits
  bool mine = true;
  unsigned long long mine_bits = 0;
  const auto b = src.bound(tmax);
  for (;;) {
    const typename Nodes::Node n = src.load(node);
    if (w && active && mine) w->nodes++;
    typename Nodes::T tl = 0, tr = 0;
    bool hl = active && n.lcnt >= 0 && src.test(n.lmn, n.lmx, b, &tl);
    bool hr = active && n.rcnt >= 0 && src.test(n.rmn, n.rmx, b, &tr);
    if (w) {
      hl = hl && mine;
      hr = hr && mine;
    }
    // leaf children first: they may retire lanes
    if (n.lcnt > 0 && hl && visit_leaf(n.lidx, n.lcnt)) {
      found = true;
      active = false;
    }
    if (n.rcnt > 0 && hr && active && visit_leaf(n.ridx, n.rcnt)) {
      found = true;
      active = false;
    }
    const bool gl = __any_sync(FULL, n.lcnt == 0 && hl && active);
    const bool gr = __any_sync(FULL, n.rcnt == 0 && hr && active);
    int next = -1;
    if (gl && gr) {
      // nearer child first for most of the searching lanes
      const unsigned both = __ballot_sync(FULL, hl && hr && active);
      const unsigned rfirst = __ballot_sync(FULL, hl && hr && active && tr < tl);
      const bool right_first = __popc(rfirst) * 2 > __popc(both);
      if (sp >= RTB_STACK) {
        if ((threadIdx.x & 31) == 0) atomicOr(err, ERR_STACK);
        return found;
      }
      if (w) {
        const bool pushed_mine = right_first ? hl : hr;
        mine_bits = pushed_mine ? (mine_bits | (1ull << sp)) : (mine_bits & ~(1ull << sp));
        mine = right_first ? hr : hl;
      }
      stack[sp++] = right_first ? n.lidx : n.ridx;
      next = right_first ? n.ridx : n.lidx;
    } else if (gl) {
      next = n.lidx;
      if (w) mine = hl;
    } else if (gr) {
      next = n.ridx;
      if (w) mine = hr;
    }
    if (!__any_sync(FULL, active)) return found;
    if (next >= 0) {
      node = next;
      continue;
    }
    if (sp == 0) return found;
    node = stack[--sp];
    if (w) mine = (mine_bits >> sp) & 1ull;
  }
}

// mesh_any for a warp of shadow rays.
__device__ __forceinline__ bool mesh_any_warp(const DMesh& M, const RayC& r, double tmin, double tmax, bool active,
                                              bool use_kd, volatile int* stack, int* err, Work* w) {
  active = active && mesh_bounds(M, r, tmin, tmax);
  return bvh_any_warp(
      mesh_nodes(M, r), tmax, active,
      [&](int first, int cnt) {
        for (int k = 0; k < cnt; k++) {
          const double2* E = M.btris + 5 * (size_t)(first + k);
          double t;
          if (w) w->tris++;
          if (tri_t(E, r, tmin, tmax, &t)) {
            if (!use_kd) return true;
            if (tri_visited(M, r, lo32(__ldg(E + 4).y), w)) return true;
          }
        }
        return false;
      },
      stack, err, w);
}

// group_hit<true> (any sphere of the run accepts within t_max) for a warp.
__device__ __forceinline__ bool group_any_warp(const DScene& S, const DSphGroup& G, const RayC& r, double tmin,
                                               double tmax, bool active, volatile int* stack, int* err, Work* w) {
  return bvh_any_warp(
      group_nodes(G, r), tmax, active,
      [&](int first, int cnt) {
        for (int k = 0; k < cnt; k++) {
          int sidx = __ldg(G.order + first + k);
          double t;
          if (w) w->spheres++;
          if (sphere_t(S.sph + 5 * (size_t)(G.first_sphere + sidx), r, tmin, tmax, &t)) return true;
        }
        return false;
      },
      stack, err, w);
}

// world.hit(ray, t_min, t_max).is_some() for a warp of rays (all 32 lanes
// call it; lanes with valid == false take part without a ray).  Objects are
// visited in scene order; the answer does not depend on the order.
__device__ __forceinline__ bool world_any_warp(const DScene& S, const RayC& r, double tmin, double tmax, bool valid,
                                               bool use_kd, volatile int* stack, int* err, Work* w) {
  bool blocked = false;
  for (int i = 0; i < S.n_obj; i++) {
    int4 ob = __ldg(S.obj + i);
    const bool live = valid && !blocked;
    double t;
    switch (ob.x) {
      case OBJ_SPHERE:
        if (live) {
          if (w) w->spheres++;
          blocked = sphere_t(S.sph + 5 * (size_t)ob.y, r, tmin, tmax, &t);
        }
        break;
      case OBJ_PLANE:
        if (live) blocked = plane_t(S.pln + 12 * (size_t)ob.y, r, tmin, tmax, &t);
        break;
      case OBJ_CUBE:
        if (live) {
          int ax;
          blocked = cube_t(S.cub[ob.y], r, tmin, tmax, &t, &ax);
        }
        break;
      case OBJ_MESH:
        if (mesh_any_warp(S.mesh[ob.y], r, tmin, tmax, live, use_kd, stack, err, w)) blocked = true;
        break;
      default:
        if (group_any_warp(S, S.grp[ob.y], r, tmin, tmax, live, stack, err, w)) blocked = true;
        break;
    }
  }
  return blocked;
}

struct HitRec {
  V3 p, n;
  int mat;
  int has_uv;
  double u, v;
};

// HitRecord::new (src/ray.rs:39-64)
__device__ __forceinline__ V3 face_normal(V3 d, V3 outward) {
  bool front = dot(d, outward) < 0.0;
  return front ? normalize(outward) : normalize(-outward);
}

// Rebuilds the winning object's HitRecord from (entry, aux, t).
__device__ __forceinline__ HitRec finalize_hit(const DScene& S, const RayC& r, const WHit& w) {
  HitRec h;
  int4 ob = __ldg(S.obj + w.ent);
  h.mat = ob.z;
  h.has_uv = 0;
  h.u = h.v = 0.0;
  double t = w.t;
  switch (ob.x) {
    case OBJ_SPHERE:
    case OBJ_SPHERE_GROUP: {
      int si = ob.x == OBJ_SPHERE ? ob.y : S.grp[ob.y].first_sphere + (w.obj - ob.w);
      const double* s = S.sph + 5 * (size_t)si;
      if (ob.x == OBJ_SPHERE_GROUP) h.mat = S.sph_mat[si];
      V3 c = mk(s[0], s[1], s[2]);
      h.p = r.o + t * r.d;
      h.n = face_normal(r.d, (h.p - c) / s[3]);
      break;
    }
    case OBJ_PLANE: {
      const double* p = S.pln + 12 * (size_t)ob.y;
      V3 n = mk(p[3], p[4], p[5]);
      h.p = r.o + t * r.d;
      h.n = face_normal(r.d, n);
      V3 rel = h.p - mk(p[0], p[1], p[2]);
      h.has_uv = 1;
      h.u = dot(rel, mk(p[6], p[7], p[8]));
      h.v = dot(rel, mk(p[9], p[10], p[11]));
      break;
    }
    case OBJ_CUBE: {
      const DCube& C = S.cub[ob.y];
      V3 lo = gemv34(C.w2l, r.o - ld3(C.c), 0.0);
      V3 dn = normalize(gemv34(C.w2l, r.d, 0.0));
      V3 lhp = lo + t * dn;
      h.p = ld3(C.c) + gemv34(C.l2w, lhp, 1.0);
      V3 ln = mk(0.0, 0.0, 0.0);
      if (w.aux == 0) ln.x = -1.0;
      if (w.aux == 1) ln.y = -1.0;
      if (w.aux == 2) ln.z = -1.0;
      V3 wn = C.identity ? ln : gemv33(C.ntr, ln);
      h.n = face_normal(r.d, wn);
      break;
    }
    default: {
      const DMesh& M = S.mesh[ob.y];
      const double2* E = M.brute + 5 * (size_t)w.aux;
      double2 q0 = E[0], q1 = E[1], q2 = E[2], q3 = E[3], q4 = E[4];
      V3 v0 = mk(q0.x, q0.y, q1.x), e1 = mk(q1.y, q2.x, q2.y), e2 = mk(q3.x, q3.y, q4.x);
      V3 hh = cross(r.d, e2);
      double a = dot(e1, hh);
      double f = 1.0 / a;
      V3 s = r.o - v0;
      double u = f * dot(s, hh);
      V3 q = cross(s, e1);
      double v = f * dot(r.d, q);
      double4 nn = M.normals[w.aux];
      V3 n = mk(nn.x, nn.y, nn.z);
      if (a < 0.0) n = -n;
      h.p = r.o + t * r.d;
      h.n = face_normal(r.d, n);
      h.has_uv = 1;
      h.u = u;
      h.v = v;
      break;
    }
  }
  return h;
}

// Camera::get_grid_color (src/camera.rs:171-254)
__device__ __forceinline__ bool grid_color(const DCam& c, V3 o, V3 d, V3* out) {
  if (!c.grid) return false;
  double p = c.pitch, half = c.half_th;
#pragma unroll
  for (int plane = 0; plane < 3; plane++) {
    int ax = plane == 0 ? 2 : (plane == 1 ? 1 : 0);
    int a1 = plane == 2 ? 1 : 0;
    int a2 = plane == 0 ? 1 : 2;
    if (fabs(d[ax]) > 1e-10) {
      double t = -o[ax] / d[ax];
      if (t > 0.0) {
        V3 ip = o + t * d;
        double m1 = fabs(rfract(ip[a1] / p));
        double m2 = fabs(rfract(ip[a2] / p));
        double d1 = rmin(m1 * p, (1.0 - m1) * p);
        double d2 = rmin(m2 * p, (1.0 - m2) * p);
        if (d1 <= half || d2 <= half) {
          *out = ld3(c.gcolor);
          return true;
        }
      }
    }
  }
  return false;
}

}  // namespace rtb
