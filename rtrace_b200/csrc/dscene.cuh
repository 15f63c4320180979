// Device-resident scene layout and the intersection routines of the render
// path.  Each routine restates one reference function in the same IEEE
// operation order; see the comments for the reference lines.
#pragma once

#include "dmath.cuh"

namespace rtb {

#ifndef RTB_INF
#define RTB_INF __longlong_as_double(0x7ff0000000000000LL)
#endif

enum { OBJ_SPHERE = 0, OBJ_PLANE = 1, OBJ_CUBE = 2, OBJ_MESH = 3 };

// Device error flags (bitmask in DFrame::err)
enum { ERR_WATCHDOG = 1, ERR_EMPTY_RANGE = 2, ERR_STACK = 4, ERR_RANGE_OVERFLOW = 8 };

// k-d tree pruning margin.  A triangle whose Moller-Trumbore t is below the
// current closest t lies inside its leaf's bounds, so the leaf's slab entry
// cannot exceed that t by more than the rounding of the two computations;
// nodes are skipped only when their entry exceeds closest * (1 + REL) + ABS.
#define RTB_PRUNE_REL 1.000001
#define RTB_PRUNE_ABS 1e-9

struct DCube {
  double c[3], half[3];
  double w2l[12];  // rows 0..2 of the world-to-local matrix
  double l2w[12];  // rows 0..2 of the local-to-world matrix
  double ntr[9];   // inverse-transpose of w2l's rotation part
  int identity;
  int pad;
};

// One mesh.  Nodes: 4 double2 each = (bmin.x, bmin.y) (bmin.z, bmax.x)
// (bmax.y, bmax.z) (split, meta); meta = int2{a, b}: internal a = right
// child, b = axis; leaf a = first entry, b = -1 - count.  Entries (leaf
// order, duplicated like the reference's index lists): 5 double2 =
// v0, e1 = v1 - v0, e2 = v2 - v0, meta int2{triangle index, degenerate}.
struct DMesh {
  double bmin[3], bmax[3];
  const double2* nodes;
  const double2* entries;
  const double2* brute;    // same entry layout, original triangle order
  const double4* normals;  // normalize(e1 x e2) per triangle
  int n_nodes;
  int n_tris;
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
  int n_obj;
  int n_lights;
  const int4* obj;  // {kind, index in its kind array, material, 0}
  const double* sph;  // 5 per sphere: cx cy cz r r*r
  const double* pln;  // 12 per plane: p, n, u axis, v axis
  const DCube* cub;
  const DMesh* mesh;
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

// Per-ray constants shared by all object tests.
struct RayC {
  V3 o, d;
  double dd;       // d.d (sphere `a`)
  V3 inv;          // 1/d per axis
  int par;         // bit a: |d[a]| < 1e-9 (k-d slabs treat the axis as parallel)
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
// test; the normal is looked up afterwards for the winning entry.
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

// MeshObject::hit with KdTree::traverse (src/ray.rs:614-649,
// src/mesh.rs:399-465).  Leaves are visited in the reference's order; a
// subtree is skipped when its bounds fail the reference's slab test (its
// leaves would all fail it) or start beyond the current closest t (none of
// its triangles can win the strict `t < closest` test).  any = true stops
// at the first accepted triangle (shadow rays only ask is_some()).
template <bool ANY>
__device__ __forceinline__ bool mesh_trace(const DMesh& M, const RayC& r, double tmin, double& closest, int& best,
                                           bool use_kd, int* err) {
  if (!mesh_bounds(M, r, tmin, closest)) return false;
  bool found = false;
  if (!use_kd) {
    for (int i = 0; i < M.n_tris; i++) {
      double t;
      if (tri_t(M.brute + 5 * (size_t)i, r, tmin, closest, &t)) {
        if (t < closest) {
          closest = t;
          best = i;
          found = true;
          if (ANY) return true;
        }
      }
    }
    return found;
  }
  if (M.n_nodes == 0) return false;
  int stack[32];
  int sp = 0;
  int node = 0;
  for (;;) {
    const double2* N = M.nodes + 4 * (size_t)node;
    double te;
    bool visit = kd_slab(N, r, &te) && !(te > closest * RTB_PRUNE_REL + RTB_PRUNE_ABS);
    if (visit) {
      double2 n3 = __ldg(N + 3);
      int ma = lo32(n3.y), mb = hi32(n3.y);
      if (mb < 0) {
        int first = ma, cnt = -1 - mb;
        for (int k = 0; k < cnt; k++) {
          double t;
          const double2* E = M.entries + 5 * (size_t)(first + k);
          if (tri_t(E, r, tmin, closest, &t)) {
            if (t < closest) {
              closest = t;
              best = first + k;
              found = true;
              if (ANY) return true;
            }
          }
        }
      } else {
        int axis = mb;
        double split = n3.x;
        double op = r.o[axis];
        int near_c, far_c;
        if (op <= split) {
          near_c = node + 1;
          far_c = ma;
        } else {
          near_c = ma;
          far_c = node + 1;
        }
        if (r.par & (1 << axis)) {
          node = near_c;
          continue;
        }
        double ts = (split - op) / r.d[axis];
        if (ts >= 0.0) {
          if (sp >= 32) {
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

struct WHit {
  int obj;   // scene object index, -1 = miss
  int aux;   // mesh entry / cube axis
  double t;
};

// World::hit (src/ray.rs:699-711): scene order, closest narrowing
__device__ __forceinline__ WHit world_closest(const DScene& S, const RayC& r, double tmin, bool use_kd, int* err) {
  double closest = RTB_INF;
  WHit h{-1, 0, 0.0};
  for (int i = 0; i < S.n_obj; i++) {
    int4 ob = __ldg(S.obj + i);
    double t;
    switch (ob.x) {
      case OBJ_SPHERE:
        if (sphere_t(S.sph + 5 * ob.y, r, tmin, closest, &t)) {
          closest = t;
          h = WHit{i, 0, t};
        }
        break;
      case OBJ_PLANE:
        if (plane_t(S.pln + 12 * ob.y, r, tmin, closest, &t)) {
          closest = t;
          h = WHit{i, 0, t};
        }
        break;
      case OBJ_CUBE: {
        int ax;
        if (cube_t(S.cub[ob.y], r, tmin, closest, &t, &ax)) {
          closest = t;
          h = WHit{i, ax, t};
        }
        break;
      }
      default: {
        int best = -1;
        if (mesh_trace<false>(S.mesh[ob.y], r, tmin, closest, best, use_kd, err)) h = WHit{i, best, closest};
        break;
      }
    }
  }
  return h;
}

// world.hit(ray, t_min, t_max).is_some(): true iff some object hits with
// t_max fixed (the per-object tests are monotone in t_max), in any order.
__device__ __forceinline__ bool world_any(const DScene& S, const RayC& r, double tmin, double tmax, bool use_kd,
                                          int* err) {
  for (int i = 0; i < S.n_obj; i++) {
    int4 ob = __ldg(S.obj + i);
    double t;
    switch (ob.x) {
      case OBJ_SPHERE:
        if (sphere_t(S.sph + 5 * ob.y, r, tmin, tmax, &t)) return true;
        break;
      case OBJ_PLANE:
        if (plane_t(S.pln + 12 * ob.y, r, tmin, tmax, &t)) return true;
        break;
      case OBJ_CUBE: {
        int ax;
        if (cube_t(S.cub[ob.y], r, tmin, tmax, &t, &ax)) return true;
        break;
      }
      default: {
        double c = tmax;
        int best;
        if (mesh_trace<true>(S.mesh[ob.y], r, tmin, c, best, use_kd, err)) return true;
        break;
      }
    }
  }
  return false;
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

// Rebuilds the winning object's HitRecord from (object, aux, t).
__device__ __forceinline__ HitRec finalize_hit(const DScene& S, const RayC& r, const WHit& w, bool use_kd) {
  HitRec h;
  int4 ob = __ldg(S.obj + w.obj);
  h.mat = ob.z;
  h.has_uv = 0;
  h.u = h.v = 0.0;
  double t = w.t;
  switch (ob.x) {
    case OBJ_SPHERE: {
      const double* s = S.sph + 5 * ob.y;
      V3 c = mk(s[0], s[1], s[2]);
      h.p = r.o + t * r.d;
      h.n = face_normal(r.d, (h.p - c) / s[3]);
      break;
    }
    case OBJ_PLANE: {
      const double* p = S.pln + 12 * ob.y;
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
      const double2* E = (use_kd ? M.entries : M.brute) + 5 * (size_t)w.aux;
      double2 q0 = E[0], q1 = E[1], q2 = E[2], q3 = E[3], q4 = E[4];
      V3 v0 = mk(q0.x, q0.y, q1.x), e1 = mk(q1.y, q2.x, q2.y), e2 = mk(q3.x, q3.y, q4.x);
      int tri = lo32(q4.y);
      V3 hh = cross(r.d, e2);
      double a = dot(e1, hh);
      double f = 1.0 / a;
      V3 s = r.o - v0;
      double u = f * dot(s, hh);
      V3 q = cross(s, e1);
      double v = f * dot(r.d, q);
      double4 nn = M.normals[tri];
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
