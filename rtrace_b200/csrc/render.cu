// Wavefront render pipeline for SeaRyanC/rtrace scenes on B200 (sm_100a)
// and the C ABI of include/rtrace_gpu.h.
//
// One render = one pass per reflection depth over a compacted ray queue:
//   k_raygen      camera rays for the three anti-aliasing modes
//                 (src/renderer.rs:445-584, 752-897)
//   k_trace       closest hit per queued ray (World::hit, src/ray.rs:699)
//   k_shade       Phong + textures + point/area-light shadow rays + fog
//                 (src/lighting.rs:9-319); reflective hits append their
//                 reflection ray to the next queue (warp ballot + one
//                 atomic per warp)
//   k_fold        the reflection recursion's blend, deepest level first
//                 (src/lighting.rs:469-493)
//   k_resolve     quincunx / sample average per pixel, outline buffers,
//                 quantisation (src/renderer.rs:552, 702, 881-886, 899-912)
//   k_outline_*   edge mask, dilation and blend (src/outline.rs:86-278)
// All arithmetic is IEEE double in the reference's operation order
// (compile with -fmad=false).

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/rtrace_gpu.h"
#include "dscene.cuh"
#include "scene_loader.hpp"

namespace rtb {

// --------------------------------------------------------------------------
// Frame state passed by value to every kernel
// --------------------------------------------------------------------------
struct RayBuf {
  double *ox, *oy, *oz, *dx, *dy, *dz;
  uint64_t* seed;
};
struct LevelBuf {
  double *r, *g, *b, *refl;
  int* child;
};

#define RTB_MAX_LEVELS 64

struct DFrame {
  DScene S;
  DCam C;
  int W, H, S_per_px, aa, max_depth, use_kd, outline, camera_mode;
  uint64_t seed;
  long long n_primary;
  long long n_corner;  // quincunx corner rays, (W+1)(H+1)
  RayBuf q[2];
  int* hobj;
  int* haux;
  double* ht;
  LevelBuf* levels;  // device array [max_depth]
  int* counts;       // device [max_depth + 1]
  // per primary ray outline data
  double *pdepth, *pnx, *pny, *pnz;
  unsigned char* phit;
  // per pixel
  double *cr, *cg, *cb;
  double *dep, *nx, *ny, *nz;
  unsigned char* valid;
  double* mask;
  unsigned char* rgb;
  double* linear;  // optional pixel colours (3 per pixel) before quantisation
  unsigned long long* stats;  // [0] shadow rays
  int* err;
  // outline parameters
  double o_wd, o_wn, o_thr, o_color[3], o_thick;
  int o_use8, o_radius;
};

// --------------------------------------------------------------------------
// Camera rays
// --------------------------------------------------------------------------
// Camera::get_ray (src/camera.rs:155-167) followed by Ray::new's normalise
__device__ __forceinline__ void camera_ray(const DCam& c, double u, double v, V3* o, V3* d) {
  V3 vp = ld3(c.llc) + u * ld3(c.hor) + v * ld3(c.ver);
  if (c.persp) {
    V3 dir = normalize(vp - ld3(c.origin));
    *o = ld3(c.origin);
    *d = normalize(dir);
  } else {
    *o = vp;
    *d = normalize(ld3(c.vdir));
  }
}

__global__ void k_raygen(DFrame F) {
  const uint64_t GOLD = 0x9E3779B97F4A7C15ULL;
  long long n = F.n_primary;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double u, v;
    uint64_t seed;
    if (F.aa == RT_AA_QUINCUNX) {
      // render_quincunx (src/renderer.rs:752-897)
      double pw = 1.0 / (double)F.W, ph = 1.0 / (double)F.H;
      if (i < F.n_corner) {
        unsigned cx = (unsigned)(i % (F.W + 1)), cy = (unsigned)(i / (F.W + 1));
        u = rclamp((double)cx * pw, 0.0, 1.0);
        v = rclamp(1.0 - (double)cy * ph, 0.0, 1.0);
        seed = F.seed * GOLD + (uint64_t)cx + (uint64_t)cy * 0x85EBCA6BULL;
      } else {
        long long j = i - F.n_corner;
        unsigned x = (unsigned)(j % F.W), y = (unsigned)(j / F.W);
        u = ((double)x + 0.5) * pw;
        v = 1.0 - ((double)y + 0.5) * ph;
        seed = F.seed * GOLD + (uint64_t)x * 0x85EBCA6BULL + (uint64_t)y * 0xC2B2AE35ULL + 0x12345678ULL;
      }
    } else {
      // render_standard (src/renderer.rs:445-584)
      long long pix = i / F.S_per_px;
      unsigned s = (unsigned)(i % F.S_per_px);
      unsigned x = (unsigned)(pix % F.W), y = (unsigned)(pix / F.W);
      double wm1 = (double)(unsigned)(F.W - 1), hm1 = (double)(unsigned)(F.H - 1);
      double pu = (double)x / wm1;
      double pv = (double)(unsigned)(F.H - 1 - y) / hm1;
      double pwid = 1.0 / wm1, phei = 1.0 / hm1;
      uint64_t pseed = F.seed * GOLD + (uint64_t)x * 0x85EBCA6BULL + (uint64_t)y * 0xC2B2AE35ULL;
      seed = pseed + (uint64_t)s * 0x1F845FEDULL;
      if (F.aa == RT_AA_NO_JITTER) {
        u = pu;
        v = pv;
      } else {
        // The pixel's StdRng stream: sample s draws u64 number 2s and 2s+1
        // (samples == 1: numbers 0 and 1), i.e. words 4s..4s+3, which sit in
        // ChaCha block s / 4.
        uint32_t key[8], blk[16];
        pcg32_key(pseed, key);
        chacha_block(key, (uint64_t)(s >> 2), 6, blk);
        int w0 = 4 * (s & 3);
        uint64_t r0 = ((uint64_t)blk[w0 + 1] << 32) | blk[w0];
        uint64_t r1 = ((uint64_t)blk[w0 + 3] << 32) | blk[w0 + 2];
        const double scale = 1.0 / 9007199254740992.0;
        double f0 = scale * (double)(r0 >> 11), f1 = scale * (double)(r1 >> 11);
        if (F.S_per_px == 1) {
          double ju = f0 - 0.5, jv = f1 - 0.5;
          u = pu + ju * pwid;
          v = pv + jv * phei;
        } else {
          const double PI = 3.141592653589793;
          double ang = 2.0 * PI * (double)s / (double)F.S_per_px;
          double phase = f0 * 2.0 * PI;
          double ra = ang + phase;
          double rad = 0.5 * f1;
          double ju = rad * cos(ra), jv = rad * sin(ra);
          u = pu + ju * pwid;
          v = pv + jv * phei;
        }
      }
    }
    V3 o, d;
    camera_ray(F.C, u, v, &o, &d);
    RayBuf q = F.q[0];
    q.ox[i] = o.x;
    q.oy[i] = o.y;
    q.oz[i] = o.z;
    q.dx[i] = d.x;
    q.dy[i] = d.y;
    q.dz[i] = d.z;
    q.seed[i] = seed;
  }
}

// --------------------------------------------------------------------------
// Closest hit
// --------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_trace(DFrame F, int level) {
  int n = F.counts[level];
  RayBuf q = F.q[level & 1];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    V3 o = mk(q.ox[i], q.oy[i], q.oz[i]);
    V3 d = mk(q.dx[i], q.dy[i], q.dz[i]);
    RayC r = make_rayc(o, d);
    WHit h = world_closest(F.S, r, 0.001, F.use_kd != 0, F.err);
    F.hobj[i] = h.obj;
    F.haux[i] = h.aux;
    F.ht[i] = h.t;
  }
}

// --------------------------------------------------------------------------
// Shading
// --------------------------------------------------------------------------
struct SMat {
  V3 c;
  double ka, kd, ks, shin;
};

// apply_texture (src/lighting.rs:9-54) + the colour parse of phong_lighting
__device__ __forceinline__ SMat effective_material(const DMat& m, const HitRec& h) {
  SMat s;
  s.c = ld3(m.color);
  s.ka = m.ambient;
  s.kd = m.diffuse;
  s.ks = m.specular;
  s.shin = m.shininess;
  if (h.has_uv) {
    if (m.texture == 1) {
      double um = fabs(rfract(h.u / m.cell_size));
      double vm = fabs(rfract(h.v / m.cell_size));
      double hw = m.half_width;
      bool onu = um <= hw || um >= (1.0 - hw);
      bool onv = vm <= hw || vm >= (1.0 - hw);
      if (onu || onv) s.c = ld3(m.grid_color);
    } else if (m.texture == 2) {
      int32_t cu = sat_i32(floor(h.u)), cv = sat_i32(floor(h.v));
      int32_t sum = (int32_t)((uint32_t)cu + (uint32_t)cv);
      if (sum % 2 != 0) {
        s.c = ld3(m.cb_color);
        s.ka = m.cb_ambient;
        s.kd = m.cb_diffuse;
        s.ks = m.cb_specular;
        s.shin = m.cb_shininess;
      }
    }
  }
  return s;
}

// diffuse + specular of one light sample (src/lighting.rs:124-141, 191-208)
__device__ __forceinline__ V3 light_term(const SMat& m, const HitRec& h, V3 ldir, V3 lc, double li, V3 view) {
  double ds = rmax(dot(h.n, ldir), 0.0);
  V3 diffuse = m.kd * ds * li * cmul(lc, m.c);
  V3 spec = mk(0.0, 0.0, 0.0);
  if (ds > 0.0) {
    V3 rd = reflect(-ldir, h.n);
    double ss = pow(rmax(dot(view, rd), 0.0), m.shin);
    spec = m.ks * ss * li * lc;
  }
  return diffuse + spec;
}

__device__ __forceinline__ int warp_alloc(int* counter, bool want) {
  unsigned m = __ballot_sync(0xffffffffu, want);
  int lane = threadIdx.x & 31;
  int base = 0;
  if (m) {
    int leader = __ffs(m) - 1;
    if (lane == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
  }
  return want ? base + __popc(m & ((1u << lane) - 1u)) : -1;
}

__global__ void __launch_bounds__(128) k_shade(DFrame F, int level) {
  const DScene& S = F.S;
  int n = F.counts[level];
  RayBuf q = F.q[level & 1];
  RayBuf qn = F.q[(level + 1) & 1];
  LevelBuf L = F.levels[level];
  bool can_reflect = (F.max_depth - level) > 1;
  V3 campos = ld3(F.C.campos);
  int stride = gridDim.x * blockDim.x;
  // uniform trip count per warp so the ballot below sees every lane
  for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
    int i = base + threadIdx.x;
    bool active = i < n;
    bool emit = false;
    V3 ro, rd;
    V3 color = mk(0.0, 0.0, 0.0);
    double refl = 0.0;
    int hitp = 0;
    uint64_t seed = 0;
    if (active) {
      V3 o = mk(q.ox[i], q.oy[i], q.oz[i]);
      V3 d = mk(q.dx[i], q.dy[i], q.dz[i]);
      seed = q.seed[i];
      WHit w{F.hobj[i], F.haux[i], F.ht[i]};
      if (w.obj < 0) {
        // miss: grid background (camera = Some) or the background colour
        V3 g;
        if (F.camera_mode && grid_color(F.C, o, d, &g)) color = g;
        else color = ld3(S.bg);
        if (level == 0 && F.outline) F.phit[i] = 0;
      } else {
        hitp = 1;
        RayC r = make_rayc(o, d);
        HitRec h = finalize_hit(S, r, w, F.use_kd != 0);
        const DMat& mat = S.mat[h.mat];
        SMat m = effective_material(mat, h);
        // phong_lighting (src/lighting.rs:220-288)
        color = m.ka * S.amb_int * cmul(ld3(S.amb_color), m.c);
        V3 view = normalize(campos - h.p);
        V3 so = h.p + 0.001 * h.n;
        for (int li = 0; li < S.n_lights; li++) {
          const DLight& L0 = S.lights[li];
          V3 lp = ld3(L0.pos), lc = ld3(L0.color);
          V3 contrib;
          if (!L0.disk) {
            // calculate_point_light_contribution (src/lighting.rs:100-142)
            V3 ldir = normalize(lp - h.p);
            double dist = norm(lp - h.p);
            RayC sr = make_rayc(so, normalize(ldir));
            if (world_any(S, sr, 0.001, dist, F.use_kd != 0, F.err)) contrib = mk(0.0, 0.0, 0.0);
            else contrib = light_term(m, h, ldir, lc, L0.intensity, view);
          } else {
            // calculate_diffuse_light_contribution (src/lighting.rs:145-217)
            uint64_t ls = seed * 0x9E3779B97F4A7C15ULL + sat_u64(h.p.x * 1000.0) * 0x85EBCA6BULL +
                          sat_u64(h.p.y * 1000.0) * 0xC2B2AE35ULL + sat_u64(h.p.z * 1000.0) * 0x6C8E9CF5ULL;
            StdRng rng;
            rng.init(ls);
            double radius = L0.diameter / 2.0;
            V3 total = mk(0.0, 0.0, 0.0);
            unsigned visible = 0;
            // gen_range(-radius..radius) panics on an empty or infinite range
            bool ok = -radius < radius;
            if (!ok) atomicOr(F.err, ERR_EMPTY_RANGE);
            if (ok && !isfinite(radius - -radius)) {
              atomicOr(F.err, ERR_RANGE_OVERFLOW);
              ok = false;
            }
            // sample_disk_light_point's basis (src/lighting.rs:75-90)
            V3 cdir = normalize(lp - h.p);
            V3 up = fabs(cdir.x) < 0.9 ? mk(1.0, 0.0, 0.0) : mk(0.0, 1.0, 0.0);
            V3 bu = normalize(cross(up, cdir));
            V3 bv = normalize(cross(cdir, bu));
            for (int smp = 0; smp < 16 && ok; smp++) {
              double dx = 0.0, dy = 0.0;
              int it = 0;
              for (;; it++) {
                if (it >= 4096 || !rng.range(-radius, radius, &dx) || !rng.range(-radius, radius, &dy)) {
                  atomicOr(F.err, ERR_WATCHDOG);
                  ok = false;
                  break;
                }
                if (dx * dx + dy * dy <= radius * radius) break;
              }
              if (!ok) break;
              V3 sp = lp + dx * bu + dy * bv;
              V3 sdir = normalize(sp - h.p);
              double dist = norm(sp - h.p);
              RayC sr = make_rayc(so, normalize(sdir));
              if (world_any(S, sr, 0.001, dist, F.use_kd != 0, F.err)) continue;
              visible++;
              total = total + light_term(m, h, sdir, lc, L0.intensity, view);
            }
            contrib = (total / 16.0) * ((double)visible / 16.0);
          }
          color = color + contrib;
        }
        // apply_fog (src/lighting.rs:297-319)
        if (S.has_fog) {
          double dist = norm(h.p - campos);
          double f;
          if (dist <= S.fog_start) f = 0.0;
          else if (dist >= S.fog_end) f = 1.0;
          else f = (dist - S.fog_start) / (S.fog_end - S.fog_start);
          f = 1.0 - exp(-S.fog_density * f);
          f = rclamp(f, 0.0, 1.0);
          color = color * (1.0 - f) + ld3(S.fog_color) * f;
        }
        if (mat.has_refl && mat.refl > 0.0 && can_reflect) {
          emit = true;
          refl = mat.refl;
          V3 vd = normalize(campos - h.p);
          ro = h.p + 0.001 * h.n;
          rd = normalize(reflect(-vd, h.n));
        }
        if (level == 0 && F.outline) {
          F.phit[i] = 1;
          F.pdepth[i] = norm(h.p - campos);
          F.pnx[i] = h.n.x;
          F.pny[i] = h.n.y;
          F.pnz[i] = h.n.z;
        }
      }
    }
    unsigned long long hits = (unsigned long long)__popc(__ballot_sync(0xffffffffu, hitp != 0));
    if ((threadIdx.x & 31) == 0 && hits) atomicAdd(&F.stats[0], hits * (unsigned long long)S.shadow_per_hit);
    int slot = warp_alloc(&F.counts[level + 1], emit);
    if (active) {
      L.r[i] = color.x;
      L.g[i] = color.y;
      L.b[i] = color.z;
      L.refl[i] = refl;
      L.child[i] = slot;
      if (emit) {
        qn.ox[slot] = ro.x;
        qn.oy[slot] = ro.y;
        qn.oz[slot] = ro.z;
        qn.dx[slot] = rd.x;
        qn.dy[slot] = rd.y;
        qn.dz[slot] = rd.z;
        qn.seed[slot] = seed;
      }
    }
  }
}

// color * (1 - r) + reflected * r, deepest level first
__global__ void k_fold(DFrame F, int level) {
  int n = F.counts[level];
  LevelBuf L = F.levels[level];
  LevelBuf C = F.levels[level + 1];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int c = L.child[i];
    if (c < 0) continue;
    double r = L.refl[i];
    double k = 1.0 - r;
    L.r[i] = L.r[i] * k + C.r[c] * r;
    L.g[i] = L.g[i] * k + C.g[c] * r;
    L.b[i] = L.b[i] * k + C.b[c] * r;
  }
}

// --------------------------------------------------------------------------
// Per-pixel resolve, outline, quantise
// --------------------------------------------------------------------------
__device__ __forceinline__ void store_rgb(const DFrame& F, long long p, V3 c) {
  F.rgb[3 * p + 0] = sat_u8(rclamp(c.x, 0.0, 1.0) * 255.0);
  F.rgb[3 * p + 1] = sat_u8(rclamp(c.y, 0.0, 1.0) * 255.0);
  F.rgb[3 * p + 2] = sat_u8(rclamp(c.z, 0.0, 1.0) * 255.0);
  if (F.linear) {
    F.linear[3 * p + 0] = c.x;
    F.linear[3 * p + 1] = c.y;
    F.linear[3 * p + 2] = c.z;
  }
}

__global__ void k_resolve(DFrame F) {
  long long np = (long long)F.W * F.H;
  LevelBuf L = F.levels[0];
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < np; p += (long long)gridDim.x * blockDim.x) {
    V3 c;
    if (F.max_depth <= 0) {
      c = mk(0.0, 0.0, 0.0);
      if (F.aa == RT_AA_QUINCUNX) {
        c = (c + c + c + c + c) / 5.0;
      } else {
        V3 t = mk(0.0, 0.0, 0.0);
        for (int s = 0; s < F.S_per_px; s++) t = t + c;
        c = t / (double)F.S_per_px;
      }
      if (F.outline) F.valid[p] = 0;
    } else if (F.aa == RT_AA_QUINCUNX) {
      long long x = p % F.W, y = p / F.W;
      long long W1 = F.W + 1;
      long long ci = F.n_corner + p;
      long long k0 = y * W1 + x, k1 = y * W1 + x + 1, k2 = (y + 1) * W1 + x, k3 = (y + 1) * W1 + x + 1;
      V3 cc = mk(L.r[ci], L.g[ci], L.b[ci]);
      V3 c0 = mk(L.r[k0], L.g[k0], L.b[k0]);
      V3 c1 = mk(L.r[k1], L.g[k1], L.b[k1]);
      V3 c2 = mk(L.r[k2], L.g[k2], L.b[k2]);
      V3 c3 = mk(L.r[k3], L.g[k3], L.b[k3]);
      c = (cc + c0 + c1 + c2 + c3) / 5.0;
    } else {
      V3 t = mk(0.0, 0.0, 0.0);
      bool have = false;
      double pd = 0.0;
      V3 pn = mk(0.0, 0.0, 0.0);
      for (int s = 0; s < F.S_per_px; s++) {
        long long i = p * F.S_per_px + s;
        t = t + mk(L.r[i], L.g[i], L.b[i]);
        if (F.outline && F.phit[i]) {
          double d = F.pdepth[i];
          if (!have || d < pd) {
            have = true;
            pd = d;
            pn = mk(F.pnx[i], F.pny[i], F.pnz[i]);
          }
        }
      }
      c = t / (double)F.S_per_px;
      if (F.outline) {
        F.valid[p] = have ? 1 : 0;
        F.dep[p] = pd;
        F.nx[p] = pn.x;
        F.ny[p] = pn.y;
        F.nz[p] = pn.z;
      }
    }
    if (F.outline) {
      F.cr[p] = c.x;
      F.cg[p] = c.y;
      F.cb[p] = c.z;
    } else {
      store_rgb(F, p, c);
    }
  }
}

// detect_edges / compute_edge_strength (src/outline.rs:113-182): one tile of
// TX x TY pixels with a one-pixel halo staged in shared memory.
#define OT_X 32
#define OT_Y 8
__global__ void __launch_bounds__(OT_X* OT_Y) k_outline_mask(DFrame F) {
  __shared__ double sd[OT_Y + 2][OT_X + 2];
  __shared__ double snx[OT_Y + 2][OT_X + 2], sny[OT_Y + 2][OT_X + 2], snz[OT_Y + 2][OT_X + 2];
  __shared__ unsigned char sv[OT_Y + 2][OT_X + 2];
  int x0 = blockIdx.x * OT_X - 1, y0 = blockIdx.y * OT_Y - 1;
  for (int k = threadIdx.y * OT_X + threadIdx.x; k < (OT_X + 2) * (OT_Y + 2); k += OT_X * OT_Y) {
    int lx = k % (OT_X + 2), ly = k / (OT_X + 2);
    int gx = x0 + lx, gy = y0 + ly;
    unsigned char v = 0;
    double d = 0, a = 0, b = 0, c = 0;
    if (gx >= 0 && gy >= 0 && gx < F.W && gy < F.H) {
      long long p = (long long)gy * F.W + gx;
      v = F.valid[p];
      d = F.dep[p];
      a = F.nx[p];
      b = F.ny[p];
      c = F.nz[p];
    }
    sv[ly][lx] = v;
    sd[ly][lx] = d;
    snx[ly][lx] = a;
    sny[ly][lx] = b;
    snz[ly][lx] = c;
  }
  __syncthreads();
  int gx = blockIdx.x * OT_X + threadIdx.x, gy = blockIdx.y * OT_Y + threadIdx.y;
  if (gx >= F.W || gy >= F.H) return;
  int lx = threadIdx.x + 1, ly = threadIdx.y + 1;
  bool cf = sv[ly][lx] != 0;
  double cd = sd[ly][lx];
  V3 cn = mk(snx[ly][lx], sny[ly][lx], snz[ly][lx]);
  // neighbour lists of get_4_neighbors / get_8_neighbors (src/outline.rs:185-224)
  int ndx[8], ndy[8], nn = 0;
  if (F.o_use8) {
    for (int dy = -1; dy <= 1; dy++)
      for (int dx = -1; dx <= 1; dx++) {
        if (dx == 0 && dy == 0) continue;
        if (gx + dx >= 0 && gy + dy >= 0) {
          ndx[nn] = dx;
          ndy[nn] = dy;
          nn++;
        }
      }
  } else {
    if (gx > 0) { ndx[nn] = -1; ndy[nn] = 0; nn++; }
    ndx[nn] = 1; ndy[nn] = 0; nn++;
    if (gy > 0) { ndx[nn] = 0; ndy[nn] = -1; nn++; }
    ndx[nn] = 0; ndy[nn] = 1; nn++;
  }
  double maxe = 0.0;
  for (int k = 0; k < nn; k++) {
    int qx = gx + ndx[k], qy = gy + ndy[k];
    bool nf = false;
    double nd = 0.0;
    V3 nnv = mk(0, 0, 0);
    if (qx < F.W && qy < F.H) {  // get_depth / get_normal bounds (src/outline.rs:68-82)
      nf = sv[ly + ndy[k]][lx + ndx[k]] != 0;
      nd = sd[ly + ndy[k]][lx + ndx[k]];
      nnv = mk(snx[ly + ndy[k]][lx + ndx[k]], sny[ly + ndy[k]][lx + ndx[k]], snz[ly + ndy[k]][lx + ndx[k]]);
    }
    double e;
    if (cf && nf) {
      double dd = fabs(cd - nd);
      double ndd = dd / rmax(cd * 0.1, 0.1);
      double dp = rclamp(dot(cn, nnv), -1.0, 1.0);
      e = F.o_wd * ndd + F.o_wn * (1.0 - dp);
    } else if (cf != nf) {
      e = F.o_wd * 2.0 + F.o_wn * 2.0;
    } else {
      e = 0.0;
    }
    maxe = rmax(maxe, e);
  }
  double m = 0.0;
  if (maxe > F.o_thr) m = (maxe - F.o_thr) / rmax(1.0 - F.o_thr, 0.001);
  F.mask[(long long)gy * F.W + gx] = m;
}

// dilate_edges + blend_colors + quantise (src/outline.rs:227-278,
// src/renderer.rs:899-912); the mask tile with a halo of `radius` pixels is
// staged in dynamic shared memory.
__global__ void __launch_bounds__(OT_X* OT_Y) k_outline_apply(DFrame F) {
  extern __shared__ double sm[];
  int R = F.o_radius;
  int TW = OT_X + 2 * R, TH = OT_Y + 2 * R;
  int x0 = blockIdx.x * OT_X - R, y0 = blockIdx.y * OT_Y - R;
  for (int k = threadIdx.y * OT_X + threadIdx.x; k < TW * TH; k += OT_X * OT_Y) {
    int lx = k % TW, ly = k / TW;
    int gx = x0 + lx, gy = y0 + ly;
    double v = 0.0;
    if (gx >= 0 && gy >= 0 && gx < F.W && gy < F.H) v = F.mask[(long long)gy * F.W + gx];
    sm[k] = v;
  }
  __syncthreads();
  int gx = blockIdx.x * OT_X + threadIdx.x, gy = blockIdx.y * OT_Y + threadIdx.y;
  if (gx >= F.W || gy >= F.H) return;
  int lx = threadIdx.x + R, ly = threadIdx.y + R;
  double ms = sm[ly * TW + lx];
  if (R > 0) {
    double th = F.o_thick;
    for (int dy = -R; dy <= R; dy++)
      for (int dx = -R; dx <= R; dx++) {
        int nx = gx + dx, ny = gy + dy;
        if (nx >= 0 && ny >= 0 && nx < F.W && ny < F.H) {
          double dist = sqrt((double)(dx * dx + dy * dy));
          if (dist <= th) {
            double fo = 1.0 - (dist / th);
            ms = rmax(ms, sm[(ly + dy) * TW + (lx + dx)] * fo);
          }
        }
      }
  }
  long long p = (long long)gy * F.W + gx;
  V3 c = mk(F.cr[p], F.cg[p], F.cb[p]);
  if (ms > 0.0) {
    double w = rclamp(rmin(ms, 1.0), 0.0, 1.0);
    c = mk(c.x * (1.0 - w) + F.o_color[0] * w, c.y * (1.0 - w) + F.o_color[1] * w, c.z * (1.0 - w) + F.o_color[2] * w);
  }
  store_rgb(F, p, c);
}

// --------------------------------------------------------------------------
// Debug / unit kernels for the parity tests
// --------------------------------------------------------------------------
__global__ void k_debug_rng(const uint64_t* seeds, long long n, int nw, uint32_t* out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    StdRng r;
    r.init(seeds[i]);
    for (int k = 0; k < nw; k++) out[i * nw + k] = r.u32();
  }
}
__global__ void k_debug_disk(const uint64_t* seeds, long long n, double radius, double* out, int* err) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    StdRng r;
    r.init(seeds[i]);
    for (int s = 0; s < 16; s++) {
      double dx = 0, dy = 0;
      int it = 0;
      for (;; it++) {
        if (it >= 4096 || !r.range(-radius, radius, &dx) || !r.range(-radius, radius, &dy)) {
          atomicOr(err, ERR_WATCHDOG);
          break;
        }
        if (dx * dx + dy * dy <= radius * radius) break;
      }
      out[i * 32 + 2 * s] = dx;
      out[i * 32 + 2 * s + 1] = dy;
    }
  }
}
__global__ void k_debug_mesh(DMesh M, int use_kd, const double* rays, long long n, double tmin, double tmax,
                             double* out, int* err) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double* rr = rays + 6 * i;
    V3 o = mk(rr[0], rr[1], rr[2]);
    V3 d = normalize(mk(rr[3], rr[4], rr[5]));
    RayC r = make_rayc(o, d);
    double closest = tmax;
    int best = -1;
    double* oo = out + 8 * i;
    if (mesh_trace<false>(M, r, tmin, closest, best, use_kd != 0, err)) {
      const double2* E = (use_kd ? M.entries : M.brute) + 5 * (size_t)best;
      double2 q0 = E[0], q1 = E[1], q2 = E[2], q3 = E[3], q4 = E[4];
      V3 e1 = mk(q1.y, q2.x, q2.y), e2 = mk(q3.x, q3.y, q4.x);
      (void)q0;
      double a = dot(e1, cross(r.d, e2));
      double4 nn = M.normals[lo32(q4.y)];
      V3 nv = mk(nn.x, nn.y, nn.z);
      if (a < 0.0) nv = -nv;
      V3 p = r.o + closest * r.d;
      V3 fn = face_normal(r.d, nv);
      oo[0] = 1.0;
      oo[1] = closest;
      oo[2] = p.x; oo[3] = p.y; oo[4] = p.z;
      oo[5] = fn.x; oo[6] = fn.y; oo[7] = fn.z;
    } else {
      for (int k = 0; k < 8; k++) oo[k] = 0.0;
    }
  }
}

}  // namespace rtb

// ==========================================================================
// Host side: context, scene upload, render orchestration, C ABI
// ==========================================================================
using namespace rtb;

namespace {

std::mutex g_err_mu;
std::string g_global_err;

template <class T>
struct DevArray {
  T* p = nullptr;
  size_t n = 0;
};

}  // namespace

struct rt_scene {
  rt_ctx* ctx = nullptr;
  int device = 0;
  std::vector<void*> allocs;
  DScene S{};
  rt_camera_config camera{};
  rt_outline_config outline{};
  int has_outline = 0;
  std::string render_error;
  std::vector<DMesh> host_meshes;  // device pointers, for the debug entry point
  std::vector<int> obj_kind, obj_index;
  bool disk_light_bad = false;
};

struct rt_ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string err;
  // scratch
  long long cap_rays = 0;
  int cap_levels = 0;
  long long cap_pixels = 0;
  std::vector<void*> scratch;
  DFrame F{};
  LevelBuf* d_levels = nullptr;
  std::vector<LevelBuf> h_levels;
  int* d_counts = nullptr;
  unsigned long long* d_stats = nullptr;
  int* d_err = nullptr;
};

namespace {

rt_status fail(rt_ctx* ctx, rt_status s, const std::string& m) {
  if (ctx) ctx->err = m;
  else {
    std::lock_guard<std::mutex> g(g_err_mu);
    g_global_err = m;
  }
  return s;
}

rt_status cuda_fail(rt_ctx* ctx, cudaError_t e, const char* what) {
  rt_status s = (e == cudaErrorMemoryAllocation) ? RT_ERR_OUT_OF_MEMORY : RT_ERR_CUDA;
  return fail(ctx, s, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                        \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
  } while (0)

template <class T>
cudaError_t dalloc(std::vector<void*>& owner, T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e == cudaSuccess) owner.push_back(*p);
  return e;
}

void free_all(std::vector<void*>& v) {
  for (void* p : v) cudaFree(p);
  v.clear();
}

// Scratch sized for n_rays queue entries per level, `levels` levels and
// n_pix pixels; kept across renders and grown on demand.
rt_status ensure_scratch(rt_ctx* ctx, long long n_rays, int levels, long long n_pix) {
  if (n_rays <= ctx->cap_rays && levels <= ctx->cap_levels && n_pix <= ctx->cap_pixels) return RT_OK;
  free_all(ctx->scratch);
  long long R = std::max(n_rays, ctx->cap_rays);
  int Lv = std::max(levels, ctx->cap_levels);
  long long P = std::max(n_pix, ctx->cap_pixels);
  DFrame& F = ctx->F;
  auto& o = ctx->scratch;
  for (int k = 0; k < 2; k++) {
    CK(dalloc(o, &F.q[k].ox, R)); CK(dalloc(o, &F.q[k].oy, R)); CK(dalloc(o, &F.q[k].oz, R));
    CK(dalloc(o, &F.q[k].dx, R)); CK(dalloc(o, &F.q[k].dy, R)); CK(dalloc(o, &F.q[k].dz, R));
    CK(dalloc(o, &F.q[k].seed, R));
  }
  CK(dalloc(o, &F.hobj, R));
  CK(dalloc(o, &F.haux, R));
  CK(dalloc(o, &F.ht, R));
  ctx->h_levels.assign(Lv + 1, LevelBuf{});
  for (int l = 0; l < Lv; l++) {
    LevelBuf& L = ctx->h_levels[l];
    CK(dalloc(o, &L.r, R)); CK(dalloc(o, &L.g, R)); CK(dalloc(o, &L.b, R));
    CK(dalloc(o, &L.refl, R)); CK(dalloc(o, &L.child, R));
  }
  CK(dalloc(o, &ctx->d_levels, Lv + 1));
  CK(cudaMemcpy(ctx->d_levels, ctx->h_levels.data(), (Lv + 1) * sizeof(LevelBuf), cudaMemcpyHostToDevice));
  CK(dalloc(o, &ctx->d_counts, Lv + 2));
  CK(dalloc(o, &F.pdepth, R)); CK(dalloc(o, &F.pnx, R)); CK(dalloc(o, &F.pny, R)); CK(dalloc(o, &F.pnz, R));
  CK(dalloc(o, &F.phit, R));
  CK(dalloc(o, &F.cr, P)); CK(dalloc(o, &F.cg, P)); CK(dalloc(o, &F.cb, P));
  CK(dalloc(o, &F.dep, P)); CK(dalloc(o, &F.nx, P)); CK(dalloc(o, &F.ny, P)); CK(dalloc(o, &F.nz, P));
  CK(dalloc(o, &F.valid, P));
  CK(dalloc(o, &F.mask, P));
  CK(dalloc(o, &F.rgb, 3 * P));
  CK(dalloc(o, &ctx->d_stats, 8));
  CK(dalloc(o, &ctx->d_err, 1));
  ctx->cap_rays = R;
  ctx->cap_levels = Lv;
  ctx->cap_pixels = P;
  return RT_OK;
}

template <class T>
rt_status upload(rt_ctx* ctx, rt_scene* sc, const std::vector<T>& h, const T** out) {
  T* p = nullptr;
  CK(dalloc(sc->allocs, &p, h.size()));
  if (!h.empty()) CK(cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  *out = p;
  return RT_OK;
}

rt_status do_upload(rt_ctx* ctx, const rt_scene_desc* d, rt_scene** out) {
  if (!d) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null scene description");
  auto sc = std::make_unique<rt_scene>();
  sc->ctx = ctx;
  sc->device = ctx->device;
  sc->camera = d->camera;
  sc->outline = d->outline;
  sc->has_outline = d->has_outline;
  sc->render_error = d->render_error ? d->render_error : "";
  DScene& S = sc->S;
  std::vector<int4> obj;
  std::vector<double> sph, pln;
  std::vector<DCube> cub;
  std::vector<DMesh> meshes;
  for (int m = 0; m < d->n_meshes; m++) {
    const rt_mesh_desc& md = d->meshes[m];
    DMesh M{};
    for (int k = 0; k < 3; k++) { M.bmin[k] = md.bounds_min[k]; M.bmax[k] = md.bounds_max[k]; }
    long long nt = md.n_triangles;
    // per-triangle entries in original order + normals
    std::vector<double2> brute((size_t)nt * 5);
    std::vector<double4> normals((size_t)nt);
    for (long long t = 0; t < nt; t++) {
      const double* v = md.vertices + 9 * t;
      V3 v0 = mk(v[0], v[1], v[2]), v1 = mk(v[3], v[4], v[5]), v2 = mk(v[6], v[7], v[8]);
      V3 e1 = v1 - v0, e2 = v2 - v0;
      V3 n = cross(e1, e2);
      int degenerate = norm(n) < 1e-8 ? 1 : 0;
      V3 nn = normalize(n);
      normals[t] = double4{nn.x, nn.y, nn.z, 0.0};
      double2* E = &brute[5 * t];
      E[0] = double2{v0.x, v0.y};
      E[1] = double2{v0.z, e1.x};
      E[2] = double2{e1.y, e1.z};
      E[3] = double2{e2.x, e2.y};
      E[4] = double2{e2.z, pack2((int)t, degenerate)};
    }
    std::vector<double2> entries((size_t)md.n_tri_index * 5);
    for (long long k = 0; k < md.n_tri_index; k++) {
      int t = md.tri_index[k];
      if (t < 0 || t >= nt) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "k-d leaf index out of range");
      for (int j = 0; j < 5; j++) entries[5 * k + j] = brute[5 * (size_t)t + j];
    }
    std::vector<double2> nodes((size_t)md.n_nodes * 4);
    for (long long k = 0; k < md.n_nodes; k++) {
      const rt_kd_node_desc& nd = md.nodes[k];
      double2* N = &nodes[4 * k];
      N[0] = double2{nd.bounds_min[0], nd.bounds_min[1]};
      N[1] = double2{nd.bounds_min[2], nd.bounds_max[0]};
      N[2] = double2{nd.bounds_max[1], nd.bounds_max[2]};
      if (nd.axis < 0) {
        if (nd.first < 0 || nd.count < 0 || (long long)nd.first + nd.count > md.n_tri_index)
          return fail(ctx, RT_ERR_INVALID_ARGUMENT, "k-d leaf range out of bounds");
        N[3] = double2{0.0, pack2(nd.first, -1 - nd.count)};
      } else {
        if (nd.axis > 2 || nd.right <= k || nd.right >= md.n_nodes)
          return fail(ctx, RT_ERR_INVALID_ARGUMENT, "k-d node layout is not preorder");
        N[3] = double2{nd.split, pack2(nd.right, nd.axis)};
      }
    }
    rt_status st;
    const double2* p;
    if ((st = upload(ctx, sc.get(), nodes, &p)) != RT_OK) return st;
    M.nodes = p;
    if ((st = upload(ctx, sc.get(), entries, &p)) != RT_OK) return st;
    M.entries = p;
    if ((st = upload(ctx, sc.get(), brute, &p)) != RT_OK) return st;
    M.brute = p;
    const double4* pn;
    if ((st = upload(ctx, sc.get(), normals, &pn)) != RT_OK) return st;
    M.normals = pn;
    M.n_nodes = (int)md.n_nodes;
    M.n_tris = (int)nt;
    meshes.push_back(M);
  }
  for (int i = 0; i < d->n_objects; i++) {
    const rt_object_desc& o = d->objects[i];
    if (o.material < 0 || o.material >= d->n_materials) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "material index out of range");
    int4 e{o.kind, 0, o.material, 0};
    if (o.kind == RT_OBJ_SPHERE) {
      e.y = (int)(sph.size() / 5);
      sph.insert(sph.end(), {o.a[0], o.a[1], o.a[2], o.radius, o.radius * o.radius});
    } else if (o.kind == RT_OBJ_PLANE) {
      e.y = (int)(pln.size() / 12);
      V3 n = mk(o.b[0], o.b[1], o.b[2]);
      V3 ua = fabs(n.x) > 0.9 ? mk(0, 1, 0) : mk(1, 0, 0);
      V3 uax = normalize(cross(ua, n));
      V3 vax = normalize(cross(n, uax));
      pln.insert(pln.end(), {o.a[0], o.a[1], o.a[2], n.x, n.y, n.z, uax.x, uax.y, uax.z, vax.x, vax.y, vax.z});
    } else if (o.kind == RT_OBJ_CUBE) {
      e.y = (int)cub.size();
      DCube C{};
      for (int k = 0; k < 3; k++) { C.c[k] = o.a[k]; C.half[k] = o.b[k] / 2.0; }
      double tm[16], inv[16];
      for (int k = 0; k < 16; k++) tm[k] = o.has_transform ? o.transform[k] : ((k % 5) == 0 ? 1.0 : 0.0);
      // Cube::new_with_transform (src/ray.rs:208-225): w2l = inverse (or identity)
      {
        // nalgebra 4x4 cofactor inverse on the column-major slice
        double m[16], iv[16];
        for (int k = 0; k < 16; k++) m[k] = tm[(k % 4) * 4 + k / 4];
        iv[0] = m[5] * m[10] * m[15] - m[5] * m[11] * m[14] - m[9] * m[6] * m[15] + m[9] * m[7] * m[14] + m[13] * m[6] * m[11] - m[13] * m[7] * m[10];
        iv[4] = -m[4] * m[10] * m[15] + m[4] * m[11] * m[14] + m[8] * m[6] * m[15] - m[8] * m[7] * m[14] - m[12] * m[6] * m[11] + m[12] * m[7] * m[10];
        iv[8] = m[4] * m[9] * m[15] - m[4] * m[11] * m[13] - m[8] * m[5] * m[15] + m[8] * m[7] * m[13] + m[12] * m[5] * m[11] - m[12] * m[7] * m[9];
        iv[12] = -m[4] * m[9] * m[14] + m[4] * m[10] * m[13] + m[8] * m[5] * m[14] - m[8] * m[6] * m[13] - m[12] * m[5] * m[10] + m[12] * m[6] * m[9];
        double det = m[0] * iv[0] + m[1] * iv[4] + m[2] * iv[8] + m[3] * iv[12];
        bool ok = o.has_transform && det != 0.0;
        if (ok) {
          iv[1] = -m[1] * m[10] * m[15] + m[1] * m[11] * m[14] + m[9] * m[2] * m[15] - m[9] * m[3] * m[14] - m[13] * m[2] * m[11] + m[13] * m[3] * m[10];
          iv[5] = m[0] * m[10] * m[15] - m[0] * m[11] * m[14] - m[8] * m[2] * m[15] + m[8] * m[3] * m[14] + m[12] * m[2] * m[11] - m[12] * m[3] * m[10];
          iv[9] = -m[0] * m[9] * m[15] + m[0] * m[11] * m[13] + m[8] * m[1] * m[15] - m[8] * m[3] * m[13] - m[12] * m[1] * m[11] + m[12] * m[3] * m[9];
          iv[13] = m[0] * m[9] * m[14] - m[0] * m[10] * m[13] - m[8] * m[1] * m[14] + m[8] * m[2] * m[13] + m[12] * m[1] * m[10] - m[12] * m[2] * m[9];
          iv[2] = m[1] * m[6] * m[15] - m[1] * m[7] * m[14] - m[5] * m[2] * m[15] + m[5] * m[3] * m[14] + m[13] * m[2] * m[7] - m[13] * m[3] * m[6];
          iv[6] = -m[0] * m[6] * m[15] + m[0] * m[7] * m[14] + m[4] * m[2] * m[15] - m[4] * m[3] * m[14] - m[12] * m[2] * m[7] + m[12] * m[3] * m[6];
          iv[10] = m[0] * m[5] * m[15] - m[0] * m[7] * m[13] - m[4] * m[1] * m[15] + m[4] * m[3] * m[13] + m[12] * m[1] * m[7] - m[12] * m[3] * m[5];
          iv[14] = -m[0] * m[5] * m[14] + m[0] * m[6] * m[13] + m[4] * m[1] * m[14] - m[4] * m[2] * m[13] - m[12] * m[1] * m[6] + m[12] * m[2] * m[5];
          iv[3] = -m[1] * m[6] * m[11] + m[1] * m[7] * m[10] + m[5] * m[2] * m[11] - m[5] * m[3] * m[10] - m[9] * m[2] * m[7] + m[9] * m[3] * m[6];
          iv[7] = m[0] * m[6] * m[11] - m[0] * m[7] * m[10] - m[4] * m[2] * m[11] + m[4] * m[3] * m[10] + m[8] * m[2] * m[7] - m[8] * m[3] * m[6];
          iv[11] = -m[0] * m[5] * m[11] + m[0] * m[7] * m[9] + m[4] * m[1] * m[11] - m[4] * m[3] * m[9] - m[8] * m[1] * m[7] + m[8] * m[3] * m[5];
          iv[15] = m[0] * m[5] * m[10] - m[0] * m[6] * m[9] - m[4] * m[1] * m[10] + m[4] * m[2] * m[9] + m[8] * m[1] * m[6] - m[8] * m[2] * m[5];
          double id = 1.0 / det;
          for (int k = 0; k < 16; k++) inv[(k % 4) * 4 + k / 4] = iv[k] * id;
        } else {
          for (int k = 0; k < 16; k++) inv[k] = (k % 5) == 0 ? 1.0 : 0.0;
        }
      }
      for (int k = 0; k < 12; k++) { C.w2l[k] = inv[k]; C.l2w[k] = tm[k]; }
      bool ident = true;
      for (int k = 0; k < 16; k++)
        if (inv[k] != ((k % 5) == 0 ? 1.0 : 0.0)) ident = false;
      C.identity = ident ? 1 : 0;
      // normal transform: nalgebra 3x3 inverse of w2l's rotation part, transposed
      double a[3][3];
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) a[r][c] = inv[4 * r + c];
      double m11 = a[1][1] * a[2][2] - a[2][1] * a[1][2];
      double m12 = a[1][0] * a[2][2] - a[2][0] * a[1][2];
      double m13 = a[1][0] * a[2][1] - a[2][0] * a[1][1];
      double det = a[0][0] * m11 - a[0][1] * m12 + a[0][2] * m13;
      double ri[3][3];
      if (det != 0.0) {
        double m21 = a[0][1] * a[2][2] - a[2][1] * a[0][2];
        double m22 = a[0][0] * a[2][2] - a[2][0] * a[0][2];
        double m23 = a[0][0] * a[2][1] - a[2][0] * a[0][1];
        double m31 = a[0][1] * a[1][2] - a[1][1] * a[0][2];
        double m32 = a[0][0] * a[1][2] - a[1][0] * a[0][2];
        double m33 = a[0][0] * a[1][1] - a[1][0] * a[0][1];
        ri[0][0] = m11 / det; ri[1][0] = -m12 / det; ri[2][0] = m13 / det;
        ri[0][1] = -m21 / det; ri[1][1] = m22 / det; ri[2][1] = -m23 / det;
        ri[0][2] = m31 / det; ri[1][2] = -m32 / det; ri[2][2] = m33 / det;
      } else {
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 3; c++) ri[r][c] = r == c ? 1.0 : 0.0;
      }
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) C.ntr[3 * r + c] = ri[c][r];
      cub.push_back(C);
    } else if (o.kind == RT_OBJ_MESH) {
      if (o.mesh < 0 || o.mesh >= d->n_meshes) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "mesh index out of range");
      e.y = o.mesh;
    } else {
      return fail(ctx, RT_ERR_INVALID_ARGUMENT, "unknown object kind");
    }
    obj.push_back(e);
    sc->obj_kind.push_back(o.kind);
    sc->obj_index.push_back(e.y);
  }
  std::vector<DMat> mats(d->n_materials);
  for (int i = 0; i < d->n_materials; i++) {
    const rt_material_desc& m = d->materials[i];
    DMat& M = mats[i];
    M = DMat{};
    for (int k = 0; k < 3; k++) M.color[k] = m.color[k];
    M.ambient = m.ambient; M.diffuse = m.diffuse; M.specular = m.specular; M.shininess = m.shininess;
    M.refl = m.reflectivity; M.has_refl = m.has_reflectivity; M.texture = m.texture;
    // the grid colour is formatted as #RRGGBB from (c * 255) as u8 and parsed
    // back (src/lighting.rs:28-36)
    for (int k = 0; k < 3; k++) M.grid_color[k] = (double)sat_u8(m.grid_line_color[k] * 255.0) / 255.0;
    M.half_width = m.grid_line_width / 2.0;
    M.cell_size = m.grid_cell_size;
    for (int k = 0; k < 3; k++) M.cb_color[k] = m.checker_color[k];
    M.cb_ambient = m.checker_ambient; M.cb_diffuse = m.checker_diffuse;
    M.cb_specular = m.checker_specular; M.cb_shininess = m.checker_shininess;
  }
  std::vector<DLight> lights(d->n_lights);
  int K = 0;
  for (int i = 0; i < d->n_lights; i++) {
    const rt_light_desc& l = d->lights[i];
    DLight& L = lights[i];
    L = DLight{};
    for (int k = 0; k < 3; k++) { L.pos[k] = l.position[k]; L.color[k] = l.color[k]; }
    L.intensity = l.intensity;
    L.disk = l.has_diameter ? 1 : 0;
    L.diameter = l.diameter;
    K += L.disk ? 16 : 1;
  }
  rt_status st;
  const int4* po;
  if ((st = upload(ctx, sc.get(), obj, &po)) != RT_OK) return st;
  S.obj = po;
  const double* pd;
  if ((st = upload(ctx, sc.get(), sph, &pd)) != RT_OK) return st;
  S.sph = pd;
  if ((st = upload(ctx, sc.get(), pln, &pd)) != RT_OK) return st;
  S.pln = pd;
  const DCube* pc;
  if ((st = upload(ctx, sc.get(), cub, &pc)) != RT_OK) return st;
  S.cub = pc;
  const DMesh* pm;
  if ((st = upload(ctx, sc.get(), meshes, &pm)) != RT_OK) return st;
  S.mesh = pm;
  const DMat* pmt;
  if ((st = upload(ctx, sc.get(), mats, &pmt)) != RT_OK) return st;
  S.mat = pmt;
  const DLight* pl;
  if ((st = upload(ctx, sc.get(), lights, &pl)) != RT_OK) return st;
  S.lights = pl;
  S.n_obj = (int)obj.size();
  S.n_lights = d->n_lights;
  for (int k = 0; k < 3; k++) {
    S.amb_color[k] = d->ambient_color[k];
    S.fog_color[k] = d->fog_color[k];
    S.bg[k] = d->background[k];
  }
  S.amb_int = d->ambient_intensity;
  S.has_fog = d->has_fog;
  S.fog_density = d->fog_density;
  S.fog_start = d->fog_start;
  S.fog_end = d->fog_end;
  S.shadow_per_hit = K;
  sc->host_meshes = meshes;
  *out = sc.release();
  return RT_OK;
}

rt_status render_impl(rt_ctx* ctx, const rt_scene* sc, const rt_render_params* P, uint8_t* rgb_out, int on_device,
                      double* linear_out, rt_stats* stats) {
  auto t0 = std::chrono::steady_clock::now();
  if (!ctx || !sc || !P) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  if (!rgb_out && !linear_out) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "no output buffer");
  if (P->anti_aliasing_mode < 0 || P->anti_aliasing_mode > 2)
    return fail(ctx, RT_ERR_INVALID_ARGUMENT, "unknown anti-aliasing mode");
  // Renderer::render (src/renderer.rs:120-317) error order
  if (P->samples == 0) return fail(ctx, RT_ERR_RENDER, "Samples must be greater than 0");
  if (P->width == 0 || P->height == 0) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "image size must be non-zero");
  CameraBasis cam;
  std::string cerr;
  double aspect = (double)P->width / (double)P->height;
  if (!make_camera(sc->camera, aspect, &cam, &cerr)) return fail(ctx, RT_ERR_RENDER, cerr);
  if (!sc->render_error.empty()) return fail(ctx, RT_ERR_RENDER, sc->render_error);
  CK(cudaSetDevice(ctx->device));

  const int W = (int)P->width, H = (int)P->height;
  const int aa = P->anti_aliasing_mode;
  const int spp = aa == RT_AA_QUINCUNX ? 1 : (int)P->samples;
  long long npix = (long long)W * H;
  long long ncorner = aa == RT_AA_QUINCUNX ? (long long)(W + 1) * (H + 1) : 0;
  long long nprim = aa == RT_AA_QUINCUNX ? ncorner + npix : npix * spp;
  if (nprim > 0x7fffffffLL) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "too many rays for one render");
  int max_depth = P->max_depth;
  int levels = std::max(1, std::min(max_depth, RTB_MAX_LEVELS));
  if (max_depth > RTB_MAX_LEVELS) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "max_depth above 64 is not supported");
  rt_status st = ensure_scratch(ctx, nprim, levels, npix);
  if (st != RT_OK) return st;

  DFrame F = ctx->F;
  F.S = sc->S;
  for (int k = 0; k < 3; k++) {
    F.C.origin[k] = cam.origin[k];
    F.C.hor[k] = cam.horizontal[k];
    F.C.ver[k] = cam.vertical[k];
    F.C.llc[k] = cam.llc[k];
    F.C.vdir[k] = cam.view_dir[k];
    F.C.campos[k] = sc->camera.position[k];
    F.C.gcolor[k] = cam.grid_color[k];
  }
  F.C.persp = cam.persp;
  F.C.grid = cam.grid_enabled;
  F.C.pitch = cam.grid_pitch;
  F.C.half_th = cam.grid_half_thickness;
  F.W = W;
  F.H = H;
  F.S_per_px = spp;
  F.aa = aa;
  F.max_depth = max_depth;
  F.use_kd = P->use_kdtree ? 1 : 0;
  F.camera_mode = aa == RT_AA_QUINCUNX ? 0 : 1;  // quincunx passes camera = None
  F.outline = (aa != RT_AA_QUINCUNX && P->outline.enabled) ? 1 : 0;
  F.seed = P->seed;
  F.n_primary = nprim;
  F.n_corner = ncorner;
  F.levels = ctx->d_levels;
  F.counts = ctx->d_counts;
  F.stats = ctx->d_stats;
  F.err = ctx->d_err;
  F.linear = nullptr;
  F.o_wd = P->outline.depth_weight;
  F.o_wn = P->outline.normal_weight;
  F.o_thr = P->outline.threshold;
  for (int k = 0; k < 3; k++) F.o_color[k] = P->outline.edge_color[k];
  F.o_thick = P->outline.line_thickness;
  F.o_use8 = P->outline.use_8_neighbors ? 1 : 0;
  F.o_radius = 0;
  if (F.outline && P->outline.line_thickness > 1.0) {
    double rr = std::ceil(P->outline.line_thickness - 1.0);
    F.o_radius = rr > 64.0 ? 64 : (int)rr;
    if (rr > 64.0) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "outline thickness above 65 is not supported");
  }
  double* d_linear = nullptr;
  std::vector<void*> tmp;
  if (linear_out) {
    cudaError_t e = dalloc(tmp, &d_linear, 3 * npix);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc(linear)");
    F.linear = d_linear;
  }
  uint8_t* d_rgb = F.rgb;
  if (rgb_out && on_device) F.rgb = rgb_out;

  cudaStream_t s = ctx->stream;
  int nsm = ctx->num_sms;
  auto blocks = [&](long long n, int bs, int per_sm) {
    long long b = (n + bs - 1) / bs;
    long long cap = (long long)nsm * per_sm;
    return (int)std::max<long long>(1, std::min(b, cap));
  };
  CK(cudaMemsetAsync(ctx->d_counts, 0, (levels + 2) * sizeof(int), s));
  int n0 = (int)nprim;
  CK(cudaMemcpyAsync(ctx->d_counts, &n0, sizeof(int), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(ctx->d_stats, 0, 8 * sizeof(unsigned long long), s));
  CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), s));
  CK(cudaEventRecord(ctx->ev0, s));
  if (max_depth > 0) {
    k_raygen<<<blocks(nprim, 256, 16), 256, 0, s>>>(F);
    for (int l = 0; l < levels; l++) {
      k_trace<<<blocks(nprim, 128, 16), 128, 0, s>>>(F, l);
      k_shade<<<blocks(nprim, 128, 16), 128, 0, s>>>(F, l);
    }
    for (int l = levels - 2; l >= 0; l--) k_fold<<<blocks(nprim, 256, 16), 256, 0, s>>>(F, l);
  }
  k_resolve<<<blocks(npix, 256, 16), 256, 0, s>>>(F);
  if (F.outline) {
    dim3 ob(OT_X, OT_Y), og((W + OT_X - 1) / OT_X, (H + OT_Y - 1) / OT_Y);
    k_outline_mask<<<og, ob, 0, s>>>(F);
    size_t shm = (size_t)(OT_X + 2 * F.o_radius) * (OT_Y + 2 * F.o_radius) * sizeof(double);
    if (shm > 48 * 1024) CK(cudaFuncSetAttribute(k_outline_apply, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
    k_outline_apply<<<og, ob, shm, s>>>(F);
  }
  CK(cudaGetLastError());
  CK(cudaEventRecord(ctx->ev1, s));
  if (rgb_out && !on_device) CK(cudaMemcpyAsync(rgb_out, d_rgb, 3 * npix, cudaMemcpyDeviceToHost, s));
  if (linear_out) CK(cudaMemcpyAsync(linear_out, d_linear, 3 * npix * sizeof(double), cudaMemcpyDeviceToHost, s));
  std::vector<int> counts(levels + 2, 0);
  unsigned long long hstats[8];
  int herr = 0;
  CK(cudaMemcpyAsync(counts.data(), ctx->d_counts, (levels + 2) * sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(hstats, ctx->d_stats, sizeof hstats, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&herr, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  cudaError_t se = cudaStreamSynchronize(s);
  free_all(tmp);
  if (se != cudaSuccess) return cuda_fail(ctx, se, "render");
  if (herr & ERR_EMPTY_RANGE) return fail(ctx, RT_ERR_RENDER, "cannot sample empty range");
  if (herr & ERR_RANGE_OVERFLOW) return fail(ctx, RT_ERR_RENDER, "UniformSampler::sample_single: range overflow");
  if (herr & (ERR_WATCHDOG | ERR_STACK))
    return fail(ctx, RT_ERR_DEVICE_WATCHDOG, herr & ERR_STACK ? "k-d traversal stack exhausted" : "rejection sampling did not terminate");
  if (stats) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    memset(stats, 0, sizeof *stats);
    if (max_depth > 0) {
      stats->primary_rays = (uint64_t)counts[0];
      uint64_t refl = 0;
      for (int l = 1; l < levels; l++) refl += (uint64_t)counts[l];
      stats->reflection_rays = refl;
      stats->shadow_rays = hstats[0];
    }
    stats->device_ms = ms;
    stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  ctx->err.clear();
  return RT_OK;
}

}  // namespace

// ==========================================================================
// C ABI
// ==========================================================================
extern "C" {

rt_status rt_ctx_create(int device, rt_ctx** out) {
  if (!out) return fail(nullptr, RT_ERR_INVALID_ARGUMENT, "null output pointer");
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    return fail(nullptr, RT_ERR_CUDA, std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "count is 0"));
  if (device < 0 || device >= n) return fail(nullptr, RT_ERR_INVALID_ARGUMENT, "device index out of range");
  auto c = std::make_unique<rt_ctx>();
  c->device = device;
  rt_ctx* ctx = nullptr;  // errors below are reported globally
  CK(cudaSetDevice(device));
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) return fail(nullptr, RT_ERR_CUDA, "device is not sm_100 class (B200 required)");
  c->num_sms = prop.multiProcessorCount;
  CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  CK(cudaEventCreate(&c->ev0));
  CK(cudaEventCreate(&c->ev1));
  *out = c.release();
  return RT_OK;
}

void rt_ctx_destroy(rt_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  free_all(ctx->scratch);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char* rt_last_error(const rt_ctx* ctx) {
  if (ctx) return ctx->err.c_str();
  std::lock_guard<std::mutex> g(g_err_mu);
  return g_global_err.c_str();
}

rt_status rt_scene_upload(rt_ctx* ctx, const rt_scene_desc* desc, rt_scene** out) {
  if (!ctx || !out) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  CK(cudaSetDevice(ctx->device));
  rt_status s = do_upload(ctx, desc, out);
  if (s == RT_OK) ctx->err.clear();
  return s;
}

rt_status rt_scene_load_json_str(rt_ctx* ctx, const char* json, rt_scene** out) {
  if (!ctx || !json || !out) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  HostScene hs;
  std::string err;
  if (!load_scene_json(json, ".", &hs, &err)) return fail(ctx, RT_ERR_SCENE, err);
  return rt_scene_upload(ctx, &hs.desc, out);
}

rt_status rt_scene_load_json_file(rt_ctx* ctx, const char* path, rt_scene** out) {
  if (!ctx || !path || !out) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  std::string text, err;
  if (!read_text_file(path, &text, &err)) return fail(ctx, RT_ERR_IO, err);
  HostScene hs;
  if (!load_scene_json(text, parent_dir(path), &hs, &err)) return fail(ctx, RT_ERR_SCENE, err);
  return rt_scene_upload(ctx, &hs.desc, out);
}

rt_status rt_scene_outline_config(rt_ctx* ctx, const rt_scene* scene, rt_outline_config* out) {
  if (!scene || !out) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  if (scene->has_outline == 2) return fail(ctx, RT_ERR_SCENE, "Invalid hex color");
  *out = scene->outline;
  out->enabled = scene->has_outline == 1 ? 1 : 0;
  return RT_OK;
}

rt_status rt_scene_camera_aspect(rt_ctx* ctx, const rt_scene* scene, double* out) {
  if (!scene || !out) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  *out = scene->camera.width / scene->camera.height;
  return RT_OK;
}

void rt_scene_free(rt_scene* scene) {
  if (!scene) return;
  cudaSetDevice(scene->device);
  free_all(scene->allocs);
  delete scene;
}

rt_status rt_render(rt_ctx* ctx, const rt_scene* scene, const rt_render_params* params, uint8_t* rgb_out,
                    int out_on_device, rt_stats* stats) {
  return render_impl(ctx, scene, params, rgb_out, out_on_device, nullptr, stats);
}

rt_status rt_render_linear(rt_ctx* ctx, const rt_scene* scene, const rt_render_params* params, uint8_t* rgb_out,
                           double* linear_out, rt_stats* stats) {
  return render_impl(ctx, scene, params, rgb_out, 0, linear_out, stats);
}

rt_status rt_debug_stdrng_u32(rt_ctx* ctx, const uint64_t* seeds, int64_t n, int32_t n_words, uint32_t* out) {
  if (!ctx || !seeds || !out || n < 0 || n_words < 0) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "bad argument");
  if (n == 0 || n_words == 0) return RT_OK;
  CK(cudaSetDevice(ctx->device));
  std::vector<void*> tmp;
  uint64_t* ds;
  uint32_t* dout;
  CK(dalloc(tmp, &ds, n));
  CK(dalloc(tmp, &dout, (size_t)n * n_words));
  CK(cudaMemcpy(ds, seeds, n * sizeof(uint64_t), cudaMemcpyHostToDevice));
  k_debug_rng<<<(int)std::min<int64_t>((n + 127) / 128, 4096), 128, 0, ctx->stream>>>(ds, n, n_words, dout);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaMemcpy(out, dout, (size_t)n * n_words * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  free_all(tmp);
  return RT_OK;
}

rt_status rt_debug_disk_offsets(rt_ctx* ctx, const uint64_t* light_seeds, int64_t n, double radius, double* out) {
  if (!ctx || !light_seeds || !out || n < 0) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "bad argument");
  if (!(-radius < radius)) return fail(ctx, RT_ERR_RENDER, "cannot sample empty range");
  if (n == 0) return RT_OK;
  CK(cudaSetDevice(ctx->device));
  std::vector<void*> tmp;
  uint64_t* ds;
  double* dout;
  int* derr;
  CK(dalloc(tmp, &ds, n));
  CK(dalloc(tmp, &dout, (size_t)n * 32));
  CK(dalloc(tmp, &derr, 1));
  CK(cudaMemset(derr, 0, sizeof(int)));
  CK(cudaMemcpy(ds, light_seeds, n * sizeof(uint64_t), cudaMemcpyHostToDevice));
  k_debug_disk<<<(int)std::min<int64_t>((n + 127) / 128, 4096), 128, 0, ctx->stream>>>(ds, n, radius, dout, derr);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  int herr = 0;
  CK(cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(out, dout, (size_t)n * 32 * sizeof(double), cudaMemcpyDeviceToHost));
  free_all(tmp);
  if (herr) return fail(ctx, RT_ERR_DEVICE_WATCHDOG, "rejection sampling did not terminate");
  return RT_OK;
}

rt_status rt_debug_mesh_hit(rt_ctx* ctx, const rt_scene* scene, int32_t object_index, int32_t use_kdtree,
                            const double* rays, int64_t n, double t_min, double t_max, double* out) {
  if (!ctx || !scene || !rays || !out || n < 0) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "bad argument");
  if (object_index < 0 || object_index >= (int)scene->obj_kind.size() || scene->obj_kind[object_index] != RT_OBJ_MESH)
    return fail(ctx, RT_ERR_INVALID_ARGUMENT, "object is not a mesh");
  if (n == 0) return RT_OK;
  CK(cudaSetDevice(ctx->device));
  DMesh M = scene->host_meshes[scene->obj_index[object_index]];
  std::vector<void*> tmp;
  double *dr, *dout;
  int* derr;
  CK(dalloc(tmp, &dr, (size_t)n * 6));
  CK(dalloc(tmp, &dout, (size_t)n * 8));
  CK(dalloc(tmp, &derr, 1));
  CK(cudaMemset(derr, 0, sizeof(int)));
  CK(cudaMemcpy(dr, rays, (size_t)n * 6 * sizeof(double), cudaMemcpyHostToDevice));
  k_debug_mesh<<<(int)std::min<int64_t>((n + 127) / 128, 4096), 128, 0, ctx->stream>>>(M, use_kdtree, dr, n, t_min, t_max,
                                                                                      dout, derr);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaMemcpy(out, dout, (size_t)n * 8 * sizeof(double), cudaMemcpyDeviceToHost));
  int herr = 0;
  CK(cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost));
  free_all(tmp);
  if (herr) return fail(ctx, RT_ERR_DEVICE_WATCHDOG, "k-d traversal stack exhausted");
  return RT_OK;
}

}  // extern "C"
