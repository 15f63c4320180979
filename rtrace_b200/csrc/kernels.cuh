// Wavefront kernels of one render.  Per reflection depth (queue level):
//   k_trace    closest hit per queued ray (World::hit, src/ray.rs:699);
//              misses get their background/grid colour here, hits are
//              compacted into the level's hit list (warp ballot + one atomic
//              per warp)
//   k_emit     per hit: light sampling (point lights: one ray; disk
//              lights: 16 ChaCha12-driven disk samples in the reference,
//              dsamp in general)
//   k_shadow   one any-hit query per shadow ray
//   k_resolve  per hit: ambient + visible contributions in the reference's
//              summation order, fog, and the reflection ray, appended to
//              the next level's queue (warp ballot + one atomic per warp)
// then, deepest level first, k_fold blends reflections into their parents
// (src/lighting.rs:469-493), and k_pixels/k_outline_* produce the image.
#pragma once

#include <cuda_fp16.h>

#include "denoise.hpp"
#include "dscene.cuh"

namespace rtb {

struct RayBuf {
  double *ox, *oy, *oz, *dx, *dy, *dz;
  uint64_t* seed;
};
struct LevelBuf {
  double *r, *g, *b, *refl;
  int* child;
};
// One shadow ray: unit direction to the light sample and its distance
// (-1: not traced), one 32-byte sector.
struct __align__(32) SRay {
  double dx, dy, dz, dist;
};
// Shadow rays of a chunk, sample-major: ray k of hit h (h relative to the
// chunk) lives at k * chunk_hits + h, so that k_emit and k_resolve (one
// thread per hit) write and read it coalesced; k_shadow's hit-major
// packets read each ray as one sector.  The visibility bytes are
// hit-major (h * K + k), so that a packet stores them contiguously.
struct ShadowBuf {
  SRay* ray;
  unsigned char* vis;
  double *ox, *oy, *oz;  // per hit: shadow-ray origin p + 0.001 n
};

#define RTB_MAX_LEVELS 64

struct DFrame {
  DScene S;
  DCam C;
  int W, H, S_per_px, aa, max_depth, use_kd, outline, camera_mode;
  // The frame buffers hold image rows [y0, y0 + H) of an image of height
  // Himg (a row band; y0 = 0 and H = Himg for a whole image).  Camera
  // coordinates and seeds use absolute rows.
  int y0, Himg;
  // Shadow rays per hit at the current level (point lights 1 each, disk
  // lights dsamp each) and the disk-light sample count; both are set per
  // level by the host.  The reference casts 16 per disk light.
  int K, dsamp;
  // Learned soft shadows (extension): at level 0 each disk light gets one
  // ray, and its visibility comes from the denoiser's vhat
  // ([plane][slot][H][W], plane = sample index within the pixel).
  int learned;
  int feat_on;          // write the feature image (and vis_aov) at level 0
  __half* feat;         // [plane][H][W][FEAT_CHANNELS]
  float* vhat;          // denoised visibility, read by k_resolve at level 0
  float* vis_aov;       // optional: per slot visible/dsamp of level-0 hits
  int n_slots;          // disk lights that are denoiser slots (<= DN_MAX_SLOTS)
  // Confidence-gated fallback (learned shadows): for a level-0 hit whose
  // estimated visibility error (vconf, layout of vhat) exceeds conf_thr on
  // some slot, those slots are shaded by the plain path.  k_fb_select lists
  // such hits in fb_list (count fbn[0]; fbn[1] counts their slots) and
  // keeps each hit's slot bits in fb_flag; launches with fb_mode set walk
  // fb_list instead of the level's hit list (fb_hit).  The list holds the
  // hits with one falling slot from the front (fbn[2] of them) and those
  // with more from the back (fbn[3], down from index n_primary - 1), so
  // that a warp's hits sample and shade the same number of lights.
  float* vconf;
  float conf_thr;
  int fb_mode;
  int* fb_list;
  int* fbn;
  unsigned char* fb_flag;
  uint64_t seed;
  long long n_primary;
  long long n_corner;  // quincunx corner rays, (W+1)(H+1)
  RayBuf q[2];
  int* hobj;  // per queued ray: World index of the hit, -1 miss
  int* haux;
  int* hent;
  double* ht;
  int* hit_ray;  // per hit slot: queued ray index
  LevelBuf* levels;  // device array [max_depth]
  int* counts;       // device: [0, L] queue sizes, [L+1 ..] hit counts per level
  int* nhits;        // device [max_depth]
  ShadowBuf sh;
  long long chunk_hits;  // hits whose shadow rays fit the shadow buffer at once
  // per primary ray outline data (pobj: World index of the hit object)
  double *pdepth, *pnx, *pny, *pnz;
  unsigned char* phit;
  int* pobj;
  // per pixel
  double *cr, *cg, *cb;
  double *dep, *nx, *ny, *nz;
  int* oid;  // per pixel: object of the nearest sample (outline object-ID term), or null
  unsigned char* valid;
  double* mask;
  unsigned char* rgb;
  double* linear;  // optional pixel colours (3 per pixel) before quantisation
  unsigned long long* stats;  // [2..5] trace work, [6..9] shadow work (nodes, tris, spheres, verify)
  int* err;
  double o_wd, o_wn, o_thr, o_color[3], o_thick, o_wid;
  int o_use8, o_radius;
};

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

__device__ __forceinline__ void warp_sum_add(unsigned long long* ctr, unsigned long long v) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(ctr, v);
}

// slot 0: trace counters (stats[2..5]), 1: shadow counters (stats[6..9])
__device__ __forceinline__ void flush_work(const DFrame& F, const Work& w, int slot) {
  unsigned long long* b = F.stats + 2 + 4 * slot;
  warp_sum_add(b + 0, w.nodes);
  warp_sum_add(b + 1, w.tris);
  warp_sum_add(b + 2, w.spheres);
  warp_sum_add(b + 3, w.verify);
}

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

// Several frames in one launch (batched small jobs): T holds the frames,
// and job j owns blocks [b0[j], b0[j + 1]) of the grid (b0[nj] = the grid
// size).  The job of this block, by binary search.
__device__ __forceinline__ int job_of_block(const int* __restrict__ b0, int nj) {
  int lo = 0, hi = nj - 1;
  const int b = (int)blockIdx.x;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (b0[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}
// queue levels of a frame: max_depth clamped to [1, RTB_MAX_LEVELS]
__device__ __forceinline__ int frame_levels(const DFrame& F) {
  return F.max_depth < 1 ? 1 : (F.max_depth > RTB_MAX_LEVELS ? RTB_MAX_LEVELS : F.max_depth);
}

// Start of a frame: queue sizes and hit counts to zero except the level-0
// queue, which holds the primary rays; work counters and the error word
// cleared.  One block of 128 threads (levels <= RTB_MAX_LEVELS).  A kernel
// rather than memsets and a host copy, so that the whole frame is device
// work a CUDA graph can hold.
__device__ __forceinline__ void frame_init_body(const DFrame& F, int levels) {
  for (int i = threadIdx.x; i < levels + 2; i += blockDim.x) F.counts[i] = i == 0 ? (int)F.n_primary : 0;
  for (int i = threadIdx.x; i < levels + 1; i += blockDim.x) F.nhits[i] = 0;
  if (threadIdx.x < 16) F.stats[threadIdx.x] = 0;
  if (threadIdx.x == 0) *F.err = 0;
  if (threadIdx.x < 4 && F.fbn) F.fbn[threadIdx.x] = 0;
}
__global__ void k_frame_init(const __grid_constant__ DFrame F, int levels) { frame_init_body(F, levels); }
// one block per frame
__global__ void k_frame_init_multi(const DFrame* __restrict__ T) {
  const DFrame& F = T[blockIdx.x];
  frame_init_body(F, frame_levels(F));
}

__device__ __forceinline__ void raygen_body(const DFrame& F, int bid, int nblk) {
  const uint64_t GOLD = 0x9E3779B97F4A7C15ULL;
  long long n = F.n_primary;
  for (long long i = bid * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)nblk * blockDim.x) {
    double u, v;
    uint64_t seed;
    if (F.aa == RT_AA_QUINCUNX) {
      // render_quincunx (src/renderer.rs:752-897)
      double pw = 1.0 / (double)F.W, ph = 1.0 / (double)F.Himg;
      if (i < F.n_corner) {
        unsigned cx = (unsigned)(i % (F.W + 1)), cy = (unsigned)(F.y0 + i / (F.W + 1));
        u = rclamp((double)cx * pw, 0.0, 1.0);
        v = rclamp(1.0 - (double)cy * ph, 0.0, 1.0);
        seed = F.seed * GOLD + (uint64_t)cx + (uint64_t)cy * 0x85EBCA6BULL;
      } else {
        long long j = i - F.n_corner;
        unsigned x = (unsigned)(j % F.W), y = (unsigned)(F.y0 + j / F.W);
        u = ((double)x + 0.5) * pw;
        v = 1.0 - ((double)y + 0.5) * ph;
        seed = F.seed * GOLD + (uint64_t)x * 0x85EBCA6BULL + (uint64_t)y * 0xC2B2AE35ULL + 0x12345678ULL;
      }
    } else {
      // render_standard (src/renderer.rs:445-584)
      long long pix = i / F.S_per_px;
      unsigned s = (unsigned)(i % F.S_per_px);
      unsigned x = (unsigned)(pix % F.W), y = (unsigned)(F.y0 + pix / F.W);
      double wm1 = (double)(unsigned)(F.W - 1), hm1 = (double)(unsigned)(F.Himg - 1);
      double pu = (double)x / wm1;
      double pv = (double)(unsigned)(F.Himg - 1 - y) / hm1;
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
__global__ void k_raygen(const __grid_constant__ DFrame F) {
  raygen_body(F, blockIdx.x, gridDim.x);
}
__global__ void k_raygen_multi(const DFrame* __restrict__ T, const int* __restrict__ b0, int nj) {
  const int j = job_of_block(b0, nj);
  const DFrame& F = T[j];
  raygen_body(F, blockIdx.x - b0[j], b0[j + 1] - b0[j]);
}


// --------------------------------------------------------------------------
// Closest hit + hit compaction; misses resolve to their background here.
// Six blocks of 128 per SM (80 registers): trace stage 0.71 ms against
// 0.75-0.78 ms unbounded (96 registers) on the bench frame.
// --------------------------------------------------------------------------
template <bool COUNT>
__device__ __forceinline__ void trace_body(const DFrame& F, int level, int bid, int nblk) {
  int n = F.counts[level];
  RayBuf q = F.q[level & 1];
  LevelBuf L = F.levels[level];
  int stride = nblk * blockDim.x;
  Work w{0, 0, 0, 0};
  for (int base = bid * blockDim.x; base < n; base += stride) {
    int i = base + threadIdx.x;
    bool active = i < n;
    bool hit = false;
    WHit h{-1, 0, 0.0, -1};
    if (active) {
      V3 o = mk(q.ox[i], q.oy[i], q.oz[i]);
      V3 d = mk(q.dx[i], q.dy[i], q.dz[i]);
      RayC r = make_rayc(o, d);
      h = world_closest(F.S, r, 0.001, F.use_kd != 0, F.err, COUNT ? &w : nullptr);
      hit = h.obj >= 0;
      if (!hit) {
        // ray_color_with_camera / ray_color miss branch (src/lighting.rs:497-505)
        V3 g;
        V3 c = (F.camera_mode && grid_color(F.C, o, d, &g)) ? g : ld3(F.S.bg);
        L.r[i] = c.x;
        L.g[i] = c.y;
        L.b[i] = c.z;
        L.refl[i] = 0.0;
        L.child[i] = -1;
        if (level == 0 && F.outline) F.phit[i] = 0;
      }
    }
    int slot = warp_alloc(&F.nhits[level], hit);
    if (hit) {
      F.hobj[slot] = h.obj;
      F.haux[slot] = h.aux;
      F.hent[slot] = h.ent;
      F.ht[slot] = h.t;
      F.hit_ray[slot] = i;
    }
  }
  if (COUNT) flush_work(F, w, 0);
}
template <bool COUNT>
__global__ void __launch_bounds__(128, 6) k_trace(const __grid_constant__ DFrame F, int level) {
  trace_body<COUNT>(F, level, blockIdx.x, gridDim.x);
}
template <bool COUNT>
__global__ void __launch_bounds__(128, 6) k_trace_multi(const DFrame* __restrict__ T, const int* __restrict__ b0, int nj, int level) {
  const int j = job_of_block(b0, nj);
  const DFrame& F = T[j];
  if (level >= frame_levels(F)) return;
  trace_body<COUNT>(F, level, blockIdx.x - b0[j], b0[j + 1] - b0[j]);
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

__device__ __forceinline__ HitRec load_hit(const DFrame& F, int level, int h, RayC* rc, uint64_t* seed) {
  RayBuf q = F.q[level & 1];
  int i = F.hit_ray[h];
  V3 o = mk(q.ox[i], q.oy[i], q.oz[i]);
  V3 d = mk(q.dx[i], q.dy[i], q.dz[i]);
  *seed = q.seed[i];
  *rc = make_rayc(o, d);
  WHit w{F.hobj[h], F.haux[h], F.ht[h], F.hent[h]};
  return finalize_hit(F.S, *rc, w);
}

// The hit at position h of the fallback list (see DFrame::fb_list).
__device__ __forceinline__ int fb_hit(const DFrame& F, long long h) {
  const long long n1 = F.fbn[2];
  return F.fb_list[h < n1 ? h : F.n_primary - 1 - (h - n1)];
}

// Light sampling for hits [c0, c1) of the level's hit list.
__device__ __forceinline__ void emit_body(const DFrame& F, int level, long long c0, int bid, int nblk) {
  const DScene& S = F.S;
  long long nh = F.fb_mode ? *F.fbn : F.nhits[level];
  long long c1 = c0 + F.chunk_hits < nh ? c0 + F.chunk_hits : nh;
  V3 campos = ld3(F.C.campos);
  unsigned long long culled = 0;  // shadow rays not traced (lights facing away)
  for (long long h = c0 + bid * (long long)blockDim.x + threadIdx.x; h < c1;
       h += (long long)nblk * blockDim.x) {
    RayC rc;
    uint64_t seed;
    const int hidx = F.fb_mode ? fb_hit(F, h) : (int)h;
    HitRec hr = load_hit(F, level, hidx, &rc, &seed);
    // fallback launches sample only the slots that fall back
    const unsigned fbmask = F.fb_mode ? (unsigned)F.fb_flag[hidx] : ~0u;
    int dslot = 0;
    // Lights the surface faces away from: the reference's light term is
    // exactly zero there (diffuse max(n . l, 0) = 0, specular only when
    // n . l > 0), so their shadow rays cannot change the image and are not
    // traced (distance -1).  A disk light qualifies when every point of the
    // disk is behind the surface: n . (centre - p) + radius < 0, with a
    // margin far above the rounding of the sample directions' dot products.
    // Not where the rays' visibility is itself an output (the denoiser's
    // features and visibility images at level 0, the fallback).
    const bool may_cull = !F.fb_mode && !(level == 0 && F.feat_on);
    const double pscale = norm(hr.p) + 1.0;
    V3 so = hr.p + 0.001 * hr.n;
    long long hl = h - c0;
    F.sh.ox[hl] = so.x;
    F.sh.oy[hl] = so.y;
    F.sh.oz[hl] = so.z;
    const long long CH = F.chunk_hits;
    long long s = hl;  // advances by CH per shadow ray
    for (int li = 0; li < S.n_lights; li++) {
      const DLight& L0 = S.lights[li];
      V3 lp = ld3(L0.pos);
      if (!L0.disk) {
        // calculate_point_light_contribution (src/lighting.rs:100-142)
        V3 lv = lp - hr.p;
        double dist = norm(lv);
        V3 ldir = lv / dist;
        const bool cull = may_cull && dot(hr.n, lv) < -1e-9 * (norm(lp) + pscale);
        culled += cull ? 1 : 0;
        F.sh.ray[s] = SRay{ldir.x, ldir.y, ldir.z, cull ? -1.0 : dist};
        s += CH;
      } else {
        // calculate_diffuse_light_contribution (src/lighting.rs:145-217),
        // sample_disk_light_point (:69-97), sample_disk_point (:57-66)
        uint64_t ls = seed * 0x9E3779B97F4A7C15ULL + sat_u64(hr.p.x * 1000.0) * 0x85EBCA6BULL +
                      sat_u64(hr.p.y * 1000.0) * 0xC2B2AE35ULL + sat_u64(hr.p.z * 1000.0) * 0x6C8E9CF5ULL;
        StdRng rng;
        rng.init(ls);
        double radius = L0.diameter / 2.0;
        // gen_range(-radius..radius) panics on an empty or infinite range
        bool ok = -radius < radius;
        if (!ok) atomicOr(F.err, ERR_EMPTY_RANGE);
        if (ok && !isfinite(radius - -radius)) {
          atomicOr(F.err, ERR_RANGE_OVERFLOW);
          ok = false;
        }
        // a slot the network is confident about: placeholder rays, never traced
        if (dslot < F.n_slots && !((fbmask >> dslot) & 1u)) ok = false;
        dslot++;
        if (ok && may_cull && dot(hr.n, lp - hr.p) + radius < -1e-9 * (norm(lp) + pscale + radius)) {
          ok = false;  // facing away from the whole disk
          culled += (unsigned long long)F.dsamp;
        }
        V3 cdir = normalize(lp - hr.p);
        V3 up = fabs(cdir.x) < 0.9 ? mk(1.0, 0.0, 0.0) : mk(0.0, 1.0, 0.0);
        V3 bu = normalize(cross(up, cdir));
        V3 bv = normalize(cross(cdir, bu));
        // One rejection-sampling attempt per iteration; an accepted attempt
        // emits the next sample.  Each lane draws exactly the numbers the
        // reference's per-sample loop draws, in the same order, but the
        // lanes of a warp stay in step (every attempt takes four words, so
        // they also refill their ChaCha buffers together) instead of each
        // sample waiting for the warp's slowest lane.
        int smp = 0, it = 0;
        while (ok && smp < F.dsamp) {
          double dx, dy;
          if (it >= 4096 || !rng.range(-radius, radius, &dx) || !rng.range(-radius, radius, &dy)) {
            atomicOr(F.err, ERR_WATCHDOG);
            ok = false;
            break;
          }
          it++;
          if (dx * dx + dy * dy <= radius * radius) {
            V3 sp = lp + dx * bu + dy * bv;
            // normalize(v) divides by norm(v): one square root for both
            V3 sv = sp - hr.p;
            double dist = norm(sv);
            V3 sdir = sv / dist;
            F.sh.ray[s] = SRay{sdir.x, sdir.y, sdir.z, dist};
            s += CH;
            smp++;
            it = 0;
          }
        }
        // after a failed range check or the watchdog, for a culled light or
        // a slot the network is confident about: never traced (one
        // direction, the light centre's, for all of the light's records)
        if (smp < F.dsamp) {
          const V3 sv = lp - hr.p;
          const V3 sdir = sv / norm(sv);
          for (; smp < F.dsamp; smp++, s += CH) F.sh.ray[s] = SRay{sdir.x, sdir.y, sdir.z, -1.0};
        }
      }
    }
  }
  warp_sum_add(F.stats + 10, culled);
}
__global__ void __launch_bounds__(128) k_emit(const __grid_constant__ DFrame F, int level, long long c0) {
  emit_body(F, level, c0, blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(128) k_emit_multi(const DFrame* __restrict__ T, const int* __restrict__ b0, int nj, int level, long long c0) {
  const int j = job_of_block(b0, nj);
  const DFrame& F = T[j];
  if (level >= frame_levels(F)) return;
  emit_body(F, level, c0, blockIdx.x - b0[j], b0[j + 1] - b0[j]);
}


// world.hit(&shadow_ray, 0.001, distance).is_some() per shadow ray.  MINB
// blocks of 128 per SM: with meshes 7 (72 registers; the icosphere frame's
// shadow stage 3.30 ms, against 3.40 at 6 and 3.50 at 8), with spheres and
// planes only 8 (64 registers; the ring frame's 21.57 -> 20.83 ms).
template <bool COUNT>
__device__ __forceinline__ void shadow_body(const DFrame& F, int level, long long c0, int bid, int nblk) {
  long long nh = F.fb_mode ? *F.fbn : F.nhits[level];
  long long c1 = c0 + F.chunk_hits < nh ? c0 + F.chunk_hits : nh;
  const int K = F.K;
  long long nhc = c1 > c0 ? c1 - c0 : 0;
  // a chunk holds at most 2^28 shadow rays (the host's cap): 32-bit indices
  const int ns = (int)(nhc * K);
  const int CH = (int)F.chunk_hits;
  Work w{0, 0, 0, 0};
  __shared__ int s_stack[4][RTB_STACK];  // one traversal stack per warp (128 threads)
  volatile int* stack = s_stack[threadIdx.x >> 5];
  // The warp steps through the rays together (world_any_warp is a warp
  // collective).  Hit-major order: the K rays of one hit point sit in
  // adjacent lanes, so a warp holds a bundle of rays from one or two points
  // towards one light, which the packet traversal shares out.
  const int stride = nblk * blockDim.x;
  for (int base = bid * blockDim.x + (threadIdx.x & ~31); base < ns; base += stride) {
    const int t = base + (threadIdx.x & 31);
    const bool have = t < ns;
    int hl = 0;
    SRay sr{0.0, 0.0, 1.0, -1.0};
    if (have) {
      hl = (int)((unsigned)t / (unsigned)K);
      const int k = t - hl * K;
      sr = F.sh.ray[k * CH + hl];
    }
    const double dist = sr.dist;
    const bool valid = have && (dist >= 0.0 || dist != dist);
    RayC r;
    if (valid) {
      // Ray::new normalises the (already unit) light direction once more
      r = make_rayc(mk(F.sh.ox[hl], F.sh.oy[hl], F.sh.oz[hl]), normalize(mk(sr.dx, sr.dy, sr.dz)));
    } else {
      r = make_rayc(mk(0.0, 0.0, 0.0), mk(0.0, 0.0, 1.0));
    }
    bool blocked = world_any_warp(F.S, r, 0.001, valid ? dist : 0.0, valid, F.use_kd != 0, stack, F.err,
                                  COUNT ? &w : nullptr);
    if (have) F.sh.vis[t] = (valid && !blocked) ? 1 : 0;
  }
  if (COUNT) flush_work(F, w, 1);
}
template <bool COUNT, int MINB>
__global__ void __launch_bounds__(128, MINB) k_shadow(const __grid_constant__ DFrame F, int level, long long c0) {
  shadow_body<COUNT>(F, level, c0, blockIdx.x, gridDim.x);
}
template <bool COUNT>
__global__ void __launch_bounds__(128, 7) k_shadow_multi(const DFrame* __restrict__ T, const int* __restrict__ b0, int nj, int level, long long c0) {
  const int j = job_of_block(b0, nj);
  const DFrame& F = T[j];
  if (level >= frame_levels(F)) return;
  shadow_body<COUNT>(F, level, c0, blockIdx.x - b0[j], b0[j + 1] - b0[j]);
}


// phong_lighting's sum, fog and the reflection ray (src/lighting.rs:220-288,
// 297-319, 437-496) for hits [c0, c1).  Eight blocks of 128 per SM (64
// registers, some spilled): the kernel streams the shadow buffer, and the
// extra warps hide more of its latency than the spills cost (bench frame
// 7.0 ms against 7.23 ms at 128 registers; 6, 10 and 12 blocks were slower).
__device__ __forceinline__ void resolve_body(const DFrame& F, int level, long long c0, int bid, int nblk) {
  const DScene& S = F.S;
  long long nh = F.fb_mode ? *F.fbn : F.nhits[level];
  long long c1 = c0 + F.chunk_hits < nh ? c0 + F.chunk_hits : nh;
  RayBuf qn = F.q[(level + 1) & 1];
  LevelBuf L = F.levels[level];
  bool can_reflect = (F.max_depth - level) > 1;
  V3 campos = ld3(F.C.campos);
  long long stride = (long long)nblk * blockDim.x;
  for (long long base = c0 + bid * (long long)blockDim.x; base < c1; base += stride) {
    long long h = base + threadIdx.x;
    bool active = h < c1;
    // the hit in the level's list (fallback launches walk fb_list); a
    // learned launch leaves the hits the fallback shades
    const int hi = active ? (F.fb_mode ? fb_hit(F, h) : (int)h) : 0;
    if (active && F.learned && level == 0 && F.fb_flag && F.fb_flag[hi]) active = false;
    // fallback launch: the slots that fall back take the plain sum, the
    // others keep the network's estimate
    const unsigned fbmask = (active && F.fb_mode) ? (unsigned)F.fb_flag[hi] : ~0u;
    bool emit = false;
    V3 ro = mk(0, 0, 0), rd = mk(0, 0, 0);
    uint64_t seed = 0;
    int i = -1;
    V3 color = mk(0.0, 0.0, 0.0);
    double refl = 0.0;
    if (active) {
      RayC rc;
      HitRec hr = load_hit(F, level, hi, &rc, &seed);
      i = F.hit_ray[hi];
      const DMat& mat = S.mat[hr.mat];
      SMat m = effective_material(mat, hr);
      color = m.ka * S.amb_int * cmul(ld3(S.amb_color), m.c);
      V3 view = normalize(campos - hr.p);
      const long long CH = F.chunk_hits;
      long long s = h - c0;  // advances by CH per shadow ray
      long long v = s * F.K;  // the ray's visibility byte
      const bool learned = level == 0 && F.learned;
      long long vix = 0;
      if (learned || (level == 0 && F.fb_mode)) {
        long long pix = i / F.S_per_px;
        vix = ((long long)(i % F.S_per_px) * DN_MAX_SLOTS * F.H) * F.W + pix;  // slot 0 of this sample
      }
      int slot = 0;
      for (int li = 0; li < S.n_lights; li++) {
        const DLight& L0 = S.lights[li];
        V3 lc = ld3(L0.color);
        V3 contrib;
        if (!L0.disk) {
          if (F.sh.vis[v]) {
            const SRay sr = F.sh.ray[s];
            contrib = light_term(m, hr, mk(sr.dx, sr.dy, sr.dz), lc, L0.intensity, view);
          } else {
            contrib = mk(0.0, 0.0, 0.0);
          }
          s += CH;
          v++;
        } else if (learned || (F.fb_mode && level == 0 && slot < F.n_slots && !((fbmask >> slot) & 1u))) {
          // extension: the light-centre term times the squared visibility
          // estimate, the expectation of the reference's
          // (sum of visible terms / n) * (visible / n)
          double vh = (double)F.vhat[vix + (long long)slot * F.H * F.W];
          vh = rclamp(vh, 0.0, 1.0);
          V3 cdir = normalize(ld3(L0.pos) - hr.p);
          contrib = light_term(m, hr, cdir, lc, L0.intensity, view) * (vh * vh);
          slot++;
          s += (long long)F.dsamp * CH;
          v += F.dsamp;
        } else {
          V3 total = mk(0.0, 0.0, 0.0);
          unsigned visible = 0;
          for (int smp = 0; smp < F.dsamp; smp++, s += CH, v++) {
            if (F.sh.vis[v]) {
              visible++;
              const SRay sr = F.sh.ray[s];
              total = total + light_term(m, hr, mk(sr.dx, sr.dy, sr.dz), lc, L0.intensity, view);
            }
          }
          const double n = (double)F.dsamp;  // 16.0 in the reference
          contrib = (total / n) * ((double)visible / n);
          // fallback of a learned render: the plain visibility replaces the
          // estimate in the visibility output
          if (F.fb_mode && level == 0 && slot < F.n_slots && F.vhat)
            F.vhat[vix + (long long)slot * F.H * F.W] = (float)visible / (float)F.dsamp;
          slot++;
        }
        color = color + contrib;
      }
      if (S.has_fog) {
        double dist = norm(hr.p - campos);
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
        V3 vd = normalize(campos - hr.p);
        ro = hr.p + 0.001 * hr.n;
        rd = normalize(reflect(-vd, hr.n));
      }
      if (level == 0 && F.outline) {
        F.phit[i] = 1;
        F.pobj[i] = F.hobj[hi];
        F.pdepth[i] = norm(hr.p - campos);
        F.pnx[i] = hr.n.x;
        F.pny[i] = hr.n.y;
        F.pnz[i] = hr.n.z;
      }
    }
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
__global__ void __launch_bounds__(128, 8) k_resolve(const __grid_constant__ DFrame F, int level, long long c0) {
  resolve_body(F, level, c0, blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(128, 8) k_resolve_multi(const DFrame* __restrict__ T, const int* __restrict__ b0, int nj, int level, long long c0) {
  const int j = job_of_block(b0, nj);
  const DFrame& F = T[j];
  if (level >= frame_levels(F)) return;
  resolve_body(F, level, c0, blockIdx.x - b0[j], b0[j + 1] - b0[j]);
}


// Confidence gate of learned shadows: every level-0 hit with an estimated
// visibility error above conf_thr on one of its slots goes to fb_list, with
// those slots' bits in fb_flag, to be shaded by the plain path.
__global__ void __launch_bounds__(128) k_fb_select(DFrame F) {
  const long long nh = F.nhits[0];
  const long long plane_px = (long long)F.H * F.W;
  for (long long base = blockIdx.x * (long long)blockDim.x; base < nh; base += (long long)gridDim.x * blockDim.x) {
    const long long h = base + threadIdx.x;
    unsigned mask = 0;
    if (h < nh) {
      const int i = F.hit_ray[h];
      const long long pix = i / F.S_per_px, plane = i % F.S_per_px;
      for (int j = 0; j < F.n_slots; j++)
        if (F.vconf[(plane * DN_MAX_SLOTS + j) * plane_px + pix] > F.conf_thr) mask |= 1u << j;
      F.fb_flag[h] = (unsigned char)mask;
    }
    const bool want = mask != 0, one = __popc(mask) == 1;
    // every lane of the warp takes part in each allocation
    warp_alloc(F.fbn, want);
    const int at1 = warp_alloc(F.fbn + 2, one);
    const int at2 = warp_alloc(F.fbn + 3, want && !one);
    if (want) F.fb_list[one ? at1 : F.n_primary - 1 - at2] = (int)h;
    const unsigned slots = __reduce_add_sync(0xffffffffu, (unsigned)__popc(mask));
    if ((threadIdx.x & 31) == 0 && slots) atomicAdd(F.fbn + 1, (int)slots);
  }
}

// Denoiser input of the level-0 hits [c0, c1): one FEAT_CHANNELS FP16
// pixel per (sample plane, pixel); misses stay zero (FEAT_VALID = 0).  Also
// the plain visibility (visible / dsamp) of each slot into vis_aov.
__global__ void __launch_bounds__(128) k_features(DFrame F, long long c0) {
  const DScene& S = F.S;
  long long nh = F.nhits[0];
  long long c1 = c0 + F.chunk_hits < nh ? c0 + F.chunk_hits : nh;
  V3 campos = ld3(F.C.campos);
  const long long plane_px = (long long)F.H * F.W;
  for (long long h = c0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; h < c1;
       h += (long long)gridDim.x * blockDim.x) {
    RayC rc;
    uint64_t seed;
    HitRec hr = load_hit(F, 0, (int)h, &rc, &seed);
    int i = F.hit_ray[h];
    long long pix = i / F.S_per_px;
    long long plane = i % F.S_per_px;
    float f[FEAT_CHANNELS];
#pragma unroll
    for (int c = 0; c < FEAT_CHANNELS; c++) f[c] = 0.f;
    f[FEAT_VALID] = 1.f;
    double d = norm(hr.p - campos);
    f[FEAT_DEPTH] = (float)(d / (d + 4.0));
    f[FEAT_NX] = (float)hr.n.x;
    f[FEAT_NX + 1] = (float)hr.n.y;
    f[FEAT_NX + 2] = (float)hr.n.z;
    long long v = (h - c0) * F.K;  // the hit's first visibility byte
    int slot = 0;
    for (int li = 0; li < S.n_lights; li++) {
      const DLight& L0 = S.lights[li];
      if (!L0.disk) {
        v++;
        continue;
      }
      unsigned visible = 0;
      for (int smp = 0; smp < F.dsamp; smp++, v++) visible += F.sh.vis[v];
      if (slot < DN_MAX_SLOTS) {
        float v = (float)visible / (float)F.dsamp;
        V3 lp = ld3(L0.pos);
        double dist = norm(lp - hr.p);
        V3 cdir = normalize(lp - hr.p);
        double cosc = rmax(dot(hr.n, cdir), 0.0);
        double ang = rclamp(0.5 * L0.diameter / dist, 0.0, 1.0);
        int b = FEAT_SLOT0 + FEAT_SLOT_STRIDE * slot;
        f[b] = v;
        f[b + 1] = (float)cosc;
        f[b + 2] = (float)ang;
        f[b + 3] = 1.f;
        if (F.vis_aov) F.vis_aov[(plane * DN_MAX_SLOTS + slot) * plane_px + pix] = v;
      }
      slot++;
    }
    __align__(16) __half hv[FEAT_CHANNELS];
#pragma unroll
    for (int c = 0; c < FEAT_CHANNELS; c++) hv[c] = __float2half_rn(f[c]);
    uint4* dst = reinterpret_cast<uint4*>(F.feat + (plane * plane_px + pix) * FEAT_CHANNELS);
    const uint4* src = reinterpret_cast<const uint4*>(hv);
    dst[0] = src[0];
    dst[1] = src[1];
  }
}

// Pixel-level feature: for each slot, the mean cast-ray visibility over the
// samples of the pixel whose primary ray hit, written into every hit
// sample's FEAT_PIXEL_VIS + slot channel, so that the network of each
// sample plane sees the pixel's other samples too.  One thread per pixel.
__global__ void __launch_bounds__(128) k_feat_pixel_mean(DFrame F) {
  const long long plane_px = (long long)F.H * F.W;
  for (long long pix = blockIdx.x * (long long)blockDim.x + threadIdx.x; pix < plane_px;
       pix += (long long)gridDim.x * blockDim.x) {
    float sum[DN_MAX_SLOTS] = {0.f, 0.f};
    int n = 0;
    for (int s = 0; s < F.S_per_px; s++) {
      const __half* f = F.feat + ((long long)s * plane_px + pix) * FEAT_CHANNELS;
      if (__half2float(f[FEAT_VALID]) > 0.f) {
        n++;
#pragma unroll
        for (int j = 0; j < DN_MAX_SLOTS; j++) sum[j] += __half2float(f[FEAT_SLOT0 + FEAT_SLOT_STRIDE * j]);
      }
    }
    if (n == 0) continue;
    for (int s = 0; s < F.S_per_px; s++) {
      __half* f = F.feat + ((long long)s * plane_px + pix) * FEAT_CHANNELS;
      if (__half2float(f[FEAT_VALID]) > 0.f) {
#pragma unroll
        for (int j = 0; j < DN_MAX_SLOTS; j++) f[FEAT_PIXEL_VIS + j] = __float2half_rn(sum[j] / (float)n);
      }
    }
  }
}

// color * (1 - r) + reflected * r, deepest level first
__device__ __forceinline__ void fold_body(const DFrame& F, int level, int bid, int nblk) {
  int n = F.counts[level];
  LevelBuf L = F.levels[level];
  LevelBuf C = F.levels[level + 1];
  for (int i = bid * blockDim.x + threadIdx.x; i < n; i += nblk * blockDim.x) {
    int c = L.child[i];
    if (c < 0) continue;
    double r = L.refl[i];
    double k = 1.0 - r;
    L.r[i] = L.r[i] * k + C.r[c] * r;
    L.g[i] = L.g[i] * k + C.g[c] * r;
    L.b[i] = L.b[i] * k + C.b[c] * r;
  }
}
__global__ void k_fold(const __grid_constant__ DFrame F, int level) {
  fold_body(F, level, blockIdx.x, gridDim.x);
}
__global__ void k_fold_multi(const DFrame* __restrict__ T, const int* __restrict__ b0, int nj, int level) {
  const int j = job_of_block(b0, nj);
  const DFrame& F = T[j];
  if (level > frame_levels(F) - 2) return;
  fold_body(F, level, blockIdx.x - b0[j], b0[j + 1] - b0[j]);
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

__device__ __forceinline__ void pixels_body(const DFrame& F, int bid, int nblk) {
  long long np = (long long)F.W * F.H;
  LevelBuf L = F.levels[0];
  for (long long p = bid * (long long)blockDim.x + threadIdx.x; p < np; p += (long long)nblk * blockDim.x) {
    V3 c;
    if (F.max_depth <= 0) {
      // ray_color returns black before any World::hit (src/lighting.rs:450-452)
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
      // (center + tl + tr + bl + br) / 5 (src/renderer.rs:873-886)
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
      // sum / samples; outline keeps the nearest sample's depth and normal
      // (src/renderer.rs:548-552, 690-702)
      V3 t = mk(0.0, 0.0, 0.0);
      bool have = false;
      double pd = 0.0;
      V3 pn = mk(0.0, 0.0, 0.0);
      int po = -1;
      for (int s = 0; s < F.S_per_px; s++) {
        long long i = p * F.S_per_px + s;
        t = t + mk(L.r[i], L.g[i], L.b[i]);
        if (F.outline && F.phit[i]) {
          double d = F.pdepth[i];
          if (!have || d < pd) {
            have = true;
            pd = d;
            pn = mk(F.pnx[i], F.pny[i], F.pnz[i]);
            po = F.pobj[i];
          }
        }
      }
      c = t / (double)F.S_per_px;
      if (F.outline) {
        F.valid[p] = have ? 1 : 0;
        if (F.oid) F.oid[p] = po;
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
__global__ void k_pixels(const __grid_constant__ DFrame F) {
  pixels_body(F, blockIdx.x, gridDim.x);
}
__global__ void k_pixels_multi(const DFrame* __restrict__ T, const int* __restrict__ b0, int nj) {
  const int j = job_of_block(b0, nj);
  const DFrame& F = T[j];
  pixels_body(F, blockIdx.x - b0[j], b0[j + 1] - b0[j]);
}


// detect_edges / compute_edge_strength (src/outline.rs:113-182): one tile of
// OT_X x OT_Y pixels with a one-pixel halo staged in shared memory.
#define OT_X 32
#define OT_Y 8
__global__ void __launch_bounds__(OT_X* OT_Y) k_outline_mask(DFrame F) {
  __shared__ double sd[OT_Y + 2][OT_X + 2];
  __shared__ double snx[OT_Y + 2][OT_X + 2], sny[OT_Y + 2][OT_X + 2], snz[OT_Y + 2][OT_X + 2];
  __shared__ unsigned char sv[OT_Y + 2][OT_X + 2];
  __shared__ int so[OT_Y + 2][OT_X + 2];
  const bool ids = F.oid && F.o_wid != 0.0;
  int x0 = blockIdx.x * OT_X - 1, y0 = blockIdx.y * OT_Y - 1;
  for (int k = threadIdx.y * OT_X + threadIdx.x; k < (OT_X + 2) * (OT_Y + 2); k += OT_X * OT_Y) {
    int lx = k % (OT_X + 2), ly = k / (OT_X + 2);
    int gx = x0 + lx, gy = y0 + ly;
    unsigned char v = 0;
    double d = 0, a = 0, b = 0, c = 0;
    int o = -1;
    if (gx >= 0 && gy >= 0 && gx < F.W && gy < F.H) {
      long long p = (long long)gy * F.W + gx;
      v = F.valid[p];
      d = F.dep[p];
      a = F.nx[p];
      b = F.ny[p];
      c = F.nz[p];
      if (ids) o = F.oid[p];
    }
    so[ly][lx] = o;
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
      // extension: different objects on either side of the edge
      if (ids && so[ly][lx] != so[ly + ndy[k]][lx + ndx[k]]) e = e + F.o_wid;
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
    c = mk(c.x * (1.0 - w) + F.o_color[0] * w, c.y * (1.0 - w) + F.o_color[1] * w,
           c.z * (1.0 - w) + F.o_color[2] * w);
  }
  store_rgb(F, p, c);
}

// k_outline_apply for radii whose mask tile does not fit in shared memory
// (outline thickness above 65): the same dilation, reading the mask from
// global memory (its neighbourhood stays in L1/L2).  One thread per pixel.
__global__ void __launch_bounds__(256) k_outline_apply_wide(DFrame F) {
  const int R = F.o_radius;
  const double th = F.o_thick;
  const long long n = (long long)F.W * F.H;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    const int gx = (int)(p % F.W), gy = (int)(p / F.W);
    double ms = F.mask[p];
    for (int dy = -R; dy <= R; dy++) {
      const int ny = gy + dy;
      if (ny < 0 || ny >= F.H) continue;
      for (int dx = -R; dx <= R; dx++) {
        const int nx = gx + dx;
        if (nx < 0 || nx >= F.W) continue;
        double dist = sqrt((double)(dx * dx + dy * dy));
        if (dist <= th) {
          double fo = 1.0 - (dist / th);
          ms = rmax(ms, __ldg(F.mask + (long long)ny * F.W + nx) * fo);
        }
      }
    }
    V3 c = mk(F.cr[p], F.cg[p], F.cb[p]);
    if (ms > 0.0) {
      double w = rclamp(rmin(ms, 1.0), 0.0, 1.0);
      c = mk(c.x * (1.0 - w) + F.o_color[0] * w, c.y * (1.0 - w) + F.o_color[1] * w,
             c.z * (1.0 - w) + F.o_color[2] * w);
    }
    store_rgb(F, p, c);
  }
}

// --------------------------------------------------------------------------
// Unit kernels for the parity tests and the FP64 rate probe
// --------------------------------------------------------------------------
// Eight independent add/multiply chains per thread; each iteration issues
// 16 FP64 add and 16 FP64 multiply instructions.
__global__ void k_fp64_rate(double* out, int iters, double a, double b) {
  double x[8], y[8];
  for (int k = 0; k < 8; k++) {
    x[k] = threadIdx.x * 1e-3 + k;
    y[k] = blockIdx.x * 1e-3 + k;
  }
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) {
      x[k] = x[k] * a + b;
      y[k] = y[k] * b + a;
    }
  }
  double s = 0;
  for (int k = 0; k < 8; k++) s += x[k] + y[k];
  if (s == 12345.678) out[0] = s;  // keeps the chains live
}
// Read bandwidth of a buffer small enough to stay in L2: 16-byte loads
// with ld.global.cg (cached in L2, not L1, so no pass is served by L1),
// four independent loads per thread in flight, `reps` passes over the
// buffer.  n16 is the buffer's size in 16-byte vectors, a multiple of
// 4 * gridDim.x * blockDim.x.
__global__ void k_l2_read(const uint4* __restrict__ buf, long long n16, int reps, unsigned* out) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  unsigned acc = 0;
  for (int r = 0; r < reps; r++) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n16; i += 4 * stride) {
      uint4 a = __ldcg(buf + i), b = __ldcg(buf + i + stride), c = __ldcg(buf + i + 2 * stride),
            d = __ldcg(buf + i + 3 * stride);
      acc ^= a.x ^ a.y ^ a.z ^ a.w ^ b.x ^ b.y ^ b.z ^ b.w ^ c.x ^ c.y ^ c.z ^ c.w ^ d.x ^ d.y ^ d.z ^ d.w;
    }
  }
  if (acc == 0x9E3779B9u) out[0] = acc;  // keeps the loads live
}
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
      for (int it = 0;; it++) {
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
// Mesh queries for the parity tests: closest hit as the renderer runs it
// (mode 0: BVH search + reference-leaf verification), the plain reference
// k-d walk (mode 1), any-hit as shadow rays run it (mode 2: packet walk),
// and for every k-d leaf the cell-based visit test against the root walk
// (mode 3: out = {leaves where they differ, where they agree, leaves the
// walk visits}).  128 threads per block; every warp steps through the
// rays together because the packet walks are warp collectives.
__global__ void __launch_bounds__(128) k_debug_mesh(DMesh M, int use_kd, int mode, const double* rays, long long n,
                                                    double tmin, double tmax, double* out, int* err) {
  __shared__ int s_stack[4][RTB_STACK];
  volatile int* stack = s_stack[threadIdx.x >> 5];
  for (long long base = blockIdx.x * (long long)blockDim.x + (threadIdx.x & ~31); base < n;
       base += (long long)gridDim.x * blockDim.x) {
    const long long i = base + (threadIdx.x & 31);
    const bool valid = i < n;
    V3 o = mk(0.0, 0.0, 0.0), d = mk(0.0, 0.0, 1.0);
    if (valid) {
      const double* rr = rays + 6 * i;
      o = mk(rr[0], rr[1], rr[2]);
      d = normalize(mk(rr[3], rr[4], rr[5]));
    }
    RayC r = make_rayc(o, d);
    double closest = tmax;
    int best = -1;
    double* oo = out + 8 * (valid ? i : 0);
    if (mode == 3) {
      // every k-d leaf: the cell-based visit test against the root walk
      if (valid) {
        double agree = 0.0, visited = 0.0, differ = 0.0;
        for (int k = 0; k < M.n_nodes; k++) {
          if (hi32(__ldg(M.nodes + 4 * (size_t)k + 3).y) >= 0) continue;
          unsigned key;
          const bool a = kd_leaf_visited_cell(M, r, k, nullptr), b = kd_leaf_visited(M, r, k, &key);
          if (a == b) agree += 1.0;
          else differ += 1.0;
          if (b) visited += 1.0;
        }
        for (int k = 0; k < 8; k++) oo[k] = 0.0;
        oo[0] = differ;
        oo[1] = agree;
        oo[2] = visited;
      }
      continue;
    }
    if (mode == 2) {
      bool any = mesh_any_warp(M, r, tmin, tmax, valid, use_kd != 0, stack, err, nullptr);
      if (valid) {
        for (int k = 0; k < 8; k++) oo[k] = 0.0;
        oo[0] = any ? 1.0 : 0.0;
      }
      continue;
    }
    bool hit = valid && (mode == 0 ? mesh_closest(M, r, tmin, closest, best, use_kd != 0, err, nullptr)
                                   : (mesh_bounds(M, r, tmin, closest) &&
                                      mesh_kd_walk<false>(M, r, tmin, closest, best, err, nullptr)));
    if (!valid) continue;
    for (int k = 0; k < 8; k++) oo[k] = 0.0;
    if (hit) {
      const double2* E = M.brute + 5 * (size_t)best;
      double2 q1 = E[1], q2 = E[2], q3 = E[3], q4 = E[4];
      V3 e1 = mk(q1.y, q2.x, q2.y), e2 = mk(q3.x, q3.y, q4.x);
      double a = dot(e1, cross(r.d, e2));
      double4 nn = M.normals[best];
      V3 nv = mk(nn.x, nn.y, nn.z);
      if (a < 0.0) nv = -nv;
      V3 p = r.o + closest * r.d;
      V3 fn = face_normal(r.d, nv);
      oo[0] = 1.0;
      oo[1] = closest;
      oo[2] = p.x;
      oo[3] = p.y;
      oo[4] = p.z;
      oo[5] = fn.x;
      oo[6] = fn.y;
      oo[7] = fn.z;
    }
  }
}

}  // namespace rtb
