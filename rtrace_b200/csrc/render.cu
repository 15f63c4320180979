// Render orchestration and the C ABI of include/rtrace_gpu.h.
//
// A render is the wavefront pipeline of kernels.cuh: camera rays, then per
// reflection depth trace -> emit -> shadow -> resolve over compacted
// queues, then the reflection fold (deepest level first), the per-pixel
// resolve and the outline post-process.  All arithmetic is IEEE double in
// the reference's operation order (compile with -fmad=false).

#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/rtrace_gpu.h"
#include "bvh_build.hpp"
#include "kd_build.hpp"
#include "mesh_prep.hpp"
#include "kernels.cuh"
#include "scene_loader.hpp"

using namespace rtb;

// A region of a scene's device block and where it is copied from at the
// flush: a host array of its own (a pinned mesh image, or a mesh array
// prepared by this upload), or the context's pinned staging buffer.
struct DirectCopy {
  size_t off, take;
  const char* src;
  size_t bytes;
};
struct StagedCopy {
  size_t off, pin_off, bytes;
};
// A host-prepared mesh whose records in mesh order, normals and occurrence
// lists the device derives from its copied arrays (derive_mesh_device), at
// the flush once the copies are queued.
struct MeshDerive {
  const double2* bvh;
  int nb;
  float4* fbvh;
  const double2* btris;
  int n;
  const double2* nodes;
  int n_nodes;
  const int* leaf_tris;
  const int2* leaf_path;
  int n_index;
  double2* cells;
  double2* brute;
  double4* normals;
  int2* occ;
  int* occ_off;
};

struct rt_scene {
  rt_ctx* ctx = nullptr;
  int device = 0;
  std::vector<void*> allocs;
  size_t uploaded_bytes = 0;
  DScene S{};
  rt_camera_config camera{};
  rt_outline_config outline{};
  int has_outline = 0;
  std::string render_error;
  std::vector<DMesh> host_meshes;       // device pointers, for the debug entry point; empty: k_shadow's
                                        // mesh-free register budget
  std::vector<int> obj_kind, obj_mesh;  // per World object
  int n_point_lights = 0, n_disk_lights = 0;
  // upload arena: one device block; small arrays are staged in the
  // context's pinned buffer, mesh arrays copied from their own host memory
  char* blk = nullptr;
  size_t blk_cap = 0, blk_used = 0, pin_used = 0;
  char* arena = nullptr;  // the scene's device block (returned to the pool when freed)
  size_t arena_bytes = 0;
  ~rt_scene();
  std::vector<DirectCopy> direct;
  std::vector<StagedCopy> staged;  // runs of the staging buffer
  std::vector<MeshDerive> derive;
};

// One captured render (RT_FLAG_CUDA_GRAPH): the launch sequence is fully
// determined by the bytes of its key (every kernel argument, grid size and
// the denoiser layers), so a render with the same key replays it.
struct GraphEntry {
  std::vector<unsigned char> key;
  cudaGraphExec_t exec = nullptr;
  uint32_t launches = 0;
  uint64_t used = 0;  // LRU tick
};

struct rt_ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<cudaEvent_t> stage_ev;
  std::string err;
  long long cap_rays = 0;
  int cap_levels = 0;
  long long cap_pixels = 0;
  long long cap_shadow = 0;   // shadow-ray entries
  long long cap_hits_sh = 0;  // per-hit shadow origins
  std::vector<void*> scratch;
  DFrame F{};
  std::vector<LevelBuf> h_levels;
  LevelBuf* d_levels = nullptr;
  int* d_counts = nullptr;
  int* d_nhits = nullptr;
  unsigned long long* d_stats = nullptr;
  int* d_err = nullptr;
  // learned soft shadows: network and its buffers (grown on demand)
  DenoiseNet net;
  std::vector<void*> dn_scratch;
  long long dn_cap = 0;  // primary samples the buffers hold
  __half* d_feat = nullptr;
  float *d_vhat = nullptr, *d_vconf = nullptr;  // visibility estimates and their error estimates
  int *d_fb_list = nullptr, *d_fbn = nullptr;   // confidence-gated fallback: hits and their count
  unsigned char* d_fb_flag = nullptr;
  std::vector<void*> dn_arena_alloc;  // the network's activations (grown on demand)
  __half* d_dn_arena = nullptr;
  size_t dn_arena_cap = 0;  // halves
  // batched rendering: lanes are child contexts (own stream and scratch)
  std::vector<rt_ctx*> lanes;
  uint32_t tuned_lanes = 0;
  // the fused group of a batch: frames of at most fuse_pixels pixels are
  // rendered together, each kernel launched once for all of them; slots
  // hold their scratch (child contexts), group_buf their frame table.
  std::vector<rt_ctx*> slots;
  uint32_t fuse_pixels = 640 * 480;
  uint64_t fuse_bytes = 16ull << 30;  // scratch the group's frames may hold together (estimated)
  int tune_bpsm[7] = {16, 64, 64, 128, 16, 16, 16};  // blocks per SM: raygen trace emit shadow resolve fold pixels
  bool tuned = false;
  void* group_buf = nullptr;
  size_t group_cap = 0;
  char* pin = nullptr;  // pinned staging of scene uploads
  size_t pin_cap = 0;
  bool borrowed_net = false;  // a lane's net points at its parent's weights
  std::vector<GraphEntry> graphs;  // captured renders, least recently used evicted
  uint64_t graph_tick = 0;
  KdArena* kd_arena = nullptr;  // device memory of k-d builds, kept between them
};

namespace {

std::mutex g_err_mu;
std::string g_global_err;

rt_status fail(rt_ctx* ctx, rt_status s, const std::string& m) {
  if (ctx) {
    ctx->err = m;
  } else {
    std::lock_guard<std::mutex> g(g_err_mu);
    g_global_err = m;
  }
  return s;
}

rt_status cuda_fail(rt_ctx* ctx, cudaError_t e, const char* what) {
  rt_status s = (e == cudaErrorMemoryAllocation) ? RT_ERR_OUT_OF_MEMORY : RT_ERR_CUDA;
  return fail(ctx, s, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                             \
  do {                                                       \
    cudaError_t e_ = (call);                                 \
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

// Captured renders name scratch buffers; they go whenever those are freed.
// Callers have synchronised the stream, so no replay is in flight.
void drop_graphs(rt_ctx* ctx) {
  for (GraphEntry& g : ctx->graphs) cudaGraphExecDestroy(g.exec);
  ctx->graphs.clear();
}

// Captured renders one context keeps (tens of kB of host and device memory
// each): enough for every job a batch lane renders, so that a repeated batch
// replays instead of cycling through a too-small LRU.
const size_t kMaxGraphs = 256;

// Shadow-ray entries kept on the device at once (33 B each, 8.9 GB at
// most).  A 1080p frame with 4 samples and 32 rays per hit fits in one
// chunk per level: at 2^26 it took four, and at every reflection level the
// three chunks beyond the level's few hits still cost their launches (about
// 0.7 ms per frame of the 1,000-sphere ring scene).
const long long kShadowCap = 1LL << 28;

rt_status ensure_scratch(rt_ctx* ctx, long long n_rays, int levels, long long n_pix, long long n_shadow,
                         long long n_hits_sh) {
  if (n_rays <= ctx->cap_rays && levels <= ctx->cap_levels && n_pix <= ctx->cap_pixels &&
      n_shadow <= ctx->cap_shadow && n_hits_sh <= ctx->cap_hits_sh)
    return RT_OK;
  CK(cudaStreamSynchronize(ctx->stream));
  long long R = std::max(n_rays, ctx->cap_rays);
  int Lv = std::max(levels, ctx->cap_levels);
  long long P = std::max(n_pix, ctx->cap_pixels);
  long long SH = std::max(n_shadow, ctx->cap_shadow), HS = std::max(n_hits_sh, ctx->cap_hits_sh);
  drop_graphs(ctx);
  free_all(ctx->scratch);
  ctx->cap_rays = ctx->cap_levels = 0;
  ctx->cap_pixels = ctx->cap_shadow = ctx->cap_hits_sh = 0;
  DFrame& F = ctx->F;
  auto& o = ctx->scratch;
  for (int k = 0; k < 2; k++) {
    CK(dalloc(o, &F.q[k].ox, R)); CK(dalloc(o, &F.q[k].oy, R)); CK(dalloc(o, &F.q[k].oz, R));
    CK(dalloc(o, &F.q[k].dx, R)); CK(dalloc(o, &F.q[k].dy, R)); CK(dalloc(o, &F.q[k].dz, R));
    CK(dalloc(o, &F.q[k].seed, R));
  }
  CK(dalloc(o, &F.hobj, R)); CK(dalloc(o, &F.haux, R)); CK(dalloc(o, &F.hent, R)); CK(dalloc(o, &F.ht, R));
  CK(dalloc(o, &F.hit_ray, R));
  ctx->h_levels.assign(Lv + 1, LevelBuf{});
  for (int l = 0; l < Lv; l++) {
    LevelBuf& L = ctx->h_levels[l];
    CK(dalloc(o, &L.r, R)); CK(dalloc(o, &L.g, R)); CK(dalloc(o, &L.b, R));
    CK(dalloc(o, &L.refl, R)); CK(dalloc(o, &L.child, R));
  }
  CK(dalloc(o, &ctx->d_levels, Lv + 1));
  CK(cudaMemcpy(ctx->d_levels, ctx->h_levels.data(), (Lv + 1) * sizeof(LevelBuf), cudaMemcpyHostToDevice));
  CK(dalloc(o, &ctx->d_counts, Lv + 2));
  CK(dalloc(o, &ctx->d_nhits, Lv + 1));
  CK(dalloc(o, &F.sh.ray, SH));
  CK(dalloc(o, &F.sh.vis, SH));
  CK(dalloc(o, &F.sh.ox, HS)); CK(dalloc(o, &F.sh.oy, HS)); CK(dalloc(o, &F.sh.oz, HS));
  CK(dalloc(o, &F.pdepth, R)); CK(dalloc(o, &F.pnx, R)); CK(dalloc(o, &F.pny, R)); CK(dalloc(o, &F.pnz, R));
  CK(dalloc(o, &F.phit, R));
  CK(dalloc(o, &F.pobj, R));
  CK(dalloc(o, &F.cr, P)); CK(dalloc(o, &F.cg, P)); CK(dalloc(o, &F.cb, P));
  CK(dalloc(o, &F.dep, P)); CK(dalloc(o, &F.nx, P)); CK(dalloc(o, &F.ny, P)); CK(dalloc(o, &F.nz, P));
  CK(dalloc(o, &F.valid, P));
  CK(dalloc(o, &F.oid, P));
  CK(dalloc(o, &F.mask, P));
  CK(dalloc(o, &F.rgb, 3 * P));
  CK(dalloc(o, &ctx->d_stats, 16));
  CK(dalloc(o, &ctx->d_err, 1));
  ctx->cap_rays = R;
  ctx->cap_levels = Lv;
  ctx->cap_pixels = P;
  ctx->cap_shadow = SH;
  ctx->cap_hits_sh = HS;
  return RT_OK;
}

// Dilation radii (ceil(thickness - 1)) up to kOutlineTileRadius stage their
// mask tile in shared memory ((32 + 2R) x (8 + 2R) doubles: 174 KB at 64);
// larger ones read the mask from global memory.  The reference has no
// limit; radii are capped where one pixel's (2R + 1)^2 loop would run for
// seconds.
constexpr int kOutlineTileRadius = 64;
constexpr double kOutlineMaxRadius = 2048.0;

// Raises k_outline_apply's dynamic shared-memory limit to at least `bytes`
// (never lowers it: batch lanes render from several host threads).
cudaError_t outline_smem_attr(int bytes) {
  static std::mutex mu;
  static int set[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> g(mu);
  if (dev < 64 && set[dev] >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(k_outline_apply, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess && dev < 64) set[dev] = bytes;
  return e;
}

// Feature image, visibility and error estimates and the fallback lists for
// n primary samples (32 + 8 + 8 + 4 + 1 bytes each).
rt_status ensure_dn_scratch(rt_ctx* ctx, long long n) {
  if (n <= ctx->dn_cap) return RT_OK;
  CK(cudaStreamSynchronize(ctx->stream));
  drop_graphs(ctx);
  free_all(ctx->dn_scratch);
  ctx->dn_cap = 0;
  auto& o = ctx->dn_scratch;
  CK(dalloc(o, &ctx->d_feat, n * FEAT_CHANNELS));
  CK(dalloc(o, &ctx->d_vhat, n * DN_MAX_SLOTS));
  CK(dalloc(o, &ctx->d_vconf, n * DN_MAX_SLOTS));
  CK(dalloc(o, &ctx->d_fb_list, n));
  CK(dalloc(o, &ctx->d_fb_flag, n));
  CK(dalloc(o, &ctx->d_fbn, 4));
  ctx->dn_cap = n;
  return RT_OK;
}

// The network's activation buffers for one run (denoise_scratch_halves).
rt_status ensure_dn_arena(rt_ctx* ctx, size_t halves) {
  if (halves <= ctx->dn_arena_cap) return RT_OK;
  CK(cudaStreamSynchronize(ctx->stream));
  drop_graphs(ctx);
  free_all(ctx->dn_arena_alloc);
  ctx->dn_arena_cap = 0;
  CK(dalloc(ctx->dn_arena_alloc, &ctx->d_dn_arena, halves));
  ctx->dn_arena_cap = halves;
  return RT_OK;
}

// Scene uploads go into one device block per scene (sized from the scene
// description by arena_open) and are copied with one asynchronous transfer
// per run of staged arrays and one per mesh array (arena_flush); arrays that
// do not fit get their own allocation.  One cudaMalloc and one cudaFree per
// scene instead of one per array.
rt_status arena_flush(rt_ctx* ctx, rt_scene* sc) {
  bool queued = false;
  if (sc->blk && sc->blk_used) {
    for (const StagedCopy& c : sc->staged)
      CK(cudaMemcpyAsync(sc->blk + c.off, ctx->pin + c.pin_off, c.bytes, cudaMemcpyHostToDevice, ctx->stream));
    for (const DirectCopy& d : sc->direct)
      if (d.bytes) CK(cudaMemcpyAsync(sc->blk + d.off, d.src, d.bytes, cudaMemcpyHostToDevice, ctx->stream));
    queued = true;
  }
  std::vector<MeshDerive> derive;
  derive.swap(sc->derive);
  for (const MeshDerive& m : derive) {
    if (!ctx->kd_arena) ctx->kd_arena = kd_arena_new();
    cudaError_t ce = cudaSuccess;
    std::string e = derive_mesh_device(m.bvh, m.nb, m.btris, m.n, m.nodes, m.n_nodes, m.leaf_tris, m.leaf_path,
                                       m.n_index, ctx->stream, ctx->kd_arena, m.fbvh, m.cells, m.brute, m.normals,
                                       m.occ, m.occ_off, &ce);
    if (!e.empty()) return cuda_fail(ctx, ce, e.c_str());
    queued = true;
  }
  if (queued) CK(cudaStreamSynchronize(ctx->stream));
  sc->direct.clear();
  sc->staged.clear();
  sc->blk = nullptr;
  sc->blk_cap = sc->blk_used = sc->pin_used = 0;
  return RT_OK;
}

// Reserves `bytes` of the arena for a host array and copies it there at
// the flush, straight from `src` (which must live until then; pinned memory
// copies fastest); a dedicated allocation and a synchronous copy when the
// arena has no room.
rt_status upload_direct(rt_ctx* ctx, rt_scene* sc, const char* src, size_t bytes, char** dev) {
  const size_t take = (std::max<size_t>(bytes, 16) + 255) & ~(size_t)255;
  if (sc->blk && sc->blk_used + take <= sc->blk_cap) {
    *dev = sc->blk + sc->blk_used;
    sc->direct.push_back(DirectCopy{sc->blk_used, take, src, bytes});
    sc->blk_used += take;
  } else {
    char* p = nullptr;
    CK(dalloc(sc->allocs, &p, take));
    if (bytes) CK(cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice));
    *dev = p;
  }
  sc->uploaded_bytes += bytes;
  return RT_OK;
}

// Freed scene blocks, kept per device for the next upload of a similar
// size (uploading and freeing a scene per frame then allocates nothing).
// Bounded: at most kPoolBlocks blocks and kPoolBytes bytes per device.
struct PoolBlock {
  int device;
  size_t bytes;
  char* ptr;
};
std::mutex g_pool_mu;
std::vector<PoolBlock> g_pool;
const size_t kPoolBlocks = 8;
const size_t kPoolBytes = (size_t)4 << 30;

char* pool_take(int device, size_t bytes, size_t* got) {
  std::lock_guard<std::mutex> g(g_pool_mu);
  int best = -1;
  for (int i = 0; i < (int)g_pool.size(); i++) {
    const PoolBlock& b = g_pool[i];
    if (b.device == device && b.bytes >= bytes && b.bytes <= 2 * bytes &&
        (best < 0 || b.bytes < g_pool[best].bytes))
      best = i;
  }
  if (best < 0) return nullptr;
  char* p = g_pool[best].ptr;
  *got = g_pool[best].bytes;
  g_pool.erase(g_pool.begin() + best);
  return p;
}

void pool_give(int device, char* p, size_t bytes) {
  {
    std::lock_guard<std::mutex> g(g_pool_mu);
    size_t n = 0, total = 0;
    for (const PoolBlock& b : g_pool)
      if (b.device == device) {
        n++;
        total += b.bytes;
      }
    if (n < kPoolBlocks && total + bytes <= kPoolBytes) {
      g_pool.push_back(PoolBlock{device, bytes, p});
      return;
    }
  }
  cudaFree(p);
}

}  // namespace

// Frees the scene's own allocations and returns its block to the pool; no
// kernel may still read the block when a later upload reuses it, hence the
// device-wide synchronisation (which cudaFree would imply as well).
rt_scene::~rt_scene() {
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  cudaDeviceSynchronize();
  free_all(allocs);
  if (arena) pool_give(device, arena, arena_bytes);
  if (prev >= 0 && prev != device) cudaSetDevice(prev);
}

namespace {

// Opens a scene block of `bytes`, of which at most `staged_bytes` are
// staged through the context's pinned buffer.
rt_status arena_open(rt_ctx* ctx, rt_scene* sc, size_t bytes, size_t staged_bytes) {
  rt_status st = arena_flush(ctx, sc);
  if (st != RT_OK) return st;
  bytes = (bytes + 255) & ~(size_t)255;
  staged_bytes = (staged_bytes + 255) & ~(size_t)255;
  size_t got = 0;
  char* b = pool_take(ctx->device, bytes, &got);
  if (!b) {
    CK(cudaMalloc((void**)&b, bytes));
    got = bytes;
  }
  sc->arena = b;
  sc->arena_bytes = got;
  if (ctx->pin_cap < staged_bytes) {
    if (ctx->pin) cudaFreeHost(ctx->pin);
    ctx->pin = nullptr;
    ctx->pin_cap = 0;
    CK(cudaMallocHost((void**)&ctx->pin, staged_bytes));
    ctx->pin_cap = staged_bytes;
  }
  sc->blk = b;
  sc->blk_cap = bytes;
  sc->blk_used = 0;
  return RT_OK;
}

template <class T>
rt_status upload(rt_ctx* ctx, rt_scene* sc, const std::vector<T>& h, const T** out) {
  const size_t bytes = h.size() * sizeof(T);
  const size_t take = (std::max<size_t>(bytes, 16) + 255) & ~(size_t)255;
  if (sc->blk && sc->blk_used + take <= sc->blk_cap && sc->pin_used + take <= ctx->pin_cap) {
    if (bytes) memcpy(ctx->pin + sc->pin_used, h.data(), bytes);
    *out = reinterpret_cast<const T*>(sc->blk + sc->blk_used);
    StagedCopy* last = sc->staged.empty() ? nullptr : &sc->staged.back();
    if (last && last->off + last->bytes == sc->blk_used && last->pin_off + last->bytes == sc->pin_used)
      last->bytes += take;  // contiguous with the previous staged array
    else
      sc->staged.push_back(StagedCopy{sc->blk_used, sc->pin_used, take});
    sc->blk_used += take;
    sc->pin_used += take;
  } else {
    T* p = nullptr;
    CK(dalloc(sc->allocs, &p, h.size()));
    if (bytes) CK(cudaMemcpy(p, h.data(), bytes, cudaMemcpyHostToDevice));
    *out = p;
  }
  sc->uploaded_bytes += bytes;
  return RT_OK;
}

// Device bytes of a scene description other than its meshes' arrays (an
// upper bound for what upload() stages).
size_t scene_staged_bound(const rt_scene_desc* d) {
  return (1 << 16) + (size_t)std::max(d->n_meshes, 0) * 256 + (size_t)std::max(d->n_objects, 0) * 512 +
         (size_t)std::max(d->n_materials, 0) * 256 + (size_t)std::max(d->n_lights, 0) * 128 + 32 * 256;
}

// Device bytes a scene description needs (an upper bound for the arena).
size_t scene_bytes_bound(const rt_scene_desc* d) {
  size_t b = 1 << 16;
  for (int m = 0; m < d->n_meshes; m++) {
    const rt_mesh_desc& md = d->meshes[m];
    size_t nt = (size_t)std::max<int64_t>(md.n_triangles, 0);
    // triangle records twice (80 B), normals (32), BVH nodes in double and
    // single precision (<= nt/2 nodes, 112 + 64 B, with a median split;
    // an SAH tree with more spills to its own allocation), k-d nodes
    // (64 + 8) and leaf cells (48), leaf entries and occurrences (4 + 8),
    // padding
    b += nt * (80 * 2 + 32 + 88) + (size_t)std::max<int64_t>(md.n_nodes, 0) * 120 +
         (size_t)std::max<int64_t>(md.n_tri_index, 0) * 12 + 8 * 256;
  }
  // objects, spheres (+ run BVHs), planes, cubes, materials, lights
  b += (size_t)std::max(d->n_objects, 0) * 512 + (size_t)std::max(d->n_materials, 0) * 256 +
       (size_t)std::max(d->n_lights, 0) * 128 + 32 * 256;
  return b;
}

// nalgebra 4x4 try_inverse: cofactors over the column-major slice, det from
// the first column, every entry scaled by 1/det.  Cube::new_with_transform
// (src/ray.rs:208-225) stores it as the world-to-local matrix.
bool inverse4(const double* tm, double* inv) {
  double m[16], iv[16];
  for (int k = 0; k < 16; k++) m[k] = tm[(k % 4) * 4 + k / 4];
  iv[0] = m[5] * m[10] * m[15] - m[5] * m[11] * m[14] - m[9] * m[6] * m[15] + m[9] * m[7] * m[14] +
          m[13] * m[6] * m[11] - m[13] * m[7] * m[10];
  iv[4] = -m[4] * m[10] * m[15] + m[4] * m[11] * m[14] + m[8] * m[6] * m[15] - m[8] * m[7] * m[14] -
          m[12] * m[6] * m[11] + m[12] * m[7] * m[10];
  iv[8] = m[4] * m[9] * m[15] - m[4] * m[11] * m[13] - m[8] * m[5] * m[15] + m[8] * m[7] * m[13] +
          m[12] * m[5] * m[11] - m[12] * m[7] * m[9];
  iv[12] = -m[4] * m[9] * m[14] + m[4] * m[10] * m[13] + m[8] * m[5] * m[14] - m[8] * m[6] * m[13] -
           m[12] * m[5] * m[10] + m[12] * m[6] * m[9];
  double det = m[0] * iv[0] + m[1] * iv[4] + m[2] * iv[8] + m[3] * iv[12];
  if (det == 0.0) return false;
  iv[1] = -m[1] * m[10] * m[15] + m[1] * m[11] * m[14] + m[9] * m[2] * m[15] - m[9] * m[3] * m[14] -
          m[13] * m[2] * m[11] + m[13] * m[3] * m[10];
  iv[5] = m[0] * m[10] * m[15] - m[0] * m[11] * m[14] - m[8] * m[2] * m[15] + m[8] * m[3] * m[14] +
          m[12] * m[2] * m[11] - m[12] * m[3] * m[10];
  iv[9] = -m[0] * m[9] * m[15] + m[0] * m[11] * m[13] + m[8] * m[1] * m[15] - m[8] * m[3] * m[13] -
          m[12] * m[1] * m[11] + m[12] * m[3] * m[9];
  iv[13] = m[0] * m[9] * m[14] - m[0] * m[10] * m[13] - m[8] * m[1] * m[14] + m[8] * m[2] * m[13] +
           m[12] * m[1] * m[10] - m[12] * m[2] * m[9];
  iv[2] = m[1] * m[6] * m[15] - m[1] * m[7] * m[14] - m[5] * m[2] * m[15] + m[5] * m[3] * m[14] +
          m[13] * m[2] * m[7] - m[13] * m[3] * m[6];
  iv[6] = -m[0] * m[6] * m[15] + m[0] * m[7] * m[14] + m[4] * m[2] * m[15] - m[4] * m[3] * m[14] -
          m[12] * m[2] * m[7] + m[12] * m[3] * m[6];
  iv[10] = m[0] * m[5] * m[15] - m[0] * m[7] * m[13] - m[4] * m[1] * m[15] + m[4] * m[3] * m[13] +
           m[12] * m[1] * m[7] - m[12] * m[3] * m[5];
  iv[14] = -m[0] * m[5] * m[14] + m[0] * m[6] * m[13] + m[4] * m[1] * m[14] - m[4] * m[2] * m[13] -
           m[12] * m[1] * m[6] + m[12] * m[2] * m[5];
  iv[3] = -m[1] * m[6] * m[11] + m[1] * m[7] * m[10] + m[5] * m[2] * m[11] - m[5] * m[3] * m[10] -
          m[9] * m[2] * m[7] + m[9] * m[3] * m[6];
  iv[7] = m[0] * m[6] * m[11] - m[0] * m[7] * m[10] - m[4] * m[2] * m[11] + m[4] * m[3] * m[10] +
          m[8] * m[2] * m[7] - m[8] * m[3] * m[6];
  iv[11] = -m[0] * m[5] * m[11] + m[0] * m[7] * m[9] + m[4] * m[1] * m[11] - m[4] * m[3] * m[9] -
           m[8] * m[1] * m[7] + m[8] * m[3] * m[5];
  iv[15] = m[0] * m[5] * m[10] - m[0] * m[6] * m[9] - m[4] * m[1] * m[10] + m[4] * m[2] * m[9] +
           m[8] * m[1] * m[6] - m[8] * m[2] * m[5];
  double id = 1.0 / det;
  for (int k = 0; k < 16; k++) inv[(k % 4) * 4 + k / 4] = iv[k] * id;
  return true;
}

// nalgebra 3x3 try_inverse (adjugate / determinant)
bool inverse3(const double a[3][3], double ri[3][3]) {
  double m11 = a[1][1] * a[2][2] - a[2][1] * a[1][2];
  double m12 = a[1][0] * a[2][2] - a[2][0] * a[1][2];
  double m13 = a[1][0] * a[2][1] - a[2][0] * a[1][1];
  double det = a[0][0] * m11 - a[0][1] * m12 + a[0][2] * m13;
  if (det == 0.0) return false;
  double m21 = a[0][1] * a[2][2] - a[2][1] * a[0][2];
  double m22 = a[0][0] * a[2][2] - a[2][0] * a[0][2];
  double m23 = a[0][0] * a[2][1] - a[2][0] * a[0][1];
  double m31 = a[0][1] * a[1][2] - a[1][1] * a[0][2];
  double m32 = a[0][0] * a[1][2] - a[1][0] * a[0][2];
  double m33 = a[0][0] * a[1][1] - a[1][0] * a[0][1];
  ri[0][0] = m11 / det;
  ri[1][0] = -m12 / det;
  ri[2][0] = m13 / det;
  ri[0][1] = -m21 / det;
  ri[1][1] = m22 / det;
  ri[2][1] = -m23 / det;
  ri[0][2] = m31 / det;
  ri[1][2] = -m32 / det;
  ri[2][2] = m33 / det;
  return true;
}

void put_bvh(const std::vector<BvhNode>& nodes, std::vector<double2>* out) {
  out->resize(nodes.size() * 7);
  for (size_t k = 0; k < nodes.size(); k++) {
    const BvhNode& n = nodes[k];
    double2* N = &(*out)[7 * k];
    N[0] = double2{n.lmin[0], n.lmin[1]};
    N[1] = double2{n.lmin[2], n.lmax[0]};
    N[2] = double2{n.lmax[1], n.lmax[2]};
    N[3] = double2{n.rmin[0], n.rmin[1]};
    N[4] = double2{n.rmin[2], n.rmax[0]};
    N[5] = double2{n.rmax[1], n.rmax[2]};
    N[6] = double2{pack2(n.lidx, n.lcnt), pack2(n.ridx, n.rcnt)};
  }
}

// A double rounded down (up) to a float: the float box holds the double one.
float float_down(double x) {
  if (x != x) return std::numeric_limits<float>::quiet_NaN();
  if (x >= (double)FLT_MAX) return FLT_MAX;
  if (x < -(double)FLT_MAX) return -std::numeric_limits<float>::infinity();
  float f = (float)x;
  return (double)f > x ? std::nextafter(f, -std::numeric_limits<float>::infinity()) : f;
}
float float_up(double x) { return -float_down(-x); }

// The single-precision copy of a BVH that the device walks test (the FNode
// layout of dscene.cuh, as mesh_prep.cu's k_prep_fbvh writes it for
// meshes): child boxes rounded outwards, references as they are, and in
// element 0 the largest |coordinate| of a present child's box (+inf when
// one is NaN, which turns the float tests off).
void put_fbvh(const std::vector<BvhNode>& nodes, std::vector<float4>* out) {
  out->assign(RTB_FBVH_HEAD + 4 * nodes.size(), float4{0.f, 0.f, 0.f, 0.f});
  float scale = 0.0f;
  for (size_t k = 0; k < nodes.size(); k++) {
    const BvhNode& n = nodes[k];
    float f[12];
    for (int a = 0; a < 3; a++) {
      f[a] = float_down(n.lmin[a]);
      f[3 + a] = float_up(n.lmax[a]);
      f[6 + a] = float_down(n.rmin[a]);
      f[9 + a] = float_up(n.rmax[a]);
    }
    for (int j = 0; j < 12; j++) {
      const float m = std::fabs(f[j]);
      if ((j < 6 ? n.lcnt : n.rcnt) >= 0 && (m > scale || m != m) && scale == scale) scale = m;
    }
    float4* F = &(*out)[RTB_FBVH_HEAD + 4 * k];
    auto bits = [](int v) {
      float x;
      memcpy(&x, &v, sizeof x);
      return x;
    };
    F[0] = float4{f[0], f[1], f[2], f[3]};
    F[1] = float4{f[4], f[5], f[6], f[7]};
    F[2] = float4{f[8], f[9], f[10], f[11]};
    F[3] = float4{bits(n.lidx), bits(n.lcnt), bits(n.ridx), bits(n.rcnt)};
  }
  (*out)[0].x = scale == scale ? scale : std::numeric_limits<float>::infinity();
}

// Everything the device needs for one mesh, computed on the host: triangle
// records in original and BVH order, normals, the reference k-d tree with
// root paths and occurrence lists, the BVH.  Pure function of the mesh
// description, so a host scene can keep it across uploads.  An upload
// copies the BVH, the BVH-order records and the k-d part; the device
// derives the records in mesh order, the normals and the occurrence lists
// from them (derive_mesh_device), so only prep_mesh(full = true) fills those.
struct MeshPrep {
  std::vector<double2> bvh, btris, brute, nodes;
  std::vector<float4> fbvh;  // the BVH in single precision (put_fbvh), which uploads copy
  std::vector<double4> normals;
  std::vector<int> leaf_tris, occ_off;
  std::vector<int2> leaf_path, occ;
  double bmin[3], bmax[3];
  int n_nodes = 0, n_tris = 0, n_index = 0;
  // Prepared on the device by the last upload: the records, normals, BVH
  // and occurrence arrays are not on the host (only the k-d part is).
  bool device_made = false;
  // Kept by a host scene, the five uploaded arrays are packed into one
  // pinned buffer (each at a 256-byte aligned offset; fbvh, btris, nodes,
  // leaf_tris, leaf_path) and the vectors released: uploads then copy the
  // image straight from pinned memory.
  static const int kImageArrays = 5;
  char* image = nullptr;
  size_t image_bytes = 0;
  size_t off[kImageArrays] = {}, len[kImageArrays] = {};
  ~MeshPrep() {
    if (image) cudaFreeHost(image);
  }
};

// Packs P's uploaded arrays into a pinned image (see MeshPrep); leaves P as
// it is if pinned memory cannot be had.
void pack_prep(MeshPrep* P) {
  const int K = MeshPrep::kImageArrays;
  const void* src[K] = {P->fbvh.data(), P->btris.data(), P->nodes.data(), P->leaf_tris.data(), P->leaf_path.data()};
  size_t n[K] = {P->fbvh.size() * sizeof(float4), P->btris.size() * sizeof(double2), P->nodes.size() * sizeof(double2),
                 P->leaf_tris.size() * sizeof(int), P->leaf_path.size() * sizeof(int2)};
  size_t total = 0;
  for (int k = 0; k < K; k++) {
    P->off[k] = total;
    P->len[k] = n[k];
    total += (std::max<size_t>(n[k], 16) + 255) & ~(size_t)255;
  }
  char* img = nullptr;
  if (cudaHostAlloc((void**)&img, total, cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  for (int k = 0; k < K; k++)
    if (n[k]) memcpy(img + P->off[k], src[k], n[k]);
  P->image = img;
  P->image_bytes = total;
  P->bvh = {};
  P->fbvh = {};
  P->btris = {};
  P->brute = {};
  P->normals = {};
  P->nodes = {};
  P->leaf_tris = {};
  P->leaf_path = {};
  P->occ = {};
  P->occ_off = {};
}

// Returns an empty string, or why the description is invalid.
// Host threads for a loop over n items (at least 64k items each).
int host_parts(long long n) {
  const long long hw = std::max(1u, std::thread::hardware_concurrency());
  return (int)std::max(1LL, std::min(hw, n / 65536));
}

// f(begin, end, part) over host_parts(n) contiguous ranges of [0, n), each
// on its own thread.
template <class F>
void parallel_ranges(long long n, F f) {
  const int parts = host_parts(n);
  if (parts == 1) {
    f(0LL, n, 0);
    return;
  }
  std::vector<std::thread> th;
  for (int p = 0; p < parts; p++) th.emplace_back([&f, n, parts, p] { f(n * p / parts, n * (p + 1) / parts, p); });
  for (auto& t : th) t.join();
}

// Triangles per mesh BVH leaf.  With single-precision box tests 4 is
// fastest on the 82k-triangle mesh frame (7.21 ms; 2: 7.31, 3: 7.26,
// 5: 7.28, 6: 7.30, 8: 7.39, 12: 7.68); with double boxes it was 8.
const int kMeshLeaf = 4;
// Meshes from this many triangles up are prepared on the device (median
// split BVH, tens of ms for millions of triangles); smaller ones on the
// host with a binned SAH BVH (about 7% fewer node visits per ray, 4% on the
// 82k-triangle mesh frame).
const long long kPrepDeviceMin = 262144;

// The part of a mesh's preparation that always runs on the host: checks,
// the reference k-d nodes packed for the device with each node's root path,
// the leaf lists.  Every leaf-list entry must name a triangle and belong to
// exactly one leaf (as in every tree KdTree::new builds).
std::string prep_mesh_kd(const rt_mesh_desc& md, MeshPrep* P) {
  for (int k = 0; k < 3; k++) {
    P->bmin[k] = md.bounds_min[k];
    P->bmax[k] = md.bounds_max[k];
  }
  long long nt = md.n_triangles;
  if (nt < 0 || md.n_nodes < 0 || md.n_tri_index < 0) return "negative count";
  if (nt > 0x3fffffffLL || md.n_nodes > 0x3fffffffLL || md.n_tri_index > 0x3fffffffLL)
    return "mesh too large";
  if ((nt > 0 && !md.vertices) || (md.n_nodes > 0 && !md.nodes) || (md.n_tri_index > 0 && !md.tri_index))
    return "null mesh array";
  std::vector<double2> nodes((size_t)md.n_nodes * 4);
  std::vector<int2> leaf_path((size_t)md.n_nodes, int2{0, 0});
  std::vector<char> covered((size_t)md.n_tri_index, 0);
  for (long long k = 0; k < md.n_nodes; k++) {
    const rt_kd_node_desc& nd = md.nodes[k];
    double2* N = &nodes[4 * k];
    N[0] = double2{nd.bounds_min[0], nd.bounds_min[1]};
    N[1] = double2{nd.bounds_min[2], nd.bounds_max[0]};
    N[2] = double2{nd.bounds_max[1], nd.bounds_max[2]};
    if (nd.axis < 0) {
      if (nd.first < 0 || nd.count < 0 || (long long)nd.first + nd.count > md.n_tri_index)
        return "k-d leaf range out of bounds";
      for (int p = 0; p < nd.count; p++)
        if (covered[nd.first + p]++) return "k-d leaves overlap";
      N[3] = double2{0.0, pack2(nd.first, -1 - nd.count)};
    } else {
      if (nd.axis > 2 || nd.right <= k + 1 || nd.right >= md.n_nodes)
        return "k-d node layout is not preorder";
      N[3] = double2{nd.split, pack2(nd.right, nd.axis)};
    }
  }
  for (char c : covered)
    if (!c) return "k-d leaf lists have entries in no leaf";
  if (md.n_nodes > 0) {
    std::vector<std::pair<int, int2>> st;  // node, {path bits, depth}
    st.push_back({0, int2{0, 0}});
    std::vector<char> seen((size_t)md.n_nodes, 0);
    while (!st.empty()) {
      int k = st.back().first;
      int2 pd = st.back().second;
      st.pop_back();
      if (seen[k]) return "k-d nodes do not form a tree";
      seen[k] = 1;
      leaf_path[k] = pd;
      const rt_kd_node_desc& nd = md.nodes[k];
      if (nd.axis >= 0) {
        if (pd.y >= 31) return "k-d tree deeper than 31 levels";
        st.push_back({k + 1, int2{pd.x, pd.y + 1}});
        st.push_back({nd.right, int2{pd.x | (1 << pd.y), pd.y + 1}});
      }
    }
  }
  std::vector<int> leaf_tris((size_t)md.n_tri_index);
  for (long long k = 0; k < md.n_tri_index; k++) {
    int t = md.tri_index[k];
    if (t < 0 || t >= nt) return "k-d leaf index out of range";
    leaf_tris[k] = t;
  }
  P->nodes = std::move(nodes);
  P->leaf_path = std::move(leaf_path);
  P->leaf_tris = std::move(leaf_tris);
  P->n_nodes = (int)md.n_nodes;
  P->n_tris = (int)nt;
  P->n_index = (int)md.n_tri_index;
  return std::string();
}

// A mesh's whole preparation on the host: the k-d part, then the triangle
// records, the triangle BVH (binned SAH, or sah = false the median split
// the device builds) and the records in BVH order; full = true also keeps
// the records in mesh order, the normals and the occurrence lists, which
// uploads derive on the device.
std::string prep_mesh(const rt_mesh_desc& md, MeshPrep* P, bool sah = true, bool full = false) {
  std::string e = prep_mesh_kd(md, P);
  if (!e.empty()) return e;
  const long long nt = md.n_triangles;
  // triangle records and normals in original order
  std::vector<double2> brute((size_t)nt * 5);
  std::vector<double4> normals(full ? (size_t)nt : 0);
  std::vector<double> tmin((size_t)nt * 3), tmax((size_t)nt * 3);
  std::vector<double> part_scale(host_parts(nt), 0.0);
  parallel_ranges(nt, [&](long long t0, long long t1, int part) {
    double scale = 0.0;
    for (long long t = t0; t < t1; t++) {
      const double* v = md.vertices + 9 * t;
      V3 v0 = mk(v[0], v[1], v[2]), v1 = mk(v[3], v[4], v[5]), v2 = mk(v[6], v[7], v[8]);
      V3 e1 = v1 - v0, e2 = v2 - v0;
      V3 n = cross(e1, e2);
      int degenerate = norm(n) < 1e-8 ? 1 : 0;  // src/ray.rs:565-567
      if (full) {
        V3 nn = normalize(n);
        normals[t] = double4{nn.x, nn.y, nn.z, 0.0};
      }
      double2* E = &brute[5 * t];
      E[0] = double2{v0.x, v0.y};
      E[1] = double2{v0.z, e1.x};
      E[2] = double2{e1.y, e1.z};
      E[3] = double2{e2.x, e2.y};
      E[4] = double2{e2.z, pack2((int)t, degenerate)};
      for (int k = 0; k < 3; k++) {
        double a = v[k], b = v[3 + k], c = v[6 + k];
        tmin[3 * t + k] = std::min(a, std::min(b, c));
        tmax[3 * t + k] = std::max(a, std::max(b, c));
        scale = std::max(scale, std::max(std::fabs(tmin[3 * t + k]), std::fabs(tmax[3 * t + k])));
      }
    }
    part_scale[part] = scale;
  });
  double scale = 0.0;
  for (double v : part_scale) scale = std::max(scale, v);
  // per-triangle occurrences (leaf node, position in the leaf), by leaf
  // node then position
  std::vector<int> occ_off;
  std::vector<int2> occ;
  if (full) {
    occ_off.assign((size_t)nt + 1, 0);
    for (int t : P->leaf_tris) occ_off[t + 1]++;
    for (long long t = 0; t < nt; t++) occ_off[t + 1] += occ_off[t];
    occ.resize((size_t)md.n_tri_index);
    std::vector<int> fill(occ_off.begin(), occ_off.end() - 1);
    for (long long k = 0; k < md.n_nodes; k++) {
      const rt_kd_node_desc& nd = md.nodes[k];
      if (nd.axis >= 0) continue;
      for (int p = 0; p < nd.count; p++) {
        int t = md.tri_index[nd.first + p];
        occ[fill[t]++] = int2{(int)k, p};
      }
    }
  }
  // triangle BVH, the candidate search structure
  std::vector<BvhNode> bnodes;
  std::vector<int32_t> order;
  if (sah)
    build_bvh_sah(tmin, tmax, kMeshLeaf, 1e-7 * (1.0 + scale), &bnodes, &order);
  else
    build_bvh(tmin, tmax, kMeshLeaf, 1e-7 * (1.0 + scale), &bnodes, &order);
  std::vector<double2> bvh, btris((size_t)nt * 5);
  if (full) put_bvh(bnodes, &bvh);
  put_fbvh(bnodes, &P->fbvh);
  parallel_ranges(nt, [&](long long k0, long long k1, int) {
    for (long long k = k0; k < k1; k++)
      for (int j = 0; j < 5; j++) btris[5 * k + j] = brute[5 * (size_t)order[k] + j];
  });
  P->bvh = std::move(bvh);
  P->btris = std::move(btris);
  if (full) {
    P->brute = std::move(brute);
    P->normals = std::move(normals);
    P->occ_off = std::move(occ_off);
    P->occ = std::move(occ);
  }
  return std::string();
}

template <class T>
rt_status upload_array(rt_ctx* ctx, rt_scene* sc, const std::vector<T>& h, const T** out) {
  char* dev = nullptr;
  rt_status st = upload_direct(ctx, sc, reinterpret_cast<const char*>(h.data()), h.size() * sizeof(T), &dev);
  *out = reinterpret_cast<const T*>(dev);
  return st;
}

// A region of the scene's block that a kernel will fill (no copy).
template <class T>
rt_status reserve(rt_ctx* ctx, rt_scene* sc, size_t count, T** dev) {
  const size_t bytes = count * sizeof(T);
  const size_t take = (std::max<size_t>(bytes, 16) + 255) & ~(size_t)255;
  if (sc->blk && sc->blk_used + take <= sc->blk_cap) {
    *dev = reinterpret_cast<T*>(sc->blk + sc->blk_used);
    sc->blk_used += take;
  } else {
    CK(dalloc(sc->allocs, dev, std::max<size_t>(count, 1)));
  }
  return RT_OK;
}

// A host array copied into the scene's block now, on the context's stream
// (for data a kernel of this upload reads).
template <class T>
rt_status upload_now(rt_ctx* ctx, rt_scene* sc, const std::vector<T>& h, const T** out) {
  T* dev = nullptr;
  rt_status st = reserve(ctx, sc, h.size(), &dev);
  if (st != RT_OK) return st;
  if (!h.empty()) CK(cudaMemcpyAsync(dev, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  sc->uploaded_bytes += h.size() * sizeof(T);
  *out = dev;
  return RT_OK;
}

// Prepares a large mesh on the device straight into the scene's block: P
// holds the k-d part (prep_mesh_kd).  keep_host: also copies the
// single-precision BVH and the BVH-order records back into P, so that
// later uploads copy them (upload_prep).
rt_status upload_prep_device(rt_ctx* ctx, rt_scene* sc, const rt_mesh_desc& md, MeshPrep* P, bool keep_host,
                             DMesh* out) {
  DMesh M{};
  for (int k = 0; k < 3; k++) {
    M.bmin[k] = P->bmin[k];
    M.bmax[k] = P->bmax[k];
  }
  M.n_nodes = P->n_nodes;
  M.n_tris = P->n_tris;
  const int n = P->n_tris, nb = bvh_internal_nodes(n, kMeshLeaf);
  rt_status st;
  double2 *bvh, *btris, *brute, *cells;
  float4* fbvh;
  double4* normals;
  int2* occ;
  int* occ_off;
  if ((st = upload_now(ctx, sc, P->nodes, &M.nodes)) != RT_OK || (st = upload_now(ctx, sc, P->leaf_tris, &M.leaf_tris)) != RT_OK ||
      (st = upload_now(ctx, sc, P->leaf_path, &M.leaf_path)) != RT_OK || (st = reserve(ctx, sc, 7 * (size_t)nb, &bvh)) != RT_OK ||
      (st = reserve(ctx, sc, RTB_FBVH_HEAD + 4 * (size_t)nb, &fbvh)) != RT_OK ||
      (st = reserve(ctx, sc, 3 * (size_t)P->n_nodes, &cells)) != RT_OK ||
      (st = reserve(ctx, sc, 5 * (size_t)n, &btris)) != RT_OK || (st = reserve(ctx, sc, 5 * (size_t)n, &brute)) != RT_OK ||
      (st = reserve(ctx, sc, (size_t)n, &normals)) != RT_OK || (st = reserve(ctx, sc, (size_t)P->n_index, &occ)) != RT_OK ||
      (st = reserve(ctx, sc, (size_t)n + 1, &occ_off)) != RT_OK)
    return st;
  if (!ctx->kd_arena) ctx->kd_arena = kd_arena_new();
  cudaError_t ce = cudaSuccess;
  std::string e = prep_mesh_device(md.vertices, n, M.nodes, P->n_nodes, M.leaf_tris, M.leaf_path, P->n_index,
                                   kMeshLeaf, ctx->stream, ctx->kd_arena,
                                   MeshPrepOut{bvh, fbvh, cells, btris, brute, normals, occ, occ_off}, &ce);
  if (ce != cudaSuccess) return cuda_fail(ctx, ce, e.c_str());
  if (!e.empty()) return fail(ctx, RT_ERR_INVALID_ARGUMENT, e);
  sc->uploaded_bytes += 9 * (size_t)n * sizeof(double);
  M.bvh = bvh;
  M.fbvh = fbvh;
  M.cells = cells;
  M.btris = btris;
  M.brute = brute;
  M.normals = normals;
  M.occ = occ;
  M.occ_off = occ_off;
  if (keep_host) {
    // what upload_prep copies; it derives the rest
    P->fbvh.resize(RTB_FBVH_HEAD + 4 * (size_t)nb);
    P->btris.resize(5 * (size_t)n);
    CK(cudaMemcpy(P->fbvh.data(), fbvh, P->fbvh.size() * sizeof(float4), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(P->btris.data(), btris, P->btris.size() * sizeof(double2), cudaMemcpyDeviceToHost));
    P->device_made = false;
  }
  *out = M;
  return RT_OK;
}

// Copies a prepared mesh into the scene's block: the BVH, the BVH-order
// records and the k-d part; the rest is derived on the device at the flush.
rt_status upload_prep(rt_ctx* ctx, rt_scene* sc, const MeshPrep& P, DMesh* out) {
  DMesh M{};
  for (int k = 0; k < 3; k++) {
    M.bmin[k] = P.bmin[k];
    M.bmax[k] = P.bmax[k];
  }
  M.n_nodes = P.n_nodes;
  M.n_tris = P.n_tris;
  rt_status st;
  if (P.image) {
    char* base = nullptr;
    if ((st = upload_direct(ctx, sc, P.image, P.image_bytes, &base)) != RT_OK) return st;
    M.fbvh = reinterpret_cast<const float4*>(base + P.off[0]);
    M.btris = reinterpret_cast<const double2*>(base + P.off[1]);
    M.nodes = reinterpret_cast<const double2*>(base + P.off[2]);
    M.leaf_tris = reinterpret_cast<const int*>(base + P.off[3]);
    M.leaf_path = reinterpret_cast<const int2*>(base + P.off[4]);
  } else {
    // not packed: each array straight from P's own memory (P outlives the flush)
    if ((st = upload_array(ctx, sc, P.fbvh, &M.fbvh)) != RT_OK || (st = upload_array(ctx, sc, P.btris, &M.btris)) != RT_OK ||
        (st = upload_array(ctx, sc, P.nodes, &M.nodes)) != RT_OK ||
        (st = upload_array(ctx, sc, P.leaf_tris, &M.leaf_tris)) != RT_OK ||
        (st = upload_array(ctx, sc, P.leaf_path, &M.leaf_path)) != RT_OK)
      return st;
  }
  const int n = P.n_tris;
  double2 *cells, *brute;
  double4* normals;
  int2* occ;
  int* occ_off;
  if ((st = reserve(ctx, sc, 3 * (size_t)P.n_nodes, &cells)) != RT_OK ||
      (st = reserve(ctx, sc, 5 * (size_t)n, &brute)) != RT_OK || (st = reserve(ctx, sc, (size_t)n, &normals)) != RT_OK ||
      (st = reserve(ctx, sc, (size_t)P.n_index, &occ)) != RT_OK ||
      (st = reserve(ctx, sc, (size_t)n + 1, &occ_off)) != RT_OK)
    return st;
  // the single-precision BVH is copied as it is: nothing to convert
  sc->derive.push_back(MeshDerive{nullptr, 0, nullptr, M.btris, n, M.nodes, P.n_nodes, M.leaf_tris, M.leaf_path,
                                  P.n_index, cells, brute, normals, occ, occ_off});
  M.cells = cells;
  M.brute = brute;
  M.normals = normals;
  M.occ = occ;
  M.occ_off = occ_off;
  *out = M;
  return RT_OK;
}


// Runs of at least this many consecutive spheres are searched through a BVH.
const int kMinSphereRun = 8;

// Uploads a scene description.  preps, when given, holds one prepared mesh
// per d->meshes entry (kept by a host scene); missing entries are prepared
// here and stored into it.
rt_status do_upload(rt_ctx* ctx, const rt_scene_desc* d, rt_scene** out,
                    std::vector<std::shared_ptr<MeshPrep>>* preps = nullptr) {
  if (!d) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null scene description");
  if (d->n_objects < 0 || d->n_materials < 0 || d->n_lights < 0 || d->n_meshes < 0)
    return fail(ctx, RT_ERR_INVALID_ARGUMENT, "negative count");
  if ((d->n_objects && !d->objects) || (d->n_materials && !d->materials) || (d->n_lights && !d->lights) ||
      (d->n_meshes && !d->meshes))
    return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null scene array");
  auto sc = std::make_unique<rt_scene>();
  sc->ctx = ctx;
  sc->device = ctx->device;
  sc->camera = d->camera;
  sc->outline = d->outline;
  sc->has_outline = d->has_outline;
  sc->render_error = d->render_error ? d->render_error : "";
  DScene& S = sc->S;
  for (int m = 0; m < d->n_meshes; m++)
    if (d->meshes[m].n_triangles < 0 || d->meshes[m].n_nodes < 0 || d->meshes[m].n_tri_index < 0)
      return fail(ctx, RT_ERR_INVALID_ARGUMENT, "negative count");
  {
    rt_status st = arena_open(ctx, sc.get(), scene_bytes_bound(d), scene_staged_bound(d));
    if (st != RT_OK) return st;
  }
  std::vector<DMesh> meshes(d->n_meshes);
  std::vector<std::shared_ptr<MeshPrep>> keep;  // the copies read them until the flush
  if (preps && preps->size() != (size_t)d->n_meshes) preps->assign(d->n_meshes, nullptr);
  for (int m = 0; m < d->n_meshes; m++) {
    const rt_mesh_desc& md = d->meshes[m];
    std::shared_ptr<MeshPrep> P = preps ? (*preps)[m] : nullptr;
    rt_status st;
    if (!P) {
      // first upload: large meshes are prepared on the device, into the block
      P = std::make_shared<MeshPrep>();
      const bool dev = md.n_triangles >= kPrepDeviceMin;
      std::string e = dev ? prep_mesh_kd(md, P.get()) : prep_mesh(md, P.get());
      if (!e.empty()) return fail(ctx, RT_ERR_INVALID_ARGUMENT, e);
      P->device_made = dev;
      if (preps) (*preps)[m] = P;
      keep.push_back(P);
      st = dev ? upload_prep_device(ctx, sc.get(), md, P.get(), false, &meshes[m])
               : upload_prep(ctx, sc.get(), *P, &meshes[m]);
    } else if (P->device_made) {
      // uploaded again: prepared on the device once more, and this time
      // the arrays stay on the host, as one pinned image for the uploads
      // after this one (pinning costs more than a copy, so the first
      // upload skips it)
      st = upload_prep_device(ctx, sc.get(), md, P.get(), true, &meshes[m]);
      if (st == RT_OK) pack_prep(P.get());
    } else {
      if (!P->image) pack_prep(P.get());
      keep.push_back(P);
      st = upload_prep(ctx, sc.get(), *P, &meshes[m]);
    }
    if (st != RT_OK) return st;
  }
  std::vector<int4> obj;
  std::vector<double> sph, pln;
  std::vector<int> sph_mat;
  std::vector<DCube> cub;
  for (int i = 0; i < d->n_objects; i++) {
    const rt_object_desc& o = d->objects[i];
    if (o.material < 0 || o.material >= d->n_materials)
      return fail(ctx, RT_ERR_INVALID_ARGUMENT, "material index out of range");
    sc->obj_kind.push_back(o.kind);
    sc->obj_mesh.push_back(o.kind == RT_OBJ_MESH ? o.mesh : -1);
    if (o.kind == RT_OBJ_SPHERE) {
      int si = (int)(sph.size() / 5);
      sph.insert(sph.end(), {o.a[0], o.a[1], o.a[2], o.radius, o.radius * o.radius});
      sph_mat.push_back(o.material);
      obj.push_back(int4{OBJ_SPHERE, si, o.material, i});
    } else if (o.kind == RT_OBJ_PLANE) {
      int pi = (int)(pln.size() / 12);
      V3 n = mk(o.b[0], o.b[1], o.b[2]);
      // Plane::hit's texture axes (src/ray.rs:161-167)
      V3 ua = fabs(n.x) > 0.9 ? mk(0, 1, 0) : mk(1, 0, 0);
      V3 uax = normalize(cross(ua, n));
      V3 vax = normalize(cross(n, uax));
      pln.insert(pln.end(), {o.a[0], o.a[1], o.a[2], n.x, n.y, n.z, uax.x, uax.y, uax.z, vax.x, vax.y, vax.z});
      obj.push_back(int4{OBJ_PLANE, pi, o.material, i});
    } else if (o.kind == RT_OBJ_CUBE) {
      DCube C{};
      for (int k = 0; k < 3; k++) {
        C.c[k] = o.a[k];
        C.half[k] = o.b[k] / 2.0;
      }
      double tm[16], inv[16];
      for (int k = 0; k < 16; k++) tm[k] = o.has_transform ? o.transform[k] : ((k % 5) == 0 ? 1.0 : 0.0);
      if (!o.has_transform || !inverse4(tm, inv))
        for (int k = 0; k < 16; k++) inv[k] = (k % 5) == 0 ? 1.0 : 0.0;
      for (int k = 0; k < 12; k++) {
        C.w2l[k] = inv[k];
        C.l2w[k] = tm[k];
      }
      bool ident = true;
      for (int k = 0; k < 16; k++)
        if (inv[k] != ((k % 5) == 0 ? 1.0 : 0.0)) ident = false;
      C.identity = ident ? 1 : 0;
      // normal transform: inverse of w2l's rotation part, transposed (src/ray.rs:474-481)
      double a[3][3], ri[3][3];
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) a[r][c] = inv[4 * r + c];
      if (!inverse3(a, ri))
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 3; c++) ri[r][c] = r == c ? 1.0 : 0.0;
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) C.ntr[3 * r + c] = ri[c][r];
      obj.push_back(int4{OBJ_CUBE, (int)cub.size(), o.material, i});
      cub.push_back(C);
    } else if (o.kind == RT_OBJ_MESH) {
      if (o.mesh < 0 || o.mesh >= d->n_meshes) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "mesh index out of range");
      obj.push_back(int4{OBJ_MESH, o.mesh, o.material, i});
    } else {
      return fail(ctx, RT_ERR_INVALID_ARGUMENT, "unknown object kind");
    }
  }
  // Long runs of consecutive spheres become one BVH group entry.
  std::vector<DSphGroup> groups;
  std::vector<int4> entries;
  for (size_t k = 0; k < obj.size();) {
    size_t e = k;
    while (e < obj.size() && obj[e].x == OBJ_SPHERE) e++;
    int run = (int)(e - k);
    if (run >= kMinSphereRun) {
      int first_sph = obj[k].y;
      std::vector<double> bmin(3 * (size_t)run), bmax(3 * (size_t)run);
      double scale = 0.0;
      for (int s = 0; s < run; s++) {
        const double* sp = &sph[5 * (size_t)(first_sph + s)];
        double r = std::fabs(sp[3]);
        for (int c = 0; c < 3; c++) {
          bmin[3 * s + c] = sp[c] - r;
          bmax[3 * s + c] = sp[c] + r;
          scale = std::max(scale, std::fabs(sp[c]) + r);
        }
      }
      std::vector<BvhNode> bn;
      std::vector<int32_t> order;
      // leaves of 4 spheres: 47.6 ms for the 1,000-sphere ring frame (1080p,
      // 4 spp) against 49.4 ms with 8 or 12
      build_bvh(bmin, bmax, 4, 1e-6 * (1.0 + scale), &bn, &order);
      std::vector<float4> fbvh;
      put_fbvh(bn, &fbvh);  // the walks test single-precision boxes only
      DSphGroup G{};
      const float4* pf;
      rt_status st = upload(ctx, sc.get(), fbvh, &pf);
      if (st != RT_OK) return st;
      G.fbvh = pf;
      std::vector<int> ord(order.begin(), order.end());
      const int* po;
      st = upload(ctx, sc.get(), ord, &po);
      if (st != RT_OK) return st;
      G.order = po;
      G.first_sphere = first_sph;
      G.first_obj = obj[k].w;
      G.count = run;
      entries.push_back(int4{OBJ_SPHERE_GROUP, (int)groups.size(), -1, obj[k].w});
      groups.push_back(G);
      k = e;
    } else if (run > 0) {
      for (size_t j = k; j < e; j++) entries.push_back(obj[j]);
      k = e;
    } else {
      entries.push_back(obj[k]);
      k++;
    }
  }
  std::vector<DMat> mats(d->n_materials);
  for (int i = 0; i < d->n_materials; i++) {
    const rt_material_desc& m = d->materials[i];
    DMat& M = mats[i];
    M = DMat{};
    for (int k = 0; k < 3; k++) M.color[k] = m.color[k];
    M.ambient = m.ambient;
    M.diffuse = m.diffuse;
    M.specular = m.specular;
    M.shininess = m.shininess;
    M.refl = m.reflectivity;
    M.has_refl = m.has_reflectivity;
    M.texture = m.texture;
    // the grid colour is formatted as #RRGGBB from (c * 255) as u8 and parsed
    // back (src/lighting.rs:28-36)
    for (int k = 0; k < 3; k++) M.grid_color[k] = (double)sat_u8(m.grid_line_color[k] * 255.0) / 255.0;
    M.half_width = m.grid_line_width / 2.0;
    M.cell_size = m.grid_cell_size;
    for (int k = 0; k < 3; k++) M.cb_color[k] = m.checker_color[k];
    M.cb_ambient = m.checker_ambient;
    M.cb_diffuse = m.checker_diffuse;
    M.cb_specular = m.checker_specular;
    M.cb_shininess = m.checker_shininess;
  }
  std::vector<DLight> lights(d->n_lights);
  int K = 0;
  for (int i = 0; i < d->n_lights; i++) {
    const rt_light_desc& l = d->lights[i];
    DLight& L = lights[i];
    L = DLight{};
    for (int k = 0; k < 3; k++) {
      L.pos[k] = l.position[k];
      L.color[k] = l.color[k];
    }
    L.intensity = l.intensity;
    L.disk = l.has_diameter ? 1 : 0;
    L.diameter = l.diameter;
    K += L.disk ? 16 : 1;
    (L.disk ? sc->n_disk_lights : sc->n_point_lights)++;
  }
  rt_status st;
  const int4* po4;
  if ((st = upload(ctx, sc.get(), entries, &po4)) != RT_OK) return st;
  S.obj = po4;
  const double* pd;
  if ((st = upload(ctx, sc.get(), sph, &pd)) != RT_OK) return st;
  S.sph = pd;
  const int* pmi;
  if ((st = upload(ctx, sc.get(), sph_mat, &pmi)) != RT_OK) return st;
  S.sph_mat = pmi;
  if ((st = upload(ctx, sc.get(), pln, &pd)) != RT_OK) return st;
  S.pln = pd;
  const DCube* pc;
  if ((st = upload(ctx, sc.get(), cub, &pc)) != RT_OK) return st;
  S.cub = pc;
  const DMesh* pm;
  if ((st = upload(ctx, sc.get(), meshes, &pm)) != RT_OK) return st;
  S.mesh = pm;
  const DSphGroup* pg;
  if ((st = upload(ctx, sc.get(), groups, &pg)) != RT_OK) return st;
  S.grp = pg;
  const DMat* pmt;
  if ((st = upload(ctx, sc.get(), mats, &pmt)) != RT_OK) return st;
  S.mat = pmt;
  const DLight* pl;
  if ((st = upload(ctx, sc.get(), lights, &pl)) != RT_OK) return st;
  S.lights = pl;
  S.n_obj = (int)entries.size();
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
  {
    rt_status st = arena_flush(ctx, sc.get());
    if (st != RT_OK) return st;
  }
  *out = sc.release();
  return RT_OK;
}

// Counts launches and, for profiling renders, records an event after each
// one so that stage times can be attributed.
struct Launcher {
  rt_ctx* ctx;
  bool timed;
  unsigned launches = 0;
  std::vector<std::pair<int, cudaEvent_t>> marks;
  int ev_used = 0;
  cudaEvent_t next_event() {
    if (ev_used >= (int)ctx->stage_ev.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      ctx->stage_ev.push_back(e);
    }
    return ctx->stage_ev[ev_used++];
  }
  void begin() {
    if (!timed) return;
    cudaEvent_t e = next_event();
    cudaEventRecord(e, ctx->stream);
    marks.push_back({-1, e});
  }
  void after(int stage) {
    launches++;
    if (!timed) return;
    cudaEvent_t e = next_event();
    cudaEventRecord(e, ctx->stream);
    marks.push_back({stage, e});
  }
  void collect(double* stage_ms) {
    for (size_t k = 1; k < marks.size(); k++) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, marks[k - 1].second, marks[k].second);
      if (marks[k].first >= 0) stage_ms[marks[k].first] += ms;
    }
  }
};

// Renders image rows [row_begin, row_end) (the whole image when they are 0
// and height) into rgb_out / linear_out, which hold those rows only.  A band
// with the outline on traces 1 + radius extra rows on each inner side: the
// edge mask of a kept row reads its neighbours' G-buffers and the dilation
// reads masks up to radius rows away, so the extra rows make every kept
// pixel's inputs those of the whole-image render.
// Optional per-sample outputs of the primary hits (device pointers).
struct AovOut {
  float* vis = nullptr;   // [plane][DN_MAX_SLOTS][H][W]
  __half* feat = nullptr; // [plane][H][W][FEAT_CHANNELS]
};

// A frame set up for a fused multi-frame launch (rt_render_batch): its
// arguments, validated as rt_render validates them, with the context's
// scratch sized and the frame's launch block filled, but nothing launched.
struct FramePlan {
  DFrame F;
  int levels = 1;
  long long nprim = 0, npix = 0, chunk = 0;
  int K = 0;
  uint8_t* rgb_out = nullptr;  // where the image goes
  int on_device = 0;
  bool direct = false;         // the kernels write rgb_out themselves
  uint8_t* d_rgb = nullptr;    // else the image in the context's scratch
  std::chrono::steady_clock::time_point t0;
};

rt_status render_impl(rt_ctx* ctx, const rt_scene* sc, const rt_render_params* P, uint32_t row_begin,
                      uint32_t row_end, uint8_t* rgb_out, int on_device, double* linear_out, rt_stats* stats,
                      const AovOut* aov = nullptr, const rt_camera_config* camera = nullptr,
                      FramePlan* plan = nullptr) {
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
  const rt_camera_config& camcfg = camera ? *camera : sc->camera;
  if (!make_camera(camcfg, aspect, &cam, &cerr)) return fail(ctx, RT_ERR_RENDER, cerr);
  if (!sc->render_error.empty()) return fail(ctx, RT_ERR_RENDER, sc->render_error);
  CK(cudaSetDevice(ctx->device));

  const int W = (int)P->width, Himg = (int)P->height;
  if (row_begin >= row_end || row_end > P->height)
    return fail(ctx, RT_ERR_INVALID_ARGUMENT, "row range must satisfy row_begin < row_end <= height");
  const int aa = P->anti_aliasing_mode;
  const bool outline = aa != RT_AA_QUINCUNX && P->outline.enabled;
  int o_radius = 0;
  if (outline && P->outline.line_thickness > 1.0) {
    double rr = std::ceil(P->outline.line_thickness - 1.0);
    if (!(rr <= kOutlineMaxRadius))
      return fail(ctx, RT_ERR_INVALID_ARGUMENT, "outline thickness above 2049 is not supported");
    o_radius = (int)rr;
  }
  const int halo = outline ? 1 + o_radius : 0;
  const int y0 = std::max(0, (int)row_begin - halo);
  const int H = std::min(Himg, (int)row_end + halo) - y0;  // rows traced
  const long long keep_off = (long long)((int)row_begin - y0) * W;
  const long long keep_pix = (long long)(row_end - row_begin) * W;
  const int spp = aa == RT_AA_QUINCUNX ? 1 : (int)P->samples;
  long long npix = (long long)W * H;
  long long ncorner = aa == RT_AA_QUINCUNX ? (long long)(W + 1) * (H + 1) : 0;
  long long nprim = aa == RT_AA_QUINCUNX ? ncorner + npix : npix * spp;
  if (nprim > 0x7fffffffLL) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "too many rays for one render");
  int max_depth = P->max_depth;
  if (max_depth > RTB_MAX_LEVELS) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "max_depth above 64 is not supported");
  int levels = std::max(1, std::min(max_depth, RTB_MAX_LEVELS));
  // Shadow rays per hit: 1 per point light, dsamp per disk light (16 in the
  // reference).  Learned shadows cast 1 per disk light at level 0.
  if (P->disk_samples > 4096) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "disk_samples above 4096 is not supported");
  const int dsamp = P->disk_samples ? (int)P->disk_samples : 16;
  const bool learned = P->learned_shadows != 0 && sc->n_disk_lights > 0;
  const bool want_aov = aov && (aov->vis || aov->feat);
  const bool full_frame = row_begin == 0 && row_end == P->height;
  if (learned || want_aov) {
    if (aa == RT_AA_QUINCUNX)
      return fail(ctx, RT_ERR_INVALID_ARGUMENT, "learned shadows and shadow AOVs need no-jitter or stochastic sampling");
    if (!full_frame) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "learned shadows and shadow AOVs render whole frames");
  }
  if (learned) {
    if (sc->n_disk_lights > DN_MAX_SLOTS)
      return fail(ctx, RT_ERR_INVALID_ARGUMENT, "learned shadows support at most two disk lights");
    if (!ctx->net.loaded()) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "learned shadows need rt_denoiser_load first");
  }
  if (P->learned_rays > 16) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "learned_rays above 16 is not supported");
  if (P->fallback_samples > 4096)
    return fail(ctx, RT_ERR_INVALID_ARGUMENT, "fallback_samples above 4096 is not supported");
  if (!(P->confidence_threshold == P->confidence_threshold))
    return fail(ctx, RT_ERR_INVALID_ARGUMENT, "confidence_threshold is NaN");
  const int lrays = learned ? (P->learned_rays ? (int)P->learned_rays : ctx->net.rays_per_light) : 0;
  const int K_full = sc->n_point_lights + sc->n_disk_lights * dsamp;
  const int K_0 = learned ? sc->n_point_lights + sc->n_disk_lights * lrays : K_full;
  // Confidence-gated fallback: level-0 hits whose estimated visibility error
  // exceeds the threshold are shaded by the plain path with fb_dsamp rays
  // per disk light.  Threshold 0: the one stored with the weights; < 0: off.
  const bool fallback = learned && ctx->net.has_conf && P->confidence_threshold >= 0.0f;
  const float conf_thr = P->confidence_threshold > 0.0f ? P->confidence_threshold : ctx->net.conf_threshold;
  const int fb_dsamp = P->fallback_samples ? (int)P->fallback_samples : dsamp;
  const int K_fb = sc->n_point_lights + sc->n_disk_lights * fb_dsamp;
  auto chunk_for = [&](int K) { return K > 0 ? std::max(1LL, std::min(nprim, kShadowCap / K)) : nprim; };
  const long long chunk_0 = chunk_for(K_0), chunk_n = chunk_for(K_full), chunk_fb = fallback ? chunk_for(K_fb) : 1;
  if (learned && chunk_0 < nprim)
    return fail(ctx, RT_ERR_INVALID_ARGUMENT, "too many primary samples for learned shadows in one pass");
  long long n_shadow = std::max(1LL, std::max(chunk_0 * std::max(K_0, 1), chunk_n * std::max(K_full, 1)));
  if (fallback) n_shadow = std::max(n_shadow, chunk_fb * std::max(K_fb, 1));
  rt_status st = ensure_scratch(ctx, nprim, levels, npix, n_shadow, std::max(std::max(chunk_0, chunk_n), chunk_fb));
  if (st != RT_OK) return st;
  if (learned || want_aov) {
    st = ensure_dn_scratch(ctx, nprim);
    if (st != RT_OK) return st;
  }
  if (learned) {
    st = ensure_dn_arena(ctx, denoise_scratch_halves(ctx->net, spp, H, W));
    if (st != RT_OK) return st;
  }

  DFrame F = ctx->F;
  F.S = sc->S;
  for (int k = 0; k < 3; k++) {
    F.C.origin[k] = cam.origin[k];
    F.C.hor[k] = cam.horizontal[k];
    F.C.ver[k] = cam.vertical[k];
    F.C.llc[k] = cam.llc[k];
    F.C.vdir[k] = cam.view_dir[k];
    F.C.campos[k] = camcfg.position[k];
    F.C.gcolor[k] = cam.grid_color[k];
  }
  F.C.persp = cam.persp;
  F.C.grid = cam.grid_enabled;
  F.C.pitch = cam.grid_pitch;
  F.C.half_th = cam.grid_half_thickness;
  F.W = W;
  F.H = H;
  F.y0 = y0;
  F.Himg = Himg;
  F.S_per_px = spp;
  F.aa = aa;
  F.max_depth = max_depth;
  F.use_kd = P->use_kdtree ? 1 : 0;
  F.camera_mode = aa == RT_AA_QUINCUNX ? 0 : 1;  // quincunx passes camera = None
  F.outline = outline ? 1 : 0;
  F.seed = P->seed;
  F.n_primary = nprim;
  F.n_corner = ncorner;
  F.levels = ctx->d_levels;
  F.counts = ctx->d_counts;
  F.nhits = ctx->d_nhits;
  F.chunk_hits = chunk_0;
  F.K = K_0;
  F.dsamp = dsamp;
  F.learned = learned ? 1 : 0;
  F.feat_on = (learned || want_aov) ? 1 : 0;
  F.feat = (aov && aov->feat) ? aov->feat : ctx->d_feat;
  F.vhat = (aov && aov->vis) ? aov->vis : ctx->d_vhat;
  F.vis_aov = (aov && aov->vis && !learned) ? aov->vis : nullptr;
  F.n_slots = std::min(sc->n_disk_lights, (int)DN_MAX_SLOTS);
  F.vconf = learned ? ctx->d_vconf : nullptr;
  F.conf_thr = conf_thr;
  F.fb_mode = 0;
  F.fb_list = fallback ? ctx->d_fb_list : nullptr;
  F.fbn = fallback ? ctx->d_fbn : nullptr;
  F.fb_flag = fallback ? ctx->d_fb_flag : nullptr;
  F.stats = ctx->d_stats;
  F.err = ctx->d_err;
  F.linear = nullptr;
  F.o_wd = P->outline.depth_weight;
  F.o_wn = P->outline.normal_weight;
  F.o_thr = P->outline.threshold;
  for (int k = 0; k < 3; k++) F.o_color[k] = P->outline.edge_color[k];
  F.o_thick = P->outline.line_thickness;
  F.o_wid = P->outline.object_id_weight;
  F.o_use8 = P->outline.use_8_neighbors ? 1 : 0;
  F.o_radius = o_radius;
  double* d_linear = nullptr;
  std::vector<void*> tmp;
  if (linear_out) {
    cudaError_t e = dalloc(tmp, &d_linear, 3 * npix);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc(linear)");
    F.linear = d_linear;
  }
  uint8_t* d_rgb = F.rgb;
  const bool direct = rgb_out && on_device && keep_off == 0 && keep_pix == npix;
  if (direct) F.rgb = rgb_out;
  if (plan) {
    // one launch block for every level (no learned level 0), one shadow
    // chunk, whole frame, no outline pass, no linear copy
    if (learned || want_aov || linear_out || F.outline || !full_frame || max_depth <= 0 || chunk_n < nprim ||
        !rgb_out)
      return fail(ctx, RT_ERR_INVALID_ARGUMENT, "this frame cannot join a fused batch group");
    plan->F = F;
    plan->levels = levels;
    plan->nprim = nprim;
    plan->npix = npix;
    plan->chunk = chunk_n;
    plan->K = K_full;
    plan->rgb_out = rgb_out;
    plan->on_device = on_device;
    plan->direct = direct;
    plan->d_rgb = d_rgb;
    plan->t0 = t0;
    return RT_OK;
  }

  const bool count = (P->flags & RT_FLAG_COUNT_WORK) != 0;
  Launcher Lc{ctx, (P->flags & RT_FLAG_STAGE_TIMES) != 0};
  cudaStream_t s = ctx->stream;
  int nsm = ctx->num_sms;
  auto blocks = [&](long long n, int bs, int per_sm) {
    long long b = (n + bs - 1) / bs;
    long long cap = (long long)nsm * per_sm;
    return (int)std::max<long long>(1, std::min(b, cap));
  };
  // k_shadow's register budget: 7 blocks per SM where the walk reaches mesh
  // leaves (triangle tests, k-d verification), 8 for spheres and planes only
  const bool mesh_scene = !sc->host_meshes.empty();
  auto launch_shadow = [&](const DFrame& Fs, int level, long long c0, int grid) {
    if (count) {
      if (mesh_scene) k_shadow<true, 7><<<grid, 128, 0, s>>>(Fs, level, c0);
      else k_shadow<true, 8><<<grid, 128, 0, s>>>(Fs, level, c0);
    } else {
      if (mesh_scene) k_shadow<false, 7><<<grid, 128, 0, s>>>(Fs, level, c0);
      else k_shadow<false, 8><<<grid, 128, 0, s>>>(Fs, level, c0);
    }
  };
  const bool o_wide = o_radius > kOutlineTileRadius;  // mask tile beyond shared memory: global-memory dilation
  const size_t o_shm = o_wide ? 0 : (size_t)(OT_X + 2 * o_radius) * (OT_Y + 2 * o_radius) * sizeof(double);
  if (F.outline && o_shm > 48 * 1024) CK(outline_smem_attr((int)o_shm));
  // The frame's device work, from queue reset to outline: launched directly,
  // or captured into a CUDA graph.  Every argument it passes comes from F
  // and the values the graph key lists below.
  auto enqueue = [&]() -> rt_status {
    k_frame_init<<<1, 128, 0, s>>>(F, levels);
    Lc.after(RT_STAGE_RAYGEN);
    if (max_depth > 0) {
      k_raygen<<<blocks(nprim, 256, 16), 256, 0, s>>>(F);
      Lc.after(RT_STAGE_RAYGEN);
      for (int l = 0; l < levels; l++) {
        // per-level shadow layout (k_emit/k_shadow/k_resolve read it from F)
        const int K = l == 0 ? K_0 : K_full;
        const long long chunk = l == 0 ? chunk_0 : chunk_n;
        F.K = K;
        F.chunk_hits = chunk;
        F.dsamp = (l == 0 && learned) ? lrays : dsamp;
        const bool feat = l == 0 && F.feat_on;
        const long long nchunks = (nprim + chunk - 1) / chunk;
        // The walks' grids hold many more blocks than stay resident (64 per
        // SM for k_trace, 128 for k_shadow), each striding over a few warps
        // of rays: blocks whose rays finish early are replaced by the block
        // scheduler, where one long-striding block per slot left its SM
        // half idle at the end.  Bench frame: 8.18 ms at 16 / 32, 7.55 ms
        // at 64 / 128; one block per 128 rays was slower (8.66 ms).
        if (count) k_trace<true><<<blocks(nprim, 128, 64), 128, 0, s>>>(F, l);
        else k_trace<false><<<blocks(nprim, 128, 64), 128, 0, s>>>(F, l);
        Lc.after(RT_STAGE_TRACE);
        if (feat) {
          CK(cudaMemsetAsync(F.feat, 0, (size_t)nprim * FEAT_CHANNELS * sizeof(__half), s));
          if (F.vis_aov) CK(cudaMemsetAsync(F.vis_aov, 0, (size_t)nprim * DN_MAX_SLOTS * sizeof(float), s));
        }
        for (long long c = 0; c < nchunks; c++) {
          long long c0 = c * chunk;
          // 64 blocks per SM as for k_trace: emit stage 0.97 ms against 1.03 ms at 16
          k_emit<<<blocks(chunk, 128, 64), 128, 0, s>>>(F, l, c0);
          Lc.after(RT_STAGE_EMIT);
          if (K > 0) {
            launch_shadow(F, l, c0, blocks(chunk * K, 128, 128));
            Lc.after(RT_STAGE_SHADOW);
          }
          if (feat) {
            k_features<<<blocks(chunk, 128, 16), 128, 0, s>>>(F, c0);
            Lc.after(RT_STAGE_DENOISE);
          }
          if (l == 0 && learned) continue;  // resolved after the denoiser (one chunk)
          k_resolve<<<blocks(chunk, 128, 16), 128, 0, s>>>(F, l, c0);
          Lc.after(RT_STAGE_RESOLVE);
        }
        if (feat) {
          k_feat_pixel_mean<<<blocks(npix, 128, 16), 128, 0, s>>>(F);
          Lc.after(RT_STAGE_DENOISE);
        }
        if (l == 0 && learned) {
          cudaError_t le = cudaSuccess;
          int nl = denoise_run(ctx->net, F.feat, spp, H, W, ctx->d_dn_arena, F.vhat, F.vconf, F.err, s, nsm, &le);
          for (int k = 0; k < nl; k++) Lc.after(RT_STAGE_DENOISE);
          if (le != cudaSuccess) return cuda_fail(ctx, le, "denoiser launch");
          if (fallback) {
            // the hits the network is not confident about: plain shading
            // with fb_dsamp rays per disk light, over the compacted list
            k_fb_select<<<blocks(nprim, 128, 16), 128, 0, s>>>(F);
            Lc.after(RT_STAGE_DENOISE);
            DFrame Fb = F;
            Fb.fb_mode = 1;
            Fb.learned = 0;
            Fb.dsamp = fb_dsamp;
            Fb.K = K_fb;
            Fb.chunk_hits = chunk_fb;
            const long long nfb_chunks = (nprim + chunk_fb - 1) / chunk_fb;  // the list holds at most nprim hits
            for (long long c = 0; c < nfb_chunks; c++) {
              const long long c0 = c * chunk_fb;
              k_emit<<<blocks(chunk_fb, 128, 64), 128, 0, s>>>(Fb, 0, c0);
              Lc.after(RT_STAGE_EMIT);
              if (K_fb > 0) {
                launch_shadow(Fb, 0, c0, blocks(chunk_fb * K_fb, 128, 128));
                Lc.after(RT_STAGE_SHADOW);
              }
              k_resolve<<<blocks(chunk_fb, 128, 16), 128, 0, s>>>(Fb, 0, c0);
              Lc.after(RT_STAGE_RESOLVE);
            }
          }
          k_resolve<<<blocks(chunk, 128, 16), 128, 0, s>>>(F, l, 0);
          Lc.after(RT_STAGE_RESOLVE);
        }
      }
      for (int l = levels - 2; l >= 0; l--) {
        k_fold<<<blocks(nprim, 256, 16), 256, 0, s>>>(F, l);
        Lc.after(RT_STAGE_FOLD);
      }
    }
    k_pixels<<<blocks(npix, 256, 16), 256, 0, s>>>(F);
    Lc.after(RT_STAGE_POST);
    if (F.outline) {
      dim3 ob(OT_X, OT_Y), og((W + OT_X - 1) / OT_X, (H + OT_Y - 1) / OT_Y);
      k_outline_mask<<<og, ob, 0, s>>>(F);
      Lc.after(RT_STAGE_POST);
      if (o_wide) k_outline_apply_wide<<<blocks(npix, 256, 8), 256, 0, s>>>(F);
      else k_outline_apply<<<og, ob, o_shm, s>>>(F);
      Lc.after(RT_STAGE_POST);
    }
    CK(cudaGetLastError());
    return RT_OK;
  };
  // CUDA graph: not with stage times (events between launches) nor with a
  // linear output (a per-call buffer, so no key would ever repeat).
  uint32_t graph_state = 0;
  if ((P->flags & RT_FLAG_CUDA_GRAPH) && !Lc.timed && !linear_out) {
    std::vector<unsigned char> key;
    auto put = [&key](const void* p, size_t n) {
      key.insert(key.end(), static_cast<const unsigned char*>(p), static_cast<const unsigned char*>(p) + n);
    };
    put(&F, sizeof F);
    const long long kl[] = {nprim, npix, chunk_0, chunk_n, levels, max_depth, K_0, K_full, lrays, dsamp,
                            learned, count, nsm, spp, H, W, (long long)o_shm, fallback, fb_dsamp, K_fb, chunk_fb};
    put(kl, sizeof kl);
    if (learned) {
      const void* ap[] = {ctx->d_dn_arena};
      put(ap, sizeof ap);
      for (const DnOp& o : ctx->net.ops) {
        const void* lp[] = {o.w, o.b};
        const int li[] = {o.kind, o.cin, o.cout, o.dil, o.act, o.src, o.src2, o.level};
        put(lp, sizeof lp);
        put(li, sizeof li);
      }
    }
    GraphEntry* hit = nullptr;
    for (GraphEntry& g : ctx->graphs)
      if (g.key == key) hit = &g;
    if (!hit) {
      cudaGraph_t g = nullptr;
      CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      rt_status es = enqueue();
      cudaError_t ce = cudaStreamEndCapture(s, &g);  // always ends the capture
      if (es != RT_OK) {
        if (g) cudaGraphDestroy(g);
        return es;
      }
      if (ce != cudaSuccess) return cuda_fail(ctx, ce, "cudaStreamEndCapture");
      cudaGraphExec_t ex = nullptr;
      ce = cudaGraphInstantiate(&ex, g, 0);
      cudaGraphDestroy(g);
      if (ce != cudaSuccess) return cuda_fail(ctx, ce, "cudaGraphInstantiate");
      if (ctx->graphs.size() >= kMaxGraphs) {
        auto lru = std::min_element(ctx->graphs.begin(), ctx->graphs.end(),
                                    [](const GraphEntry& a, const GraphEntry& b) { return a.used < b.used; });
        cudaGraphExecDestroy(lru->exec);
        ctx->graphs.erase(lru);
      }
      ctx->graphs.push_back(GraphEntry{std::move(key), ex, Lc.launches, 0});
      hit = &ctx->graphs.back();
      graph_state = 1;
    } else {
      Lc.launches = hit->launches;
      graph_state = 2;
    }
    hit->used = ++ctx->graph_tick;
    CK(cudaEventRecord(ctx->ev0, s));
    CK(cudaGraphLaunch(hit->exec, s));
  } else {
    CK(cudaEventRecord(ctx->ev0, s));
    Lc.begin();
    rt_status es = enqueue();
    if (es != RT_OK) return es;
  }
  CK(cudaEventRecord(ctx->ev1, s));
  if (rgb_out && !direct)
    CK(cudaMemcpyAsync(rgb_out, d_rgb + 3 * keep_off, 3 * keep_pix,
                       on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
  if (linear_out)
    CK(cudaMemcpyAsync(linear_out, d_linear + 3 * keep_off, 3 * keep_pix * sizeof(double), cudaMemcpyDeviceToHost,
                       s));
  std::vector<int> counts(levels + 2, 0), nh(levels + 1, 0);
  unsigned long long hstats[16];
  int herr = 0;
  CK(cudaMemcpyAsync(counts.data(), ctx->d_counts, (levels + 2) * sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(nh.data(), ctx->d_nhits, (levels + 1) * sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(hstats, ctx->d_stats, sizeof hstats, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&herr, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  int hfb[2] = {0, 0};  // fallback hits, fallback slots
  if (fallback) CK(cudaMemcpyAsync(hfb, ctx->d_fbn, sizeof hfb, cudaMemcpyDeviceToHost, s));
  cudaError_t se = cudaStreamSynchronize(s);
  free_all(tmp);
  if (se != cudaSuccess) return cuda_fail(ctx, se, "render");
  if (herr & ERR_EMPTY_RANGE) return fail(ctx, RT_ERR_RENDER, "cannot sample empty range");
  if (herr & ERR_RANGE_OVERFLOW) return fail(ctx, RT_ERR_RENDER, "UniformSampler::sample_single: range overflow");
  if (herr & DN_ERR_WAIT) return fail(ctx, RT_ERR_DEVICE_WATCHDOG, "denoiser: a tensor-core wait timed out");
  if (herr & (ERR_WATCHDOG | ERR_STACK))
    return fail(ctx, RT_ERR_DEVICE_WATCHDOG,
                herr & ERR_STACK ? "traversal stack exhausted" : "rejection sampling did not terminate");
  if (stats) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    memset(stats, 0, sizeof *stats);
    if (max_depth > 0) {
      stats->primary_rays = (uint64_t)counts[0];
      uint64_t refl = 0, hits = 0;
      for (int l = 1; l < levels; l++) refl += (uint64_t)counts[l];
      for (int l = 0; l < levels; l++) hits += (uint64_t)nh[l];
      stats->reflection_rays = refl;
      stats->hits = hits;
      // fallback hits recast their point lights and fb_dsamp rays per slot
      // that falls back
      stats->shadow_rays = (uint64_t)nh[0] * (uint64_t)K_0 + (hits - (uint64_t)nh[0]) * (uint64_t)K_full +
                           (uint64_t)hfb[0] * (uint64_t)sc->n_point_lights + (uint64_t)hfb[1] * (uint64_t)fb_dsamp;
      stats->fallback_hits = (uint64_t)hfb[0];
      stats->fallback_lights = (uint64_t)hfb[1];
      stats->shadow_rays_untraced = hstats[10];
      stats->trace_nodes = hstats[2];
      stats->trace_triangles = hstats[3];
      stats->trace_spheres = hstats[4];
      stats->trace_verifications = hstats[5];
      stats->shadow_nodes = hstats[6];
      stats->shadow_triangles = hstats[7];
      stats->shadow_spheres = hstats[8];
      stats->shadow_verifications = hstats[9];
    }
    stats->kernel_launches = Lc.launches;
    stats->graph = graph_state;
    stats->device_ms = ms;
    Lc.collect(stats->stage_ms);
    stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  ctx->err.clear();
  return RT_OK;
}

// Kernel kinds of a fused launch, their block sizes and the work that sizes
// their grids.
enum { FK_RAYGEN, FK_TRACE, FK_EMIT, FK_SHADOW, FK_RESOLVE, FK_FOLD, FK_PIXELS, FK_COUNT };
const int kFusedBlock[FK_COUNT] = {256, 128, 128, 128, 128, 256, 256};

// The fused group of a batch on `lane`: every frame is planned on its own
// slot (scratch; render_impl's checks), then each kernel of the wavefront is
// launched once for all frames over a device table of their launch blocks.
// Kernel kind k gets about nsm * tune_bpsm[k] blocks in all, shared out in
// proportion to each frame's work bound; each frame's blocks stride over its
// own rays.  The sequence is captured as a CUDA graph and replayed when the
// same group (frames, buffers, grid split) comes again.  Frames that cannot
// join (rare: the eligibility test in rt_render_batch mirrors render_impl's)
// render on their slot the usual way.
rt_status run_fused(rt_ctx* parent, rt_ctx* lane, rt_job* jobs, const std::vector<uint32_t>& idx,
                    std::vector<std::string>& errs, double* group_ms) {
  rt_ctx* ctx = lane;  // CK reports failures on the lane
  *group_ms = 0.0;
  const size_t n = idx.size();
  while (parent->slots.size() < n) {
    rt_ctx* l = nullptr;
    rt_status st = rt_ctx_create(parent->device, &l);
    if (st != RT_OK) return fail(parent, st, "creating a batch slot: " + std::string(rt_last_error(nullptr)));
    l->borrowed_net = true;
    parent->slots.push_back(l);
  }
  std::vector<FramePlan> plans(n);
  std::vector<size_t> ok;
  for (size_t k = 0; k < n; k++) {
    rt_job& J = jobs[idx[k]];
    rt_ctx* sl = parent->slots[k];
    memset(&J.stats, 0, sizeof J.stats);
    if (!J.scene || !J.rgb_out) {
      J.status = RT_ERR_INVALID_ARGUMENT;
      errs[idx[k]] = "null scene or output";
      continue;
    }
    J.status = render_impl(sl, J.scene, &J.params, 0, J.params.height, J.rgb_out, J.out_on_device, nullptr, nullptr,
                           nullptr, J.camera, &plans[k]);
    if (J.status == RT_OK) {
      // whatever set-up the plan queued on the slot's stream precedes the
      // fused launch, which runs on the lane's stream
      cudaError_t se = cudaStreamSynchronize(sl->stream);
      if (se != cudaSuccess) return cuda_fail(parent, se, "batch slot set-up");
      ok.push_back(k);
    } else if (sl->err == "this frame cannot join a fused batch group") {
      J.status = render_impl(sl, J.scene, &J.params, 0, J.params.height, J.rgb_out, J.out_on_device, nullptr,
                             &J.stats, nullptr, J.camera);
      if (J.status != RT_OK) errs[idx[k]] = sl->err;
    } else {
      errs[idx[k]] = sl->err;
    }
  }
  if (ok.empty()) return RT_OK;
  const int nj = (int)ok.size();
  CK(cudaSetDevice(lane->device));
  // host image of the table: frames, then (nj + 1) first blocks per kind
  const size_t frames_bytes = ((sizeof(DFrame) * nj + 255) / 256) * 256;
  const size_t bytes = frames_bytes + sizeof(int) * (size_t)FK_COUNT * (nj + 1);
  std::vector<unsigned char> host(bytes, 0);
  DFrame* T = reinterpret_cast<DFrame*>(host.data());
  int* b0 = reinterpret_cast<int*>(host.data() + frames_bytes);
  int Lmax = 1;
  for (int j = 0; j < nj; j++) {
    T[j] = plans[ok[j]].F;
    Lmax = std::max(Lmax, plans[ok[j]].levels);
  }
  const int nsm = lane->num_sms;
  int total[FK_COUNT];
  for (int k = 0; k < FK_COUNT; k++) {
    std::vector<double> w(nj);
    double sum = 0.0;
    for (int j = 0; j < nj; j++) {
      const FramePlan& pl = plans[ok[j]];
      const double v = k == FK_SHADOW ? (double)pl.chunk * std::max(pl.K, 1)
                       : (k == FK_EMIT || k == FK_RESOLVE) ? (double)pl.chunk
                       : k == FK_PIXELS ? (double)pl.npix : (double)pl.nprim;
      w[j] = v;
      sum += v;
    }
    const double budget = (double)nsm * parent->tune_bpsm[k];
    int at = 0;
    for (int j = 0; j < nj; j++) {
      b0[k * (nj + 1) + j] = at;
      const long long most = std::max(1LL, (long long)((w[j] + kFusedBlock[k] - 1) / kFusedBlock[k]));
      const long long want = std::max(1LL, (long long)std::llround(budget * w[j] / std::max(sum, 1.0)));
      at += (int)std::min(most, want);
    }
    b0[k * (nj + 1) + nj] = at;
    total[k] = at;
  }
  if (bytes > parent->group_cap) {
    CK(cudaStreamSynchronize(lane->stream));
    if (parent->group_buf) cudaFree(parent->group_buf);
    parent->group_buf = nullptr;
    parent->group_cap = 0;
    cudaError_t e = cudaMalloc(&parent->group_buf, bytes * 2);
    if (e != cudaSuccess) return cuda_fail(parent, e, "cudaMalloc(batch group table)");
    parent->group_cap = bytes * 2;
  }
  const DFrame* dT = reinterpret_cast<const DFrame*>(parent->group_buf);
  const int* db0 = reinterpret_cast<const int*>(static_cast<unsigned char*>(parent->group_buf) + frames_bytes);
  auto B = [&](int k) { return db0 + k * (nj + 1); };
  cudaStream_t s = lane->stream;
  CK(cudaMemcpyAsync(parent->group_buf, host.data(), bytes, cudaMemcpyHostToDevice, s));
  uint32_t launches = 0;
  auto enqueue = [&]() -> rt_status {
    k_frame_init_multi<<<nj, 128, 0, s>>>(dT);
    k_raygen_multi<<<total[FK_RAYGEN], 256, 0, s>>>(dT, B(FK_RAYGEN), nj);
    launches = 2;
    for (int l = 0; l < Lmax; l++) {
      k_trace_multi<false><<<total[FK_TRACE], 128, 0, s>>>(dT, B(FK_TRACE), nj, l);
      k_emit_multi<<<total[FK_EMIT], 128, 0, s>>>(dT, B(FK_EMIT), nj, l, 0);
      k_shadow_multi<false><<<total[FK_SHADOW], 128, 0, s>>>(dT, B(FK_SHADOW), nj, l, 0);
      k_resolve_multi<<<total[FK_RESOLVE], 128, 0, s>>>(dT, B(FK_RESOLVE), nj, l, 0);
      launches += 4;
    }
    for (int l = Lmax - 2; l >= 0; l--) {
      k_fold_multi<<<total[FK_FOLD], 256, 0, s>>>(dT, B(FK_FOLD), nj, l);
      launches++;
    }
    k_pixels_multi<<<total[FK_PIXELS], 256, 0, s>>>(dT, B(FK_PIXELS), nj);
    launches++;
    CK(cudaGetLastError());
    return RT_OK;
  };
  // graph: keyed by the table image (frames with their buffers, grid split)
  std::vector<unsigned char> key(host.begin(), host.end());
  const char tag[] = "fused";
  key.insert(key.end(), tag, tag + sizeof tag);
  GraphEntry* hit = nullptr;
  for (GraphEntry& g : lane->graphs)
    if (g.key == key) hit = &g;
  uint32_t graph_state = 2;
  if (!hit) {
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    rt_status es = enqueue();
    cudaError_t ce = cudaStreamEndCapture(s, &g);
    if (es != RT_OK) {
      if (g) cudaGraphDestroy(g);
      return es;
    }
    if (ce != cudaSuccess) return cuda_fail(lane, ce, "cudaStreamEndCapture");
    cudaGraphExec_t ex = nullptr;
    ce = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) return cuda_fail(lane, ce, "cudaGraphInstantiate");
    if (lane->graphs.size() >= kMaxGraphs) {
      auto lru = std::min_element(lane->graphs.begin(), lane->graphs.end(),
                                  [](const GraphEntry& a, const GraphEntry& b) { return a.used < b.used; });
      cudaGraphExecDestroy(lru->exec);
      lane->graphs.erase(lru);
    }
    lane->graphs.push_back(GraphEntry{std::move(key), ex, launches, 0});
    hit = &lane->graphs.back();
    graph_state = 1;
  }
  hit->used = ++lane->graph_tick;
  CK(cudaEventRecord(lane->ev0, s));
  CK(cudaGraphLaunch(hit->exec, s));
  CK(cudaEventRecord(lane->ev1, s));
  // per frame: image, queue sizes, hit counts, error word
  struct Back {
    std::vector<int> counts, nh;
    int err = 0;
    unsigned long long untraced = 0;
  };
  std::vector<Back> back(nj);
  for (int j = 0; j < nj; j++) {
    const FramePlan& pl = plans[ok[j]];
    rt_ctx* sl = parent->slots[ok[j]];
    if (!pl.direct)
      CK(cudaMemcpyAsync(pl.rgb_out, pl.d_rgb, 3 * pl.npix,
                         pl.on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
    back[j].counts.assign(pl.levels + 2, 0);
    back[j].nh.assign(pl.levels + 1, 0);
    CK(cudaMemcpyAsync(back[j].counts.data(), sl->d_counts, (pl.levels + 2) * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(back[j].nh.data(), sl->d_nhits, (pl.levels + 1) * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&back[j].err, sl->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&back[j].untraced, sl->d_stats + 10, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  }
  cudaError_t se = cudaStreamSynchronize(s);
  if (se != cudaSuccess) return cuda_fail(lane, se, "fused batch group");
  float ms = 0.f;
  cudaEventElapsedTime(&ms, lane->ev0, lane->ev1);
  *group_ms = ms;
  for (int j = 0; j < nj; j++) {
    const FramePlan& pl = plans[ok[j]];
    rt_job& J = jobs[idx[ok[j]]];
    const int herr = back[j].err;
    std::string msg;
    rt_status st = RT_OK;
    if (herr & ERR_EMPTY_RANGE) st = RT_ERR_RENDER, msg = "cannot sample empty range";
    else if (herr & ERR_RANGE_OVERFLOW) st = RT_ERR_RENDER, msg = "UniformSampler::sample_single: range overflow";
    else if (herr & (ERR_WATCHDOG | ERR_STACK))
      st = RT_ERR_DEVICE_WATCHDOG,
      msg = herr & ERR_STACK ? "traversal stack exhausted" : "rejection sampling did not terminate";
    J.status = st;
    if (st != RT_OK) {
      errs[idx[ok[j]]] = msg;
      continue;
    }
    rt_stats& S = J.stats;
    memset(&S, 0, sizeof S);
    S.primary_rays = (uint64_t)back[j].counts[0];
    uint64_t refl = 0, hits = 0;
    for (int l = 1; l < pl.levels; l++) refl += (uint64_t)back[j].counts[l];
    for (int l = 0; l < pl.levels; l++) hits += (uint64_t)back[j].nh[l];
    S.reflection_rays = refl;
    S.hits = hits;
    S.shadow_rays = hits * (uint64_t)pl.K;
    S.shadow_rays_untraced = back[j].untraced;
    S.kernel_launches = launches;  // shared by the group
    S.graph = graph_state;
    S.device_ms = ms;  // the group's time, shared by its frames
    S.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - pl.t0).count();
  }
  return RT_OK;
}

}  // namespace

// Meshes from this many triangles up build their k-d tree on the device when
// a load has a context; smaller ones build faster on the host.
const size_t kKdDeviceMin = 16384;

KdBuildHook device_kd_hook(rt_ctx* ctx) {
  KdBuildHook h;
  h.min_triangles = kKdDeviceMin;
  h.build = [ctx](const double* v, size_t n, std::vector<rt_kd_node_desc>* nodes, std::vector<int32_t>* idx) {
    if (!ctx->kd_arena) ctx->kd_arena = kd_arena_new();
    cudaError_t ce = cudaSuccess;
    return kd_build_device(v, (int64_t)n, ctx->stream, ctx->kd_arena, nodes, idx, &ce);
  };
  return h;
}

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
    return fail(nullptr, RT_ERR_CUDA,
                std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "count is 0"));
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
  for (rt_ctx* l : ctx->lanes) rt_ctx_destroy(l);
  ctx->lanes.clear();
  for (rt_ctx* l : ctx->slots) rt_ctx_destroy(l);
  ctx->slots.clear();
  if (ctx->group_buf) cudaFree(ctx->group_buf);
  ctx->group_buf = nullptr;
  if (ctx->pin) cudaFreeHost(ctx->pin);
  ctx->pin = nullptr;
  drop_graphs(ctx);
  free_all(ctx->scratch);
  free_all(ctx->dn_scratch);
  free_all(ctx->dn_arena_alloc);
  if (ctx->kd_arena) kd_arena_free(ctx->kd_arena);
  if (!ctx->borrowed_net) denoise_free(&ctx->net);
  for (cudaEvent_t e : ctx->stage_ev) cudaEventDestroy(e);
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
  CK(cudaSetDevice(ctx->device));
  HostScene hs;
  std::string err;
  KdBuildHook kd = device_kd_hook(ctx);
  if (!load_scene_json(json, ".", &hs, &err, &kd)) return fail(ctx, RT_ERR_SCENE, err);
  return rt_scene_upload(ctx, &hs.desc, out);
}

rt_status rt_scene_load_json_file(rt_ctx* ctx, const char* path, rt_scene** out) {
  if (!ctx || !path || !out) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  CK(cudaSetDevice(ctx->device));
  std::string text, err;
  if (!read_text_file(path, &text, &err)) return fail(ctx, RT_ERR_IO, err);
  HostScene hs;
  KdBuildHook kd = device_kd_hook(ctx);
  if (!load_scene_json(text, parent_dir(path), &hs, &err, &kd)) return fail(ctx, RT_ERR_SCENE, err);
  return rt_scene_upload(ctx, &hs.desc, out);
}

struct rt_kd_tree {
  std::vector<rt_kd_node_desc> nodes;
  std::vector<int32_t> idx;
};

rt_status rt_kd_build(rt_ctx* ctx, const double* vertices, int64_t n_triangles, rt_kd_tree** out) {
  if (!out || (n_triangles > 0 && !vertices) || n_triangles < 0)
    return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null or invalid argument");
  *out = nullptr;
  auto t = std::make_unique<rt_kd_tree>();
  std::string e;
  if (ctx) {
    CK(cudaSetDevice(ctx->device));
    cudaError_t ce = cudaSuccess;
    if (!ctx->kd_arena) ctx->kd_arena = kd_arena_new();
    e = kd_build_device(vertices, n_triangles, ctx->stream, ctx->kd_arena, &t->nodes, &t->idx, &ce);
    if (ce != cudaSuccess) return cuda_fail(ctx, ce, e.c_str());
  } else {
    e = kd_build_host(vertices, (size_t)n_triangles, &t->nodes, &t->idx);
  }
  if (!e.empty()) return fail(ctx, RT_ERR_SCENE, e);
  if (ctx) ctx->err.clear();
  *out = t.release();
  return RT_OK;
}

const rt_kd_node_desc* rt_kd_tree_nodes(const rt_kd_tree* t, int64_t* n_nodes) {
  if (n_nodes) *n_nodes = t ? (int64_t)t->nodes.size() : 0;
  return t && !t->nodes.empty() ? t->nodes.data() : nullptr;
}

const int32_t* rt_kd_tree_index(const rt_kd_tree* t, int64_t* n_index) {
  if (n_index) *n_index = t ? (int64_t)t->idx.size() : 0;
  return t && !t->idx.empty() ? t->idx.data() : nullptr;
}

void rt_kd_tree_free(rt_kd_tree* t) { delete t; }

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
  delete scene;
}

struct rt_host_scene {
  HostScene hs;
  // the meshes' device data prepared on the host, kept for later uploads
  // (a host scene never changes after loading)
  std::mutex mu;
  std::vector<std::shared_ptr<MeshPrep>> prep;
};

rt_status rt_host_scene_load_json_file(const char* path, rt_host_scene** out) {
  return rt_host_scene_load_json_file_on(nullptr, path, out);
}

rt_status rt_host_scene_load_json_file_on(rt_ctx* ctx, const char* path, rt_host_scene** out) {
  if (!path || !out) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (ctx) CK(cudaSetDevice(ctx->device));
  std::string text, err;
  if (!read_text_file(path, &text, &err)) return fail(ctx, RT_ERR_IO, err);
  auto h = std::make_unique<rt_host_scene>();
  KdBuildHook kd;
  if (ctx) kd = device_kd_hook(ctx);
  if (!load_scene_json(text, parent_dir(path), &h->hs, &err, ctx ? &kd : nullptr))
    return fail(ctx, RT_ERR_SCENE, err);
  if (ctx) ctx->err.clear();
  *out = h.release();
  return RT_OK;
}

rt_status rt_host_scene_upload(rt_ctx* ctx, rt_host_scene* hs, rt_scene** out) {
  if (!ctx || !hs || !out) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  CK(cudaSetDevice(ctx->device));
  std::lock_guard<std::mutex> g(hs->mu);
  rt_status s = do_upload(ctx, &hs->hs.desc, out, &hs->prep);
  if (s == RT_OK) ctx->err.clear();
  return s;
}

rt_status rt_auto_cameras_json_file(const char* path, rt_camera_config* out) {
  if (!path || !out) return fail(nullptr, RT_ERR_INVALID_ARGUMENT, "null argument");
  std::string text, err;
  if (!read_text_file(path, &text, &err)) return fail(nullptr, RT_ERR_IO, err);
  if (!auto_cameras(text, parent_dir(path), out, &err)) return fail(nullptr, RT_ERR_SCENE, err);
  return RT_OK;
}

rt_status rt_auto_cameras_json_str(const char* json, rt_camera_config* out) {
  if (!json || !out) return fail(nullptr, RT_ERR_INVALID_ARGUMENT, "null argument");
  std::string err;
  if (!auto_cameras(json, ".", out, &err)) return fail(nullptr, RT_ERR_SCENE, err);
  return RT_OK;
}

rt_status rt_host_scene_load_json_str(const char* json, rt_host_scene** out) {
  return rt_host_scene_load_json_str_on(nullptr, json, out);
}

rt_status rt_host_scene_load_json_str_on(rt_ctx* ctx, const char* json, rt_host_scene** out) {
  if (!json || !out) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (ctx) CK(cudaSetDevice(ctx->device));
  std::string err;
  auto h = std::make_unique<rt_host_scene>();
  KdBuildHook kd;
  if (ctx) kd = device_kd_hook(ctx);
  if (!load_scene_json(json, ".", &h->hs, &err, ctx ? &kd : nullptr)) return fail(ctx, RT_ERR_SCENE, err);
  if (ctx) ctx->err.clear();
  *out = h.release();
  return RT_OK;
}

const rt_scene_desc* rt_host_scene_desc(const rt_host_scene* hs) { return hs ? &hs->hs.desc : nullptr; }

void rt_host_scene_free(rt_host_scene* hs) { delete hs; }

rt_status rt_scene_device_bytes(rt_ctx* ctx, const rt_scene* scene, uint64_t* out) {
  if (!scene || !out) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  *out = scene->uploaded_bytes;
  return RT_OK;
}

rt_status rt_debug_fp64_rate(rt_ctx* ctx, double* gops) {
  if (!ctx || !gops) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  CK(cudaSetDevice(ctx->device));
  std::vector<void*> tmp;
  double* d;
  CK(dalloc(tmp, &d, 1));
  const int blocks = ctx->num_sms * 8, threads = 256, iters = 4096;
  k_fp64_rate<<<blocks, threads, 0, ctx->stream>>>(d, 64, 1.0000001, 1e-9);  // warm-up
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  k_fp64_rate<<<blocks, threads, 0, ctx->stream>>>(d, iters, 1.0000001, 1e-9);
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  free_all(tmp);
  double ops = (double)blocks * threads * iters * 32.0;
  *gops = ops / (ms * 1e-3) / 1e9;
  return RT_OK;
}

}  // extern "C"

namespace rtb {
// Context access for the training entry points (dn_train.cu).
cudaStream_t ctx_stream(rt_ctx* ctx) { return ctx->stream; }
int ctx_device(rt_ctx* ctx) { return ctx->device; }
int ctx_num_sms(rt_ctx* ctx) { return ctx->num_sms; }
rt_status ctx_fail(rt_ctx* ctx, rt_status st, const std::string& msg) { return fail(ctx, st, msg); }
}  // namespace rtb

extern "C" {

rt_status rt_debug_l2_read_bandwidth(rt_ctx* ctx, uint64_t bytes, int32_t reps, double* gbs) {
  if (!ctx || !gbs || reps <= 0) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument or reps <= 0");
  CK(cudaSetDevice(ctx->device));
  const int threads = 512, blocks = ctx->num_sms * 4;
  const uint64_t unit = 16ull * 4 * threads * blocks;  // one pass of every thread's four loads
  uint64_t n_units = bytes / unit;
  if (n_units == 0 || bytes > (1ull << 31)) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "buffer size out of range");
  std::vector<void*> tmp;
  uint4* buf;
  unsigned* sink;
  CK(dalloc(tmp, &buf, n_units * unit / 16));
  CK(dalloc(tmp, &sink, 1));
  CK(cudaMemsetAsync(buf, 1, n_units * unit, ctx->stream));
  long long n16 = (long long)(n_units * unit / 16);
  k_l2_read<<<blocks, threads, 0, ctx->stream>>>(buf, n16, 2, sink);  // warm-up: the buffer enters L2
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  k_l2_read<<<blocks, threads, 0, ctx->stream>>>(buf, n16, reps, sink);
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  free_all(tmp);
  *gbs = (double)n_units * unit * reps / (ms * 1e-3) / 1e9;
  return RT_OK;
}

namespace {
// Checks the arguments of the outline entry points and fills the frame
// fields the outline kernels read.
rt_status outline_frame(rt_ctx* ctx, uint32_t width, uint32_t height, const double* r, const double* g,
                        const double* b, const uint8_t* valid, const double* depth, const double* nx,
                        const double* ny, const double* nz, const rt_outline_config* cfg, uint8_t* rgb_out,
                        DFrame* F) {
  if (!ctx || !r || !g || !b || !valid || !depth || !nx || !ny || !nz || !cfg || !rgb_out)
    return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  if (width == 0 || height == 0 || (uint64_t)width * height > 0x7fffffffULL)
    return fail(ctx, RT_ERR_INVALID_ARGUMENT, "bad image size");
  *F = DFrame{};
  F->W = (int)width;
  F->H = (int)height;
  F->cr = const_cast<double*>(r);
  F->cg = const_cast<double*>(g);
  F->cb = const_cast<double*>(b);
  F->valid = const_cast<unsigned char*>(valid);
  F->dep = const_cast<double*>(depth);
  F->nx = const_cast<double*>(nx);
  F->ny = const_cast<double*>(ny);
  F->nz = const_cast<double*>(nz);
  F->rgb = rgb_out;
  F->linear = nullptr;
  F->o_wd = cfg->depth_weight;
  F->o_wn = cfg->normal_weight;
  F->o_thr = cfg->threshold;
  for (int k = 0; k < 3; k++) F->o_color[k] = cfg->edge_color[k];
  F->o_thick = cfg->line_thickness;
  F->o_wid = 0.0;  // no object buffer here
  F->oid = nullptr;
  F->o_use8 = cfg->use_8_neighbors ? 1 : 0;
  F->o_radius = 0;
  if (cfg->line_thickness > 1.0) {
    double rr = std::ceil(cfg->line_thickness - 1.0);
    if (!(rr <= kOutlineMaxRadius))
      return fail(ctx, RT_ERR_INVALID_ARGUMENT, "outline thickness above 2049 is not supported");
    F->o_radius = (int)rr;
  }
  return RT_OK;
}

rt_status launch_outline(rt_ctx* ctx, const DFrame& F) {
  dim3 ob(OT_X, OT_Y), og((F.W + OT_X - 1) / OT_X, (F.H + OT_Y - 1) / OT_Y);
  k_outline_mask<<<og, ob, 0, ctx->stream>>>(F);
  if (F.o_radius > kOutlineTileRadius) {
    const long long n = (long long)F.W * F.H;
    const int nb = (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, (long long)ctx->num_sms * 8));
    k_outline_apply_wide<<<nb, 256, 0, ctx->stream>>>(F);
  } else {
    size_t shm = (size_t)(OT_X + 2 * F.o_radius) * (OT_Y + 2 * F.o_radius) * sizeof(double);
    if (shm > 48 * 1024) CK(outline_smem_attr((int)shm));
    k_outline_apply<<<og, ob, shm, ctx->stream>>>(F);
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  return RT_OK;
}
}  // namespace

rt_status rt_outline_apply(rt_ctx* ctx, uint32_t width, uint32_t height, const double* r, const double* g,
                           const double* b, const uint8_t* valid, const double* depth, const double* nx,
                           const double* ny, const double* nz, const rt_outline_config* config, uint8_t* rgb_out) {
  DFrame F;
  rt_status st = outline_frame(ctx, width, height, r, g, b, valid, depth, nx, ny, nz, config, rgb_out, &F);
  if (st != RT_OK) return st;
  CK(cudaSetDevice(ctx->device));
  std::vector<void*> tmp;
  CK(dalloc(tmp, &F.mask, (size_t)width * height));  // edge-strength scratch
  st = launch_outline(ctx, F);
  free_all(tmp);
  if (st == RT_OK) ctx->err.clear();
  return st;
}

// Scratch of rt_outline_apply_noalloc: the per-pixel edge strengths.  One
// copy per device, alive for the life of the process; host code must not
// use the symbol as an address (it is a host-side shadow), only the device
// address that cudaGetSymbolAddress returns.
static __device__ __align__(256) double g_outline_mask[RT_OUTLINE_NOALLOC_MAX_PIXELS];

namespace {
// The device address of g_outline_mask on the current device (ctx's, made
// current by the caller).  Looked up on every call rather than cached, so
// that an address never outlives the context it came from (a device reset
// or a new primary context gives the array a new address).
rt_status noalloc_mask(rt_ctx* ctx, double** out) {
  double* p = nullptr;
  CK(cudaGetSymbolAddress((void**)&p, g_outline_mask));
  if (!p) return fail(ctx, RT_ERR_CUDA, "cudaGetSymbolAddress returned a null address");
  *out = p;
  return RT_OK;
}
}  // namespace

rt_status rt_outline_apply_noalloc(rt_ctx* ctx, uint32_t width, uint32_t height, const double* r,
                                   const double* g, const double* b, const uint8_t* valid, const double* depth,
                                   const double* nx, const double* ny, const double* nz,
                                   const rt_outline_config* config, uint8_t* rgb_out) {
  DFrame F;
  rt_status st = outline_frame(ctx, width, height, r, g, b, valid, depth, nx, ny, nz, config, rgb_out, &F);
  if (st != RT_OK) return st;
  if ((uint64_t)width * height > RT_OUTLINE_NOALLOC_MAX_PIXELS)
    return fail(ctx, RT_ERR_INVALID_ARGUMENT,
                "image larger than the static outline scratch (RT_OUTLINE_NOALLOC_MAX_PIXELS = 4194304 pixels)");
  CK(cudaSetDevice(ctx->device));
  st = noalloc_mask(ctx, &F.mask);
  if (st != RT_OK) return st;
  st = launch_outline(ctx, F);
  if (st == RT_OK) ctx->err.clear();
  return st;
}

rt_status rt_render(rt_ctx* ctx, const rt_scene* scene, const rt_render_params* params, uint8_t* rgb_out,
                    int out_on_device, rt_stats* stats) {
  if (!params) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  return render_impl(ctx, scene, params, 0, params->height, rgb_out, out_on_device, nullptr, stats);
}

rt_status rt_render_rows(rt_ctx* ctx, const rt_scene* scene, const rt_render_params* params, uint32_t row_begin,
                         uint32_t row_end, uint8_t* rgb_out, int out_on_device, rt_stats* stats) {
  if (!rgb_out) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "no output buffer");
  return render_impl(ctx, scene, params, row_begin, row_end, rgb_out, out_on_device, nullptr, stats);
}

rt_status rt_batch_assign(const double* costs, uint32_t n, uint32_t lanes, uint32_t* lane_of_job) {
  if ((n && (!costs || !lane_of_job)) || lanes == 0 || lanes > 64)
    return fail(nullptr, RT_ERR_INVALID_ARGUMENT, "rt_batch_assign: bad arguments (lanes must be 1..64)");
  std::vector<uint32_t> order(n);
  for (uint32_t i = 0; i < n; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return costs[a] > costs[b]; });
  std::vector<double> load(lanes, 0.0);
  for (uint32_t i : order) {
    uint32_t best = 0;
    for (uint32_t l = 1; l < lanes; l++)
      if (load[l] < load[best]) best = l;
    load[best] += costs[i];
    lane_of_job[i] = best;
  }
  return RT_OK;
}

rt_status rt_render_batch(rt_ctx* ctx, rt_job* jobs, uint32_t n, uint32_t lanes, rt_batch_stats* stats) {
  if (!ctx) return fail(nullptr, RT_ERR_INVALID_ARGUMENT, "null context");
  if (n && !jobs) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null jobs");
  if (lanes == 0) lanes = ctx->tuned_lanes ? ctx->tuned_lanes : 4;
  if (lanes > 16) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "at most 16 lanes");
  lanes = std::max(1u, std::min(lanes, std::max(n, 1u)));
  auto t0 = std::chrono::steady_clock::now();
  // lanes: child contexts on the same device, sharing the parent's denoiser
  while (ctx->lanes.size() < lanes) {
    rt_ctx* l = nullptr;
    rt_status st = rt_ctx_create(ctx->device, &l);
    if (st != RT_OK) return fail(ctx, st, "creating a batch lane: " + std::string(rt_last_error(nullptr)));
    l->borrowed_net = true;
    ctx->lanes.push_back(l);
  }
  for (uint32_t k = 0; k < lanes; k++) {
    rt_ctx* l = ctx->lanes[k];
    l->net.ops = ctx->net.ops;
    l->net.param_count = ctx->net.param_count;
    l->net.rays_per_light = ctx->net.rays_per_light;
    l->net.has_conf = ctx->net.has_conf;
    l->net.conf_threshold = ctx->net.conf_threshold;
    l->net.allocs.clear();
  }
  // estimated rays per job -> lanes, longest first; small frames that can
  // share launches form the fused group, which lane 0 renders first
  std::vector<double> cost(n, 0.0);
  std::vector<uint32_t> fused;
  std::vector<char> in_group(n, 0);
  std::vector<double> scratch(n, 0.0);  // estimated scratch bytes of a fused frame
  for (uint32_t i = 0; i < n; i++) {
    const rt_render_params& P = jobs[i].params;
    const rt_scene* sc = jobs[i].scene;
    double spp = P.anti_aliasing_mode == RT_AA_QUINCUNX ? 2.0 : (double)std::max(1u, P.samples);
    int ds = P.disk_samples ? (int)P.disk_samples : 16;
    double K = sc ? (double)(sc->n_point_lights + sc->n_disk_lights * ds) : 0.0;
    cost[i] = (double)P.width * P.height * spp * (1.0 + K);
    // fused group: whole small frames on the plain path, one shadow chunk,
    // no outline pass, no profiling
    const double nprim = P.anti_aliasing_mode == RT_AA_QUINCUNX
                             ? (double)(P.width + 1) * (P.height + 1) + (double)P.width * P.height
                             : (double)P.width * P.height * std::max(1u, P.samples);
    const bool outline = P.outline.enabled && P.anti_aliasing_mode != RT_AA_QUINCUNX;
    if (ctx->fuse_pixels && sc && jobs[i].rgb_out && (uint64_t)P.width * P.height <= ctx->fuse_pixels &&
        !P.learned_shadows && !outline && P.max_depth > 0 && P.max_depth <= RTB_MAX_LEVELS && P.samples > 0 &&
        !(P.flags & (RT_FLAG_STAGE_TIMES | RT_FLAG_COUNT_WORK)) && nprim * std::max(K, 1.0) <= (double)kShadowCap) {
      // a fused frame keeps all its scratch at once: per primary ray the
      // queues, hit records, per-level colours and outline data, its whole
      // shadow buffer (K rays of 33 bytes, 24 bytes of origin per hit), and
      // about 80 bytes per pixel
      const double levels = std::max(1, std::min(P.max_depth, RTB_MAX_LEVELS));
      scratch[i] = nprim * (173.0 + 36.0 * levels + 33.0 * K + 24.0) + (double)P.width * P.height * 80.0;
      fused.push_back(i);
    }
  }
  // the smallest frames first, while the estimated scratch fits the budget
  std::stable_sort(fused.begin(), fused.end(), [&](uint32_t a, uint32_t b) { return scratch[a] < scratch[b]; });
  {
    double used = 0.0;
    size_t keep = 0;
    while (keep < fused.size() && used + scratch[fused[keep]] <= (double)ctx->fuse_bytes) used += scratch[fused[keep++]];
    fused.resize(keep);
    for (uint32_t i : fused) in_group[i] = 1;
  }
  if (fused.size() < 2) {  // one frame gains nothing from fusion
    fused.clear();
    std::fill(in_group.begin(), in_group.end(), 0);
  }
  std::vector<std::vector<uint32_t>> per_lane(lanes);
  {
    // longest processing time first onto the least-loaded lane; lane 0
    // starts with the fused group's estimated cost
    std::vector<double> load(lanes, 0.0);
    for (uint32_t i : fused) load[0] += cost[i];
    std::vector<uint32_t> order;
    for (uint32_t i = 0; i < n; i++)
      if (!in_group[i]) order.push_back(i);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cost[a] > cost[b]; });
    for (uint32_t i : order) {
      uint32_t best = 0;
      for (uint32_t k = 1; k < lanes; k++)
        if (load[k] < load[best]) best = k;
      per_lane[best].push_back(i);
      load[best] += cost[i];
    }
  }
  std::vector<std::string> errs(n);
  std::vector<double> lane_ms(lanes, 0.0);
  rt_status group_st = RT_OK;
  std::string group_err;
  double group_ms = 0.0;  // device time of the fused group (shared by its frames)
  auto run_lane = [&](uint32_t k) {
    rt_ctx* l = ctx->lanes[k];
    if (k == 0 && !fused.empty()) {
      group_st = run_fused(ctx, l, jobs, fused, errs, &group_ms);
      if (group_st != RT_OK) group_err = l->err.empty() ? ctx->err : l->err;
      lane_ms[0] += group_ms;
    }
    for (uint32_t i : per_lane[k]) {
      rt_job& J = jobs[i];
      memset(&J.stats, 0, sizeof J.stats);
      if (!J.scene || !J.rgb_out) {
        J.status = RT_ERR_INVALID_ARGUMENT;
        errs[i] = "null scene or output";
        continue;
      }
      J.status = render_impl(l, J.scene, &J.params, 0, J.params.height, J.rgb_out, J.out_on_device, nullptr, &J.stats,
                             nullptr, J.camera);
      if (J.status != RT_OK) errs[i] = l->err;
      lane_ms[k] += J.stats.device_ms;
    }
  };
  std::vector<std::thread> threads;
  for (uint32_t k = 1; k < lanes; k++) threads.emplace_back(run_lane, k);
  run_lane(0);
  for (auto& t : threads) t.join();
  if (group_st != RT_OK) return fail(ctx, group_st, "fused batch group: " + group_err);
  rt_status first = RT_OK;
  std::string msg;
  uint64_t rays = 0;
  double dev = 0.0;
  for (uint32_t i = 0; i < n; i++) {
    if (jobs[i].status != RT_OK && first == RT_OK) {
      first = (rt_status)jobs[i].status;
      msg = "job " + std::to_string(i) + ": " + errs[i];
    }
    rays += jobs[i].stats.primary_rays + jobs[i].stats.reflection_rays + jobs[i].stats.shadow_rays;
    if (!in_group[i]) dev += jobs[i].stats.device_ms;
  }
  dev += group_ms;
  if (stats) {
    memset(stats, 0, sizeof *stats);
    stats->jobs = n;
    stats->lanes = lanes;
    stats->rays = rays;
    stats->device_ms = dev;
    stats->busiest_lane_ms = *std::max_element(lane_ms.begin(), lane_ms.end());
    stats->wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  if (first != RT_OK) return fail(ctx, first, msg);
  ctx->err.clear();
  return RT_OK;
}

rt_status rt_batch_get_tuning(rt_ctx* ctx, rt_batch_tuning* out) {
  if (!ctx || !out) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  memset(out, 0, sizeof *out);
  out->lanes = ctx->tuned_lanes ? ctx->tuned_lanes : 4;
  out->fuse_pixels = ctx->fuse_pixels;
  out->fuse_bytes = ctx->fuse_bytes;
  for (int k = 0; k < 7; k++) out->blocks_per_sm[k] = ctx->tune_bpsm[k];
  return RT_OK;
}

rt_status rt_batch_set_tuning(rt_ctx* ctx, const rt_batch_tuning* t) {
  if (!ctx || !t) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  if (t->lanes < 1 || t->lanes > 16) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "lanes must be 1..16");
  for (int k = 0; k < 7; k++)
    if (t->blocks_per_sm[k] < 1 || t->blocks_per_sm[k] > 1024)
      return fail(ctx, RT_ERR_INVALID_ARGUMENT, "blocks_per_sm must be 1..1024");
  ctx->tuned_lanes = t->lanes;
  ctx->fuse_pixels = t->fuse_pixels;
  ctx->fuse_bytes = t->fuse_bytes;
  for (int k = 0; k < 7; k++) ctx->tune_bpsm[k] = t->blocks_per_sm[k];
  return RT_OK;
}

rt_status rt_batch_autotune_ex(rt_ctx* ctx, rt_job* jobs, uint32_t n, rt_batch_tuning* out) {
  if (!ctx) return fail(nullptr, RT_ERR_INVALID_ARGUMENT, "null context");
  rt_batch_tuning cur;
  rt_status st = rt_batch_get_tuning(ctx, &cur);
  if (st != RT_OK) return st;
  uint32_t trials = 0;
  auto measure = [&](const rt_batch_tuning& t, double* ms) -> rt_status {
    rt_status s2 = rt_batch_set_tuning(ctx, &t);
    if (s2 != RT_OK) return s2;
    rt_batch_stats bs;
    s2 = rt_render_batch(ctx, jobs, n, t.lanes, &bs);  // first run with a new group captures its graph
    if (s2 != RT_OK) return s2;
    s2 = rt_render_batch(ctx, jobs, n, t.lanes, &bs);
    if (s2 != RT_OK) return s2;
    trials++;
    *ms = bs.wall_ms;
    return RT_OK;
  };
  {
    // warm-up with the most lanes: creates the lanes and slots and sizes
    // their scratch, so that the timed runs allocate nothing
    rt_batch_tuning w = cur;
    w.lanes = 8;
    double ms;
    st = measure(w, &ms);
    if (st != RT_OK) return st;
  }
  double best_ms;
  st = measure(cur, &best_ms);
  if (st != RT_OK) return st;
  // coordinate search: lanes, then the fused group's size limit, then the
  // grid budget (blocks per SM) of each fused kernel kind
  auto try_values = [&](auto set, std::initializer_list<long long> vals) -> rt_status {
    for (long long v : vals) {
      rt_batch_tuning t = cur;
      set(t, v);
      if (memcmp(&t, &cur, sizeof t) == 0) continue;
      double ms;
      rt_status s2 = measure(t, &ms);
      if (s2 != RT_OK) return s2;
      if (ms < best_ms) {
        best_ms = ms;
        cur = t;
      }
    }
    return RT_OK;
  };
  st = try_values([](rt_batch_tuning& t, long long v) { t.lanes = (uint32_t)v; }, {1, 2, 4, 8});
  if (st != RT_OK) return st;
  st = try_values([](rt_batch_tuning& t, long long v) { t.fuse_pixels = (uint32_t)v; },
                  {0, 256 * 256, 640 * 480, 1280 * 720});
  if (st != RT_OK) return st;
  const std::initializer_list<long long> grid_vals[7] = {{8, 16, 32}, {16, 32, 64, 128}, {16, 32, 64, 128},
                                                         {32, 64, 128, 256}, {8, 16, 32, 64}, {8, 16, 32},
                                                         {8, 16, 32}};
  if (cur.fuse_pixels) {
    for (int k : {1, 3, 2, 4}) {  // the walks first, then emit and resolve
      st = try_values([k](rt_batch_tuning& t, long long v) { t.blocks_per_sm[k] = (int32_t)v; }, grid_vals[k]);
      if (st != RT_OK) return st;
    }
  }
  st = rt_batch_set_tuning(ctx, &cur);
  if (st != RT_OK) return st;
  ctx->tuned = true;
  if (out) {
    *out = cur;
    out->best_ms = best_ms;
    out->trials = trials;
  }
  return RT_OK;
}

rt_status rt_batch_autotune(rt_ctx* ctx, rt_job* jobs, uint32_t n, uint32_t* best_lanes) {
  rt_batch_tuning t;
  rt_status st = rt_batch_autotune_ex(ctx, jobs, n, &t);
  if (st == RT_OK && best_lanes) *best_lanes = t.lanes;
  return st;
}

rt_status rt_denoiser_load(rt_ctx* ctx, const void* blob, size_t bytes) {
  if (!ctx) return fail(nullptr, RT_ERR_INVALID_ARGUMENT, "null context");
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  drop_graphs(ctx);
  for (rt_ctx* l : ctx->lanes) {
    CK(cudaStreamSynchronize(l->stream));
    drop_graphs(l);
  }
  std::string e = denoise_load(blob, bytes, &ctx->net);
  if (!e.empty()) return fail(ctx, RT_ERR_INVALID_ARGUMENT, e);
  ctx->err.clear();
  return RT_OK;
}

rt_status rt_denoiser_run(rt_ctx* ctx, const uint16_t* features, uint32_t planes, uint32_t height, uint32_t width,
                          float* visibility, float* confidence, double* device_ms) {
  if (!ctx) return fail(nullptr, RT_ERR_INVALID_ARGUMENT, "null context");
  if (!features || !visibility) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  if (!ctx->net.loaded()) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "no denoiser weights loaded");
  if (planes == 0 || height == 0 || width == 0 || (uint64_t)planes * height * width > 0x7fffffffULL)
    return fail(ctx, RT_ERR_INVALID_ARGUMENT, "bad feature image size");
  if (((uintptr_t)features & 15) != 0) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "features must be 16-byte aligned");
  CK(cudaSetDevice(ctx->device));
  long long n = (long long)planes * height * width;
  rt_status st = ensure_dn_scratch(ctx, n);
  if (st != RT_OK) return st;
  st = ensure_dn_arena(ctx, denoise_scratch_halves(ctx->net, (int)planes, (int)height, (int)width));
  if (st != RT_OK) return st;
  // the scratch error word is shared with renders on this context
  if (!ctx->d_err) {
    st = ensure_scratch(ctx, 1, 1, 1, 1, 1);
    if (st != RT_OK) return st;
  }
  CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
  cudaError_t le = cudaSuccess;
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  denoise_run(ctx->net, reinterpret_cast<const __half*>(features), (int)planes, (int)height, (int)width,
              ctx->d_dn_arena, visibility, confidence, ctx->d_err, ctx->stream, ctx->num_sms, &le);
  if (le != cudaSuccess) return cuda_fail(ctx, le, "denoiser launch");
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  int herr = 0;
  CK(cudaMemcpyAsync(&herr, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (device_ms) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    *device_ms = ms;
  }
  if (herr & DN_ERR_WAIT) return fail(ctx, RT_ERR_DEVICE_WATCHDOG, "denoiser: a tensor-core wait timed out");
  ctx->err.clear();
  return RT_OK;
}

rt_status rt_render_shadow_aov(rt_ctx* ctx, const rt_scene* scene, const rt_render_params* params, uint8_t* rgb_out,
                               float* vis, uint16_t* features, rt_stats* stats) {
  if (!params) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  if (features && ((uintptr_t)features & 15) != 0)
    return fail(ctx, RT_ERR_INVALID_ARGUMENT, "features must be 16-byte aligned");
  AovOut aov;
  aov.vis = vis;
  aov.feat = reinterpret_cast<__half*>(features);
  std::vector<uint8_t> sink;
  if (!rgb_out) {
    sink.resize((size_t)params->width * params->height * 3);
    rgb_out = sink.data();
  }
  return render_impl(ctx, scene, params, 0, params->height, rgb_out, 0, nullptr, stats, &aov);
}

rt_status rt_render_linear(rt_ctx* ctx, const rt_scene* scene, const rt_render_params* params, uint8_t* rgb_out,
                           double* linear_out, rt_stats* stats) {
  if (!params) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  return render_impl(ctx, scene, params, 0, params->height, rgb_out, 0, linear_out, stats);
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
  if (!std::isfinite(radius - -radius))
    return fail(ctx, RT_ERR_RENDER, "UniformSampler::sample_single: range overflow");
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

rt_status rt_debug_mesh_prep(rt_ctx* ctx, const rt_mesh_desc* md, uint32_t* mismatch) {
  if (!ctx || !md || !mismatch) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "null argument");
  *mismatch = 0;
  if (md->n_triangles <= kMeshLeaf) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "mesh too small for the device preparation");
  CK(cudaSetDevice(ctx->device));
  MeshPrep H, D;
  std::string e = prep_mesh(*md, &H, false, true);
  if (!e.empty()) return fail(ctx, RT_ERR_INVALID_ARGUMENT, e);
  e = prep_mesh_kd(*md, &D);
  if (!e.empty()) return fail(ctx, RT_ERR_INVALID_ARGUMENT, e);
  const int n = D.n_tris, nb = bvh_internal_nodes(n, kMeshLeaf);
  std::vector<void*> tmp;
  double2 *dn, *bvh, *btris, *brute, *cells;
  float4* fbvh;
  double4* normals;
  int *dl, *occ_off;
  int2 *occ, *dp;
  cudaError_t ce = cudaSuccess;
  if ((ce = dalloc(tmp, &dn, D.nodes.size())) != cudaSuccess || (ce = dalloc(tmp, &dl, D.leaf_tris.size())) != cudaSuccess ||
      (ce = dalloc(tmp, &dp, D.leaf_path.size())) != cudaSuccess ||
      (ce = dalloc(tmp, &cells, 3 * (size_t)D.n_nodes)) != cudaSuccess ||
      (ce = dalloc(tmp, &bvh, 7 * (size_t)nb)) != cudaSuccess || (ce = dalloc(tmp, &fbvh, RTB_FBVH_HEAD + 4 * (size_t)nb)) != cudaSuccess ||
      (ce = dalloc(tmp, &btris, 5 * (size_t)n)) != cudaSuccess ||
      (ce = dalloc(tmp, &brute, 5 * (size_t)n)) != cudaSuccess || (ce = dalloc(tmp, &normals, (size_t)n)) != cudaSuccess ||
      (ce = dalloc(tmp, &occ, (size_t)D.n_index)) != cudaSuccess || (ce = dalloc(tmp, &occ_off, (size_t)n + 1)) != cudaSuccess) {
    free_all(tmp);
    return cuda_fail(ctx, ce, "cudaMalloc");
  }
  // on the context's stream (non-blocking), which the preparations below use
  cudaMemcpyAsync(dn, D.nodes.data(), D.nodes.size() * sizeof(double2), cudaMemcpyHostToDevice, ctx->stream);
  cudaMemcpyAsync(dl, D.leaf_tris.data(), D.leaf_tris.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream);
  cudaMemcpyAsync(dp, D.leaf_path.data(), D.leaf_path.size() * sizeof(int2), cudaMemcpyHostToDevice, ctx->stream);
  if (!ctx->kd_arena) ctx->kd_arena = kd_arena_new();
  e = prep_mesh_device(md->vertices, n, dn, D.n_nodes, dl, dp, D.n_index, kMeshLeaf, ctx->stream, ctx->kd_arena,
                       MeshPrepOut{bvh, fbvh, cells, btris, brute, normals, occ, occ_off}, &ce);
  if (!e.empty()) {
    free_all(tmp);
    return ce != cudaSuccess ? cuda_fail(ctx, ce, e.c_str()) : fail(ctx, RT_ERR_INVALID_ARGUMENT, e);
  }
  auto same = [](const void* dev, const void* host, size_t bytes) {
    std::vector<char> h(bytes);
    if (bytes) cudaMemcpy(h.data(), dev, bytes, cudaMemcpyDeviceToHost);
    return !bytes || memcmp(h.data(), host, bytes) == 0;
  };
  uint32_t m = 0;
  if (H.bvh.size() != 7 * (size_t)nb || !same(bvh, H.bvh.data(), H.bvh.size() * sizeof(double2))) m |= 1;
  if (!same(btris, H.btris.data(), H.btris.size() * sizeof(double2))) m |= 2;
  if (!same(brute, H.brute.data(), H.brute.size() * sizeof(double2))) m |= 4;
  if (!same(normals, H.normals.data(), H.normals.size() * sizeof(double4))) m |= 8;
  if (!same(occ, H.occ.data(), H.occ.size() * sizeof(int2))) m |= 16;
  if (!same(occ_off, H.occ_off.data(), H.occ_off.size() * sizeof(int))) m |= 32;
  // the single-precision BVH the walks test: the device's conversion
  // (k_prep_fbvh) against the host's (put_fbvh), scale element included
  if (H.fbvh.size() != RTB_FBVH_HEAD + 4 * (size_t)nb || !same(fbvh, H.fbvh.data(), H.fbvh.size() * sizeof(float4))) m |= 128;
  // the arrays an upload of the host preparation derives on the device,
  // from the host's BVH-order records, into the same buffers
  cudaStream_t s = ctx->stream;
  if ((ce = cudaMemcpyAsync(btris, H.btris.data(), H.btris.size() * sizeof(double2), cudaMemcpyHostToDevice, s)) ==
          cudaSuccess &&
      (ce = cudaMemsetAsync(brute, 0xff, H.brute.size() * sizeof(double2), s)) == cudaSuccess &&
      (ce = cudaMemsetAsync(normals, 0xff, H.normals.size() * sizeof(double4), s)) == cudaSuccess &&
      (ce = cudaMemsetAsync(occ, 0xff, H.occ.size() * sizeof(int2), s)) == cudaSuccess &&
      (ce = cudaMemsetAsync(occ_off, 0xff, H.occ_off.size() * sizeof(int), s)) == cudaSuccess) {
    e = derive_mesh_device(bvh, nb, btris, n, dn, D.n_nodes, dl, dp, D.n_index, s, ctx->kd_arena, fbvh, cells, brute,
                           normals, occ, occ_off, &ce);
    if (e.empty() && (ce = cudaStreamSynchronize(s)) == cudaSuccess &&
        (!same(brute, H.brute.data(), H.brute.size() * sizeof(double2)) ||
         !same(normals, H.normals.data(), H.normals.size() * sizeof(double4)) ||
         !same(occ, H.occ.data(), H.occ.size() * sizeof(int2)) ||
         !same(occ_off, H.occ_off.data(), H.occ_off.size() * sizeof(int))))
      m |= 64;
  }
  if (ce != cudaSuccess) {
    free_all(tmp);
    return cuda_fail(ctx, ce, "mesh derivation check");
  }
  ce = cudaGetLastError();
  free_all(tmp);
  if (ce != cudaSuccess) return cuda_fail(ctx, ce, "mesh preparation check");
  *mismatch = m;
  ctx->err.clear();
  return RT_OK;
}

rt_status rt_debug_mesh_hit(rt_ctx* ctx, const rt_scene* scene, int32_t object_index, int32_t use_kdtree,
                            const double* rays, int64_t n, double t_min, double t_max, double* out) {
  if (!ctx || !scene || !rays || !out || n < 0) return fail(ctx, RT_ERR_INVALID_ARGUMENT, "bad argument");
  if (object_index < 0 || object_index >= (int)scene->obj_kind.size() ||
      scene->obj_kind[object_index] != RT_OBJ_MESH)
    return fail(ctx, RT_ERR_INVALID_ARGUMENT, "object is not a mesh");
  // bit 0: use_kdtree as the Renderer field; bits 1-2: the query
  // (0 closest hit, 1 the plain k-d walk, 2 any hit, 3 the k-d leaf visit
  // tests compared)
  int mode = (use_kdtree >> 1) & 3;
  if (n == 0) return RT_OK;
  CK(cudaSetDevice(ctx->device));
  DMesh M = scene->host_meshes[scene->obj_mesh[object_index]];
  std::vector<void*> tmp;
  double *dr, *dout;
  int* derr;
  CK(dalloc(tmp, &dr, (size_t)n * 6));
  CK(dalloc(tmp, &dout, (size_t)n * 8));
  CK(dalloc(tmp, &derr, 1));
  CK(cudaMemset(derr, 0, sizeof(int)));
  CK(cudaMemcpy(dr, rays, (size_t)n * 6 * sizeof(double), cudaMemcpyHostToDevice));
  k_debug_mesh<<<(int)std::min<int64_t>((n + 127) / 128, 4096), 128, 0, ctx->stream>>>(
      M, use_kdtree & 1, mode, dr, n, t_min, t_max, dout, derr);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaMemcpy(out, dout, (size_t)n * 8 * sizeof(double), cudaMemcpyDeviceToHost));
  int herr = 0;
  CK(cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost));
  free_all(tmp);
  if (herr) return fail(ctx, RT_ERR_DEVICE_WATCHDOG, "traversal stack exhausted");
  return RT_OK;
}

}  // extern "C"
