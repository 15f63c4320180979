// A large mesh's device search data computed on the device, with the same
// bytes as the host preparation:
//   * triangle records and normals (one thread per triangle, the same
//     double operations as the host);
//   * the triangle BVH.  A median split makes the tree's shape a function
//     of the triangle count alone, so the host lays out every level's
//     segments (node ranges of the primitive order) up front, and each
//     level is one stable radix sort of the whole order by (segment, rank
//     of the centroid on the segment's widest centroid axis; ties by id)
//     plus two bounds reductions; nothing waits for the device until the
//     end.  Leaves end in id order (the host builder's canonical layout);
//   * the k-d occurrence lists: every leaf entry as (triangle, leaf,
//     position), stably sorted by triangle.
// For a mesh prepared on the host, the arrays that follow from its BVH-order
// records and its k-d tree (records in mesh order, normals, occurrences)
// are derived here too, so an upload copies only the rest.
// Sorts and scans are CUB's device-wide radix sort and scan.
#include "mesh_prep.hpp"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <climits>
#include <map>
#include <vector>

#include "dmath.cuh"

namespace rtb {
namespace {

constexpr int SEG_LANE = 32;                // primitives one lane folds
constexpr int SEG_CHUNK = 32 * SEG_LANE;    // primitives one warp folds

int grid_for(long long n, int bs) { return (int)std::max<long long>(1, std::min<long long>((n + bs - 1) / bs, 148LL * 16)); }

int bits_for(long long n) {  // bits to hold values 0 .. n - 1
  int b = 1;
  while ((1LL << b) < n) b++;
  return b;
}

// std::min / std::max as the host builder calls them: the second operand
// when it compares below (above), so a NaN operand in second place is
// ignored.
__device__ __forceinline__ double smin(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double smax(double a, double b) { return a < b ? b : a; }

// Records: brute[5t..5t+4] = {v0, e1, e2, (t, degenerate)} packed in
// double2s, normals[t] = normalize(e1 x e2), box[6t..] = min, max of the
// vertices, cen[3t..] = box centre; scale = max |coordinate| (as bits:
// non-negative doubles order like their encodings).
__global__ void k_prep_records(const double* __restrict__ v, int n, double2* __restrict__ brute,
                               double4* __restrict__ normals, double* __restrict__ box, double* __restrict__ cen,
                               unsigned long long* __restrict__ scale_bits) {
  double scale = 0.0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const double* p = v + 9 * (long long)t;
    V3 v0 = mk(p[0], p[1], p[2]), v1 = mk(p[3], p[4], p[5]), v2 = mk(p[6], p[7], p[8]);
    V3 e1 = v1 - v0, e2 = v2 - v0;
    V3 nrm = cross(e1, e2);
    int degenerate = norm(nrm) < 1e-8 ? 1 : 0;  // src/ray.rs:565-567
    V3 nn = normalize(nrm);
    normals[t] = double4{nn.x, nn.y, nn.z, 0.0};
    double2* E = brute + 5 * (long long)t;
    E[0] = double2{v0.x, v0.y};
    E[1] = double2{v0.z, e1.x};
    E[2] = double2{e1.y, e1.z};
    E[3] = double2{e2.x, e2.y};
    E[4] = double2{e2.z, pack2(t, degenerate)};
    for (int k = 0; k < 3; k++) {
      const double a = p[k], b = p[3 + k], c = p[6 + k];
      const double lo = smin(a, smin(b, c)), hi = smax(a, smax(b, c));
      box[6 * (long long)t + k] = lo;
      box[6 * (long long)t + 3 + k] = hi;
      cen[3 * (long long)t + k] = 0.5 * (lo + hi);
      scale = smax(scale, smax(fabs(lo), fabs(hi)));
    }
  }
  for (int o = 16; o > 0; o >>= 1) scale = smax(scale, __shfl_down_sync(0xffffffffu, scale, o));
  if ((threadIdx.x & 31) == 0) atomicMax(scale_bits, (unsigned long long)dbits(scale));
}

// Centroid on one axis (-0 as +0: the host compares them equal) and the
// identity permutation, to rank the centroids.
__global__ void k_prep_axis_keys(const double* __restrict__ cen, int n, int axis, double* __restrict__ key,
                                 int* __restrict__ val) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double c = cen[3 * (long long)i + axis];
    key[i] = c == 0.0 ? 0.0 : c;
    val[i] = i;
  }
}

// rank[id] = position of id in the (centroid, id) order.
__global__ void k_prep_rank(const int* __restrict__ sorted, int n, int* __restrict__ rank) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) rank[sorted[i]] = i;
}

__global__ void k_prep_iota(int* __restrict__ e, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) e[i] = i;
}

__device__ __forceinline__ int seg_of(const int* __restrict__ start, int S, int p) {
  int lo = 0, hi = S;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (start[mid] <= p) lo = mid;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ void warp_bounds(double v[6]) {
  for (int o = 1; o < 32; o <<= 1)
    for (int a = 0; a < 3; a++) {
      v[a] = smin(v[a], __shfl_down_sync(0xffffffffu, v[a], o));
      v[3 + a] = smax(v[3 + a], __shfl_down_sync(0xffffffffu, v[3 + a], o));
    }
}

// Bounds of segments of the primitive order, phase 1: warp w folds chunk w
// (chunks of segment q are cstart[q] .. cstart[q+1]-1).  src holds `width`
// doubles per primitive: 6 (a box: min xyz, max xyz) or 3 (a point).
__global__ void k_prep_seg_chunks(const int* __restrict__ perm, const int* __restrict__ start,
                                  const int* __restrict__ cstart, int S, int nch, const double* __restrict__ src,
                                  int width, double* __restrict__ part) {
  const int w = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (w >= nch) return;  // uniform across the warp
  const int q = seg_of(cstart, S, w);
  const int b = start[q] + (w - cstart[q]) * SEG_CHUNK;
  const int e = min(start[q + 1], b + SEG_CHUNK);
  const double INF = __longlong_as_double(0x7ff0000000000000LL);
  double v[6] = {INF, INF, INF, -INF, -INF, -INF};
  const int lb = b + lane * SEG_LANE, le = min(e, lb + SEG_LANE);
  for (int p = lb; p < le; p++) {
    const double* x = src + (long long)width * perm[p];
    for (int a = 0; a < 3; a++) {
      v[a] = smin(v[a], x[a]);
      v[3 + a] = smax(v[3 + a], x[width == 6 ? 3 + a : a]);
    }
  }
  warp_bounds(v);
  if (lane == 0)
    for (int a = 0; a < 6; a++) part[6 * (long long)w + a] = v[a];
}

// Phase 2: warp q folds segment q's chunks.
__global__ void k_prep_seg_bounds(const int* __restrict__ cstart, int S, const double* __restrict__ part,
                                  double* __restrict__ out) {
  const int q = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (q >= S) return;
  const double INF = __longlong_as_double(0x7ff0000000000000LL);
  double v[6] = {INF, INF, INF, -INF, -INF, -INF};
  const int c0 = cstart[q], c1 = cstart[q + 1], per = (c1 - c0 + 31) / 32;
  const int lb = c0 + lane * per, le = min(c1, lb + per);
  for (int c = lb; c < le; c++)
    for (int a = 0; a < 3; a++) {
      v[a] = smin(v[a], part[6 * (long long)c + a]);
      v[3 + a] = smax(v[3 + a], part[6 * (long long)c + 3 + a]);
    }
  warp_bounds(v);
  if (lane == 0)
    for (int a = 0; a < 6; a++) out[6 * (long long)q + a] = v[a];
}

// Sort key of each position of the order: its segment in the high bits and,
// in a segment that splits, the rank of its centroid on the segment's
// widest centroid axis (the host's choice: the first axis of largest
// extent); 0 in a leaf, which keeps its order.
__global__ void k_prep_keys(const int* __restrict__ perm, int n, const int* __restrict__ start,
                            const int* __restrict__ splits, int S, const double* __restrict__ cb,
                            const int* __restrict__ rank, int rank_bits, unsigned long long* __restrict__ key) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int q = seg_of(start, S, p);
    unsigned long long r = 0;
    if (splits[q]) {
      const double* c = cb + 6 * (long long)q;
      int axis = 0;
      for (int k = 1; k < 3; k++)
        if (c[3 + k] - c[k] > c[3 + axis] - c[axis]) axis = k;
      r = (unsigned)rank[(long long)axis * n + perm[p]];
    }
    key[p] = ((unsigned long long)q << rank_bits) | r;
  }
}

// Leaves' canonical order: segment, then primitive id.
__global__ void k_prep_leaf_keys(const int* __restrict__ perm, int n, const int* __restrict__ start, int S,
                                 int id_bits, unsigned long long* __restrict__ key) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
    key[p] = ((unsigned long long)seg_of(start, S, p) << id_bits) | (unsigned)perm[p];
}

// One internal node per entry of `nodes`: {me, left segment, right
// segment, left ref idx, left ref count, right ref idx, right ref count}.
// Child boxes are the next level's segment bounds, padded.
__global__ void k_prep_nodes(const int* __restrict__ nodes, int m, const double* __restrict__ nb,
                             const unsigned long long* __restrict__ scale_bits, double2* __restrict__ bvh) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    const int* d = nodes + 7 * (long long)i;
    const double pad = 1e-7 * (1.0 + bitsd(*scale_bits));
    const double* L = nb + 6 * (long long)d[1];
    const double* R = nb + 6 * (long long)d[2];
    double2* N = bvh + 7 * (long long)d[0];
    N[0] = double2{L[0] - pad, L[1] - pad};
    N[1] = double2{L[2] - pad, L[3] + pad};
    N[2] = double2{L[4] + pad, L[5] + pad};
    N[3] = double2{R[0] - pad, R[1] - pad};
    N[4] = double2{R[2] - pad, R[3] + pad};
    N[5] = double2{R[4] + pad, R[5] + pad};
    N[6] = double2{pack2(d[3], d[4]), pack2(d[5], d[6])};
  }
}

__global__ void k_prep_gather(const int* __restrict__ order, int n, const double2* __restrict__ brute,
                              double2* __restrict__ btris) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 5LL * n; i += (long long)gridDim.x * blockDim.x)
    btris[i] = brute[5 * (long long)order[i / 5] + i % 5];
}

// Single-precision copy of a BVH (FNode layout): child boxes rounded
// outwards, child references as they are, and in fbvh[0].x the largest
// |coordinate| of any present child's box, by atomicMax on the bits
// (non-negative floats order like their encodings; fbvh[0] zeroed first).
__global__ void k_prep_fbvh(const double2* __restrict__ bvh, int nb, float4* __restrict__ fbvh) {
  float scale = 0.0f;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nb; k += gridDim.x * blockDim.x) {
    const double2* N = bvh + 7 * (long long)k;
    double b[12];
    for (int j = 0; j < 6; j++) {
      const double2 v = N[j];
      b[2 * j] = v.x;
      b[2 * j + 1] = v.y;
    }
    const double2 refs = N[6];
    float f[12];
    for (int j = 0; j < 12; j++) {
      // b: lmn xyz, lmx xyz, rmn xyz, rmx xyz
      const bool lower = (j / 3) % 2 == 0;
      f[j] = lower ? __double2float_rd(b[j]) : __double2float_ru(b[j]);
    }
    for (int j = 0; j < 12; j++) {
      const float m = fabsf(f[j]);
      // present children only; a NaN coordinate makes the scale NaN
      if (hi32(j < 6 ? refs.x : refs.y) >= 0 && (m > scale || m != m) && scale == scale) scale = m;
    }
    float4* F = fbvh + RTB_FBVH_HEAD + 4 * (long long)k;
    F[0] = make_float4(f[0], f[1], f[2], f[3]);
    F[1] = make_float4(f[4], f[5], f[6], f[7]);
    F[2] = make_float4(f[8], f[9], f[10], f[11]);
    F[3] = make_float4(__int_as_float(lo32(refs.x)), __int_as_float(hi32(refs.x)), __int_as_float(lo32(refs.y)),
                       __int_as_float(hi32(refs.y)));
  }
  // a NaN scale becomes +inf, which disables the float tests (RayF::all)
  if (scale != scale) scale = __int_as_float(0x7f800000);
  atomicMax(reinterpret_cast<unsigned*>(fbvh), __float_as_uint(scale));
}

// Records in BVH order back to mesh order (each record carries its triangle
// id), with each triangle's normal normalize(e1 x e2) from the record's
// edges, the operations the host and k_prep_records perform.
__global__ void k_prep_unpermute(const double2* __restrict__ btris, int n, double2* __restrict__ brute,
                                 double4* __restrict__ normals) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double2 r[5];
    for (int k = 0; k < 5; k++) r[k] = btris[5 * (long long)i + k];
    const int t = lo32(r[4].y);
    if ((unsigned)t >= (unsigned)n) continue;  // not a record of this mesh
    for (int k = 0; k < 5; k++) brute[5 * (long long)t + k] = r[k];
    const V3 e1 = mk(r[1].y, r[2].x, r[2].y), e2 = mk(r[3].x, r[3].y, r[4].x);
    const V3 nn = normalize(cross(e1, e2));
    normals[t] = double4{nn.x, nn.y, nn.z, 0.0};
  }
}

// The cell of each k-d leaf from the splits on its root path (leaf_path:
// bit j = right at depth j): per axis, lo = the largest split the path
// turns right at and hi = the smallest it turns left at (-inf / +inf when
// there is none), so the leaf's cell is lo < p <= hi.  A leaf whose path
// meets a NaN split, or does not lead to it, gets a NaN lo, which sends
// callers back to the walk.  Internal nodes get the same mark.
__global__ void k_prep_cells(const double2* __restrict__ kd, int nk, const int2* __restrict__ leaf_path,
                             double2* __restrict__ cells) {
  const double INF = __longlong_as_double(0x7ff0000000000000LL);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nk; k += gridDim.x * blockDim.x) {
    double lo[3] = {-INF, -INF, -INF}, hi[3] = {INF, INF, INF};
    bool ok = hi32(kd[4 * (long long)k + 3].y) < 0;  // leaves only
    if (ok) {
      const int2 pd = leaf_path[k];
      int node = 0;
      for (int j = 0; ok && j < pd.y && j < 31; j++) {
        const double2 n3 = kd[4 * (long long)node + 3];
        const int right = lo32(n3.y), axis = hi32(n3.y);
        const double split = n3.x;
        if (axis < 0 || axis > 2 || split != split) {
          ok = false;
          break;
        }
        if ((pd.x >> j) & 1) {
          lo[axis] = fmax(lo[axis], split);
          node = right;
        } else {
          hi[axis] = fmin(hi[axis], split);
          node = node + 1;
        }
        if (node < 0 || node >= nk) ok = false;
      }
      ok = ok && node == k;
    }
    if (!ok) lo[0] = __longlong_as_double(0x7ff8000000000000LL);
    double2* C = cells + 3 * (long long)k;
    C[0] = double2{lo[0], lo[1]};
    C[1] = double2{lo[2], hi[0]};
    C[2] = double2{hi[1], hi[2]};
  }
}

// Leaf entries per k-d node (0 for internal nodes).
__global__ void k_prep_leaf_counts(const double2* __restrict__ kd, int nk, int* __restrict__ cnt) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nk; k += gridDim.x * blockDim.x) {
    const int h = hi32(kd[4 * (long long)k + 3].y);
    cnt[k] = h < 0 ? -1 - h : 0;
  }
}

// Every leaf entry in (leaf, position) order as (triangle, {leaf, position}),
// and the per-triangle occurrence counts.
__global__ void k_prep_occ_entries(const double2* __restrict__ kd, int nk, const int* __restrict__ eoff,
                                   const int* __restrict__ leaf_tris, unsigned* __restrict__ tkey,
                                   unsigned long long* __restrict__ val, int* __restrict__ tcount) {
  const int k = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (k >= nk) return;
  const double w = kd[4 * (long long)k + 3].y;
  const int h = hi32(w);
  if (h >= 0) return;
  const int first = lo32(w), count = -1 - h;
  for (int p = lane; p < count; p += 32) {
    const int t = leaf_tris[first + p];
    tkey[eoff[k] + p] = (unsigned)t;
    val[eoff[k] + p] = (unsigned long long)(unsigned)k | ((unsigned long long)(unsigned)p << 32);
    atomicAdd(tcount + t, 1);
  }
}

// Tree shape: count(n) internal nodes below a segment of n primitives.
struct Shape {
  int leaf;
  std::map<int, int> memo;
  int count(int n) {
    if (n <= leaf) return 0;
    auto it = memo.find(n);
    if (it != memo.end()) return it->second;
    const int c = 1 + count(n / 2) + count(n - n / 2);
    memo[n] = c;
    return c;
  }
};

struct Seg {
  int off, n, node;  // node: preorder index when it splits, -1 for a leaf
};

// CUB temporary storage from the arena, grown on demand (an outgrown block
// stays in the arena until the next reset).
struct CubTemp {
  KdArena& A;
  void* p = nullptr;
  size_t cap = 0;
  cudaError_t need(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    char* t = nullptr;
    cudaError_t e = A.get(&t, bytes);
    if (e == cudaSuccess) {
      p = t;
      cap = bytes;
    }
    return e;
  }
};

// The k-d occurrence lists: every leaf entry (leaf, position) stably sorted
// by triangle, so each triangle's entries stay in (leaf, position) order,
// and occ_off[t] = the first entry of triangle t (n + 1 offsets).  Queued
// on s.
cudaError_t occ_device(const double2* d_kd_nodes, int nk, const int* d_leaf_tris, int n_index, int n,
                       cudaStream_t s, KdArena& A, CubTemp& temp, int2* occ, int* occ_off) {
#define OCK(call)                          \
  do {                                     \
    cudaError_t e_ = (call);               \
    if (e_ != cudaSuccess) return e_;      \
  } while (0)
  const int BS = 256;
  int *d_cnt, *d_eoff, *d_tcount;
  unsigned* d_tkey[2];
  unsigned long long* d_val;
  OCK(A.get(&d_cnt, (size_t)nk + 1));
  OCK(A.get(&d_eoff, (size_t)nk + 1));
  OCK(A.get(&d_tcount, (size_t)n + 1));
  OCK(A.get(&d_tkey[0], (size_t)n_index));
  OCK(A.get(&d_tkey[1], (size_t)n_index));
  OCK(A.get(&d_val, (size_t)n_index));
  OCK(cudaMemsetAsync(d_tcount, 0, (n + 1) * sizeof(int), s));
  OCK(cudaMemsetAsync(d_cnt + nk, 0, sizeof(int), s));
  if (nk > 0) k_prep_leaf_counts<<<grid_for(nk, BS), BS, 0, s>>>(d_kd_nodes, nk, d_cnt);
  OCK(cudaGetLastError());
  size_t tb = 0;
  OCK(cub::DeviceScan::ExclusiveSum(nullptr, tb, d_cnt, d_eoff, nk + 1, s));
  OCK(temp.need(tb));
  tb = temp.cap;
  OCK(cub::DeviceScan::ExclusiveSum(temp.p, tb, d_cnt, d_eoff, nk + 1, s));
  if (nk > 0)
    k_prep_occ_entries<<<(int)((32LL * nk + 255) / 256), 256, 0, s>>>(d_kd_nodes, nk, d_eoff, d_leaf_tris,
                                                                        d_tkey[0], d_val, d_tcount);
  OCK(cudaGetLastError());
  const int tri_bits = bits_for(n);
  unsigned long long* occ64 = reinterpret_cast<unsigned long long*>(occ);
  tb = 0;
  OCK(cub::DeviceRadixSort::SortPairs(nullptr, tb, d_tkey[0], d_tkey[1], d_val, occ64, n_index, 0, tri_bits, s));
  OCK(temp.need(tb));
  tb = temp.cap;
  OCK(cub::DeviceRadixSort::SortPairs(temp.p, tb, d_tkey[0], d_tkey[1], d_val, occ64, n_index, 0, tri_bits, s));
  tb = 0;
  OCK(cub::DeviceScan::ExclusiveSum(nullptr, tb, d_tcount, occ_off, n + 1, s));
  OCK(temp.need(tb));
  tb = temp.cap;
  OCK(cub::DeviceScan::ExclusiveSum(temp.p, tb, d_tcount, occ_off, n + 1, s));
#undef OCK
  return cudaSuccess;
}

}  // namespace

int bvh_internal_nodes(int n, int leaf) {
  Shape sh{leaf, {}};
  return std::max(1, sh.count(n));
}

std::string prep_mesh_device(const double* h_vertices, int n, const double2* d_kd_nodes, int n_kd_nodes,
                             const int* d_leaf_tris, const int2* d_leaf_path, int n_index, int leaf, cudaStream_t s,
                             KdArena* arena, const MeshPrepOut& out, cudaError_t* cuda_err) {
  *cuda_err = cudaSuccess;
  if (n <= leaf) return "mesh too small for the device preparation";
#define PCK(call)                                                               \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      *cuda_err = e_;                                                           \
      return std::string("mesh preparation: " #call ": ") + cudaGetErrorString(e_); \
    }                                                                           \
  } while (0)
  KdArena& A = *arena;
  A.reset();
  const int BS = 256;
  // ---- records, boxes, centroids, scale
  double *d_vertices, *d_box, *d_cen;
  unsigned long long* d_scale;
  PCK(A.get(&d_vertices, 9 * (size_t)n));
  PCK(cudaMemcpyAsync(d_vertices, h_vertices, 9 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s));
  PCK(A.get(&d_box, 6 * (size_t)n));
  PCK(A.get(&d_cen, 3 * (size_t)n));
  PCK(A.get(&d_scale, 1));
  PCK(cudaMemsetAsync(d_scale, 0, sizeof(unsigned long long), s));
  k_prep_records<<<grid_for(n, BS), BS, 0, s>>>(d_vertices, n, out.brute, out.normals, d_box, d_cen, d_scale);
  PCK(cudaGetLastError());

  // ---- centroid ranks per axis (position in (centroid, id) order)
  const int rank_bits = bits_for(n);
  int *d_rank, *d_perm[2], *d_ival;
  unsigned long long *d_key[2];
  double *d_dkey[2];
  PCK(A.get(&d_rank, 3 * (size_t)n));
  for (int b = 0; b < 2; b++) {
    PCK(A.get(&d_perm[b], (size_t)n));
    PCK(A.get(&d_key[b], (size_t)n));
  }
  d_dkey[0] = reinterpret_cast<double*>(d_key[0]);
  d_dkey[1] = reinterpret_cast<double*>(d_key[1]);
  PCK(A.get(&d_ival, (size_t)n));
  void* d_temp = nullptr;
  size_t temp_cap = 0;
  auto temp = [&](size_t bytes) -> cudaError_t {
    if (bytes <= temp_cap) return cudaSuccess;
    char* t = nullptr;
    cudaError_t e = A.get(&t, bytes);  // the old block stays in the arena until the build ends
    if (e == cudaSuccess) {
      d_temp = t;
      temp_cap = bytes;
    }
    return e;
  };
  for (int a = 0; a < 3; a++) {
    k_prep_axis_keys<<<grid_for(n, BS), BS, 0, s>>>(d_cen, n, a, d_dkey[0], d_ival);
    PCK(cudaGetLastError());
    size_t tb = 0;
    PCK(cub::DeviceRadixSort::SortPairs(nullptr, tb, d_dkey[0], d_dkey[1], d_ival, d_perm[0], n, 0, 64, s));
    PCK(temp(tb));
    tb = temp_cap;
    PCK(cub::DeviceRadixSort::SortPairs(d_temp, tb, d_dkey[0], d_dkey[1], d_ival, d_perm[0], n, 0, 64, s));
    k_prep_rank<<<grid_for(n, BS), BS, 0, s>>>(d_perm[0], n, d_rank + (size_t)a * n);
    PCK(cudaGetLastError());
  }

  // ---- the BVH, level by level; the host plans every level's segments,
  // and every level takes its own buffers from the arena, so nothing waits
  // for the device until the end
  Shape shape{leaf, {}};
  std::vector<Seg> cur{{0, n, 0}};
  // bounds of the segments `start` of the current order into out6
  auto seg_bounds = [&](const std::vector<int>& start, const int* d_st, const double* src, int width,
                        double* out6) -> cudaError_t {
    const int S = (int)start.size() - 1;
    std::vector<int> cstart(S + 1, 0);
    for (int q = 0; q < S; q++) cstart[q + 1] = cstart[q] + (start[q + 1] - start[q] + SEG_CHUNK - 1) / SEG_CHUNK;
    const int nch = cstart[S];
    int* d_cs = nullptr;
    double* d_part = nullptr;
    cudaError_t e;
    if ((e = A.get(&d_cs, (size_t)S + 1)) != cudaSuccess || (e = A.get(&d_part, 6 * (size_t)nch)) != cudaSuccess)
      return e;
    e = cudaMemcpyAsync(d_cs, cstart.data(), (S + 1) * sizeof(int), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    k_prep_seg_chunks<<<(int)((32LL * nch + 255) / 256), 256, 0, s>>>(d_perm[0], d_st, d_cs, S, nch, src, width,
                                                                       d_part);
    k_prep_seg_bounds<<<(int)((32LL * S + 255) / 256), 256, 0, s>>>(d_cs, S, d_part, out6);
    return cudaGetLastError();
  };
  auto upload = [&](const std::vector<int>& h, int** d) -> cudaError_t {
    cudaError_t e = A.get(d, h.size());
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice, s);
  };
  k_prep_iota<<<grid_for(n, BS), BS, 0, s>>>(d_perm[0], n);
  PCK(cudaGetLastError());
  for (;;) {
    const int S = (int)cur.size();
    bool any = false;
    for (const Seg& g : cur) any |= g.node >= 0;
    std::vector<int> start(S + 1);
    for (int q = 0; q < S; q++) start[q] = cur[q].off;
    start[S] = n;
    int* d_start = nullptr;
    PCK(upload(start, &d_start));
    if (!any) {
      // leaves to id order; the result is the primitive order
      k_prep_leaf_keys<<<grid_for(n, BS), BS, 0, s>>>(d_perm[0], n, d_start, S, rank_bits, d_key[0]);
      PCK(cudaGetLastError());
      size_t tb = 0;
      const int end_bit = rank_bits + bits_for(S);
      PCK(cub::DeviceRadixSort::SortPairs(nullptr, tb, d_key[0], d_key[1], d_perm[0], d_perm[1], n, 0, end_bit, s));
      PCK(temp(tb));
      tb = temp_cap;
      PCK(cub::DeviceRadixSort::SortPairs(d_temp, tb, d_key[0], d_key[1], d_perm[0], d_perm[1], n, 0, end_bit, s));
      std::swap(d_perm[0], d_perm[1]);
      break;
    }
    std::vector<int> splits(S);
    std::vector<Seg> next;
    std::vector<int> nodes;  // 7 per splitting segment (see k_prep_nodes)
    for (int q = 0; q < S; q++) {
      const Seg& g = cur[q];
      splits[q] = g.node >= 0;
      if (g.node < 0) {
        next.push_back(g);
        continue;
      }
      const int mid = g.n / 2;
      const Seg l{g.off, mid, mid > leaf ? g.node + 1 : -1};
      const Seg r{g.off + mid, g.n - mid, g.n - mid > leaf ? g.node + 1 + shape.count(mid) : -1};
      const int lq = (int)next.size();
      next.push_back(l);
      next.push_back(r);
      nodes.insert(nodes.end(), {g.node, lq, lq + 1, l.node >= 0 ? l.node : l.off, l.node >= 0 ? 0 : l.n,
                                 r.node >= 0 ? r.node : r.off, r.node >= 0 ? 0 : r.n});
    }
    // centroid bounds of this level's segments, then the split sort
    int* d_splits = nullptr;
    double* d_cb = nullptr;
    PCK(upload(splits, &d_splits));
    PCK(A.get(&d_cb, 6 * (size_t)S));
    PCK(seg_bounds(start, d_start, d_cen, 3, d_cb));
    k_prep_keys<<<grid_for(n, BS), BS, 0, s>>>(d_perm[0], n, d_start, d_splits, S, d_cb, d_rank, rank_bits,
                                               d_key[0]);
    PCK(cudaGetLastError());
    size_t tb = 0;
    const int end_bit = rank_bits + bits_for(S);
    PCK(cub::DeviceRadixSort::SortPairs(nullptr, tb, d_key[0], d_key[1], d_perm[0], d_perm[1], n, 0, end_bit, s));
    PCK(temp(tb));
    tb = temp_cap;
    PCK(cub::DeviceRadixSort::SortPairs(d_temp, tb, d_key[0], d_key[1], d_perm[0], d_perm[1], n, 0, end_bit, s));
    std::swap(d_perm[0], d_perm[1]);
    // the children's boxes, then this level's nodes
    const int S2 = (int)next.size();
    std::vector<int> nstart(S2 + 1);
    for (int q = 0; q < S2; q++) nstart[q] = next[q].off;
    nstart[S2] = n;
    int *d_nstart = nullptr, *d_nodes = nullptr;
    double* d_nb = nullptr;
    PCK(upload(nstart, &d_nstart));
    PCK(A.get(&d_nb, 6 * (size_t)S2));
    PCK(seg_bounds(nstart, d_nstart, d_box, 6, d_nb));
    PCK(upload(nodes, &d_nodes));
    const int m = (int)nodes.size() / 7;
    k_prep_nodes<<<grid_for(m, BS), BS, 0, s>>>(d_nodes, m, d_nb, d_scale, out.bvh);
    PCK(cudaGetLastError());
    cur.swap(next);
  }
  k_prep_gather<<<grid_for(5LL * n, BS), BS, 0, s>>>(d_perm[0], n, out.brute, out.btris);
  PCK(cudaGetLastError());

  // ---- the single-precision BVH, the k-d leaf cells
  const int nb = bvh_internal_nodes(n, leaf);
  PCK(cudaMemsetAsync(out.fbvh, 0, RTB_FBVH_HEAD * sizeof(float4), s));
  k_prep_fbvh<<<grid_for(nb, BS), BS, 0, s>>>(out.bvh, nb, out.fbvh);
  if (n_kd_nodes > 0)
    k_prep_cells<<<grid_for(n_kd_nodes, BS), BS, 0, s>>>(d_kd_nodes, n_kd_nodes, d_leaf_path, out.cells);
  PCK(cudaGetLastError());

  // ---- k-d occurrences
  CubTemp occ_temp{A};
  PCK(occ_device(d_kd_nodes, n_kd_nodes, d_leaf_tris, n_index, n, s, A, occ_temp, out.occ, out.occ_off));
  PCK(cudaStreamSynchronize(s));
#undef PCK
  return "";
}

std::string derive_mesh_device(const double2* d_bvh, int nb, const double2* d_btris, int n,
                               const double2* d_kd_nodes, int n_kd_nodes, const int* d_leaf_tris,
                               const int2* d_leaf_path, int n_index, cudaStream_t s, KdArena* arena, float4* fbvh,
                               double2* cells, double2* brute, double4* normals, int2* occ, int* occ_off,
                               cudaError_t* cuda_err) {
  *cuda_err = cudaSuccess;
  KdArena& A = *arena;
  A.reset();
  const int BS = 256;
  cudaError_t e = cudaSuccess;
  if (d_bvh && fbvh && nb > 0) {
    e = cudaMemsetAsync(fbvh, 0, RTB_FBVH_HEAD * sizeof(float4), s);
    if (e == cudaSuccess) k_prep_fbvh<<<grid_for(nb, BS), BS, 0, s>>>(d_bvh, nb, fbvh);
  }
  if (e == cudaSuccess && n_kd_nodes > 0)
    k_prep_cells<<<grid_for(n_kd_nodes, BS), BS, 0, s>>>(d_kd_nodes, n_kd_nodes, d_leaf_path, cells);
  if (e == cudaSuccess && n > 0) k_prep_unpermute<<<grid_for(n, BS), BS, 0, s>>>(d_btris, n, brute, normals);
  if (e == cudaSuccess) e = cudaGetLastError();
  CubTemp temp{A};
  if (e == cudaSuccess) e = occ_device(d_kd_nodes, n_kd_nodes, d_leaf_tris, n_index, n, s, A, temp, occ, occ_off);
  if (e != cudaSuccess) {
    *cuda_err = e;
    return std::string("mesh arrays from the records: ") + cudaGetErrorString(e);
  }
  return "";
}

}  // namespace rtb
