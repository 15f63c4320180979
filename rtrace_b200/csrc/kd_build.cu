// KdTree::new(triangles, 16, 10) (src/mesh.rs:75-197) on the device, one
// depth of the tree at a time.
//
// The reference builds recursively (build_recursive, src/mesh.rs:125-197).
// A node at depth d with more than 10 triangles and d < 16:
//   - stable-sorts its list by triangle centre on axis d % 3,
//   - takes the centre of element n/2 as the split,
//   - sends every triangle whose box starts at or below the split left and
//     every one whose box ends above it right, both in sorted order
//     (straddlers go both ways),
//   - moves one triangle across when a side is empty,
//   - recurses left, then right.
// A node's bounds are the union of its list's triangle boxes.
//
// Nodes of one depth are independent, so a whole depth is built at once:
//   1. one stable radix sort of the whole depth by (node, centre rank): the
//      centres of each axis are ranked once (equal centres, -0 and +0
//      included, share a rank), and a leaf's entries all get rank 0 so that
//      its list keeps its order,
//   2. each node's split, left/right flags and their exclusive scans,
//   3. one scatter into the next depth's lists,
//   4. the children's bounds, reduced in list order, so that the sign of a
//      zero bound is the one the host's sequential fmin/fmax fold keeps.
// The host keeps each depth's list offsets (at most 2^16 nodes a depth),
// lays the nodes out in preorder from subtree sizes, and a last kernel
// gathers the leaf lists in that order.
//
// The sorts and the scans are CUB's device-wide radix sort and scan (header
// source in the CUDA toolkit); the rest is the kernels below.
#include "kd_build.hpp"

#include <cub/device/device_scan.cuh>
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <climits>
#include <memory>

namespace rtb {
namespace {

constexpr int KD_MAX_DEPTH = 16;  // KdTree::new(triangles, 16, 10)
constexpr int KD_LEAF = 10;
constexpr int RED_LANE = 32;                 // entries one lane folds for the bounds
constexpr int RED_CHUNK = 32 * RED_LANE;     // entries one warp folds

const char* kNanPanic = "called `Option::unwrap()` on a `None` value";

// glibc fmin / fmax, which the host builder's fold calls: a NaN argument is
// ignored and a tie keeps the first argument (fmin(-0, +0) = -0,
// fmin(+0, -0) = +0).  The fold then selects the first minimal element in
// list order, and any reduction that keeps operands in list order
// reproduces it.
__device__ __forceinline__ double fmin_first(double a, double b) { return (b < a || a != a) ? b : a; }
__device__ __forceinline__ double fmax_first(double a, double b) { return (b > a || a != a) ? b : a; }

// Node of level entry p: the k with off[k] <= p < off[k + 1].
__device__ __forceinline__ int node_of(const int* __restrict__ off, int K, int p) {
  int lo = 0, hi = K;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (off[mid] <= p) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Per triangle: Triangle::center, cen[3i + a] = (v0 + v1 + v2) / 3, and its
// box, box[6i + a] = min, box[6i + 3 + a] = max (folded from v0 as the host
// builder does).
__global__ void k_kd_tri_prep(const double* __restrict__ v, long long n, double* __restrict__ cen,
                              double* __restrict__ box) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double* t = v + 9 * i;
    for (int a = 0; a < 3; a++) {
      const double p0 = t[a], p1 = t[3 + a], p2 = t[6 + a];
      box[6 * i + a] = fmin_first(fmin_first(p0, p1), p2);
      box[6 * i + 3 + a] = fmax_first(fmax_first(p0, p1), p2);
      cen[3 * i + a] = (p0 + p1 + p2) / 3.0;
    }
  }
}

__global__ void k_kd_iota(int* __restrict__ e, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) e[i] = i;
}

// Centre on one axis, -0 as +0 (the reference sorts with partial_cmp, under
// which they are equal; a radix sort would order them), for ranking.
__global__ void k_kd_axis_keys(const double* __restrict__ cen, int n, int axis, double* __restrict__ key,
                               int* __restrict__ val) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double c = cen[3 * (long long)i + axis];
    key[i] = c == 0.0 ? 0.0 : c;
    val[i] = i;
  }
}

// 1 where a sorted centre differs from the one before it (NaN differs from
// everything, so each NaN gets its own rank).
__global__ void k_kd_rank_heads(const double* __restrict__ key, int n, int* __restrict__ head) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    head[i] = i == 0 || !(key[i] == key[i - 1]);
}

// rank[tri] = number of distinct centres below it.
__global__ void k_kd_rank_scatter(const int* __restrict__ tri, const int* __restrict__ incl, int n,
                                  int* __restrict__ rank) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) rank[tri[i]] = incl[i] - 1;
}

// Sort key of each entry: its node in the high bits, its centre's rank on
// this depth's axis in the low rank_bits (0 in a leaf, whose list keeps its
// order).  A NaN centre in a splitting node raises the flag: the
// reference's unwrap panics on it.
__global__ void k_kd_keys(const int* __restrict__ e, int m, const int* __restrict__ off, const int* __restrict__ child,
                          int K, const double* __restrict__ cen, const int* __restrict__ rank, int axis, int rank_bits,
                          unsigned long long* __restrict__ key, int* __restrict__ flags) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < m; p += gridDim.x * blockDim.x) {
    const int k = node_of(off, K, p);
    unsigned long long r = 0;
    if (child[k] >= 0) {
      const int t = e[p];
      const double c = cen[3 * (long long)t + axis];
      if (c != c) atomicOr(flags, 1);
      r = (unsigned)rank[t];
    }
    key[p] = ((unsigned long long)k << rank_bits) | r;
  }
}

// Split of each splitting node: the centre of its sorted element n/2.
__global__ void k_kd_split(const int* __restrict__ off, const int* __restrict__ child, int K,
                           const int* __restrict__ sorted, const double* __restrict__ cen, int axis,
                           double* __restrict__ split) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
    double s = 0.0;
    if (child[k] >= 0) {
      const int c = off[k + 1] - off[k];
      s = cen[3 * (long long)sorted[off[k] + c / 2] + axis];
    }
    split[k] = s;
  }
}

// Left flag: the box starts at or below the split; right flag: it ends
// above it.  Entry m (one past the end) is 0 so that the exclusive scans
// carry the totals.
__global__ void k_kd_flags(const int* __restrict__ sorted, int m, const int* __restrict__ off,
                           const int* __restrict__ child, int K, const double* __restrict__ box, int axis,
                           const double* __restrict__ split, int* __restrict__ fl, int* __restrict__ fr) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= m; p += gridDim.x * blockDim.x) {
    int l = 0, r = 0;
    if (p < m) {
      const int k = node_of(off, K, p);
      if (child[k] >= 0) {
        const double* b = box + 6 * (long long)sorted[p];
        l = b[axis] <= split[k];
        r = b[3 + axis] > split[k];
      }
    }
    fl[p] = l;
    fr[p] = r;
  }
}

// Child list sizes of each splitting node, with the reference's empty-side
// rule (src/mesh.rs:174-178): an empty left list takes the right list's
// last triangle (mode 1), an empty right list the left list's last (mode 2).
__global__ void k_kd_children(const int* __restrict__ off, const int* __restrict__ child, int K,
                              const int* __restrict__ gl, const int* __restrict__ gr, int* __restrict__ cc,
                              int* __restrict__ mode, int* __restrict__ flags) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
    const int c = child[k];
    if (c < 0) continue;
    int nl = gl[off[k + 1]] - gl[off[k]], nr = gr[off[k + 1]] - gr[off[k]];
    int md = 0;
    if (nl == 0 && nr == 0) {
      atomicOr(flags, 2);  // only a NaN box can do this, and its centre is NaN too
    } else if (nl == 0) {
      md = 1;
      nl = 1;
      nr -= 1;
    } else if (nr == 0) {
      md = 2;
      nr = 1;
      nl -= 1;
    }
    cc[c] = nl;
    cc[c + 1] = nr;
    mode[k] = md;
  }
}

// Writes each splitting node's entries into its children's lists, in
// sorted order, at their ranks among the node's left / right entries.
__global__ void k_kd_scatter(const int* __restrict__ sorted, int m, const int* __restrict__ off,
                             const int* __restrict__ child, int K, const int* __restrict__ fl,
                             const int* __restrict__ fr, const int* __restrict__ gl, const int* __restrict__ gr,
                             const int* __restrict__ mode, const int* __restrict__ coff, int* __restrict__ next) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < m; p += gridDim.x * blockDim.x) {
    const int k = node_of(off, K, p);
    const int c = child[k];
    if (c < 0) continue;
    const int t = sorted[p], b = off[k], en = off[k + 1];
    const int lo = coff[c], ro = coff[c + 1];
    if (fl[p]) {
      const int r = gl[p] - gl[b], n = gl[en] - gl[b];
      if (mode[k] == 2 && r == n - 1) next[ro] = t;
      else next[lo + r] = t;
    }
    if (fr[p]) {
      const int r = gr[p] - gr[b], n = gr[en] - gr[b];
      if (mode[k] == 1 && r == n - 1) next[lo] = t;
      else next[ro + r] = t;
    }
  }
}

// Folds lane values in lane order; lane 0 ends with the fold of all 32.
__device__ __forceinline__ void warp_fold_bounds(double v[6]) {
  for (int o = 1; o < 32; o <<= 1)
    for (int a = 0; a < 3; a++) {
      const double dn = __shfl_down_sync(0xffffffffu, v[a], o);
      const double dx = __shfl_down_sync(0xffffffffu, v[3 + a], o);
      v[a] = fmin_first(v[a], dn);
      v[3 + a] = fmax_first(v[3 + a], dx);
    }
}

// Bounds, phase 1: warp w folds chunk w, up to RED_CHUNK consecutive
// entries of one node (chunks of node k are cstart[k] .. cstart[k+1]-1),
// each lane RED_LANE consecutive entries in order.
__global__ void k_kd_bounds_chunks(const int* __restrict__ e, const int* __restrict__ off,
                                   const int* __restrict__ cstart, int K, int nchunks,
                                   const double* __restrict__ box, double* __restrict__ part) {
  const int w = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (w >= nchunks) return;  // uniform across the warp
  const int k = node_of(cstart, K, w);
  const int b = off[k] + (w - cstart[k]) * RED_CHUNK;
  const int en = min(off[k + 1], b + RED_CHUNK);
  const double INF = __longlong_as_double(0x7ff0000000000000LL);
  double v[6] = {INF, INF, INF, -INF, -INF, -INF};
  const int lb = b + lane * RED_LANE, le = min(en, lb + RED_LANE);
  for (int p = lb; p < le; p++) {
    const double* x = box + 6 * (long long)e[p];
    for (int a = 0; a < 3; a++) {
      v[a] = fmin_first(v[a], x[a]);
      v[3 + a] = fmax_first(v[3 + a], x[3 + a]);
    }
  }
  warp_fold_bounds(v);
  if (lane == 0)
    for (int a = 0; a < 6; a++) part[6 * (long long)w + a] = v[a];
}

// Bounds, phase 2: warp k folds node k's chunk results in order.  An empty
// list has bounds 0 (KdTree::compute_bounds of an empty list).
__global__ void k_kd_bounds_nodes(const int* __restrict__ cstart, int K, const double* __restrict__ part,
                                  double* __restrict__ bnd) {
  const int k = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (k >= K) return;
  const int c0 = cstart[k], c1 = cstart[k + 1];
  if (c0 == c1) {
    if (lane < 6) bnd[6 * (long long)k + lane] = 0.0;
    return;
  }
  const double INF = __longlong_as_double(0x7ff0000000000000LL);
  double v[6] = {INF, INF, INF, -INF, -INF, -INF};
  const int per = (c1 - c0 + 31) / 32;
  const int lb = c0 + lane * per, le = min(c1, lb + per);
  for (int c = lb; c < le; c++)
    for (int a = 0; a < 3; a++) {
      v[a] = fmin_first(v[a], part[6 * (long long)c + a]);
      v[3 + a] = fmax_first(v[3 + a], part[6 * (long long)c + 3 + a]);
    }
  warp_fold_bounds(v);
  if (lane == 0)
    for (int a = 0; a < 6; a++) bnd[6 * (long long)k + a] = v[a];
}

// Copies leaf k's list (dest[k] >= 0) to the final index array.
__global__ void k_kd_gather_leaves(const int* __restrict__ e, const int* __restrict__ off,
                                   const int* __restrict__ dest, int K, int* __restrict__ idx) {
  const int k = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (k >= K || dest[k] < 0) return;
  for (int i = off[k] + lane; i < off[k + 1]; i += 32) idx[dest[k] + (i - off[k])] = e[i];
}

struct Level {
  int K = 0, m = 0;
  std::vector<int> off;    // K + 1 list offsets
  std::vector<int> child;  // left child's index in the next level, -1 for a leaf
  int* d_e = nullptr;      // the lists, node after node
  std::vector<double> bnd, split;  // 6 and 1 per node, read back from the device
};

int grid_for(long long n, int bs) { return (int)std::max<long long>(1, std::min<long long>((n + bs - 1) / bs, 148LL * 16)); }

}  // namespace

KdArena* kd_arena_new() { return new KdArena(); }
void kd_arena_free(KdArena* a) { delete a; }

std::string kd_build_device(const double* h_vertices, int64_t n, cudaStream_t s, KdArena* arena,
                            std::vector<rt_kd_node_desc>* nodes, std::vector<int32_t>* idx, cudaError_t* cuda_err) {
  nodes->clear();
  idx->clear();
  *cuda_err = cudaSuccess;
  if (n <= 0) return "";  // make_mesh builds no tree for an empty mesh
  if (n > INT_MAX / 2) return "mesh too large for the device k-d build";
#define KCK(call)                                                            \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess) {                                                 \
      *cuda_err = e_;                                                        \
      return std::string("k-d build: " #call ": ") + cudaGetErrorString(e_); \
    }                                                                        \
  } while (0)
  std::unique_ptr<KdArena> own;
  if (!arena) {
    own.reset(new KdArena());
    arena = own.get();
  }
  KdArena& A = *arena;
  A.reset();
  const int BS = 256;
  const int KMAX = 1 << KD_MAX_DEPTH;  // nodes of the deepest level
  double *d_vert = nullptr, *d_cen = nullptr, *d_box = nullptr;
  KCK(A.get(&d_vert, 9 * (size_t)n));
  KCK(A.get(&d_cen, 3 * (size_t)n));
  KCK(A.get(&d_box, 6 * (size_t)n));
  KCK(cudaMemcpyAsync(d_vert, h_vertices, 9 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s));
  k_kd_tri_prep<<<grid_for(n, BS), BS, 0, s>>>(d_vert, n, d_cen, d_box);
  KCK(cudaGetLastError());

  // node-sized buffers (one level at a time; two of the offsets and bounds,
  // for the level being split and the one being made)
  int *d_flags, *d_child, *d_mode, *d_cc, *d_coff, *d_cstart, *d_off[2];
  double *d_split, *d_bnd[2];
  KCK(A.get(&d_flags, 1));
  KCK(A.get(&d_child, KMAX));
  KCK(A.get(&d_mode, KMAX));
  KCK(A.get(&d_cc, KMAX + 1));
  KCK(A.get(&d_coff, KMAX + 1));
  KCK(A.get(&d_cstart, KMAX + 1));
  KCK(A.get(&d_split, KMAX));
  for (int b = 0; b < 2; b++) {
    KCK(A.get(&d_off[b], KMAX + 1));
    KCK(A.get(&d_bnd[b], 6 * (size_t)KMAX));
  }
  KCK(cudaMemsetAsync(d_flags, 0, sizeof(int), s));

  // entry-sized scratch, replaced by larger arrays when a level's lists
  // outgrow it (the lists at most double from one level to the next)
  size_t cap = 0, part_cap = 0, temp_cap = 0;
  unsigned long long *d_kin = nullptr, *d_kout = nullptr;
  double* d_part = nullptr;
  int *d_sorted = nullptr, *d_fl = nullptr, *d_fr = nullptr, *d_gl = nullptr, *d_gr = nullptr;
  void* d_temp = nullptr;
  auto grow_scratch = [&](size_t m) -> cudaError_t {
    if (m <= cap) return cudaSuccess;
    const size_t c = std::max(m, 2 * cap);
    cudaError_t e;
    if ((e = A.get(&d_kin, c)) != cudaSuccess || (e = A.get(&d_kout, c)) != cudaSuccess ||
        (e = A.get(&d_sorted, c)) != cudaSuccess || (e = A.get(&d_fl, c + 1)) != cudaSuccess ||
        (e = A.get(&d_fr, c + 1)) != cudaSuccess || (e = A.get(&d_gl, c + 1)) != cudaSuccess ||
        (e = A.get(&d_gr, c + 1)) != cudaSuccess)
      return e;
    cap = c;
    return cudaSuccess;
  };
  auto grow_temp = [&](size_t bytes) -> cudaError_t {
    if (bytes <= temp_cap) return cudaSuccess;
    char* t = nullptr;
    cudaError_t e = A.get(&t, 2 * bytes);
    if (e != cudaSuccess) return e;
    d_temp = t;
    temp_cap = 2 * bytes;
    return cudaSuccess;
  };
  // bounds of a level's nodes from its lists, into bnd (asynchronous)
  auto level_bounds = [&](const Level& L, const int* off, double* bnd) -> cudaError_t {
    std::vector<int> cstart(L.K + 1, 0);
    for (int k = 0; k < L.K; k++) cstart[k + 1] = cstart[k] + (L.off[k + 1] - L.off[k] + RED_CHUNK - 1) / RED_CHUNK;
    const int nch = cstart[L.K];
    if ((size_t)nch > part_cap) {
      const size_t c = std::max((size_t)nch, 2 * part_cap);
      cudaError_t e = A.get(&d_part, 6 * c);
      if (e != cudaSuccess) return e;
      part_cap = c;
    }
    cudaError_t e = cudaMemcpyAsync(d_cstart, cstart.data(), (L.K + 1) * sizeof(int), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    if (nch > 0)
      k_kd_bounds_chunks<<<(int)((32LL * nch + 255) / 256), 256, 0, s>>>(L.d_e, off, d_cstart, L.K, nch, d_box,
                                                                         d_part);
    k_kd_bounds_nodes<<<(int)((32LL * L.K + 255) / 256), 256, 0, s>>>(d_cstart, L.K, d_part, bnd);
    return cudaGetLastError();
  };

  // rank of every centre among its axis's centres (equal centres share one)
  int rank_bits = 1;
  while ((1LL << rank_bits) < n) rank_bits++;
  int* d_rank = nullptr;
  KCK(A.get(&d_rank, 3 * (size_t)n));
  KCK(grow_scratch(5 * (size_t)n / 2));  // room for the lists of most meshes
  for (int a = 0; a < 3; a++) {
    double* kin = reinterpret_cast<double*>(d_kin);
    double* kout = reinterpret_cast<double*>(d_kout);
    k_kd_axis_keys<<<grid_for(n, BS), BS, 0, s>>>(d_cen, (int)n, a, kin, d_fl);
    KCK(cudaGetLastError());
    size_t tb = 0, t2 = 0;
    KCK(cub::DeviceRadixSort::SortPairs(nullptr, tb, kin, kout, d_fl, d_fr, (int)n, 0, 64, s));
    KCK(cub::DeviceScan::InclusiveSum(nullptr, t2, d_gl, d_gr, (int)n, s));
    KCK(grow_temp(std::max(tb, t2)));
    tb = temp_cap;
    KCK(cub::DeviceRadixSort::SortPairs(d_temp, tb, kin, kout, d_fl, d_fr, (int)n, 0, 64, s));
    k_kd_rank_heads<<<grid_for(n, BS), BS, 0, s>>>(kout, (int)n, d_gl);
    KCK(cudaGetLastError());
    tb = temp_cap;
    KCK(cub::DeviceScan::InclusiveSum(d_temp, tb, d_gl, d_gr, (int)n, s));
    k_kd_rank_scatter<<<grid_for(n, BS), BS, 0, s>>>(d_fr, d_gr, (int)n, d_rank + (size_t)a * n);
    KCK(cudaGetLastError());
  }

  std::vector<Level> levels(1);
  {
    Level& L0 = levels[0];
    L0.K = 1;
    L0.m = (int)n;
    L0.off = {0, (int)n};
    KCK(A.get(&L0.d_e, (size_t)n));
    KCK(cudaMemcpyAsync(d_off[0], L0.off.data(), 2 * sizeof(int), cudaMemcpyHostToDevice, s));
    k_kd_iota<<<grid_for(n, BS), BS, 0, s>>>(L0.d_e, (int)n);
    KCK(cudaGetLastError());
    KCK(level_bounds(L0, d_off[0], d_bnd[0]));
  }

  for (int d = 0;; d++) {
    const int cur = d & 1, nxt = cur ^ 1;
    Level& L = levels[d];
    const int K = L.K, m = L.m, axis = d % 3;
    L.child.assign(K, -1);
    int J = 0;
    for (int k = 0; k < K; k++)
      if (d < KD_MAX_DEPTH && L.off[k + 1] - L.off[k] > KD_LEAF) L.child[k] = 2 * J++;
    L.bnd.resize(6 * (size_t)K);
    if (J == 0) {
      L.split.assign(K, 0.0);
      KCK(cudaMemcpyAsync(L.bnd.data(), d_bnd[cur], L.bnd.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
      break;
    }
    if (2LL * m > INT_MAX) return "k-d tree too large for the device build";
    KCK(grow_scratch((size_t)m));
    KCK(cudaMemcpyAsync(d_child, L.child.data(), K * sizeof(int), cudaMemcpyHostToDevice, s));
    KCK(cudaMemsetAsync(d_cc + 2 * J, 0, sizeof(int), s));

    int node_bits = 1;
    while ((1 << node_bits) < K) node_bits++;
    const int end_bit = rank_bits + node_bits;
    k_kd_keys<<<grid_for(m, BS), BS, 0, s>>>(L.d_e, m, d_off[cur], d_child, K, d_cen, d_rank + (size_t)axis * n,
                                             axis, rank_bits, d_kin, d_flags);
    KCK(cudaGetLastError());
    size_t tb = 0, t2 = 0, t3 = 0;
    KCK(cub::DeviceRadixSort::SortPairs(nullptr, tb, d_kin, d_kout, L.d_e, d_sorted, m, 0, end_bit, s));
    KCK(cub::DeviceScan::ExclusiveSum(nullptr, t2, d_fl, d_gl, m + 1, s));
    KCK(cub::DeviceScan::ExclusiveSum(nullptr, t3, d_cc, d_coff, 2 * J + 1, s));
    KCK(grow_temp(std::max(tb, std::max(t2, t3))));
    tb = temp_cap;
    KCK(cub::DeviceRadixSort::SortPairs(d_temp, tb, d_kin, d_kout, L.d_e, d_sorted, m, 0, end_bit, s));
    k_kd_split<<<grid_for(K, BS), BS, 0, s>>>(d_off[cur], d_child, K, d_sorted, d_cen, axis, d_split);
    k_kd_flags<<<grid_for((long long)m + 1, BS), BS, 0, s>>>(d_sorted, m, d_off[cur], d_child, K, d_box, axis, d_split,
                                                            d_fl, d_fr);
    KCK(cudaGetLastError());
    tb = temp_cap;
    KCK(cub::DeviceScan::ExclusiveSum(d_temp, tb, d_fl, d_gl, m + 1, s));
    tb = temp_cap;
    KCK(cub::DeviceScan::ExclusiveSum(d_temp, tb, d_fr, d_gr, m + 1, s));
    k_kd_children<<<grid_for(K, BS), BS, 0, s>>>(d_off[cur], d_child, K, d_gl, d_gr, d_cc, d_mode, d_flags);
    KCK(cudaGetLastError());
    tb = temp_cap;
    KCK(cub::DeviceScan::ExclusiveSum(d_temp, tb, d_cc, d_coff, 2 * J + 1, s));

    // the one wait of a level: the children's offsets, the checks, this
    // level's splits and bounds
    Level next;
    next.K = 2 * J;
    next.off.resize(2 * J + 1);
    L.split.resize(K);
    int hflags = 0;
    KCK(cudaMemcpyAsync(next.off.data(), d_coff, (2 * J + 1) * sizeof(int), cudaMemcpyDeviceToHost, s));
    KCK(cudaMemcpyAsync(&hflags, d_flags, sizeof(int), cudaMemcpyDeviceToHost, s));
    KCK(cudaMemcpyAsync(L.split.data(), d_split, K * sizeof(double), cudaMemcpyDeviceToHost, s));
    KCK(cudaMemcpyAsync(L.bnd.data(), d_bnd[cur], L.bnd.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    KCK(cudaStreamSynchronize(s));
    if (hflags & 1) return kNanPanic;
    if (hflags & 2) return "k-d build: a node with neither a left nor a right triangle";
    next.m = next.off[2 * J];
    KCK(A.get(&next.d_e, (size_t)next.m));
    KCK(cudaMemcpyAsync(d_off[nxt], next.off.data(), (next.K + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
    k_kd_scatter<<<grid_for(m, BS), BS, 0, s>>>(d_sorted, m, d_off[cur], d_child, K, d_fl, d_fr, d_gl, d_gr, d_mode,
                                                d_coff, next.d_e);
    KCK(cudaGetLastError());
    KCK(level_bounds(next, d_off[nxt], d_bnd[nxt]));
    levels.push_back(std::move(next));
  }

  // preorder layout: subtree node counts and leaf entries bottom-up, then
  // each node's position and its leaves' first entry top-down
  const int D = (int)levels.size();
  std::vector<std::vector<int>> size(D), ent(D), pre(D), base(D);
  for (int d = D - 1; d >= 0; d--) {
    const Level& L = levels[d];
    size[d].resize(L.K);
    ent[d].resize(L.K);
    for (int k = 0; k < L.K; k++) {
      const int c = L.child[k];
      if (c < 0) {
        size[d][k] = 1;
        ent[d][k] = L.off[k + 1] - L.off[k];
      } else {
        size[d][k] = 1 + size[d + 1][c] + size[d + 1][c + 1];
        ent[d][k] = ent[d + 1][c] + ent[d + 1][c + 1];
      }
    }
  }
  for (int d = 0; d < D; d++) {
    pre[d].assign(levels[d].K, 0);
    base[d].assign(levels[d].K, 0);
  }
  for (int d = 0; d + 1 < D; d++) {
    const Level& L = levels[d];
    for (int k = 0; k < L.K; k++) {
      const int c = L.child[k];
      if (c < 0) continue;
      pre[d + 1][c] = pre[d][k] + 1;
      base[d + 1][c] = base[d][k];
      pre[d + 1][c + 1] = pre[d][k] + 1 + size[d + 1][c];
      base[d + 1][c + 1] = base[d][k] + ent[d + 1][c];
    }
  }
  const int N = size[0][0], total = ent[0][0];
  // the leaves' lists, gathered into preorder: every level's offsets and
  // destinations in one upload, one gather launch per level
  std::vector<int> all_off, all_dest;
  std::vector<size_t> at(D);
  for (int d = 0; d < D; d++) {
    const Level& L = levels[d];
    at[d] = all_off.size();
    all_off.insert(all_off.end(), L.off.begin(), L.off.end());
    for (int k = 0; k < L.K; k++) all_dest.push_back(L.child[k] < 0 ? base[d][k] : -1);
    all_dest.push_back(-1);  // keeps the two arrays' per-level starts equal
  }
  int *d_all_off, *d_all_dest, *d_idx;
  KCK(A.get(&d_all_off, all_off.size()));
  KCK(A.get(&d_all_dest, all_dest.size()));
  KCK(A.get(&d_idx, (size_t)total));
  KCK(cudaMemcpyAsync(d_all_off, all_off.data(), all_off.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  KCK(cudaMemcpyAsync(d_all_dest, all_dest.data(), all_dest.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  for (int d = 0; d < D; d++) {
    const Level& L = levels[d];
    k_kd_gather_leaves<<<(int)((32LL * L.K + 255) / 256), 256, 0, s>>>(L.d_e, d_all_off + at[d],
                                                                        d_all_dest + at[d], L.K, d_idx);
  }
  KCK(cudaGetLastError());
  idx->resize(total);
  KCK(cudaMemcpyAsync(idx->data(), d_idx, (size_t)total * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  nodes->assign(N, rt_kd_node_desc{});
  for (int d = 0; d < D; d++) {
    const Level& L = levels[d];
    for (int k = 0; k < L.K; k++) {
      rt_kd_node_desc& nd = (*nodes)[pre[d][k]];
      for (int a = 0; a < 3; a++) {
        nd.bounds_min[a] = L.bnd[6 * (size_t)k + a];
        nd.bounds_max[a] = L.bnd[6 * (size_t)k + 3 + a];
      }
      const int c = L.child[k];
      if (c < 0) {
        nd.axis = -1;
        nd.first = base[d][k];
        nd.count = L.off[k + 1] - L.off[k];
      } else {
        nd.axis = d % 3;
        nd.split = L.split[k];
        nd.right = pre[d + 1][c + 1];
      }
    }
  }
  KCK(cudaStreamSynchronize(s));
#undef KCK
  return "";
}

}  // namespace rtb
