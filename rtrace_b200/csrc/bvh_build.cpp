// Binary BVH builds: top-down, split at the median centroid of the widest
// centroid axis (build_bvh) or at the binned surface-area optimum
// (build_bvh_sah); leaves of at most `leaf_size` primitives.
#include "bvh_build.hpp"

#include <algorithm>
#include <cmath>
#include <future>
#include <limits>
#include <map>
#include <thread>

namespace rtb {
namespace {

// Subtrees of at least kParallelMin primitives in the top kParallelDepth
// levels are built on their own threads; their loops over primitives are
// split across threads above kSplitLoop primitives.
constexpr int kParallelMin = 8192;
constexpr int kParallelDepth = 6;
constexpr int kSplitLoop = 1 << 18;

// f(begin, end, part) over `parts` contiguous ranges of [0, n), on threads.
template <class F>
void split_loop(int n, int parts, F f) {
  std::vector<std::thread> th;
  for (int p = 1; p < parts; p++) th.emplace_back([&f, n, parts, p] { f(n / parts * p, p + 1 == parts ? n : n / parts * (p + 1), p); });
  f(0, n / parts, 0);
  for (auto& t : th) t.join();
}

// A primitive as the build moves it: its box and centroid travel with it,
// so every loop over a node's primitives reads memory in order.
struct Prim {
  double c[3], lo[3], hi[3];
  int32_t id;
};

struct Builder {
  int leaf;
  double pad;
  int hw = 1;

  // Internal nodes of the subtree over n primitives: a median split makes
  // it a function of n alone, and halving from the root size reaches at
  // most two sizes a level, all tabulated (read-only) before the build.
  std::vector<std::pair<int, int32_t>> counts;
  int32_t tabulate(int n, std::map<int, int32_t>& m) {
    if (n <= leaf) return 0;
    auto it = m.find(n);
    if (it != m.end()) return it->second;
    const int32_t c = 1 + tabulate(n / 2, m) + tabulate(n - n / 2, m);
    m[n] = c;
    return c;
  }
  void prepare(int n) {
    std::map<int, int32_t> m;
    tabulate(n, m);
    counts.assign(m.begin(), m.end());
  }
  int32_t count(int n) const {
    if (n <= leaf) return 0;
    auto it = std::lower_bound(counts.begin(), counts.end(), std::make_pair(n, (int32_t)0));
    return it->second;
  }

  // Bounds of p[0, n): of the boxes (box = true) or of the centroids;
  // split across threads for large n.
  void bounds(const Prim* p, int n, bool box, double mn[3], double mx[3]) const {
    const double inf = std::numeric_limits<double>::infinity();
    auto run = [&](int i0, int i1, double lo[3], double hi[3]) {
      for (int k = 0; k < 3; k++) { lo[k] = inf; hi[k] = -inf; }
      for (int i = i0; i < i1; i++)
        for (int k = 0; k < 3; k++) {
          lo[k] = std::min(lo[k], box ? p[i].lo[k] : p[i].c[k]);
          hi[k] = std::max(hi[k], box ? p[i].hi[k] : p[i].c[k]);
        }
    };
    if (n >= kSplitLoop && hw > 1) {
      std::vector<double> lo(3 * hw), hi(3 * hw);
      split_loop(n, hw, [&](int i0, int i1, int q) { run(i0, i1, &lo[3 * q], &hi[3 * q]); });
      for (int k = 0; k < 3; k++) { mn[k] = inf; mx[k] = -inf; }
      for (int q = 0; q < hw; q++)
        for (int k = 0; k < 3; k++) {
          mn[k] = std::min(mn[k], lo[3 * q + k]);
          mx[k] = std::max(mx[k], hi[3 * q + k]);
        }
    } else {
      run(0, n, mn, mx);
    }
  }

  void box(const Prim* p, int n, double mn[3], double mx[3]) const {
    bounds(p, n, true, mn, mx);
    for (int k = 0; k < 3; k++) { mn[k] -= pad; mx[k] += pad; }
  }

  // Builds the subtree over p[0, n) into out[me, me + count(n)) in
  // preorder (left subtree, then right) and returns the reference to it:
  // (node, 0) or, for a leaf, (first primitive, count).
  std::pair<int32_t, int32_t> build(Prim* p, int n, int32_t base, BvhNode* out, int32_t me, int depth) {
    if (n <= leaf) return {base, n};
    double cmin[3], cmax[3];
    bounds(p, n, false, cmin, cmax);
    int axis = 0;
    for (int k = 1; k < 3; k++)
      if (cmax[k] - cmin[k] > cmax[axis] - cmin[axis]) axis = k;
    int mid = n / 2;
    std::nth_element(p, p + mid, p + n, [axis](const Prim& a, const Prim& b) {
      return a.c[axis] < b.c[axis] || (a.c[axis] == b.c[axis] && a.id < b.id);
    });
    BvhNode nd{};
    box(p, mid, nd.lmin, nd.lmax);
    box(p + mid, n - mid, nd.rmin, nd.rmax);
    const int32_t lme = me + 1, rme = me + 1 + count(mid);
    std::pair<int32_t, int32_t> l, r;
    if (n >= kParallelMin && depth < kParallelDepth) {
      auto fut = std::async(std::launch::async, [&] { return build(p, mid, base, out, lme, depth + 1); });
      r = build(p + mid, n - mid, base + mid, out, rme, depth + 1);
      l = fut.get();
    } else {
      l = build(p, mid, base, out, lme, depth + 1);
      r = build(p + mid, n - mid, base + mid, out, rme, depth + 1);
    }
    nd.lidx = l.first;
    nd.lcnt = l.second;
    nd.ridx = r.first;
    nd.rcnt = r.second;
    out[me] = nd;
    return {me, 0};
  }
};


// Binned SAH build: 16 centroid bins per axis; a node splits at the bin
// boundary with the smallest (left area x count + right area x count), the
// first such on axis x, y, z in that order; a node whose centroids cannot
// be binned apart splits at its median primitive id.  Leaves hold at most
// `leaf` primitives.  The split sets depend only on the primitives, never
// on their order, so the tree is deterministic.
struct SahBuilder {
  int leaf;
  double pad;
  static double area(const double mn[3], const double mx[3]) {
    const double dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
    return dx * dy + dy * dz + dz * dx;
  }
  static void bounds(const Prim* p, int n, double mn[3], double mx[3]) {
    const double inf = std::numeric_limits<double>::infinity();
    for (int k = 0; k < 3; k++) { mn[k] = inf; mx[k] = -inf; }
    for (int i = 0; i < n; i++)
      for (int k = 0; k < 3; k++) {
        mn[k] = std::min(mn[k], p[i].lo[k]);
        mx[k] = std::max(mx[k], p[i].hi[k]);
      }
  }
  // Subtree over p[0, n) appended to out in preorder (node, left subtree,
  // right subtree); returns its reference (node index in out, 0) or, for a
  // leaf, (first primitive, count).
  std::pair<int32_t, int32_t> build(Prim* p, int n, int32_t base, std::vector<BvhNode>& out, int depth) {
    if (n <= leaf) return {base, n};
    const double inf = std::numeric_limits<double>::infinity();
    double cmin[3] = {inf, inf, inf}, cmax[3] = {-inf, -inf, -inf};
    for (int i = 0; i < n; i++)
      for (int k = 0; k < 3; k++) {
        cmin[k] = std::min(cmin[k], p[i].c[k]);
        cmax[k] = std::max(cmax[k], p[i].c[k]);
      }
    constexpr int B = 16;
    double best = inf;
    int best_axis = -1, best_b = -1;
    for (int a = 0; a < 3; a++) {
      const double ext = cmax[a] - cmin[a];
      if (!(ext > 0)) continue;
      int cnt[B] = {};
      double bmn[B][3], bmx[B][3];
      for (int b = 0; b < B; b++)
        for (int k = 0; k < 3; k++) { bmn[b][k] = inf; bmx[b][k] = -inf; }
      for (int i = 0; i < n; i++) {
        const int b = std::min(std::max((int)((p[i].c[a] - cmin[a]) / ext * B), 0), B - 1);
        cnt[b]++;
        for (int k = 0; k < 3; k++) {
          bmn[b][k] = std::min(bmn[b][k], p[i].lo[k]);
          bmx[b][k] = std::max(bmx[b][k], p[i].hi[k]);
        }
      }
      double rmn[B][3], rmx[B][3];
      int rc[B] = {};
      double mn[3] = {inf, inf, inf}, mx[3] = {-inf, -inf, -inf};
      int c = 0;
      for (int b = B - 1; b > 0; b--) {
        for (int k = 0; k < 3; k++) { mn[k] = std::min(mn[k], bmn[b][k]); mx[k] = std::max(mx[k], bmx[b][k]); }
        c += cnt[b];
        for (int k = 0; k < 3; k++) { rmn[b][k] = mn[k]; rmx[b][k] = mx[k]; }
        rc[b] = c;
      }
      for (int k = 0; k < 3; k++) { mn[k] = inf; mx[k] = -inf; }
      c = 0;
      for (int b = 0; b < B - 1; b++) {
        for (int k = 0; k < 3; k++) { mn[k] = std::min(mn[k], bmn[b][k]); mx[k] = std::max(mx[k], bmx[b][k]); }
        c += cnt[b];
        if (c == 0 || rc[b + 1] == 0) continue;
        const double cost = area(mn, mx) * c + area(rmn[b + 1], rmx[b + 1]) * rc[b + 1];
        if (cost < best) {
          best = cost;
          best_axis = a;
          best_b = b;
        }
      }
    }
    int mid;
    if (best_axis >= 0) {
      const int a = best_axis;
      const double ext = cmax[a] - cmin[a];
      mid = (int)(std::partition(p, p + n, [&](const Prim& q) {
                    return std::min(std::max((int)((q.c[a] - cmin[a]) / ext * B), 0), B - 1) <= best_b;
                  }) - p);
    } else {
      mid = n / 2;
      std::nth_element(p, p + mid, p + n, [](const Prim& x, const Prim& y) { return x.id < y.id; });
    }
    const int32_t me = (int32_t)out.size();
    out.emplace_back();
    BvhNode nd{};
    bounds(p, mid, nd.lmin, nd.lmax);
    bounds(p + mid, n - mid, nd.rmin, nd.rmax);
    for (int k = 0; k < 3; k++) {
      nd.lmin[k] -= pad;
      nd.lmax[k] += pad;
      nd.rmin[k] -= pad;
      nd.rmax[k] += pad;
    }
    std::pair<int32_t, int32_t> l, r;
    if (n >= kParallelMin && depth < kParallelDepth) {
      // both subtrees on threads into their own lists, appended left then
      // right: the sequential build's preorder
      std::vector<BvhNode> lo, ro;
      auto fut = std::async(std::launch::async, [&] { return build(p, mid, base, lo, depth + 1); });
      r = build(p + mid, n - mid, base + mid, ro, depth + 1);
      l = fut.get();
      auto append = [&](std::vector<BvhNode>& sub, std::pair<int32_t, int32_t>& ref) {
        const int32_t off = (int32_t)out.size();
        for (BvhNode& c : sub) {
          if (c.lcnt == 0) c.lidx += off;
          if (c.rcnt == 0) c.ridx += off;
          out.push_back(c);
        }
        if (ref.second == 0) ref.first += off;
      };
      append(lo, l);
      append(ro, r);
    } else {
      l = build(p, mid, base, out, depth + 1);
      r = build(p + mid, n - mid, base + mid, out, depth + 1);
    }
    nd.lidx = l.first;
    nd.lcnt = l.second;
    nd.ridx = r.first;
    nd.rcnt = r.second;
    out[me] = nd;
    return {me, 0};
  }
};

}  // namespace

void build_bvh(const std::vector<double>& bmin, const std::vector<double>& bmax, int leaf_size, double pad,
               std::vector<BvhNode>* nodes, std::vector<int32_t>* order) {
  size_t n = bmin.size() / 3;
  nodes->clear();
  order->resize(n);
  Builder b{leaf_size, pad};
  b.hw = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<Prim> prims(n);
  for (size_t i = 0; i < n; i++) {
    Prim& q = prims[i];
    for (int k = 0; k < 3; k++) {
      q.lo[k] = bmin[3 * i + k];
      q.hi[k] = bmax[3 * i + k];
      q.c[k] = 0.5 * (q.lo[k] + q.hi[k]);
    }
    q.id = (int32_t)i;
  }
  BvhNode root{};
  if (n == 0) {
    root.lcnt = -1;
    root.rcnt = -1;
    nodes->push_back(root);
    return;
  }
  if ((int)n <= leaf_size) {
    b.box(prims.data(), (int)n, root.lmin, root.lmax);
    root.lidx = 0;
    root.lcnt = (int32_t)n;
    root.rcnt = -1;
    nodes->push_back(root);
    for (size_t i = 0; i < n; i++) (*order)[i] = (int32_t)i;
    return;
  }
  b.prepare((int)n);
  nodes->resize(b.count((int)n));
  b.build(prims.data(), (int)n, 0, nodes->data(), 0, 0);
  for (size_t i = 0; i < n; i++) (*order)[i] = prims[i].id;
  // each leaf's primitives in id order: a canonical layout (the device
  // builder makes the same one; the order within a leaf changes no result)
  for (const BvhNode& nd : *nodes) {
    if (nd.lcnt > 0) std::sort(order->begin() + nd.lidx, order->begin() + nd.lidx + nd.lcnt);
    if (nd.rcnt > 0) std::sort(order->begin() + nd.ridx, order->begin() + nd.ridx + nd.rcnt);
  }
}

void build_bvh_sah(const std::vector<double>& bmin, const std::vector<double>& bmax, int leaf_size, double pad,
                   std::vector<BvhNode>* nodes, std::vector<int32_t>* order) {
  const size_t n = bmin.size() / 3;
  nodes->clear();
  order->resize(n);
  std::vector<Prim> prims(n);
  for (size_t i = 0; i < n; i++) {
    for (int k = 0; k < 3; k++) {
      prims[i].lo[k] = bmin[3 * i + k];
      prims[i].hi[k] = bmax[3 * i + k];
      prims[i].c[k] = 0.5 * (prims[i].lo[k] + prims[i].hi[k]);
    }
    prims[i].id = (int32_t)i;
  }
  if ((int)n <= leaf_size) {  // the median builder's single-leaf and empty layouts
    build_bvh(bmin, bmax, leaf_size, pad, nodes, order);
    return;
  }
  SahBuilder b{leaf_size, pad};
  b.build(prims.data(), (int)n, 0, *nodes, 0);
  for (size_t i = 0; i < n; i++) (*order)[i] = prims[i].id;
  for (const BvhNode& nd : *nodes) {
    if (nd.lcnt > 0) std::sort(order->begin() + nd.lidx, order->begin() + nd.lidx + nd.lcnt);
    if (nd.rcnt > 0) std::sort(order->begin() + nd.ridx, order->begin() + nd.ridx + nd.rcnt);
  }
}

}  // namespace rtb
