// Binary BVH build: top-down, split at the median centroid of the widest
// centroid axis, leaves of at most `leaf_size` primitives.
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

}  // namespace rtb
