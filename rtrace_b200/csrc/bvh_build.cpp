// Binary BVH build: top-down, split at the median centroid of the widest
// centroid axis, leaves of at most `leaf_size` primitives.
#include "bvh_build.hpp"

#include <algorithm>
#include <cmath>
#include <future>
#include <limits>

namespace rtb {
namespace {

// Subtrees of at least kParallelMin primitives in the top kParallelDepth
// levels are built on their own threads (up to 2^kParallelDepth at once).
constexpr int kParallelMin = 8192;
constexpr int kParallelDepth = 4;

struct Builder {
  const std::vector<double>& bmin;
  const std::vector<double>& bmax;
  int leaf;
  double pad;
  std::vector<double> cen;

  void box(const int32_t* ids, int n, double mn[3], double mx[3]) const {
    const double inf = std::numeric_limits<double>::infinity();
    for (int k = 0; k < 3; k++) { mn[k] = inf; mx[k] = -inf; }
    for (int i = 0; i < n; i++)
      for (int k = 0; k < 3; k++) {
        mn[k] = std::min(mn[k], bmin[3 * (size_t)ids[i] + k]);
        mx[k] = std::max(mx[k], bmax[3 * (size_t)ids[i] + k]);
      }
    for (int k = 0; k < 3; k++) { mn[k] -= pad; mx[k] += pad; }
  }

  // Builds the subtree over ids[0, n) whose root box was already stored by
  // the parent.  Returns the child reference (idx, cnt).
  std::pair<int32_t, int32_t> build(int32_t* ids, int n, int32_t base, std::vector<BvhNode>& out, int depth) {
    if (n <= leaf) return {base, n};
    const double inf = std::numeric_limits<double>::infinity();
    double cmin[3] = {inf, inf, inf}, cmax[3] = {-inf, -inf, -inf};
    for (int i = 0; i < n; i++)
      for (int k = 0; k < 3; k++) {
        cmin[k] = std::min(cmin[k], cen[3 * (size_t)ids[i] + k]);
        cmax[k] = std::max(cmax[k], cen[3 * (size_t)ids[i] + k]);
      }
    int axis = 0;
    for (int k = 1; k < 3; k++)
      if (cmax[k] - cmin[k] > cmax[axis] - cmin[axis]) axis = k;
    int mid = n / 2;
    std::nth_element(ids, ids + mid, ids + n, [&](int32_t a, int32_t b) {
      double ca = cen[3 * (size_t)a + axis], cb = cen[3 * (size_t)b + axis];
      return ca < cb || (ca == cb && a < b);
    });
    int32_t me = (int32_t)out.size();
    out.emplace_back();
    BvhNode nd{};
    box(ids, mid, nd.lmin, nd.lmax);
    box(ids + mid, n - mid, nd.rmin, nd.rmax);
    std::pair<int32_t, int32_t> l, r;
    if (n >= kParallelMin && depth < kParallelDepth) {
      // the two subtrees on two threads, into their own node lists, then
      // appended left then right: the node order of the sequential build
      std::vector<BvhNode> lo, ro;
      auto fut = std::async(std::launch::async, [&] { return build(ids, mid, base, lo, depth + 1); });
      r = build(ids + mid, n - mid, base + mid, ro, depth + 1);
      l = fut.get();
      auto append = [&](std::vector<BvhNode>& sub, std::pair<int32_t, int32_t>& ref) {
        int32_t off = (int32_t)out.size();
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
      l = build(ids, mid, base, out, depth + 1);
      r = build(ids + mid, n - mid, base + mid, out, depth + 1);
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
  for (size_t i = 0; i < n; i++) (*order)[i] = (int32_t)i;
  Builder b{bmin, bmax, leaf_size, pad, {}};
  b.cen.resize(3 * n);
  for (size_t i = 0; i < 3 * n; i++) b.cen[i] = 0.5 * (bmin[i] + bmax[i]);
  BvhNode root{};
  if (n == 0) {
    root.lcnt = -1;
    root.rcnt = -1;
    nodes->push_back(root);
    return;
  }
  if ((int)n <= leaf_size) {
    b.box(order->data(), (int)n, root.lmin, root.lmax);
    root.lidx = 0;
    root.lcnt = (int32_t)n;
    root.rcnt = -1;
    nodes->push_back(root);
    return;
  }
  b.build(order->data(), (int)n, 0, *nodes, 0);
}

}  // namespace rtb
