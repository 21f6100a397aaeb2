/*
 * bvh.cpp - top-down binned SAH builder (Wald, "On fast construction of
 * SAH-based bounding volume hierarchies", 2007) with a median-split fallback
 * that bounds the depth for the device's fixed traversal stack.
 */
#include "bvh.h"

#include <algorithm>
#include <array>
#include <thread>
#include <cmath>
#include <limits>

namespace ssolb {

namespace {

struct Box {
  double lo[3], hi[3];
  void reset()
  {
    for(int c = 0; c < 3; ++c) {
      lo[c] = std::numeric_limits<double>::max();
      hi[c] = -std::numeric_limits<double>::max();
    }
  }
  void grow(const double* l, const double* h)
  {
    for(int c = 0; c < 3; ++c) {
      lo[c] = std::min(lo[c], l[c]);
      hi[c] = std::max(hi[c], h[c]);
    }
  }
  double area() const
  {
    const double d[3] = {std::max(0.0, hi[0] - lo[0]),
                         std::max(0.0, hi[1] - lo[1]),
                         std::max(0.0, hi[2] - lo[2])};
    return 2 * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
  }
};

struct Task {
  int begin, end; /* range of prims */
  int node, slot; /* parent slot to fill: node*2 + k */
  int depth;
};

Box bounds(const std::vector<PrimBox>& p, int b, int e)
{
  Box box;
  box.reset();
  for(int i = b; i < e; ++i) box.grow(p[i].lo, p[i].hi);
  return box;
}

double centroid(const PrimBox& p, int axis)
{ return 0.5 * (p.lo[axis] + p.hi[axis]); }

/* Returns the split position in [b, e) or -1 to make a leaf. One pass
 * bins the centroids of [b, e) on all three axes at once (centroids are
 * precomputed in `c`, kept in the order of `p`). */
int split(std::vector<PrimBox>& p, std::vector<std::array<double, 3>>& c, int b, int e,
          const BvhBuildParams& prm, int depth)
{
  const int n = e - b;
  if(n <= prm.max_leaf) return -1;
  /* Depth cap: a large leaf is slower but keeps the traversal stack bounded */
  if(depth >= prm.max_depth - 1) return -1;
  Box cb;
  cb.reset();
  for(int i = b; i < e; ++i) cb.grow(c[i].data(), c[i].data());
  const bool force_median = depth >= prm.max_depth - 10;
  /* Small ranges: exact SAH over the centroid order on each axis (binning's
   * fixed cost per node dominates there, and the exact sweep is at least as
   * good a split) */
  constexpr int EXACT_MAX = 32;
  if(!force_median && n <= EXACT_MAX) {
    int ord[3][EXACT_MAX];
    double best = std::numeric_limits<double>::max();
    int best_a = -1, best_k = -1;
    for(int a = 0; a < 3; ++a) {
      for(int i = 0; i < n; ++i) ord[a][i] = b + i;
      std::sort(ord[a], ord[a] + n, [&](int x, int y) {
        return c[x][a] < c[y][a] || (c[x][a] == c[y][a] && x < y);
      });
      double right_area[EXACT_MAX];
      Box acc;
      acc.reset();
      for(int k = n - 1; k > 0; --k) {
        acc.grow(p[ord[a][k]].lo, p[ord[a][k]].hi);
        right_area[k] = acc.area();
      }
      acc.reset();
      for(int k = 0; k < n - 1; ++k) {
        acc.grow(p[ord[a][k]].lo, p[ord[a][k]].hi);
        const double cost = acc.area() * (k + 1) + right_area[k + 1] * (n - k - 1);
        if(cost < best) { best = cost; best_a = a; best_k = k; }
      }
    }
    PrimBox tp[EXACT_MAX];
    std::array<double, 3> tc[EXACT_MAX];
    for(int i = 0; i < n; ++i) { tp[i] = p[ord[best_a][i]]; tc[i] = c[ord[best_a][i]]; }
    for(int i = 0; i < n; ++i) { p[b + i] = tp[i]; c[b + i] = tc[i]; }
    return b + best_k + 1;
  }
  double best_cost = std::numeric_limits<double>::max();
  int best_axis = -1, best_bin = -1;
  constexpr int MAX_BINS = 64;
  const int nb = std::min(std::max(prm.bins, 2), MAX_BINS);
  double scale[3];
  for(int a = 0; a < 3; ++a) {
    const double ext = cb.hi[a] - cb.lo[a];
    scale[a] = ext > 0 ? nb / ext : 0;
  }
  if(!force_median) {
    Box bin[3][MAX_BINS];
    int cnt[3][MAX_BINS];
    for(int a = 0; a < 3; ++a)
      for(int k = 0; k < nb; ++k) { bin[a][k].reset(); cnt[a][k] = 0; }
    for(int i = b; i < e; ++i) {
      for(int a = 0; a < 3; ++a) {
        int k = (int)((c[i][a] - cb.lo[a]) * scale[a]);
        k = std::min(std::max(k, 0), nb - 1);
        bin[a][k].grow(p[i].lo, p[i].hi);
        ++cnt[a][k];
      }
    }
    for(int axis = 0; axis < 3; ++axis) {
      if(!(scale[axis] > 0)) continue;
      double right_area[MAX_BINS] = {};
      int right_cnt[MAX_BINS] = {};
      Box acc;
      acc.reset();
      int m = 0;
      for(int k = nb - 1; k > 0; --k) {
        acc.grow(bin[axis][k].lo, bin[axis][k].hi);
        m += cnt[axis][k];
        right_area[k] = acc.area();
        right_cnt[k] = m;
      }
      acc.reset();
      m = 0;
      for(int k = 0; k < nb - 1; ++k) {
        acc.grow(bin[axis][k].lo, bin[axis][k].hi);
        m += cnt[axis][k];
        if(!m || !right_cnt[k + 1]) continue;
        const double cost = acc.area() * m + right_area[k + 1] * right_cnt[k + 1];
        if(cost < best_cost) {
          best_cost = cost;
          best_axis = axis;
          best_bin = k;
        }
      }
    }
  }
  /* Partition p and c together */
  auto swap_items = [&](int x, int y) {
    std::swap(p[x], p[y]);
    std::swap(c[x], c[y]);
  };
  if(best_axis >= 0) {
    const double lo = cb.lo[best_axis], sc = scale[best_axis];
    int l = b, r = e - 1;
    while(l <= r) {
      int k = (int)((c[l][best_axis] - lo) * sc);
      k = std::min(std::max(k, 0), nb - 1);
      if(k <= best_bin) ++l;
      else swap_items(l, r--);
    }
    if(l > b && l < e) return l;
  }
  /* Median split along the largest centroid extent */
  int axis = 0;
  double ext = -1;
  for(int k = 0; k < 3; ++k) {
    if(cb.hi[k] - cb.lo[k] > ext) { ext = cb.hi[k] - cb.lo[k]; axis = k; }
  }
  const int m = b + n / 2;
  std::vector<int> order(n);
  for(int i = 0; i < n; ++i) order[i] = b + i;
  std::nth_element(order.begin(), order.begin() + n / 2, order.end(),
    [&](int x, int y) { return c[x][axis] < c[y][axis]; });
  std::vector<PrimBox> tp(n);
  std::vector<std::array<double, 3>> tc(n);
  for(int i = 0; i < n; ++i) { tp[i] = p[order[i]]; tc[i] = c[order[i]]; }
  std::copy(tp.begin(), tp.end(), p.begin() + b);
  std::copy(tc.begin(), tc.end(), c.begin() + b);
  return m;
}

} /* namespace */

namespace {

/* Node arrays under construction; node ids are local to the builder */
struct Builder {
  std::vector<double> lo, hi;
  std::vector<int32_t> child, count;
  std::vector<uint32_t> refs;
  int depth = 0;
  int new_node()
  {
    const int id = (int)(child.size() / 2);
    lo.resize(lo.size() + 6, 0);
    hi.resize(hi.size() + 6, 0);
    child.resize(child.size() + 2, 0);
    count.resize(count.size() + 2, 0);
    return id;
  }
  void set_slot(int slot, const Box& b, int c, int n)
  {
    for(int k = 0; k < 3; ++k) {
      lo[(size_t)slot * 3 + k] = b.lo[k];
      hi[(size_t)slot * 3 + k] = b.hi[k];
    }
    child[slot] = c;
    count[slot] = n;
  }
};

/* Expands tasks top down on the calling thread */
void run_tasks(std::vector<PrimBox>& prims, std::vector<std::array<double, 3>>& cent,
               const BvhBuildParams& prm, Builder& B, std::vector<Task> stack)
{
  while(!stack.empty()) {
    const Task t = stack.back();
    stack.pop_back();
    B.depth = std::max(B.depth, t.depth + 1);
    const Box b = bounds(prims, t.begin, t.end);
    const int s = split(prims, cent, t.begin, t.end, prm, t.depth);
    if(s < 0) {
      const int first = (int)B.refs.size();
      for(int i = t.begin; i < t.end; ++i) B.refs.push_back(prims[i].ref);
      B.set_slot(t.node * 2 + t.slot, b, first, t.end - t.begin);
    } else {
      const int id = B.new_node();
      B.set_slot(t.node * 2 + t.slot, b, id, 0);
      stack.push_back({t.begin, s, id, 0, t.depth + 1});
      stack.push_back({s, t.end, id, 1, t.depth + 1});
    }
  }
}

/* Ranges below this many primitives are built by one thread */
constexpr int PAR_MIN = 1024;

/* Threads for the part of `nsub` primitives out of `n`: in proportion, at
 * least 1, leaving at least 1 for the rest */
int share(int threads, int nsub, int n)
{
  const int t = (int)((long long)threads * nsub / n);
  return std::min(std::max(t, 1), threads - 1);
}

/* Append builder L's tree to B: L's node 0 stands for B's slot (node,
 * slot), L's node j > 0 becomes a new node of B, and L's leaf references
 * move by the references B already holds */
void merge_into(Builder& B, const Builder& L, int node, int slot)
{
  const int base = (int)(B.child.size() / 2);
  const int ref_base = (int)B.refs.size();
  const size_t nl = L.child.size() / 2;
  auto fix = [&](int c, int cnt) { return cnt == 0 ? c - 1 + base : cnt > 0 ? c + ref_base : c; };
  /* L's nodes 1.. in bulk: boxes and counts as they are, children moved */
  B.lo.insert(B.lo.end(), L.lo.begin() + 6, L.lo.end());
  B.hi.insert(B.hi.end(), L.hi.begin() + 6, L.hi.end());
  B.count.insert(B.count.end(), L.count.begin() + 2, L.count.end());
  B.child.reserve(B.child.size() + 2 * (nl - 1));
  for(size_t ls = 2; ls < 2 * nl; ++ls) B.child.push_back(fix(L.child[ls], L.count[ls]));
  const size_t ps = (size_t)node * 2 + slot;
  for(int c = 0; c < 3; ++c) {
    B.lo[ps * 3 + c] = L.lo[c];
    B.hi[ps * 3 + c] = L.hi[c];
  }
  B.count[ps] = L.count[0];
  B.child[ps] = fix(L.child[0], L.count[0]);
  B.refs.insert(B.refs.end(), L.refs.begin(), L.refs.end());
  B.depth = std::max(B.depth, L.depth);
}

/* The tree of task t (absolute depth t.depth) in a builder of its own whose
 * node 0 stands for the task's parent slot. A range of at least PAR_MIN
 * primitives with 2 or more threads is split here, and its two halves are
 * built at once on two threads that share `threads` in proportion to their
 * sizes; the rest is built top down by one thread. Ranges are disjoint, so
 * the threads partition the shared arrays without overlap. */
Builder build_sub(std::vector<PrimBox>& prims, std::vector<std::array<double, 3>>& cent,
                  const BvhBuildParams& prm, const Task& t, int threads)
{
  Builder L;
  L.new_node();
  Task tt = t;
  tt.node = 0;
  tt.slot = 0;
  const int n = t.end - t.begin;
  if(threads < 2 || n < PAR_MIN) {
    run_tasks(prims, cent, prm, L, {tt});
    return L;
  }
  L.depth = std::max(L.depth, t.depth + 1);
  const Box b = bounds(prims, t.begin, t.end);
  const int s = split(prims, cent, t.begin, t.end, prm, t.depth);
  if(s < 0) {
    const int first = (int)L.refs.size();
    for(int i = t.begin; i < t.end; ++i) L.refs.push_back(prims[i].ref);
    L.set_slot(0, b, first, n);
    return L;
  }
  const int id = L.new_node();
  L.set_slot(0, b, id, 0);
  const Task tl = {t.begin, s, id, 0, t.depth + 1}, tr = {s, t.end, id, 1, t.depth + 1};
  const int thl = share(threads, s - t.begin, n);
  Builder right;
  std::thread th([&] { right = build_sub(prims, cent, prm, tr, threads - thl); });
  Builder left = build_sub(prims, cent, prm, tl, thl);
  th.join();
  merge_into(L, left, id, 0);
  merge_into(L, right, id, 1);
  return L;
}

} /* namespace */

void build_bvh(std::vector<PrimBox> prims, const BvhBuildParams& prm,
               BvhResult& out)
{
  out = BvhResult();
  Builder B;
  /* Node 0 is the root; its two slots hold the two top-level children */
  const int root = B.new_node();
  const int n = (int)prims.size();
  if(n == 0) {
    Box empty;
    empty.reset();
    B.set_slot(root * 2 + 0, empty, 0, -1);
    B.set_slot(root * 2 + 1, empty, 0, -1);
    out.lo = std::move(B.lo);
    out.hi = std::move(B.hi);
    out.child = std::move(B.child);
    out.count = std::move(B.count);
    out.primrefs.push_back(0);
    return;
  }
  std::vector<std::array<double, 3>> cent(prims.size());
  for(size_t i = 0; i < prims.size(); ++i)
    for(int a = 0; a < 3; ++a) cent[i][a] = centroid(prims[i], a);
  int m = split(prims, cent, 0, n, prm, 0);
  if(m < 0) {
    /* Whole scene in one leaf; the second slot is an empty box */
    Box empty;
    empty.reset();
    for(int i = 0; i < n; ++i) B.refs.push_back(prims[i].ref);
    B.set_slot(root * 2 + 0, bounds(prims, 0, n), 0, n);
    B.set_slot(root * 2 + 1, empty, 0, -1);
    B.depth = 1;
  } else {
    const Task t0 = {0, m, root, 0, 1}, t1 = {m, n, root, 1, 1};
    const int threads = std::max(1, prm.threads);
    if(threads == 1 || n < PAR_MIN) {
      run_tasks(prims, cent, prm, B, {t0, t1});
    } else {
      /* The two halves on two threads, each splitting its thread share
       * further (build_sub); the splits are the same, so is the tree */
      const int th0 = share(threads, m, n);
      Builder r1;
      std::thread th([&] { r1 = build_sub(prims, cent, prm, t1, threads - th0); });
      Builder r0 = build_sub(prims, cent, prm, t0, th0);
      th.join();
      merge_into(B, r0, root, 0);
      merge_into(B, r1, root, 1);
    }
  }
  out.lo = std::move(B.lo);
  out.hi = std::move(B.hi);
  out.child = std::move(B.child);
  out.count = std::move(B.count);
  out.primrefs = std::move(B.refs);
  out.depth = B.depth;
}

template<class R> static R round_down(double x)
{
  R r = (R)x;
  if((double)r > x) r = std::nextafter(r, -std::numeric_limits<R>::max());
  return r;
}
template<class R> static R round_up(double x)
{
  R r = (R)x;
  if((double)r < x) r = std::nextafter(r, std::numeric_limits<R>::max());
  return r;
}

template<class R> std::vector<DNode<R>> bvh_nodes(const BvhResult& b)
{
  const size_t nnodes = b.child.size() / 2;
  std::vector<DNode<R>> nodes(nnodes);
  for(size_t i = 0; i < nnodes; ++i) {
    for(int k = 0; k < 2; ++k) {
      const size_t s = i * 2 + k;
      for(int c = 0; c < 3; ++c) {
        const double lo = b.lo[s * 3 + c], hi = b.hi[s * 3 + c];
        if(lo > hi) { /* empty slot (count < 0): never entered */
          nodes[i].lo[k][c] = R(0);
          nodes[i].hi[k][c] = R(0);
        } else {
          nodes[i].lo[k][c] = round_down<R>(lo);
          nodes[i].hi[k][c] = round_up<R>(hi);
        }
      }
      /* A one-primitive leaf holds its prim reference itself (no indirection
       * through primrefs on the device) */
      nodes[i].child[k] = b.count[s] == 1 ? (int32_t)b.primrefs[(size_t)b.child[s]]
                                          : b.child[s];
      nodes[i].count[k] = b.count[s];
    }
  }
  return nodes;
}

template<class R> void round_box_outward(const PrimBox& b, R out[6])
{
  for(int c = 0; c < 3; ++c) {
    out[c] = round_down<R>(b.lo[c]);
    out[3 + c] = round_up<R>(b.hi[c]);
  }
}

template void round_box_outward<float>(const PrimBox&, float*);
template void round_box_outward<double>(const PrimBox&, double*);
template std::vector<DNode<float>> bvh_nodes<float>(const BvhResult&);
template std::vector<DNode<double>> bvh_nodes<double>(const BvhResult&);

} /* namespace ssolb */
