/*
 * check_bvh.cpp - host check of the binned-SAH builder (bvh.cpp): for a set
 * of primitive boxes read from stdin ("lo_x lo_y lo_z hi_x hi_y hi_z" per
 * line), build the tree with 1, 4 and 16 threads and leaf sizes 1 and 4,
 * and check that every primitive sits in exactly one leaf, that every slot's
 * box holds what lies below it, that the depth is at most 30, and that the
 * thread count changes neither the depth, the node count nor the SAH cost.
 * Prints "ok" and the figures, or the first failure (exit status 1).
 */
#include "bvh.h"

#include <cmath>
#include <cstdio>
#include <iostream>
#include <vector>

using namespace ssolb;

namespace {

double half_area(const double* lo, const double* hi)
{
  double d[3];
  for(int c = 0; c < 3; ++c) d[c] = hi[c] > lo[c] ? hi[c] - lo[c] : 0;
  return d[0] * d[1] + d[1] * d[2] + d[2] * d[0];
}

/* Walk slot s: check its box holds every primitive below it and mark them;
 * returns false on a violation */
bool walk(const BvhResult& r, const std::vector<PrimBox>& prims, size_t s,
          std::vector<int>& seen, int depth, int& maxd)
{
  const int cnt = r.count[s];
  if(cnt < 0) return true;
  const double* lo = &r.lo[3 * s];
  const double* hi = &r.hi[3 * s];
  auto inside = [&](const PrimBox& p) {
    for(int c = 0; c < 3; ++c)
      if(p.lo[c] < lo[c] || p.hi[c] > hi[c]) return false;
    return true;
  };
  if(cnt > 0) {
    maxd = depth > maxd ? depth : maxd;
    for(int i = 0; i < cnt; ++i) {
      const uint32_t ref = r.primrefs[(size_t)r.child[s] + i];
      if(ref >= prims.size() || !inside(prims[ref])) return false;
      ++seen[ref];
    }
    return true;
  }
  const size_t node = (size_t)r.child[s];
  if(node == 0 || node >= r.child.size() / 2) return false;
  for(int k = 0; k < 2; ++k) {
    const size_t cs = 2 * node + k;
    if(r.count[cs] >= 0)
      for(int c = 0; c < 3; ++c)
        if(r.lo[3 * cs + c] < lo[c] || r.hi[3 * cs + c] > hi[c]) return false;
    if(!walk(r, prims, cs, seen, depth + 1, maxd)) return false;
  }
  return true;
}

double sah(const BvhResult& r)
{
  double total = 0, root = 0;
  const size_t nn = r.child.size() / 2;
  for(size_t i = 0; i < nn; ++i) {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for(int k = 0; k < 2; ++k) {
      const size_t s = 2 * i + k;
      if(r.count[s] < 0) continue;
      for(int c = 0; c < 3; ++c) {
        lo[c] = std::fmin(lo[c], r.lo[3 * s + c]);
        hi[c] = std::fmax(hi[c], r.hi[3 * s + c]);
      }
      if(r.count[s] > 0) total += r.count[s] * half_area(&r.lo[3 * s], &r.hi[3 * s]);
    }
    const double a = half_area(lo, hi);
    if(i == 0) root = a;
    total += 1.2 * a;
  }
  return root > 0 ? total / root : total;
}

} /* namespace */

int main()
{
  std::vector<PrimBox> prims;
  PrimBox b;
  while(std::cin >> b.lo[0] >> b.lo[1] >> b.lo[2] >> b.hi[0] >> b.hi[1] >> b.hi[2]) {
    b.ref = (uint32_t)prims.size();
    prims.push_back(b);
  }
  for(int leaf : {1, 4}) {
    double cost1 = 0;
    size_t nodes1 = 0;
    int depth1 = 0;
    for(int threads : {1, 4, 16}) {
      BvhBuildParams p;
      p.max_leaf = leaf;
      p.threads = threads;
      BvhResult r;
      build_bvh(prims, p, r);
      std::vector<int> seen(prims.size(), 0);
      int maxd = 0;
      if(!walk(r, prims, 0, seen, 1, maxd) || !walk(r, prims, 1, seen, 1, maxd)) {
        printf("box or index violation (leaf %d, threads %d)\n", leaf, threads);
        return 1;
      }
      for(size_t i = 0; i < seen.size(); ++i)
        if(seen[i] != 1) {
          printf("primitive %zu in %d leaves (leaf %d, threads %d)\n", i, seen[i], leaf, threads);
          return 1;
        }
      if(r.depth > 30 || maxd > r.depth) {
        printf("depth %d (walked %d) (leaf %d, threads %d)\n", r.depth, maxd, leaf, threads);
        return 1;
      }
      const double cost = sah(r);
      if(threads == 1) {
        cost1 = cost;
        nodes1 = r.child.size() / 2;
        depth1 = r.depth;
      } else if(std::fabs(cost - cost1) > 1e-9 * cost1 || r.child.size() / 2 != nodes1
             || r.depth != depth1) {
        printf("threads %d differ: cost %.9f / %.9f nodes %zu / %zu depth %d / %d\n", threads,
               cost, cost1, r.child.size() / 2, nodes1, r.depth, depth1);
        return 1;
      }
    }
    printf("ok leaf %d: nodes %zu depth %d cost %.4f\n", leaf, nodes1, depth1, cost1);
  }
  return 0;
}
