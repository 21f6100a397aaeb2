/*
 * lbvh.cu - device-built linear BVH over a snapshot's primitive boxes
 * (Karras, "Maximizing Parallelism in the Construction of BVHs, Octrees,
 * and k-d Trees", HPG 2012), emitted in the DNode layout the traversal reads.
 *
 * It replaces, on the device, the per-solve Star-3D view build of the
 * reference (src/ssol_scene.c:347-433, s3d_scene_view_create at :410-413).
 * Seven steps on one stream; the host reads the height histogram back once,
 * to size the per-height launches:
 *   1. centroid bounds of the primitive boxes (one block);
 *   2. 30-bit Morton code of each centroid in those bounds (10 bits per axis);
 *   3. stable LSD radix sort of (code, primitive) pairs, 4 passes of 8 bits,
 *      in one block of 1024 threads: per 1024-element tile each warp ranks
 *      its lanes by digit with __match_any_sync, the tile's digit offsets
 *      come from a prefix over the warps, so equal codes keep their input
 *      order and the tree is the same on every run;
 *   4. one thread per internal node finds its key range and split from the
 *      sorted codes (longest common prefix, with the sorted position breaking
 *      ties between equal codes); internal node 0 is the root; leaves are
 *      single primitives (count 1, the child field holds the primitive
 *      reference itself);
 *   5. one thread per leaf walks toward the root writing each child box into
 *      its parent's slot; the second thread to reach a node (an atomic
 *      arrival count) merges the node's two slots and goes on, the first
 *      stops, so no thread waits on another. The same walk computes each
 *      node's SAH cost, height and internal-node count;
 *   6. treelet restructuring for a lower SAH cost (Karras and Aila, HPG
 *      2013): the nodes grouped by height, then one launch per height, lowest
 *      first, one warp per node, whose lanes share the dynamic program over
 *      the treelet's leaf subsets; the root's height is the tree depth, which
 *      the host reads back to check the traversal stack bound;
 *   7. the internal nodes are renumbered depth first, slot 0 first, so that
 *      a node's first child follows it in memory.
 */
#include "kernels.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>

namespace ssolb {

namespace {

template<class R> __device__ __forceinline__ R rmax();
template<> __device__ __forceinline__ float rmax<float>() { return FLT_MAX; }
template<> __device__ __forceinline__ double rmax<double>() { return DBL_MAX; }

constexpr int SORT_THREADS = 1024;
constexpr int SORT_WARPS = SORT_THREADS / 32;

/* Spread the low 10 bits of v to every third bit */
__device__ __forceinline__ uint32_t spread3(uint32_t v)
{
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

template<class R>
__device__ __forceinline__ R centroid(const R* box, int i, int c)
{
  return (R)0.5 * (box[6 * i + c] + box[6 * i + 3 + c]);
}

/* Step 1: bounds of the centroids, one block */
template<class R>
__global__ void __launch_bounds__(SORT_THREADS) lbvh_bounds(const R* box, int n, R* cb)
{
  __shared__ R red[6][SORT_WARPS];
  R lo[3], hi[3];
  for(int c = 0; c < 3; ++c) {
    lo[c] = centroid(box, 0, c);
    hi[c] = lo[c];
  }
  for(int i = threadIdx.x; i < n; i += blockDim.x)
    for(int c = 0; c < 3; ++c) {
      const R x = centroid(box, i, c);
      lo[c] = fmin(lo[c], x);
      hi[c] = fmax(hi[c], x);
    }
  for(int o = 16; o > 0; o >>= 1)
    for(int c = 0; c < 3; ++c) {
      lo[c] = fmin(lo[c], __shfl_xor_sync(0xffffffffu, lo[c], o));
      hi[c] = fmax(hi[c], __shfl_xor_sync(0xffffffffu, hi[c], o));
    }
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if(lane == 0)
    for(int c = 0; c < 3; ++c) {
      red[c][w] = lo[c];
      red[3 + c][w] = hi[c];
    }
  __syncthreads();
  if(threadIdx.x < 6) {
    const int q = threadIdx.x;
    R v = red[q][0];
    for(int k = 1; k < (int)(blockDim.x >> 5); ++k)
      v = q < 3 ? fmin(v, red[q][k]) : fmax(v, red[q][k]);
    cb[q] = v;
  }
}

/* Step 2: Morton codes; vals are the primitives' input positions */
template<class R>
__global__ void lbvh_morton(const R* box, int n, const R* cb, uint32_t* keys, uint32_t* vals)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n) return;
  uint32_t q[3];
  for(int c = 0; c < 3; ++c) {
    const R ext = cb[3 + c] - cb[c];
    const R t = ext > (R)0 ? (centroid(box, i, c) - cb[c]) / ext : (R)0;
    const R s = t * (R)1024;
    q[c] = s <= (R)0 ? 0u : s >= (R)1023 ? 1023u : (uint32_t)s;
  }
  keys[i] = (spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2]);
  vals[i] = (uint32_t)i;
}

/* Step 3: stable radix sort in one block; (k0, v0) in and out, (k1, v1)
 * scratch */
__global__ void __launch_bounds__(SORT_THREADS) lbvh_sort
  (uint32_t* k0, uint32_t* v0, uint32_t* k1, uint32_t* v1, int n)
{
  __shared__ uint32_t wcnt[SORT_WARPS][256];
  __shared__ uint32_t base[256];
  __shared__ uint32_t tile_total[256];
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  const unsigned lt = (1u << lane) - 1u;
  for(int pass = 0; pass < 4; ++pass) {
    const int shift = 8 * pass;
    const uint32_t* sk = pass & 1 ? k1 : k0;
    const uint32_t* sv = pass & 1 ? v1 : v0;
    uint32_t* dk = pass & 1 ? k0 : k1;
    uint32_t* dv = pass & 1 ? v0 : v1;
    if(tid < 256) tile_total[tid] = 0;
    __syncthreads();
    for(int i = tid; i < n; i += SORT_THREADS) atomicAdd(&tile_total[(sk[i] >> shift) & 255u], 1u);
    __syncthreads();
    if(tid < 32) {
      /* exclusive scan of the 256 digit counts by one warp, 8 per lane */
      uint32_t c[8], s = 0;
      for(int k = 0; k < 8; ++k) { c[k] = tile_total[8 * lane + k]; s += c[k]; }
      uint32_t inc = s;
      for(int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if(lane >= o) inc += y;
      }
      uint32_t run = inc - s;
      for(int k = 0; k < 8; ++k) { base[8 * lane + k] = run; run += c[k]; }
    }
    __syncthreads();
    for(int t0 = 0; t0 < n; t0 += SORT_THREADS) {
      const int i = t0 + tid;
      const bool valid = i < n;
      const uint32_t key = valid ? sk[i] : 0u, val = valid ? sv[i] : 0u;
      const uint32_t d = (key >> shift) & 255u;
      uint32_t* flat = &wcnt[0][0];
      for(int k = tid; k < SORT_WARPS * 256; k += SORT_THREADS) flat[k] = 0;
      __syncthreads();
      /* invalid lanes group under 256, which no digit takes */
      const unsigned peers = __match_any_sync(0xffffffffu, valid ? d : 256u);
      const uint32_t rank = __popc(peers & lt);
      if(valid && rank == 0) wcnt[w][d] = __popc(peers);
      __syncthreads();
      if(tid < 256) {
        uint32_t s = 0;
        for(int k = 0; k < SORT_WARPS; ++k) {
          const uint32_t c = wcnt[k][tid];
          wcnt[k][tid] = s;
          s += c;
        }
        tile_total[tid] = s;
      }
      __syncthreads();
      if(valid) {
        const uint32_t pos = base[d] + wcnt[w][d] + rank;
        dk[pos] = key;
        dv[pos] = val;
      }
      __syncthreads();
      if(tid < 256) base[tid] += tile_total[tid];
      __syncthreads();
    }
  }
}

/* Longest common prefix of sorted keys i and j (-1 outside [0, n)); equal
 * keys compare their positions, as if each key carried its position in its
 * low 32 bits */
__device__ __forceinline__ int lcp(const uint32_t* k, int n, int i, int j)
{
  if(j < 0 || j >= n) return -1;
  const uint32_t a = k[i], b = k[j];
  return a == b ? 32 + __clz(i ^ j) : __clz(a ^ b);
}

/* Step 4: internal node i of n - 1. parent[] holds (parent << 1) | slot:
 * entries [0, n - 1) for internal nodes, [n - 1, 2n - 1) for leaves. */
template<class R>
__global__ void lbvh_nodes(const uint32_t* keys, const uint32_t* vals, const uint32_t* ref,
                           int n, DNode<R>* nodes, int32_t* parent)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n - 1) return;
  const int d = lcp(keys, n, i, i + 1) - lcp(keys, n, i, i - 1) > 0 ? 1 : -1;
  const int dmin = lcp(keys, n, i, i - d);
  int lmax = 2;
  while(lcp(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for(int t = lmax >> 1; t >= 1; t >>= 1)
    if(lcp(keys, n, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dnode = lcp(keys, n, i, j);
  int s = 0;
  for(int t = l;;) {
    t = (t + 1) >> 1;
    if(lcp(keys, n, i, i + (s + t) * d) > dnode) s += t;
    if(t == 1) break;
  }
  const int g = i + s * d + (d < 0 ? -1 : 0);
  const int lo = min(i, j), hi = max(i, j);
  DNode<R>& N = nodes[i];
  const int c[2] = {g, g + 1};
  const bool leaf[2] = {lo == g, hi == g + 1};
  for(int k = 0; k < 2; ++k) {
    if(leaf[k]) {
      N.child[k] = (int32_t)ref[vals[c[k]]];
      N.count[k] = 1;
      parent[(n - 1) + c[k]] = (i << 1) | k;
    } else {
      N.child[k] = c[k];
      N.count[k] = 0;
      parent[c[k]] = (i << 1) | k;
    }
  }
  if(i == 0) parent[0] = -1;
}

template<class R>
__device__ __forceinline__ void put_slot(DNode<R>& N, int k, const R lo[3], const R hi[3])
{
  for(int c = 0; c < 3; ++c) {
    N.lo[k][c] = lo[c];
    N.hi[k][c] = hi[c];
  }
}

/* Surface-area heuristic: a node costs C_NODE x its surface area (a ray
 * that reaches it tests both child boxes), a primitive C_PRIM x its box's
 * (Karras and Aila's constants; areas are half surface areas, the factor
 * cancels) */
constexpr float C_NODE = 1.2f, C_PRIM = 1.0f;
constexpr int TREELET = 6; /* leaves of a restructured treelet (7 gave a 0.2 % lower SAH
                              * cost on the field for 3x the work) */

template<class R>
__device__ __forceinline__ float half_area(const R lo[3], const R hi[3])
{
  const float dx = (float)(hi[0] - lo[0]), dy = (float)(hi[1] - lo[1]),
              dz = (float)(hi[2] - lo[2]);
  return dx * dy + dy * dz + dz * dx;
}

/* Per internal node: SAH cost, height, internal nodes in its subtree
 * (itself included) and parent link ((parent << 1) | slot; entries
 * [n - 1, 2n - 1) are the leaves') */
struct Aux {
  float* cost;
  int32_t* height;
  int32_t* ninner;
  int32_t* parent;
};

/* A treelet leaf: a slot's box, what it holds (a primitive, count 1, or a
 * subtree, count 0), and the subtree's cost, height and internal nodes */
template<class R> struct TLeaf {
  R lo[3], hi[3];
  int32_t child, count;
  float cost;
  int height, ninner;
};

/* Slot k of node N as written by other threads of this launch: read past L1 */
template<class R>
__device__ __forceinline__ void read_slot(const DNode<R>& N, int k, const Aux& A, TLeaf<R>& L)
{
  for(int c = 0; c < 3; ++c) {
    L.lo[c] = __ldcg(&N.lo[k][c]);
    L.hi[c] = __ldcg(&N.hi[k][c]);
  }
  L.child = __ldcg(&N.child[k]);
  L.count = __ldcg(&N.count[k]);
  if(L.count == 0) {
    L.cost = __ldcg(&A.cost[L.child]);
    L.height = __ldcg(&A.height[L.child]);
    L.ninner = __ldcg(&A.ninner[L.child]);
  } else {
    L.cost = C_PRIM * half_area(L.lo, L.hi);
    L.height = 0;
    L.ninner = 0;
  }
}

template<class R>
__device__ __forceinline__ void union_of(const TLeaf<R>* L, int S, R lo[3], R hi[3])
{
  for(int c = 0; c < 3; ++c) { lo[c] = rmax<R>(); hi[c] = -rmax<R>(); }
  for(int i = 0; S; ++i, S >>= 1)
    if(S & 1)
      for(int c = 0; c < 3; ++c) {
        lo[c] = fmin(lo[c], L[i].lo[c]);
        hi[c] = fmax(hi[c], L[i].hi[c]);
      }
}

/* Rewrite the internal nodes of a treelet (root first, then inner[1..]) to
 * the binary tree over its nl leaves that part[] describes (part[S]: the
 * subset holding S's lowest leaf), and set their parent links, costs (c[]),
 * heights and internal node counts. The root keeps its index and box; the
 * leaves' subtrees are untouched. */
template<class R>
__device__ void rebuild_treelet(DNode<R>* nodes, const Aux& A, const TLeaf<R>* L, int nl,
                                const int* inner, const float* c, const uint8_t* part)
{
  int nset[TREELET - 1], nidx[TREELET - 1], kid[TREELET - 1][2];
  int hh[TREELET - 1], nn[TREELET - 1];
  int cnt = 1, next = 1;
  nset[0] = (1 << nl) - 1;
  nidx[0] = inner[0];
  for(int q = 0; q < cnt; ++q) {
    const int nd = nidx[q];
    DNode<R>& N = nodes[nd];
    const int S = nset[q];
    const int T[2] = {part[S], S ^ part[S]};
    for(int k = 0; k < 2; ++k) {
      R lo[3], hi[3];
      if(__popc(T[k]) == 1) {
        const int i = __ffs(T[k]) - 1;
        put_slot(N, k, L[i].lo, L[i].hi);
        N.child[k] = L[i].child;
        N.count[k] = L[i].count;
        if(L[i].count == 0) A.parent[L[i].child] = (nd << 1) | k;
        kid[q][k] = -1 - i;
      } else {
        const int m = inner[next++];
        union_of(L, T[k], lo, hi);
        put_slot(N, k, lo, hi);
        N.child[k] = m;
        N.count[k] = 0;
        A.parent[m] = (nd << 1) | k;
        nset[cnt] = T[k];
        nidx[cnt] = m;
        kid[q][k] = cnt++;
      }
    }
  }
  for(int q = cnt - 1; q >= 0; --q) {
    int hm = 0, sum = 1;
    for(int k = 0; k < 2; ++k) {
      const int e = kid[q][k];
      hm = max(hm, e >= 0 ? hh[e] : L[-1 - e].height);
      sum += e >= 0 ? nn[e] : L[-1 - e].ninner;
    }
    hh[q] = 1 + hm;
    nn[q] = sum;
    A.cost[nidx[q]] = c[nset[q]];
    A.height[nidx[q]] = hh[q];
    A.ninner[nidx[q]] = nn[q];
  }
}

constexpr int MAX_LEVELS = 128;

/* Internal nodes grouped by height (one block): level_first[h] .. [h + 1]
 * of level_nodes; *maxh the largest height present. Nodes of one height
 * are never ancestors of one another, so their treelets are disjoint. */
__global__ void __launch_bounds__(SORT_THREADS) lbvh_levels
  (const int32_t* height, int m, int32_t* level_first, int32_t* level_nodes, int32_t* maxh)
{
  __shared__ uint32_t cnt[MAX_LEVELS], cur[MAX_LEVELS];
  const int tid = threadIdx.x;
  for(int h = tid; h < MAX_LEVELS; h += SORT_THREADS) cnt[h] = 0;
  __syncthreads();
  for(int i = tid; i < m; i += SORT_THREADS)
    atomicAdd(&cnt[min(max(height[i], 0), MAX_LEVELS - 1)], 1u);
  __syncthreads();
  if(tid == 0) {
    uint32_t run = 0;
    int mh = 0;
    for(int h = 0; h < MAX_LEVELS; ++h) {
      level_first[h] = (int32_t)run;
      cur[h] = run;
      run += cnt[h];
      if(cnt[h]) mh = h;
    }
    level_first[MAX_LEVELS] = (int32_t)run;
    *maxh = mh;
  }
  __syncthreads();
  for(int i = tid; i < m; i += SORT_THREADS)
    level_nodes[atomicAdd(&cur[min(max(height[i], 0), MAX_LEVELS - 1)], 1u)] = i;
}

constexpr int TREELET_WARPS = 4;

/* Treelet restructuring (Karras and Aila, "Fast Parallel Construction of
 * High-Quality Bounding Volume Hierarchies", HPG 2013) of the nodes of one
 * height, one warp per node, heights in increasing order (one launch each),
 * so that a node's subtree is final when its treelet is formed. Lane 0
 * refreshes the node's cost, height and node count from its slots (its
 * descendants may have changed), then grows a treelet of up to TREELET
 * leaves by opening the leaf of largest area that is a subtree; the lanes
 * then find the binary tree over those leaves of lowest SAH cost by dynamic
 * programming over their subsets, all subsets of one size at a time; lane 0
 * rewrites the treelet's internal nodes to it if it is cheaper. */
template<class R>
__global__ void __launch_bounds__(32 * TREELET_WARPS) lbvh_treelets
  (DNode<R>* nodes, const Aux A, const int32_t* level_first, const int32_t* level_nodes,
   int level, int32_t* depth)
{
  __shared__ TLeaf<R> Ls[TREELET_WARPS][TREELET];
  __shared__ float cs[TREELET_WARPS][1 << TREELET];
  __shared__ uint8_t ps[TREELET_WARPS][1 << TREELET];
  __shared__ int inner_s[TREELET_WARPS][TREELET - 1];
  __shared__ int nl_s[TREELET_WARPS];
  __shared__ float cur_s[TREELET_WARPS];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int first = level_first[level], count = level_first[level + 1] - first;
  TLeaf<R>* L = Ls[w];
  float* c = cs[w];
  uint8_t* part = ps[w];
  for(int t = blockIdx.x * TREELET_WARPS + w; t < count; t += gridDim.x * TREELET_WARPS) {
    const int root = level_nodes[first + t];
    if(lane == 0) {
      read_slot(nodes[root], 0, A, L[0]);
      read_slot(nodes[root], 1, A, L[1]);
      R lo[3], hi[3];
      union_of(L, 3, lo, hi);
      const float cur = C_NODE * half_area(lo, hi) + L[0].cost + L[1].cost;
      const int h = 1 + max(L[0].height, L[1].height);
      A.cost[root] = cur;
      A.height[root] = h;
      A.ninner[root] = 1 + L[0].ninner + L[1].ninner;
      if(root == 0) *depth = h;
      int nl = 2, ni = 1;
      inner_s[w][0] = root;
      while(nl < TREELET) {
        int best = -1;
        float ba = -1.f;
        for(int i = 0; i < nl; ++i)
          if(L[i].count == 0) {
            const float a = half_area(L[i].lo, L[i].hi);
            if(a > ba) { ba = a; best = i; }
          }
        if(best < 0) break;
        const int nd = L[best].child;
        inner_s[w][ni++] = nd;
        read_slot(nodes[nd], 1, A, L[nl]);
        read_slot(nodes[nd], 0, A, L[best]);
        ++nl;
      }
      nl_s[w] = nl;
      cur_s[w] = cur;
    }
    __syncwarp();
    const int nl = nl_s[w];
    if(nl >= 3) {
      const int full = (1 << nl) - 1;
      for(int S = lane + 1; S <= full; S += 32)
        if(__popc(S) == 1) c[S] = L[__ffs(S) - 1].cost;
      __syncwarp();
      for(int k = 2; k <= nl; ++k) {
        for(int S = lane + 1; S <= full; S += 32) {
          if(__popc(S) != k) continue;
          R lo[3], hi[3];
          union_of(L, S, lo, hi);
          /* each partition once: the part holding S's lowest leaf */
          const int low = S & -S;
          float bc = 3.4e38f;
          int bp = low;
          for(int P = (S - 1) & S; P; P = (P - 1) & S) {
            if(!(P & low)) continue;
            const float v = c[P] + c[S ^ P];
            if(v < bc) { bc = v; bp = P; }
          }
          c[S] = C_NODE * half_area(lo, hi) + bc;
          part[S] = (uint8_t)bp;
        }
        __syncwarp();
      }
      if(lane == 0 && c[full] < cur_s[w] * (1.f - 1e-5f)) {
        rebuild_treelet(nodes, A, L, nl, inner_s[w], c, part);
        if(root == 0) *depth = A.height[0];
      }
    }
    __syncwarp();
  }
}

/* Step 5: boxes, SAH costs, heights and internal node counts, one thread
 * per leaf; flags start at zero */
template<class R>
__global__ void lbvh_boxes(const R* box, const uint32_t* vals, int n, DNode<R>* nodes,
                           const Aux A, uint32_t* flags, int32_t* depth)
{
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if(j >= n) return;
  const int src = (int)vals[j];
  R lo[3], hi[3];
  for(int c = 0; c < 3; ++c) {
    lo[c] = box[6 * src + c];
    hi[c] = box[6 * src + 3 + c];
  }
  int p = A.parent[(n - 1) + j];
  int node = p >> 1, slot = p & 1, h = 0, nin = 0;
  float my_cost = C_PRIM * half_area(lo, hi);
  put_slot(nodes[node], slot, lo, hi);
  for(;;) {
    /* publish this slot (and what is known below it) before arriving */
    __threadfence();
    if(atomicAdd(&flags[node], 1u) == 0u) return;
    __threadfence();
    /* both slots are final: the sibling's box, cost and height were written
     * by the thread that arrived first, read past L1 */
    DNode<R>& N = nodes[node];
    TLeaf<R> sib;
    read_slot(N, 1 - slot, A, sib);
    for(int c = 0; c < 3; ++c) {
      lo[c] = fmin(lo[c], sib.lo[c]);
      hi[c] = fmax(hi[c], sib.hi[c]);
    }
    h = 1 + max(h, sib.height);
    nin = 1 + nin + sib.ninner;
    my_cost = C_NODE * half_area(lo, hi) + my_cost + sib.cost;
    A.cost[node] = my_cost;
    A.height[node] = h;
    A.ninner[node] = nin;
    if(node == 0) {
      *depth = h;
      return;
    }
    p = A.parent[node];
    node = p >> 1;
    slot = p & 1;
    put_slot(nodes[node], slot, lo, hi);
  }
}

/* Step 6: depth-first order of the internal nodes (slot 0 first), as the
 * host builder numbers them, so that a node's first child follows it in
 * memory: a node's index is the sum, over the path from the root, of one
 * per step plus, where the path takes slot 1, the internal nodes of the
 * slot-0 subtree it passes by */
template<class R>
__global__ void lbvh_order(const DNode<R>* nodes, const int32_t* parent, const int32_t* ninner,
                           int n, int32_t* newidx)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n - 1) return;
  int x = 0, node = i;
  while(node != 0) {
    const int p = parent[node];
    const int par = p >> 1;
    x += 1;
    if(p & 1) {
      const DNode<R>& P = nodes[par];
      if(P.count[0] == 0) x += ninner[P.child[0]];
    }
    node = par;
  }
  newidx[i] = x;
}

template<class R>
__global__ void lbvh_permute(const DNode<R>* src, DNode<R>* dst, const int32_t* newidx, int n)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n - 1) return;
  DNode<R> N = src[i];
  for(int k = 0; k < 2; ++k)
    if(N.count[k] == 0) N.child[k] = newidx[N.child[k]];
  dst[newidx[i]] = N;
}

template<class R>
int launch_lbvh(const LbvhArgs& A, void* stream)
{
  const cudaStream_t s = (cudaStream_t)stream;
  const int n = A.n;
  if(n < 2) return (int)cudaErrorInvalidValue;
  const R* box = (const R*)A.box;
  R* cb = (R*)A.cbounds;
  DNode<R>* nodes = (DNode<R>*)A.nodes;
  uint32_t* k0 = A.keys;
  uint32_t* k1 = A.keys + n;
  uint32_t* v0 = A.vals;
  uint32_t* v1 = A.vals + n;
  if(cudaMemsetAsync(A.flags, 0, sizeof(uint32_t) * (size_t)(n - 1), s) != cudaSuccess)
    return (int)cudaGetLastError();
  lbvh_bounds<R><<<1, SORT_THREADS, 0, s>>>(box, n, cb);
  const unsigned g = (unsigned)((n + 255) / 256);
  lbvh_morton<R><<<g, 256, 0, s>>>(box, n, cb, k0, v0);
  lbvh_sort<<<1, SORT_THREADS, 0, s>>>(k0, v0, k1, v1, n);
  lbvh_nodes<R><<<g, 256, 0, s>>>(k0, v0, A.ref, n, nodes, A.parent);
  const Aux aux = {A.cost, A.height, A.ninner, A.parent};
  lbvh_boxes<R><<<g, 256, 0, s>>>(box, v0, n, nodes, aux, A.flags, A.depth);
  if(A.optimize && n >= 3) {
    /* the heights decide how many levels to launch and how wide */
    lbvh_levels<<<1, SORT_THREADS, 0, s>>>(A.height, n - 1, A.level_first, A.level_nodes,
                                           A.level_first + MAX_LEVELS + 1);
    int32_t lf[MAX_LEVELS + 2];
    if(cudaMemcpyAsync(lf, A.level_first, sizeof(lf), cudaMemcpyDeviceToHost, s) != cudaSuccess
    || cudaStreamSynchronize(s) != cudaSuccess)
      return (int)cudaGetLastError();
    const int maxh = lf[MAX_LEVELS + 1];
    if(maxh < MAX_LEVELS - 1)
      for(int h = 2; h <= maxh; ++h) {
        const int cnt = lf[h + 1] - lf[h];
        if(cnt <= 0) continue;
        const unsigned blocks = (unsigned)std::min(
          (cnt + TREELET_WARPS - 1) / TREELET_WARPS, 148 * 8);
        lbvh_treelets<R><<<blocks, 32 * TREELET_WARPS, 0, s>>>(nodes, aux, A.level_first,
                                                               A.level_nodes, h, A.depth);
      }
  }
  DNode<R>* tmp = (DNode<R>*)A.tmp_nodes;
  lbvh_order<R><<<g, 256, 0, s>>>(nodes, A.parent, A.ninner, n, A.newidx);
  lbvh_permute<R><<<g, 256, 0, s>>>(nodes, tmp, A.newidx, n);
  if(cudaMemcpyAsync(nodes, tmp, sizeof(DNode<R>) * (size_t)(n - 1), cudaMemcpyDeviceToDevice,
                     s) != cudaSuccess)
    return (int)cudaGetLastError();
  return (int)cudaGetLastError();
}

} /* namespace */

size_t lbvh_scratch_bytes(int n)
{
  const size_t m = n > 0 ? (size_t)n : 0;
  /* centroid bounds (6 doubles), depth (one int, padded), a copy of the
   * nodes (sized for FP64), keys and vals (2n each), parent (2n), flags,
   * heights, costs, internal node counts, new indices and nodes by level (n
   * each), level offsets and the largest height */
  return 6 * sizeof(double) + 16 + sizeof(DNode<double>) * m
    + sizeof(uint32_t) * (2 * m + 2 * m + 2 * m + 6 * m) + sizeof(int32_t) * (MAX_LEVELS + 2);
}

void lbvh_bind_scratch(LbvhArgs& A, void* scratch)
{
  const size_t m = A.n > 0 ? (size_t)A.n : 0;
  /* the doubles first, so that they are 8-byte aligned */
  unsigned char* p = (unsigned char*)scratch;
  A.cbounds = p;
  p += 6 * sizeof(double);
  A.depth = (int32_t*)p;
  p += 16;
  A.tmp_nodes = p;
  p += sizeof(DNode<double>) * m;
  A.keys = (uint32_t*)p;
  p += sizeof(uint32_t) * 2 * m;
  A.vals = (uint32_t*)p;
  p += sizeof(uint32_t) * 2 * m;
  A.parent = (int32_t*)p;
  p += sizeof(int32_t) * 2 * m;
  A.flags = (uint32_t*)p;
  p += sizeof(uint32_t) * m;
  A.height = (int32_t*)p;
  p += sizeof(int32_t) * m;
  A.cost = (float*)p;
  p += sizeof(float) * m;
  A.ninner = (int32_t*)p;
  p += sizeof(int32_t) * m;
  A.newidx = (int32_t*)p;
  p += sizeof(int32_t) * m;
  A.level_nodes = (int32_t*)p;
  p += sizeof(int32_t) * m;
  A.level_first = (int32_t*)p;
}

int launch_lbvh_f32(const LbvhArgs& A, void* stream) { return launch_lbvh<float>(A, stream); }
int launch_lbvh_f64(const LbvhArgs& A, void* stream) { return launch_lbvh<double>(A, stream); }

} /* namespace ssolb */
