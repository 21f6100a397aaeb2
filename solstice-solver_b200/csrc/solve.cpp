/*
 * solve.cpp - ssol_solve and the plan API: snapshot -> HBM upload ->
 * realisation launches -> tally readback -> estimator.
 *
 * Orchestration of src/ssol_solver.c:1132-1361: argument checks, scene
 * views, sun samplers, the parallel loop (here: kernel launches), the merge
 * of per-thread tallies (here: the device already holds one set of sums),
 * the failure rule and the RNG end state.
 */
#include "flatten.h"
#include "kernels.h"
#include "objects.h"
#include "snapshot.h"

#define SSOL_SHARED_BUILD
#include "../../include/ssol_b200.h"

#include <cuda_runtime_api.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <atomic>
#include <thread>

using namespace ssolb;

/*******************************************************************************
 * Device binding
 ******************************************************************************/
static res_T device_bind(ssol_device* dev)
{
  if(dev->stream) return RES_OK;
  int ndev = 0;
  if(cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    dev->log_error("no CUDA device available.\n");
    return RES_UNKNOWN_ERR;
  }
  int cur = 0;
  cudaGetDevice(&cur);
  dev->cuda_device = cur;
  cudaStream_t s;
  if(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
    return RES_UNKNOWN_ERR;
  dev->stream = s;
  return RES_OK;
}

/* Host threads for the work of one scene (its BVH subtrees) */
static int host_threads()
{
  const unsigned hw = std::thread::hardware_concurrency();
  return (int)std::min(16u, std::max(1u, hw));
}

/* Runs f(0..n-1) on the host's hardware threads (the calling thread
 * included); used for per-item host work of batches */
template<class F> static void parallel_for(size_t n, F&& f)
{
  const unsigned hw = std::thread::hardware_concurrency();
  const size_t nt = std::max<size_t>(1, std::min<size_t>(hw ? hw : 1, n));
  if(nt <= 1) { for(size_t i = 0; i < n; ++i) f(i); return; }
  std::atomic<size_t> next{0};
  auto work = [&]() {
    for(size_t i = next.fetch_add(1); i < n; i = next.fetch_add(1)) f(i);
  };
  std::vector<std::thread> pool;
  pool.reserve(nt - 1);
  for(size_t t = 1; t < nt; ++t) pool.emplace_back(work);
  work();
  for(std::thread& t : pool) t.join();
}

/* Device blocks released by plans and batches are kept for the next solve
 * on the same device: cudaFree unmaps memory and its cost varies by tens of
 * milliseconds, which a loop of ssol_solve calls would pay every time. A
 * released block is reused by a request of at most its size and at least a
 * quarter of it; at most 8 blocks and 4 GiB are kept. */
namespace {
struct MemCache {
  std::mutex lock;
  std::vector<std::pair<void*, size_t>> blocks;
  std::vector<std::pair<void*, size_t>> pinned; /* page-locked host blocks */
};
constexpr size_t CACHE_BLOCKS = 8;
constexpr size_t CACHE_BYTES = size_t(16) << 30;
constexpr size_t PINNED_BLOCKS = 4;
constexpr size_t PINNED_BYTES = size_t(2) << 30;
}

static MemCache* mem_cache(ssol_device* dev)
{
  if(!dev->mem_cache) dev->mem_cache = new (std::nothrow) MemCache();
  return static_cast<MemCache*>(dev->mem_cache);
}

/* Page-locked host blocks (tally read-back of batches) are kept for reuse
 * like device blocks: locking hundreds of megabytes takes longer than the
 * read-back itself */
static cudaError_t host_alloc(ssol_device* dev, void** p, size_t bytes)
{
  MemCache* c = mem_cache(dev);
  if(c) {
    std::lock_guard<std::mutex> g(c->lock);
    size_t best = c->pinned.size();
    for(size_t i = 0; i < c->pinned.size(); ++i) {
      const size_t cap = c->pinned[i].second;
      if(cap >= bytes && cap / 4 <= bytes
      && (best == c->pinned.size() || cap < c->pinned[best].second))
        best = i;
    }
    if(best < c->pinned.size()) {
      *p = c->pinned[best].first;
      c->pinned.erase(c->pinned.begin() + (long)best);
      return cudaSuccess;
    }
  }
  return cudaMallocHost(p, bytes);
}

static void host_free(ssol_device* dev, void* p, size_t bytes)
{
  if(!p) return;
  MemCache* c = mem_cache(dev);
  if(!c) { cudaFreeHost(p); return; }
  std::lock_guard<std::mutex> g(c->lock);
  c->pinned.emplace_back(p, bytes);
  size_t total = 0;
  for(const auto& b : c->pinned) total += b.second;
  while(c->pinned.size() > PINNED_BLOCKS || total > PINNED_BYTES) {
    total -= c->pinned.front().second;
    cudaFreeHost(c->pinned.front().first);
    c->pinned.erase(c->pinned.begin());
  }
}

static cudaError_t dev_alloc(ssol_device* dev, void** p, size_t bytes)
{
  MemCache* c = dev ? static_cast<MemCache*>(dev->mem_cache) : nullptr;
  if(c) {
    std::lock_guard<std::mutex> g(c->lock);
    size_t best = c->blocks.size();
    for(size_t i = 0; i < c->blocks.size(); ++i) {
      const size_t cap = c->blocks[i].second;
      if(cap >= bytes && cap / 4 <= bytes
      && (best == c->blocks.size() || cap < c->blocks[best].second))
        best = i;
    }
    if(best < c->blocks.size()) {
      *p = c->blocks[best].first;
      c->blocks.erase(c->blocks.begin() + (long)best);
      return cudaSuccess;
    }
  }
  cudaError_t e = cudaMalloc(p, bytes);
  if(e != cudaSuccess && c) {
    /* Out of memory: give the cached blocks back and try once more */
    cudaGetLastError();
    std::lock_guard<std::mutex> g(c->lock);
    for(const auto& blk : c->blocks) cudaFree(blk.first);
    c->blocks.clear();
    e = cudaMalloc(p, bytes);
  }
  return e;
}

/* Work still queued on the block finishes first (a cudaFree would have
 * synchronised too) */
static void dev_free(ssol_device* dev, void* p, size_t bytes)
{
  if(!p) return;
  if(!dev) { cudaFree(p); return; }
  cudaDeviceSynchronize();
  if(!dev->mem_cache) dev->mem_cache = new (std::nothrow) MemCache();
  MemCache* c = static_cast<MemCache*>(dev->mem_cache);
  if(!c) { cudaFree(p); return; }
  std::lock_guard<std::mutex> g(c->lock);
  c->blocks.emplace_back(p, bytes);
  size_t total = 0;
  for(const auto& b : c->blocks) total += b.second;
  while(c->blocks.size() > CACHE_BLOCKS || total > CACHE_BYTES) {
    total -= c->blocks.front().second;
    cudaFree(c->blocks.front().first);
    c->blocks.erase(c->blocks.begin());
  }
}

void ssolb_device_release_gpu(ssol_device* dev)
{
  if(dev->mem_cache) {
    MemCache* c = static_cast<MemCache*>(dev->mem_cache);
    for(const auto& b : c->blocks) cudaFree(b.first);
    for(const auto& b : c->pinned) cudaFreeHost(b.first);
    delete c;
    dev->mem_cache = nullptr;
  }
  if(dev->stream) {
    cudaStreamDestroy((cudaStream_t)dev->stream);
    dev->stream = nullptr;
  }
}

/*******************************************************************************
 * Plan
 ******************************************************************************/
namespace {

/* One contiguous device allocation holding several arrays */
struct Blob {
  std::vector<unsigned char> host;
  std::vector<size_t> offsets;
  template<class T> size_t add(const std::vector<T>& v)
  {
    size_t off = (host.size() + 255) & ~size_t(255);
    host.resize(off + v.size() * sizeof(T));
    if(!v.empty()) std::memcpy(host.data() + off, v.data(), v.size() * sizeof(T));
    offsets.push_back(off);
    return off;
  }
};

struct TallyLayout {
  size_t global, rcv, samp, samp_rcv, prim, nb_samples, counters, stats, total;
};

} /* namespace */

/* The BVH builder values ssol_b200_options accepts */
static bool builder_ok(int b)
{
  return b == SSOL_B200_BVH_AUTO || b == SSOL_B200_BVH_SAH || b == SSOL_B200_BVH_LBVH;
}

struct ssol_b200_plan {
  RefCount ref;
  ssol_device* dev = nullptr;
  ssol_scene* scn = nullptr;
  ssol_b200_options opt = SSOL_B200_OPTIONS_DEFAULT;
  FlatMeta meta;
  int nrcv = 0, nsampled = 0;
  void* d_scene = nullptr;
  void* d_tally = nullptr;
  size_t scene_bytes = 0;
  size_t scene_alloc = 0;
  int bvh_depth = 0; /* levels of internal nodes of the BVH */
  bool bvh_device = false; /* built on the device */
  unsigned long long bvh_nodes = 0;
  TallyLayout tl{};
  DScene<float> s32{};
  DScene<double> s64{};
  DTallies t{};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double kernel_ms = 0;
  bool timing_valid = false;
  /* The snapshot of a device-built tree, kept for a host SAH tree built
   * while the first realisations run (plan_swap_sah), and that tree */
  std::unique_ptr<FlatScene<float>> keep32;
  std::unique_ptr<FlatScene<double>> keep64;
  void* d_bvh2 = nullptr;
  size_t bvh2_alloc = 0;
};

/* Default register budget: 3 blocks of 256 threads per SM (80 registers) in
 * FP32, whose feature variants spill little there and gain from 24 warps
 * per SM (field 532 against 483 Mpaths/s at 2, beam-down 174 against 167);
 * 2 in FP64, whose registers are twice as wide */
static int default_min_blocks(ssol_b200_precision p)
{
  return p == SSOL_B200_FP32 ? 3 : 2;
}

static TallyLayout tally_layout(int nrcv, int nsampled, int nprim_slots)
{
  TallyLayout tl;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off = (off + bytes + 255) & ~size_t(255);
    return o;
  };
  tl.global = take(NGLOBAL * 2 * sizeof(double));
  tl.rcv = take((size_t)nrcv * NRCV_Q * 2 * sizeof(double));
  tl.samp = take((size_t)nsampled * 4 * sizeof(double));
  tl.samp_rcv = take((size_t)nsampled * nrcv * NRCV_Q * 2 * sizeof(double));
  tl.prim = take((size_t)nprim_slots * NRCV_Q * 2 * sizeof(double));
  tl.nb_samples = take((size_t)nsampled * sizeof(unsigned long long));
  tl.counters = take(8 * sizeof(unsigned long long));
  tl.stats = take(sizeof(DStats));
  tl.total = off;
  return tl;
}

static DTallies bind_tallies(const TallyLayout& tl, unsigned char* base)
{
  DTallies t;
  t.global = (double*)(base + tl.global);
  t.rcv = (double*)(base + tl.rcv);
  t.samp = (double*)(base + tl.samp);
  t.samp_rcv = (double*)(base + tl.samp_rcv);
  t.prim = (double*)(base + tl.prim);
  t.nb_samples = (unsigned long long*)(base + tl.nb_samples);
  t.counters = (unsigned long long*)(base + tl.counters);
  t.stats = (DStats*)(base + tl.stats);
  return t;
}

static void fill_sums(double dst[10][2], const double* src);

/* Estimator of `nreal` realisations from host copies of one tally layout
 * (the merge step of src/ssol_solver.c:1254-1333 is already done on the
 * device; this only maps slots back to instances) */
static res_T make_estimator
  (ssol_device* dev, ssol_scene* scn, const FlatMeta& meta,
   const TallyLayout& tl, const unsigned char* base, uint64_t nreal,
   const ssp_rng* rng, uint64_t rng_advance, const DStats* st,
   double kernel_ms, size_t scene_bytes, size_t max_failed,
   ssol_estimator** out)
{
  const int nrcv = (int)meta.rcv.size();
  const int nsampled = (int)meta.sampled.size();
  const double* g = (const double*)(base + tl.global);
  const double* rcv = (const double*)(base + tl.rcv);
  const double* samp = (const double*)(base + tl.samp);
  const double* samp_rcv = (const double*)(base + tl.samp_rcv);
  const double* prim = (const double*)(base + tl.prim);
  const unsigned long long* nbs =
    (const unsigned long long*)(base + tl.nb_samples);
  const unsigned long long* cnt =
    (const unsigned long long*)(base + tl.counters);

  ssol_estimator* e = new (std::nothrow) ssol_estimator();
  if(!e) return RES_MEM_ERR;
  ssol_device_ref_get(dev);
  e->dev = dev;
  const size_t failed = (size_t)cnt[0];
  e->failed_count = failed;
  e->realisation_count = (size_t)nreal - std::min<size_t>(failed, nreal);
  /* `nreal` counts the realisations that ran: an early stop leaves the
   * rest unstarted, as the reference's loop skips them once its error flag
   * is set (src/ssol_solver.c:1229) */
  for(int q = 0; q < NGLOBAL; ++q) {
    e->global[q][0] = g[2 * q];
    e->global[q][1] = g[2 * q + 1];
  }
  e->sampled_area = meta.sampled_area;

  /* Receivers are pre-registered like create_mc_receivers
   * (src/ssol_estimator.c:30-60) */
  for(const ssol_instance* inst : scn->instances) {
    if(inst->receiver_mask) e->receivers[inst].inst = inst;
  }
  for(int r = 0; r < nrcv; ++r) {
    const FlatMeta::RcvSide& rs = meta.rcv[r];
    fill_sums(e->receivers[rs.inst].side[rs.side].q,
              rcv + (size_t)r * NRCV_Q * 2);
  }
  for(const FlatMeta::PrimRange& pr : meta.prims) {
    const FlatMeta::RcvSide& rs = meta.rcv[pr.rcv_slot];
    std::vector<double>& v = e->receivers[rs.inst].side[rs.side].prims[pr.shape];
    v.assign(prim + (size_t)pr.base * NRCV_Q * 2,
             prim + (size_t)(pr.base + pr.ntris) * NRCV_Q * 2);
  }
  for(int si = 0; si < nsampled; ++si) {
    SampEntry& se = e->sampled[meta.sampled[si]];
    se.cos[0] = samp[si * 4 + 0];
    se.cos[1] = samp[si * 4 + 1];
    se.shadow[0] = samp[si * 4 + 2];
    se.shadow[1] = samp[si * 4 + 3];
    se.nb_samples = (size_t)nbs[si];
    for(int r = 0; r < nrcv; ++r) {
      const double* src = samp_rcv + ((size_t)si * nrcv + r) * NRCV_Q * 2;
      bool any = false;
      for(int q = 0; q < NRCV_Q * 2 && !any; ++q) any = src[q] != 0;
      if(!any) continue;
      const FlatMeta::RcvSide& rs = meta.rcv[r];
      RcvEntry& re = se.by_receiver[rs.inst];
      re.inst = rs.inst;
      fill_sums(re.side[rs.side].q, src);
    }
  }
  e->kernel_ms = kernel_ms;
  e->stats[0] = st->rays;
  e->stats[1] = st->node_visits;
  e->stats[2] = st->tri_tests;
  e->stats[3] = st->quad_tests;
  e->stats[4] = st->bounces;
  e->stats[5] = st->paths;
  e->killed = cnt[1];
  e->scene_bytes = scene_bytes;
  e->tally_bytes = tl.total;

  /* End state: the next realisation index (src/ssol_estimator.c:368-418) */
  res_T res = ssolb_rng_clone_advanced(rng, rng_advance, &e->rng);
  if(res != RES_OK) {
    ssol_estimator_ref_put(e);
    return res;
  }
  *out = e;
  /* Too many failed paths: RES_BAD_OP with a valid estimator
   * (src/ssol_solver.c:1240-1245, 1340) */
  if(failed > 0 && failed >= max_failed) {
    dev->log_error("Too many unexpected radiative paths.\n");
    return RES_BAD_OP;
  }
  return RES_OK;
}

template<class R>
static void bind_scene(DScene<R>& S, const FlatScene<R>& f, const Blob& b,
                       unsigned char* base, size_t i0 = 0)
{
  size_t i = i0;
  auto ptr = [&](void) { return base + b.offsets[i++]; };
  S.nodes = (const DNode<R>*)ptr();
  S.primrefs = (const uint32_t*)ptr();
  S.tris = (const DTri<R>*)ptr();
  S.quads = (const DQuadric<R>*)ptr();
  S.carvings = (const DCarving*)ptr();
  S.carve_verts = (const R*)ptr();
  S.sinsts = (const DShadedInst*)ptr();
  S.mtls = (const DMaterial*)ptr();
  S.media = (const DMedium*)ptr();
  S.spectra = (const DSpectrum*)ptr();
  S.spec_wl = (const double*)ptr();
  S.spec_val = (const double*)ptr();
  S.shader_tab = (const R*)ptr();
  S.shader_wl = (const double*)ptr();
  S.samp = (const DSampTri<R>*)ptr();
  S.alias_prob = (const float*)ptr();
  S.alias_idx = (const int32_t*)ptr();
  S.wl_nodes = (const double*)ptr();
  S.wl_pdf = (const double*)ptr();
  S.wl_cdf = (const double*)ptr();
  S.tshade = (const DTriShade<R>*)ptr();
  S.bake_tab = (const R*)ptr();
  if(f.tshade.empty()) S.tshade = nullptr;
  S.shader_nodes = (int32_t)f.shader_wl.size();
  S.nsamp = (int32_t)f.samp.size();
  S.sun_type = f.sun_type;
  for(int c = 0; c < 3; ++c) S.sun_dir[c] = f.sun_dir[c];
  for(int c = 0; c < 9; ++c) S.sun_basis[c] = f.sun_basis[c];
  S.sun_param = f.sun_param;
  for(int c = 0; c < 8; ++c) S.buie[c] = f.buie[c];
  S.dni = f.dni;
  S.wl_count = (int32_t)f.wl_nodes.size();
  S.air_medium = f.air_medium;
  S.area_proxy = f.meta.sampled_area_proxy;
  S.area_rt = f.meta.sampled_area;
  S.nrcv = (int32_t)f.meta.rcv.size();
  S.nsampled = (int32_t)f.meta.sampled.size();
  S.nprim_slots = f.meta.nprim_slots;
}

/* Every index the kernel dereferences, checked on the host before upload */
template<class R>
static bool validate(const FlatScene<R>& f, bool need_samp = true)
{
  const int64_t nnodes = (int64_t)f.nodes.size();
  const int64_t nrefs = (int64_t)f.bvh.primrefs.size();
  if(nnodes < 1) return false;
  /* A device-built tree's nodes are written on the device from the
   * primitive references checked here, its depth is checked once built */
  if(f.device_bvh) {
    if(f.prim_ref.size() < 2 || (size_t)nnodes != f.prim_ref.size() - 1
    || f.prim_box.size() != 6 * f.prim_ref.size() || f.prim_ref.size() > (1u << 28))
      return false;
    for(uint32_t ref : f.prim_ref) {
      const uint32_t i = primref_index(ref);
      if(primref_kind(ref) == PRIM_TRIANGLE ? i >= f.tris.size() : i >= f.quads.size())
        return false;
    }
  }
  /* the traversal defers at most depth - 1 nodes on its 32-entry stack */
  if(!f.device_bvh && f.bvh.depth > 30) return false;
  for(const DNode<R>& n : f.nodes) {
    if(f.device_bvh) break;
    for(int k = 0; k < 2; ++k) {
      if(n.count[k] == 0) {
        if(n.child[k] <= 0 || n.child[k] >= nnodes) return false;
      } else if(n.count[k] == 1) {
        const uint32_t ref = (uint32_t)n.child[k];
        const uint32_t i = primref_index(ref);
        if(primref_kind(ref) == PRIM_TRIANGLE ? i >= f.tris.size() : i >= f.quads.size())
          return false;
      } else if(n.count[k] > 0) {
        if(n.child[k] < 0 || (int64_t)n.child[k] + n.count[k] > nrefs) return false;
      }
    }
  }
  if(!f.tshade.empty()) {
    if(f.tshade.size() != f.tris.size()) return false;
    const int64_t block = 6 * (int64_t)f.shader_wl.size();
    for(const DTriShade<R>& t : f.tshade)
      for(int k = 0; k < 2; ++k)
        if(t.bake[k] < -1 || (t.bake[k] >= 0 && t.bake[k] + block > (int64_t)f.bake_tab.size()))
          return false;
  }
  for(uint32_t ref : f.bvh.primrefs) {
    const uint32_t i = primref_index(ref);
    if(primref_kind(ref) == PRIM_TRIANGLE ? i >= f.tris.size() : i >= f.quads.size())
      return false;
  }
  const int64_t nsi = (int64_t)f.sinsts.size();
  const int nrcv = (int)f.meta.rcv.size();
  const int nsampled = (int)f.meta.sampled.size();
  for(const DTri<R>& t : f.tris)
    if(t.sinst < 0 || t.sinst >= nsi) return false;
  for(const DQuadric<R>& q : f.quads) {
    if(q.sinst < 0 || q.sinst >= nsi) return false;
    if(q.carve_first < 0
    || (size_t)q.carve_first + (size_t)q.carve_count > f.carvings.size()) return false;
  }
  for(const DCarving& c : f.carvings)
    if(c.first < 0 || (size_t)(c.first + c.count) * 2 > f.carve_verts.size()) return false;
  for(const DShadedInst& si : f.sinsts) {
    for(int k = 0; k < 2; ++k) {
      if(si.mtl[k] < 0 || si.mtl[k] >= (int)f.mtls.size()) return false;
      if(si.rcv_slot[k] >= nrcv) return false;
      if(si.prim_base[k] >= 0 && si.rcv_slot[k] < 0) return false;
    }
    if(si.sampled >= nsampled) return false;
    if(si.is_punched && (si.quadric < 0 || si.quadric >= (int)f.quads.size())) return false;
  }
  for(const DMaterial& m : f.mtls) {
    const int nm = (int)f.media.size();
    if(m.in_medium < 0 || m.in_medium >= nm || m.out_medium < 0
    || m.out_medium >= nm || m.slab_medium < 0 || m.slab_medium >= nm)
      return false;
    if(m.table < 0 || (size_t)m.table + 2 * f.shader_wl.size() > f.shader_tab.size())
      return false;
  }
  for(const DMedium& m : f.media)
    for(const DData* d : {&m.extinction, &m.refractive_index})
      if(d->spectrum >= (int)f.spectra.size()) return false;
  for(const DSpectrum& sp : f.spectra)
    if(sp.count < 1 || (size_t)(sp.first + sp.count) > f.spec_wl.size()) return false;
  const int64_t nsamp = (int64_t)f.samp.size();
  if((need_samp && nsamp < 1) || f.alias_prob.size() != f.samp.size()
  || f.alias_idx.size() != f.samp.size()) return false;
  for(int32_t a : f.alias_idx) if(a < 0 || a >= nsamp) return false;
  for(const DSampTri<R>& t : f.samp) {
    if(t.sinst < 0 || t.sinst >= nsi) return false;
    if(f.sinsts[t.sinst].sampled < 0) return false;
    if(t.gid >= (int64_t)f.tris.size()) return false;
  }
  /* per-primitive slots stay inside the tally array */
  for(const FlatMeta::PrimRange& pr : f.meta.prims)
    if(pr.base < 0 || pr.base + pr.ntris > f.meta.nprim_slots) return false;
  if(f.air_medium < 0 || f.air_medium >= (int)f.media.size()) return false;
  if(f.wl_nodes.empty() || f.wl_cdf.size() != f.wl_nodes.size()) return false;
  return true;
}

template<class R>
static void add_scene(Blob& b, const FlatScene<R>& f)
{
  b.add(f.nodes);
  b.add(f.bvh.primrefs);
  b.add(f.tris);
  b.add(f.quads);
  b.add(f.carvings);
  b.add(f.carve_verts);
  b.add(f.sinsts);
  b.add(f.mtls);
  b.add(f.media);
  b.add(f.spectra);
  b.add(f.spec_wl);
  b.add(f.spec_val);
  b.add(f.shader_tab);
  b.add(f.shader_wl);
  b.add(f.samp);
  b.add(f.alias_prob);
  b.add(f.alias_idx);
  b.add(f.wl_nodes);
  b.add(f.wl_pdf);
  b.add(f.wl_cdf);
  b.add(f.tshade);
  b.add(f.bake_tab);
}

static int launch_lbvh_r(const LbvhArgs& A, void* s, float) { return launch_lbvh_f32(A, s); }
static int launch_lbvh_r(const LbvhArgs& A, void* s, double) { return launch_lbvh_f64(A, s); }

/* Snapshot upload; a device-built BVH is built here, after the copy, on the
 * device's stream, and its depth read back. RES_BAD_OP: the tree is deeper
 * than the traversal stack allows (the caller rebuilds on the host). */
template<class R>
static res_T upload(ssol_b200_plan* p, const FlatScene<R>& f, DScene<R>& S)
{
  Blob b;
  add_scene(b, f);
  size_t o_box = 0, o_ref = 0, o_scratch = 0, bytes = b.host.size() + 256;
  const int nprims = (int)f.prim_ref.size();
  if(f.device_bvh) {
    o_box = b.add(f.prim_box);
    o_ref = b.add(f.prim_ref);
    o_scratch = (b.host.size() + 255) & ~size_t(255);
    bytes = o_scratch + lbvh_scratch_bytes(nprims) + 256;
  }
  const cudaStream_t st = (cudaStream_t)p->dev->stream;
  if(dev_alloc(p->dev, &p->d_scene, bytes) != cudaSuccess) return RES_MEM_ERR;
  p->scene_alloc = bytes;
  if(cudaMemcpyAsync(p->d_scene, b.host.data(), b.host.size(),
                     cudaMemcpyHostToDevice, st) != cudaSuccess)
    return RES_UNKNOWN_ERR;
  p->scene_bytes = b.host.size();
  bind_scene(S, f, b, (unsigned char*)p->d_scene);
  if(f.device_bvh) {
    unsigned char* base = (unsigned char*)p->d_scene;
    LbvhArgs A = {};
    A.n = nprims;
    A.box = base + o_box;
    A.ref = (const uint32_t*)(base + o_ref);
    A.nodes = base + b.offsets[0];
    A.optimize = 1;
    lbvh_bind_scratch(A, base + o_scratch);
    if(launch_lbvh_r(A, st, R()) != 0) return RES_UNKNOWN_ERR;
    int32_t depth = 0;
    if(cudaMemcpyAsync(&depth, A.depth, sizeof(depth), cudaMemcpyDeviceToHost, st)
       != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
      return RES_UNKNOWN_ERR;
    p->bvh_depth = depth;
    if(depth < 1 || depth > 30) return RES_BAD_OP;
  }
  return RES_OK;
}

/*******************************************************************************
 * Device snapshots for the renderers (render.cpp)
 ******************************************************************************/
cudaError_t ssolb_dev_alloc(ssol_device* dev, void** p, size_t bytes)
{ return dev_alloc(dev, p, bytes); }

void ssolb_dev_free(ssol_device* dev, void* p, size_t bytes)
{ dev_free(dev, p, bytes); }

template<class R>
static res_T snapshot_upload(ssol_device* dev, const FlatScene<R>& f, DScene<R>& S,
                             DeviceSnapshot& out)
{
  Blob b;
  add_scene(b, f);
  out.alloc = b.host.size() + 256;
  if(dev_alloc(dev, &out.d_scene, out.alloc) != cudaSuccess) {
    out.d_scene = nullptr;
    return RES_MEM_ERR;
  }
  if(cudaMemcpyAsync(out.d_scene, b.host.data(), b.host.size(), cudaMemcpyHostToDevice,
                     (cudaStream_t)dev->stream) != cudaSuccess)
    return RES_UNKNOWN_ERR;
  out.bytes = b.host.size();
  bind_scene(S, f, b, (unsigned char*)out.d_scene);
  return RES_OK;
}

res_T ssolb_snapshot_create
  (ssol_scene* scn, const ssol_b200_options* options, DeviceSnapshot& out)
{
  out = DeviceSnapshot();
  const ssol_b200_options opt = options ? *options : SSOL_B200_OPTIONS_DEFAULT;
  if(opt.precision != SSOL_B200_FP32 && opt.precision != SSOL_B200_FP64)
    return RES_BAD_ARG;
  if(opt.bvh_leaf_size < 0 || !builder_ok(opt.bvh_builder)) return RES_BAD_ARG;
  BvhBuildParams bp;
  bp.max_leaf = opt.bvh_leaf_size ? opt.bvh_leaf_size : 1;
  bp.threads = host_threads();
  out.precision = opt.precision;
  std::unique_ptr<FlatScene<float>> f32;
  std::unique_ptr<FlatScene<double>> f64;
  res_T res;
  if(opt.precision == SSOL_B200_FP32) {
    f32.reset(new FlatScene<float>());
    res = flatten_scene(scn, bp, *f32, true);
  } else {
    f64.reset(new FlatScene<double>());
    res = flatten_scene(scn, bp, *f64, true);
  }
  if(res != RES_OK) return res;
  if(f32 ? !validate(*f32, false) : !validate(*f64, false)) {
    scn->dev->log_error("inconsistent device scene snapshot.\n");
    return RES_UNKNOWN_ERR;
  }
  res = device_bind(scn->dev);
  if(res != RES_OK) return res;
  res = f32 ? snapshot_upload(scn->dev, *f32, out.s32, out)
            : snapshot_upload(scn->dev, *f64, out.s64, out);
  if(res != RES_OK) ssolb_snapshot_release(scn->dev, out);
  return res;
}

void ssolb_snapshot_release(ssol_device* dev, DeviceSnapshot& s)
{
  dev_free(dev, s.d_scene, s.alloc);
  s.d_scene = nullptr;
  s.alloc = 0;
}

static void plan_release(ssol_b200_plan* p)
{
  dev_free(p->dev, p->d_scene, p->scene_alloc);
  dev_free(p->dev, p->d_tally, p->tl.total);
  dev_free(p->dev, p->d_bvh2, p->bvh2_alloc);
  if(p->ev0) cudaEventDestroy(p->ev0);
  if(p->ev1) cudaEventDestroy(p->ev1);
  if(p->scn) ssol_scene_ref_put(p->scn);
  ssol_device* dev = p->dev;
  delete p;
  if(dev) ssol_device_ref_put(dev);
}

extern "C" res_T ssol_b200_plan_ref_get(ssol_b200_plan* p)
{
  if(!p) return RES_BAD_ARG;
  p->ref.get();
  return RES_OK;
}

extern "C" res_T ssol_b200_plan_ref_put(ssol_b200_plan* p)
{
  if(!p) return RES_BAD_ARG;
  if(p->ref.put()) plan_release(p);
  return RES_OK;
}

/* keep_flat: with a device-built tree, the plan keeps its snapshot for
 * plan_swap_sah */
static res_T plan_create_impl
  (ssol_scene* scn, const ssol_b200_options* options, ssol_b200_plan** out,
   bool keep_flat)
{
  if(!scn || !out) return RES_BAD_ARG;
  ssol_b200_options opt = options ? *options : SSOL_B200_OPTIONS_DEFAULT;
  if(opt.precision != SSOL_B200_FP32 && opt.precision != SSOL_B200_FP64)
    return RES_BAD_ARG;
  if(opt.block_size < 0 || opt.block_size > 256 || opt.grid_blocks < 0
  || opt.waves < 0 || opt.bvh_leaf_size < 0)
    return RES_BAD_ARG;
  if(opt.block_size == 0) opt.block_size = 256;
  if(opt.block_size % 32) return RES_BAD_ARG;
  if(opt.bvh_leaf_size == 0) opt.bvh_leaf_size = 1;
  if(opt.max_segments == 0) opt.max_segments = 1000000ull;
  if(opt.min_blocks_per_sm < 0 || opt.min_blocks_per_sm > 3) return RES_BAD_ARG;
  if(opt.min_blocks_per_sm == 0) opt.min_blocks_per_sm = default_min_blocks(opt.precision);
  if(!builder_ok(opt.bvh_builder)) return RES_BAD_ARG;
  /* a plan does not know how many realisations it will trace */
  if(opt.bvh_builder == SSOL_B200_BVH_AUTO) opt.bvh_builder = SSOL_B200_BVH_SAH;
  if(opt.bvh_builder == SSOL_B200_BVH_LBVH) opt.bvh_leaf_size = 1;

  BvhBuildParams bp;
  bp.max_leaf = opt.bvh_leaf_size;
  bp.threads = host_threads();
  bp.device = opt.bvh_builder == SSOL_B200_BVH_LBVH;

  /* Snapshot on the host first: argument errors need no GPU */
  std::unique_ptr<FlatScene<float>> f32;
  std::unique_ptr<FlatScene<double>> f64;
  res_T res;
  if(opt.precision == SSOL_B200_FP32) {
    f32.reset(new FlatScene<float>());
    res = flatten_scene(scn, bp, *f32);
  } else {
    f64.reset(new FlatScene<double>());
    res = flatten_scene(scn, bp, *f64);
  }
  if(res != RES_OK) return res;
  if(f32 ? !validate(*f32) : !validate(*f64)) {
    scn->dev->log_error("inconsistent device scene snapshot.\n");
    return RES_UNKNOWN_ERR;
  }

  res = device_bind(scn->dev);
  if(res != RES_OK) return res;

  ssol_b200_plan* p = new (std::nothrow) ssol_b200_plan();
  if(!p) return RES_MEM_ERR;
  ssol_device_ref_get(scn->dev);
  p->dev = scn->dev;
  ssol_scene_ref_get(scn);
  p->scn = scn;
  p->opt = opt;
  p->bvh_device = f32 ? f32->device_bvh : f64->device_bvh;
  p->bvh_depth = f32 ? f32->bvh.depth : f64->bvh.depth;
  p->bvh_nodes = f32 ? f32->nodes.size() : f64->nodes.size();
  if(f32) {
    p->meta = f32->meta;
    res = upload(p, *f32, p->s32);
  } else {
    p->meta = f64->meta;
    res = upload(p, *f64, p->s64);
  }
  if(res == RES_BAD_OP) {
    /* A device-built tree too deep for the traversal stack: the host SAH
     * builder bounds its depth */
    plan_release(p);
    scn->dev->log_warning("device BVH deeper than 30 levels; built on the host instead.\n");
    opt.bvh_builder = SSOL_B200_BVH_SAH;
    return ssol_b200_plan_create(scn, &opt, out);
  }
  if(res != RES_OK) { plan_release(p); return res; }
  p->nrcv = (int)p->meta.rcv.size();
  p->nsampled = (int)p->meta.sampled.size();

  /* Tallies: FP64 sums, then integer counters */
  p->tl = tally_layout(p->nrcv, p->nsampled, p->meta.nprim_slots);
  if(dev_alloc(p->dev, &p->d_tally, p->tl.total) != cudaSuccess) {
    plan_release(p);
    return RES_MEM_ERR;
  }
  p->t = bind_tallies(p->tl, (unsigned char*)p->d_tally);
  cudaEventCreate(&p->ev0);
  cudaEventCreate(&p->ev1);
  if(keep_flat && p->bvh_device) {
    p->keep32 = std::move(f32);
    p->keep64 = std::move(f64);
  }
  *out = p;
  return ssol_b200_plan_reset(p, nullptr);
}

extern "C" res_T ssol_b200_plan_create
  (ssol_scene* scn, const ssol_b200_options* options, ssol_b200_plan** out)
{
  return plan_create_impl(scn, options, out, false);
}

static cudaStream_t plan_stream(ssol_b200_plan* p, void* stream)
{
  return stream ? (cudaStream_t)stream : (cudaStream_t)p->dev->stream;
}

/* What an abort request copies: a pinned word holding 1 and a non-blocking
 * stream, per device, made on the first request, so that plans themselves
 * allocate nothing for it */
struct AbortChannel {
  unsigned long long* one = nullptr;
  cudaStream_t stream = nullptr;
};

static bool abort_channel(int dev, AbortChannel& out)
{
  static AbortChannel channels[64];
  static std::mutex lock;
  if(dev < 0 || dev >= 64) return false;
  std::lock_guard<std::mutex> g(lock);
  AbortChannel& c = channels[dev];
  if(!c.one) {
    if(cudaMallocHost((void**)&c.one, sizeof(unsigned long long)) != cudaSuccess) {
      c.one = nullptr;
      return false;
    }
    *c.one = 1;
  }
  if(!c.stream && cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess) {
    c.stream = nullptr;
    return false;
  }
  out = c;
  return true;
}

extern "C" res_T ssol_b200_plan_abort(ssol_b200_plan* p)
{
  if(!p) return RES_BAD_ARG;
  /* The plan's device, whatever device is current on the calling thread */
  const int dev = p->dev->cuda_device;
  int cur = -1;
  if(cudaGetDevice(&cur) != cudaSuccess) return RES_UNKNOWN_ERR;
  if(cur != dev && cudaSetDevice(dev) != cudaSuccess) return RES_UNKNOWN_ERR;
  AbortChannel c;
  const bool ok = abort_channel(dev, c);
  if(!ok) {
    if(cur != dev) cudaSetDevice(cur);
    return RES_UNKNOWN_ERR;
  }
  /* A copy, not a kernel: it runs beside the plan's persistent kernels */
  const bool copied = cudaMemcpyAsync(p->t.counters + 5, c.one, sizeof(unsigned long long),
                                      cudaMemcpyHostToDevice, c.stream) == cudaSuccess
    && cudaStreamSynchronize(c.stream) == cudaSuccess;
  if(cur != dev) cudaSetDevice(cur);
  return copied ? RES_OK : RES_UNKNOWN_ERR;
}

extern "C" res_T ssol_b200_plan_reset(ssol_b200_plan* p, void* stream)
{
  if(!p) return RES_BAD_ARG;
  if(cudaMemsetAsync(p->d_tally, 0, p->tl.total, plan_stream(p, stream))
     != cudaSuccess)
    return RES_UNKNOWN_ERR;
  p->kernel_ms = 0;
  p->timing_valid = false;
  return RES_OK;
}

/* keep_start: the launch continues the previous one in the kernel timing
 * (the start event is not recorded again) */
static res_T plan_launch
  (ssol_b200_plan* p, const ssp_rng* rng, const uint64_t first,
   const uint64_t count, void* stream, const DTrack* track,
   const unsigned long long max_failed = ~0ull, bool keep_start = false)
{
  if(!p || !rng) return RES_BAD_ARG;
  if(!count) return RES_OK;
  const cudaStream_t s = plan_stream(p, stream);
  LaunchConfig cfg;
  cfg.block_size = p->opt.block_size;
  cfg.grid_blocks = p->opt.grid_blocks;
  cfg.waves = p->opt.waves;
  cfg.max_segments = p->opt.max_segments;
  cfg.min_blocks = p->opt.min_blocks_per_sm;
  cfg.max_failed = max_failed;
  cfg.abortable = true;
  cfg.features = p->meta.features;
  cfg.count_work = p->opt.count_work != 0;
  const uint64_t start = rng->position + first;
  if(!keep_start || !p->timing_valid) cudaEventRecord(p->ev0, s);
  const int err = p->opt.precision == SSOL_B200_FP32
    ? launch_realisations_f32(p->s32, p->t, rng->seed, start, count, cfg, s, track)
    : launch_realisations_f64(p->s64, p->t, rng->seed, start, count, cfg, s, track);
  cudaEventRecord(p->ev1, s);
  if(err != 0) {
    p->dev->log_error("kernel launch failed: %s\n",
                      cudaGetErrorString((cudaError_t)err));
    return RES_UNKNOWN_ERR;
  }
  p->timing_valid = true;
  return RES_OK;
}

extern "C" res_T ssol_b200_plan_launch
  (ssol_b200_plan* p, const ssp_rng* rng, const uint64_t first,
   const uint64_t count, void* stream)
{
  return plan_launch(p, rng, first, count, stream, nullptr);
}

/* Replace a plan's device-built tree by the host SAH tree of the same
 * primitive boxes, built on the calling thread while the plan's launches
 * already queued run on the device's tree. Both trees give the same closest
 * hits, so later launches only trace faster. The new nodes go to a buffer
 * of their own; launches take the scene by value, so the queued ones keep
 * the old tree. No-op for a plan without a kept snapshot, or when the host
 * tree would be too deep. */
template<class R>
static res_T swap_sah(ssol_b200_plan* p, const FlatScene<R>& f, DScene<R>& S)
{
  const size_t n = f.prim_ref.size();
  std::vector<PrimBox> boxes(n);
  for(size_t i = 0; i < n; ++i) {
    for(int c = 0; c < 3; ++c) {
      boxes[i].lo[c] = (double)f.prim_box[6 * i + c];
      boxes[i].hi[c] = (double)f.prim_box[6 * i + 3 + c];
    }
    boxes[i].ref = f.prim_ref[i];
  }
  BvhBuildParams bp;
  bp.max_leaf = 1;
  bp.threads = host_threads();
  BvhResult r;
  build_bvh(std::move(boxes), bp, r);
  if(r.depth > 30) return RES_OK;
  const std::vector<DNode<R>> nodes = bvh_nodes<R>(r);
  Blob b;
  const size_t o_nodes = b.add(nodes);
  const size_t o_refs = b.add(r.primrefs);
  const size_t bytes = b.host.size() + 256;
  if(dev_alloc(p->dev, &p->d_bvh2, bytes) != cudaSuccess) {
    p->d_bvh2 = nullptr;
    return RES_OK; /* keep tracing on the device's tree */
  }
  p->bvh2_alloc = bytes;
  if(cudaMemcpyAsync(p->d_bvh2, b.host.data(), b.host.size(), cudaMemcpyHostToDevice,
                     (cudaStream_t)p->dev->stream) != cudaSuccess)
    return RES_UNKNOWN_ERR;
  unsigned char* base = (unsigned char*)p->d_bvh2;
  S.nodes = (const DNode<R>*)(base + o_nodes);
  S.primrefs = (const uint32_t*)(base + o_refs);
  p->bvh_device = false;
  p->bvh_depth = r.depth;
  p->bvh_nodes = nodes.size();
  return RES_OK;
}

static res_T plan_swap_sah(ssol_b200_plan* p)
{
  res_T res = RES_OK;
  if(p->keep32) res = swap_sah(p, *p->keep32, p->s32);
  else if(p->keep64) res = swap_sah(p, *p->keep64, p->s64);
  p->keep32.reset();
  p->keep64.reset();
  return res;
}

static void fill_sums(double dst[10][2], const double* src)
{
  for(int q = 0; q < 10; ++q) {
    dst[q][0] = src[2 * q];
    dst[q][1] = src[2 * q + 1];
  }
}

extern "C" res_T ssol_b200_plan_finish
  (ssol_b200_plan* p, const ssp_rng* rng, const uint64_t nreal,
   const size_t max_failed, void* stream, ssol_estimator** out)
{
  if(!p || !rng || !out) return RES_BAD_ARG;
  const cudaStream_t s = plan_stream(p, stream);
  std::vector<unsigned char> h(p->tl.total);
  if(cudaMemcpyAsync(h.data(), p->d_tally, p->tl.total,
                     cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return RES_UNKNOWN_ERR;
  const cudaError_t err = cudaStreamSynchronize(s);
  if(err != cudaSuccess) {
    p->dev->log_error("device error: %s\n", cudaGetErrorString(err));
    return RES_UNKNOWN_ERR;
  }
  if(p->timing_valid) {
    float ms = 0;
    if(cudaEventElapsedTime(&ms, p->ev0, p->ev1) == cudaSuccess)
      p->kernel_ms = ms;
  }
  /* Realisations that ran: fewer than asked for after an early stop */
  const DStats* st = (const DStats*)(h.data() + p->tl.stats);
  const uint64_t ran = std::min<uint64_t>(nreal, st->paths);
  res_T res = make_estimator(p->dev, p->scn, p->meta, p->tl, h.data(), ran, rng,
                             nreal, st, p->kernel_ms, p->scene_bytes, max_failed, out);
  if(*out) {
    (*out)->bvh_nodes = p->bvh_nodes;
    (*out)->bvh_depth = (unsigned long long)p->bvh_depth;
    (*out)->bvh_device = p->bvh_device ? 1ull : 0ull;
  }
  const unsigned long long* cnt = (const unsigned long long*)(h.data() + p->tl.counters);
  if(res == RES_OK && cnt[5]) {
    p->dev->log_error("the solve was aborted: %llu of %llu realisations ran.\n",
                      (unsigned long long)ran, (unsigned long long)nreal);
    res = RES_BAD_OP;
  }
  return res;
}

extern "C" res_T ssol_b200_autotune
  (ssol_scene* scn, const ssp_rng* rng, const uint64_t trial_paths,
   ssol_b200_options* options, double* best_ms)
{
  if(!scn || !rng || !options || !trial_paths) return RES_BAD_ARG;
  static const int leaves[] = {1, 2, 4};
  static const int blocks[] = {128, 256};
  static const int budgets[] = {1, 2, 3};
  static const int waves[] = {1, 2};
  const ssol_b200_options base = *options;
  ssol_b200_options best_opt = base;
  double best = DBL_MAX;
  for(const int leaf : leaves) {
    /* a device-built tree has one primitive per leaf */
    if(base.bvh_builder == SSOL_B200_BVH_LBVH && leaf != 1) continue;
    ssol_b200_options o = base;
    o.bvh_leaf_size = leaf;
    o.grid_blocks = 0;
    ssol_b200_plan* plan = nullptr;
    res_T res = ssol_b200_plan_create(scn, &o, &plan);
    if(res != RES_OK) return res;
    const cudaStream_t s = plan_stream(plan, nullptr);
    for(const int blk : blocks)
      for(const int mb : budgets)
        for(const int wv : waves) {
          plan->opt.block_size = blk;
          plan->opt.min_blocks_per_sm = mb;
          plan->opt.waves = wv;
          float ms = 0;
          for(int k = 0; k < 2 && res == RES_OK; ++k) {
            res = ssol_b200_plan_launch(plan, rng, 0, trial_paths, s);
            if(res == RES_OK && cudaStreamSynchronize(s) != cudaSuccess)
              res = RES_UNKNOWN_ERR;
            if(res == RES_OK && k == 1
            && cudaEventElapsedTime(&ms, plan->ev0, plan->ev1) != cudaSuccess)
              res = RES_UNKNOWN_ERR;
          }
          if(res != RES_OK) { ssol_b200_plan_ref_put(plan); return res; }
          if(ms < best) {
            best = ms;
            best_opt = plan->opt;
          }
        }
    ssol_b200_plan_ref_put(plan);
  }
  /* the tuner picks the launch shape and the leaf size, not the builder (a
   * plan resolves the default builder to the host one) */
  best_opt.precision = base.precision;
  best_opt.max_segments = base.max_segments;
  best_opt.bvh_builder = base.bvh_builder;
  *options = best_opt;
  if(best_ms) *best_ms = best;
  return RES_OK;
}

/* Affine inverse of a 3x4 column-major transform (rotation/scale + translation) */
static bool invert_affine(const double* T, double* W)
{
  const double a = T[0], b = T[3], c = T[6];
  const double d = T[1], e = T[4], f = T[7];
  const double g = T[2], h = T[5], i = T[8];
  const double det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
  if(!(std::fabs(det) > 0)) return false;
  const double inv[9] = {(e * i - f * h) / det, (c * h - b * i) / det, (b * f - c * e) / det,
                         (f * g - d * i) / det, (a * i - c * g) / det, (c * d - a * f) / det,
                         (d * h - e * g) / det, (b * g - a * h) / det, (a * e - b * d) / det};
  /* W row-major 3x4: local = inv (x - t) */
  for(int r = 0; r < 3; ++r) {
    W[4 * r + 0] = inv[3 * r + 0];
    W[4 * r + 1] = inv[3 * r + 1];
    W[4 * r + 2] = inv[3 * r + 2];
    W[4 * r + 3] = -(inv[3 * r + 0] * T[9] + inv[3 * r + 1] * T[10] + inv[3 * r + 2] * T[11]);
  }
  return true;
}

extern "C" res_T ssol_solve_adjoint
  (ssol_scene* scn, const ssp_rng* rng, const size_t n,
   ssol_instance* const* helios, const size_t nh, const ssol_b200_adjoint_map* map,
   const ssol_b200_options* options, ssol_b200_adjoint_result* result,
   double* d_absorbed, double* d_spillage, double* flux_map)
{
  if(!scn || !rng || !n || !map || !map->receiver || !result) return RES_BAD_ARG;
  if(nh && (!helios || !d_absorbed || !d_spillage)) return RES_BAD_ARG;
  if(!map->nx || !map->ny || !(map->upper[0] > map->lower[0])
  || !(map->upper[1] > map->lower[1]) || !(map->edge_band >= 0)
  || !map->receiver->receiver_mask)
    return RES_BAD_ARG;
  /* Instance indices in attach order, as the device scene numbers them */
  const std::vector<ssol_instance*>& insts = scn->instances;
  int rcv_index = -1;
  std::vector<int> slot(insts.size(), -1);
  for(size_t i = 0; i < insts.size(); ++i)
    if(insts[i] == map->receiver) rcv_index = (int)i;
  if(rcv_index < 0) return RES_BAD_ARG;
  std::vector<double> axes(9 * nh);
  for(size_t k = 0; k < nh; ++k) {
    size_t i = 0;
    while(i < insts.size() && insts[i] != helios[k]) ++i;
    if(i == insts.size() || slot[i] >= 0 || (int)i == rcv_index) return RES_BAD_ARG;
    slot[i] = (int)k;
    const double* T = helios[k]->transform;
    double* a = axes.data() + 9 * k;
    a[0] = T[9]; a[1] = T[10]; a[2] = T[11];
    for(int c = 0; c < 2; ++c) {
      const double* col = T + 3 * c;
      const double len = std::sqrt(col[0] * col[0] + col[1] * col[1] + col[2] * col[2]);
      if(!(len > 0)) return RES_BAD_ARG;
      for(int q = 0; q < 3; ++q) a[3 + 3 * c + q] = col[q] / len;
    }
  }
  double W[12];
  if(!invert_affine(map->receiver->transform, W)) return RES_BAD_ARG;

  ssol_b200_plan* plan = nullptr;
  res_T res = ssol_b200_plan_create(scn, options, &plan);
  if(res != RES_OK) return res;
  const cudaStream_t s = plan_stream(plan, nullptr);
  const size_t ncell = (size_t)map->nx * map->ny;
  const size_t bytes = (insts.size() * sizeof(int) + 255) / 256 * 256
    + (9 * nh + ncell + 3 + 4 * nh) * sizeof(double) + 4 * sizeof(unsigned long long);
  char* dbuf = nullptr;
  if(cudaMalloc((void**)&dbuf, bytes) != cudaSuccess) {
    ssol_b200_plan_ref_put(plan);
    return RES_MEM_ERR;
  }
  int* d_slot = reinterpret_cast<int*>(dbuf);
  double* d_axes = reinterpret_cast<double*>(dbuf + (insts.size() * sizeof(int) + 255) / 256 * 256);
  double* d_map = d_axes + 9 * nh;
  double* d_sums = d_map + ncell;
  double* d_gabs = d_sums + 3;
  double* d_gspill = d_gabs + 2 * nh;
  unsigned long long* d_cnt = reinterpret_cast<unsigned long long*>(d_gspill + 2 * nh);

  AdjointArgs A;
  A.inst_slot = d_slot;
  A.axes = d_axes;
  A.rcv_instance = rcv_index;
  A.rcv_side = (map->receiver->receiver_mask & SSOL_FRONT) ? 1 : 2;
  A.rcv_mtl = (size_t)rcv_index < plan->meta.inst_mtl.size()
    ? plan->meta.inst_mtl[rcv_index][A.rcv_side - 1] : -1;
  if(A.rcv_mtl < 0) {
    ssol_b200_plan_ref_put(plan);
    cudaFree(dbuf);
    return RES_BAD_ARG;
  }
  for(int q = 0; q < 12; ++q) A.w2l[q] = W[q];
  const double cw = (map->upper[0] - map->lower[0]) / map->nx;
  const double ch = (map->upper[1] - map->lower[1]) / map->ny;
  A.lower[0] = map->lower[0];
  A.lower[1] = map->lower[1];
  A.upper[0] = map->upper[0];
  A.upper[1] = map->upper[1];
  A.edge = map->edge_band > 0 ? map->edge_band : 0.5 * std::min(cw, ch);
  A.inv_cell[0] = 1.0 / cw;
  A.inv_cell[1] = 1.0 / ch;
  A.nx = (int)map->nx;
  A.ny = (int)map->ny;
  A.map = d_map;
  A.sums = d_sums;
  A.grad_abs = d_gabs;
  A.grad_spill = d_gspill;
  A.counters = d_cnt;
  A.target = map->target;
  A.inv_n = 1.0 / (double)n;
  A.map_scale = 1.0 / ((double)n * cw * ch);

  std::vector<double> h_map(ncell), h_sums(3);
  unsigned long long h_cnt[4] = {0, 0, 0, 0};
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  bool ok = cudaMemsetAsync(dbuf, 0, bytes, s) == cudaSuccess
    && cudaMemcpyAsync(d_slot, slot.data(), insts.size() * sizeof(int),
                       cudaMemcpyHostToDevice, s) == cudaSuccess
    && (!nh || cudaMemcpyAsync(d_axes, axes.data(), 9 * nh * sizeof(double),
                               cudaMemcpyHostToDevice, s) == cudaSuccess)
    && cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess
    && cudaEventRecord(e0, s) == cudaSuccess;
  const bool f32 = plan->opt.precision == SSOL_B200_FP32;
  for(int pass = 0; ok && pass < (nh ? 2 : 1); ++pass) {
    const int err = f32
      ? launch_adjoint_f32(plan->s32, A, rng->seed, rng->position, n, pass, s)
      : launch_adjoint_f64(plan->s64, A, rng->seed, rng->position, n, pass, s);
    ok = err == 0;
  }
  ok = ok && cudaEventRecord(e1, s) == cudaSuccess
    && cudaMemcpyAsync(h_map.data(), d_map, ncell * sizeof(double),
                       cudaMemcpyDeviceToHost, s) == cudaSuccess
    && cudaMemcpyAsync(h_sums.data(), d_sums, 3 * sizeof(double),
                       cudaMemcpyDeviceToHost, s) == cudaSuccess
    && cudaMemcpyAsync(h_cnt, d_cnt, sizeof(h_cnt), cudaMemcpyDeviceToHost, s) == cudaSuccess
    && (!nh || (cudaMemcpyAsync(d_absorbed, d_gabs, 2 * nh * sizeof(double),
                                cudaMemcpyDeviceToHost, s) == cudaSuccess
             && cudaMemcpyAsync(d_spillage, d_gspill, 2 * nh * sizeof(double),
                                cudaMemcpyDeviceToHost, s) == cudaSuccess))
    && cudaStreamSynchronize(s) == cudaSuccess;
  float ms = 0;
  if(ok) cudaEventElapsedTime(&ms, e0, e1);
  if(e0) cudaEventDestroy(e0);
  if(e1) cudaEventDestroy(e1);
  cudaFree(dbuf);
  ssol_b200_plan_ref_put(plan);
  if(!ok) return RES_UNKNOWN_ERR;

  const double mean = h_sums[0] / (double)n;
  const double var = std::max(0.0, h_sums[1] / (double)n - mean * mean);
  result->absorbed = mean;
  result->absorbed_se = std::sqrt(var / (double)n);
  result->hits = (unsigned long long)h_sums[2];
  result->kernel_ms = ms;
  result->rays = h_cnt[0];
  result->node_visits = h_cnt[1];
  result->triangle_tests = h_cnt[2];
  result->quadric_tests = h_cnt[3];
  double spill = 0;
  for(size_t c = 0; c < ncell; ++c) {
    const double m = h_map[c] * A.map_scale;
    spill += (m - map->target) * (m - map->target);
    if(flux_map) flux_map[c] = m;
  }
  result->spillage = spill;
  return RES_OK;
}

extern "C" res_T ssol_b200_plan_get_stats
  (const ssol_b200_plan* p, ssol_b200_stats* s)
{
  if(!p || !s) return RES_BAD_ARG;
  std::memset(s, 0, sizeof(*s));
  s->kernel_ms = p->kernel_ms;
  s->scene_bytes = p->scene_bytes;
  s->tally_bytes = p->tl.total;
  s->bvh_nodes = p->bvh_nodes;
  s->bvh_depth = (unsigned long long)p->bvh_depth;
  s->bvh_device = p->bvh_device ? 1ull : 0ull;
  return RES_OK;
}

/*******************************************************************************
 * Tallies across GPUs: the FP64 sums region of a tally block runs from its
 * global sums to the end of its per-primitive sums, the 64-bit counts region
 * from the per-sampled sample counts to the end of the launch statistics.
 * Padding between the arrays of a region is zero and stays zero when
 * regions are added, so that two blocks of the same scene add element-wise.
 ******************************************************************************/
static void tally_regions(const TallyLayout& tl, size_t* nsums, size_t* ncounts)
{
  *nsums = (tl.nb_samples - tl.global) / sizeof(double);
  *ncounts = (tl.total - tl.nb_samples) / sizeof(unsigned long long);
}

extern "C" res_T ssol_b200_plan_get_tallies
  (ssol_b200_plan* p, double** sums, size_t* nsums, uint64_t** counts,
   size_t* ncounts)
{
  if(!p || !sums || !nsums || !counts || !ncounts) return RES_BAD_ARG;
  unsigned char* base = (unsigned char*)p->d_tally;
  *sums = (double*)(base + p->tl.global);
  *counts = (uint64_t*)(base + p->tl.nb_samples);
  tally_regions(p->tl, nsums, ncounts);
  return RES_OK;
}

/* Host snapshot metadata of `scn` (receiver slots, sampled instances,
 * primitive ranges): what gives a tally block its layout */
static res_T scene_meta(ssol_scene* scn, FlatMeta& meta, TallyLayout& tl)
{
  /* the slots only: no tree is built (the device builder's snapshot keeps
   * the primitive boxes and builds nothing on the host) */
  BvhBuildParams bp;
  bp.threads = host_threads();
  bp.device = true;
  FlatScene<float> f;
  res_T res = flatten_scene(scn, bp, f);
  if(res != RES_OK) return res;
  meta = f.meta;
  tl = tally_layout((int)meta.rcv.size(), (int)meta.sampled.size(), meta.nprim_slots);
  return RES_OK;
}

extern "C" res_T ssol_b200_tallies_size
  (ssol_scene* scn, size_t* nsums, size_t* ncounts)
{
  if(!scn || !nsums || !ncounts) return RES_BAD_ARG;
  FlatMeta meta;
  TallyLayout tl;
  const res_T res = scene_meta(scn, meta, tl);
  if(res != RES_OK) return res;
  tally_regions(tl, nsums, ncounts);
  return RES_OK;
}

extern "C" res_T ssol_b200_estimator_create_from_tallies
  (ssol_scene* scn, const ssp_rng* rng, const uint64_t nreal,
   const size_t max_failed, const double* sums, const size_t nsums,
   const uint64_t* counts, const size_t ncounts, ssol_estimator** out)
{
  if(!scn || !rng || !sums || !counts || !out) return RES_BAD_ARG;
  *out = nullptr;
  FlatMeta meta;
  TallyLayout tl;
  res_T res = scene_meta(scn, meta, tl);
  if(res != RES_OK) return res;
  size_t ns = 0, nc = 0;
  tally_regions(tl, &ns, &nc);
  if(nsums != ns || ncounts != nc) {
    scn->dev->log_error("tallies of %zu sums and %zu counts; this scene's have "
                        "%zu and %zu.\n", nsums, ncounts, ns, nc);
    return RES_BAD_ARG;
  }
  std::vector<unsigned char> block(tl.total, 0);
  std::memcpy(block.data() + tl.global, sums, nsums * sizeof(double));
  std::memcpy(block.data() + tl.nb_samples, counts, ncounts * sizeof(uint64_t));
  const DStats* st = (const DStats*)(block.data() + tl.stats);
  /* As ssol_b200_plan_finish: realisations that ran, when counted */
  const uint64_t ran = st->paths ? std::min<uint64_t>(nreal, st->paths) : nreal;
  return make_estimator(scn->dev, scn, meta, tl, block.data(), ran, rng, nreal, st,
                        0.0, 0, max_failed, out);
}


/*******************************************************************************
 * Batches: many scenes, one persistent launch (see ssol_b200.h)
 ******************************************************************************/
struct ssol_b200_batch {
  RefCount ref;
  ssol_device* dev = nullptr;
  std::vector<ssol_scene*> scenes;
  ssol_b200_options opt = SSOL_B200_OPTIONS_DEFAULT;
  std::vector<FlatMeta> meta;
  std::vector<TallyLayout> tl;
  std::vector<size_t> tally_off; /* item tallies inside d_tally */
  size_t tally_total = 0;
  size_t scene_bytes = 0;
  void* d_scene = nullptr; /* item scene arrays, then the DScene array */
  void* d_tally = nullptr; /* item tallies, DTallies array, prefix, firsts,
                              work counter and launch stats */
  unsigned long long* d_prefix = nullptr;
  unsigned long long* d_firsts = nullptr;
  unsigned long long* d_next = nullptr; /* per-item work counters */
  DStats* d_stats = nullptr;
  double* d_gather = nullptr; /* per item: global sums and failures */
  const void* d_scenes = nullptr;
  const DTallies* d_tallies = nullptr;
  std::vector<unsigned long long> done; /* realisations launched per item */
  std::vector<unsigned long long> h_prefix, h_firsts;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  cudaStream_t graph_stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double kernel_ms = 0;
  bool timing_valid = false;
  uint64_t h_seed = 0;
  void* h_tally = nullptr; /* pinned tally read-back, allocated on first finish */
  size_t scene_alloc = 0, tally_alloc = 0; /* bytes of d_scene, d_tally */
  /* Coherent order: sampled triangles per item, their histogram bins (all
   * items), per item its first bin and its segment stride (in d_tally), and
   * the presort's scratch (20 B per realisation, grown on demand) */
  std::vector<uint32_t> nsamp;
  uint32_t nbins = 0;
  uint32_t* d_bin_base = nullptr;
  uint32_t* d_hist = nullptr;
  uint32_t* d_bin_off = nullptr;
  uint32_t* d_mul = nullptr;
  std::vector<uint32_t> h_mul;
  void* d_sort = nullptr;
  size_t sort_alloc = 0;
  unsigned long long sort_cap = 0; /* realisations the scratch holds */
  bool graph_sorted = false; /* order the captured graph runs in */
};

static void batch_release(ssol_b200_batch* b)
{
  if(b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
  if(b->graph) cudaGraphDestroy(b->graph);
  dev_free(b->dev, b->d_scene, b->scene_alloc);
  dev_free(b->dev, b->d_tally, b->tally_alloc);
  dev_free(b->dev, b->d_sort, b->sort_alloc);
  host_free(b->dev, b->h_tally, b->tally_total);
  if(b->ev0) cudaEventDestroy(b->ev0);
  if(b->ev1) cudaEventDestroy(b->ev1);
  for(ssol_scene* s : b->scenes) ssol_scene_ref_put(s);
  ssol_device* dev = b->dev;
  delete b;
  if(dev) ssol_device_ref_put(dev);
}

extern "C" res_T ssol_b200_batch_ref_get(ssol_b200_batch* b)
{
  if(!b) return RES_BAD_ARG;
  b->ref.get();
  return RES_OK;
}

extern "C" res_T ssol_b200_batch_ref_put(ssol_b200_batch* b)
{
  if(!b) return RES_BAD_ARG;
  if(b->ref.put()) batch_release(b);
  return RES_OK;
}

template<class R>
static res_T batch_upload(ssol_b200_batch* b, std::vector<FlatScene<R>>& f)
{
  /* Each item's arrays are laid out in a blob of its own, on the host
   * threads; the blobs sit one after the other (256-byte aligned) in one
   * device block, followed by the DScene array */
  const size_t n = f.size();
  std::vector<Blob> blobs(n);
  parallel_for(n, [&](size_t i) { add_scene(blobs[i], f[i]); });
  std::vector<size_t> base_off(n);
  size_t total = 0;
  for(size_t i = 0; i < n; ++i) {
    base_off[i] = total;
    total = (total + blobs[i].host.size() + 255) & ~size_t(255);
  }
  const size_t s_off = total;
  total += n * sizeof(DScene<R>);
  if(dev_alloc(b->dev, &b->d_scene, total + 256) != cudaSuccess) {
    b->d_scene = nullptr;
    return RES_MEM_ERR;
  }
  b->scene_alloc = total + 256;
  unsigned char* base = (unsigned char*)b->d_scene;
  std::vector<DScene<R>> S(n);
  const cudaStream_t st = (cudaStream_t)b->dev->stream;
  for(size_t i = 0; i < n; ++i) {
    bind_scene(S[i], f[i], blobs[i], base + base_off[i]);
    if(!blobs[i].host.empty()
    && cudaMemcpyAsync(base + base_off[i], blobs[i].host.data(), blobs[i].host.size(),
                       cudaMemcpyHostToDevice, st) != cudaSuccess)
      return RES_UNKNOWN_ERR;
  }
  if(cudaMemcpyAsync(base + s_off, S.data(), n * sizeof(DScene<R>),
                     cudaMemcpyHostToDevice, st) != cudaSuccess)
    return RES_UNKNOWN_ERR;
  if(cudaStreamSynchronize(st) != cudaSuccess) return RES_UNKNOWN_ERR;
  b->scene_bytes = total;
  b->d_scenes = base + s_off;
  return RES_OK;
}

static res_T batch_tallies(ssol_b200_batch* b);

extern "C" res_T ssol_b200_batch_create
  (ssol_scene* const* scenes, const size_t nscenes,
   const ssol_b200_options* options, ssol_b200_batch** out)
{
  if(!scenes || !nscenes || !out || nscenes > (size_t)INT32_MAX)
    return RES_BAD_ARG;
  for(size_t i = 0; i < nscenes; ++i) if(!scenes[i]) return RES_BAD_ARG;
  ssol_b200_options opt = options ? *options : SSOL_B200_OPTIONS_DEFAULT;
  if(opt.precision != SSOL_B200_FP32 && opt.precision != SSOL_B200_FP64)
    return RES_BAD_ARG;
  if(opt.block_size < 0 || opt.block_size > 256 || opt.grid_blocks < 0
  || opt.waves < 0 || opt.bvh_leaf_size < 0 || opt.min_blocks_per_sm < 0
  || opt.min_blocks_per_sm > 3 || !builder_ok(opt.bvh_builder))
    return RES_BAD_ARG;
  if(opt.block_size == 0) opt.block_size = 256;
  if(opt.block_size % 32) return RES_BAD_ARG;
  if(opt.bvh_leaf_size == 0) opt.bvh_leaf_size = 1;
  if(opt.max_segments == 0) opt.max_segments = 1000000ull;
  if(opt.min_blocks_per_sm == 0) opt.min_blocks_per_sm = default_min_blocks(opt.precision);

  ssol_device* dev = scenes[0]->dev;
  ssol_b200_batch* b = new (std::nothrow) ssol_b200_batch();
  if(!b) return RES_MEM_ERR;
  ssol_device_ref_get(dev);
  b->dev = dev;
  for(size_t i = 0; i < nscenes; ++i) {
    ssol_scene_ref_get(scenes[i]);
    b->scenes.push_back(scenes[i]);
  }
  b->opt = opt;
  BvhBuildParams bp;
  bp.max_leaf = opt.bvh_leaf_size;

  /* Host snapshots first: argument errors need no GPU */
  res_T res;
  std::vector<FlatScene<float>> f32;
  std::vector<FlatScene<double>> f64;
  /* Snapshots of the items in parallel on the host threads */
  std::vector<res_T> item_res(nscenes, RES_OK);
  if(opt.precision == SSOL_B200_FP32) {
    f32.resize(nscenes);
    parallel_for(nscenes, [&](size_t i) {
      item_res[i] = flatten_scene(scenes[i], bp, f32[i]);
      if(item_res[i] == RES_OK && !validate(f32[i])) item_res[i] = RES_UNKNOWN_ERR;
    });
  } else {
    f64.resize(nscenes);
    parallel_for(nscenes, [&](size_t i) {
      item_res[i] = flatten_scene(scenes[i], bp, f64[i]);
      if(item_res[i] == RES_OK && !validate(f64[i])) item_res[i] = RES_UNKNOWN_ERR;
    });
  }
  for(size_t i = 0; i < nscenes; ++i) {
    if(item_res[i] != RES_OK) { batch_release(b); return item_res[i]; }
    b->meta.push_back(f32.empty() ? f64[i].meta : f32[i].meta);
    b->nsamp.push_back((uint32_t)(f32.empty() ? f64[i].samp.size() : f32[i].samp.size()));
  }
  res = device_bind(dev);
  if(res == RES_OK)
    res = opt.precision == SSOL_B200_FP32 ? batch_upload(b, f32) : batch_upload(b, f64);
  if(res != RES_OK) { batch_release(b); return res; }
  res = batch_tallies(b);
  if(res != RES_OK) { batch_release(b); return res; }
  *out = b;
  return ssol_b200_batch_reset(b, nullptr);
}

/* Tallies of every item (b->meta filled), then the batch bookkeeping */
static res_T batch_tallies(ssol_b200_batch* b)
{
  ssol_device* dev = b->dev;
  const size_t nscenes = b->scenes.size();
  size_t off = 0;
  for(size_t i = 0; i < nscenes; ++i) {
    const FlatMeta& m = b->meta[i];
    b->tl.push_back(tally_layout((int)m.rcv.size(), (int)m.sampled.size(),
                                 m.nprim_slots));
    b->tally_off.push_back(off);
    off += b->tl.back().total;
  }
  b->tally_total = off;
  const size_t o_tallies = off;
  off = (off + nscenes * sizeof(DTallies) + 255) & ~size_t(255);
  const size_t o_prefix = off;
  off = (off + (nscenes + 1) * sizeof(unsigned long long) + 255) & ~size_t(255);
  const size_t o_firsts = off;
  off = (off + nscenes * sizeof(unsigned long long) + 255) & ~size_t(255);
  const size_t o_next = off;
  off = (off + nscenes * sizeof(unsigned long long) + 255) & ~size_t(255);
  const size_t o_stats = off;
  off += (sizeof(DStats) + 255) & ~size_t(255);
  const size_t o_gather = off;
  off += (13 * nscenes * sizeof(double) + 255) & ~size_t(255);
  /* Coherent order: per item its first histogram bin and segment stride,
   * then the histogram and its ranges */
  std::vector<uint32_t> bin_base(nscenes, 0);
  uint64_t nbins = 0;
  for(size_t i = 0; i < nscenes; ++i) {
    bin_base[i] = (uint32_t)nbins;
    nbins += i < b->nsamp.size() ? b->nsamp[i] : 0;
  }
  if(nbins > 0x7fffffffull) nbins = 0; /* no coherent order */
  b->nbins = (uint32_t)nbins;
  const size_t o_bin_base = off;
  off += (nscenes * sizeof(uint32_t) + 255) & ~size_t(255);
  const size_t o_mul = off;
  off += (nscenes * sizeof(uint32_t) + 255) & ~size_t(255);
  const size_t o_hist = off;
  off += ((size_t)nbins * sizeof(uint32_t) + 255) & ~size_t(255);
  const size_t o_bin_off = off;
  off += ((size_t)nbins * sizeof(uint32_t) + 255) & ~size_t(255);
  if(dev_alloc(dev, &b->d_tally, off) != cudaSuccess) {
    b->d_tally = nullptr;
    return RES_MEM_ERR;
  }
  b->tally_alloc = off;
  unsigned char* base = (unsigned char*)b->d_tally;
  std::vector<DTallies> T(nscenes);
  for(size_t i = 0; i < nscenes; ++i)
    T[i] = bind_tallies(b->tl[i], base + b->tally_off[i]);
  b->d_tallies = (const DTallies*)(base + o_tallies);
  b->d_prefix = (unsigned long long*)(base + o_prefix);
  b->d_firsts = (unsigned long long*)(base + o_firsts);
  b->d_next = (unsigned long long*)(base + o_next);
  b->d_stats = (DStats*)(base + o_stats);
  b->d_gather = (double*)(base + o_gather);
  b->d_bin_base = (uint32_t*)(base + o_bin_base);
  b->d_mul = (uint32_t*)(base + o_mul);
  b->d_hist = (uint32_t*)(base + o_hist);
  b->d_bin_off = (uint32_t*)(base + o_bin_off);
  b->h_mul.assign(nscenes, 1u);
  const cudaStream_t s = (cudaStream_t)dev->stream;
  if(cudaMemcpyAsync((void*)b->d_tallies, T.data(), nscenes * sizeof(DTallies),
                     cudaMemcpyHostToDevice, s) != cudaSuccess
  || cudaMemcpyAsync(b->d_bin_base, bin_base.data(), nscenes * sizeof(uint32_t),
                     cudaMemcpyHostToDevice, s) != cudaSuccess
  || cudaStreamSynchronize(s) != cudaSuccess)
    return RES_UNKNOWN_ERR;
  b->done.assign(nscenes, 0);
  b->h_prefix.assign(nscenes + 1, 0);
  b->h_firsts.assign(nscenes, 0);
  cudaEventCreate(&b->ev0);
  cudaEventCreate(&b->ev1);
  return RES_OK;
}

/* Tracking batches (see ssol_b200_batch_create_tracking): one snapshot of
 * the scene uploaded once; per item (sun position) device copies of its
 * triangles, sampled triangles and BVH nodes, the tracked heliostats turned
 * toward the item's sun and the BVH refitted on the device; every other
 * array is shared by the items */
template<class R>
static res_T tracking_upload
  (ssol_b200_batch* b, FlatScene<R>& f, ssol_instance* const* helio, size_t nhelio,
   const double* aims, const std::vector<double>& dirs, const ssol_b200_sun_position* suns)
{
  ssol_device* dev = b->dev;
  const size_t nitems = b->scenes.size();
  /* Tracked triangles: each heliostat's mesh ranges, with local vertices */
  std::vector<double> helio_data(6 * nhelio);
  std::vector<int32_t> tri_helio, tri_index, tri_samp;
  std::vector<double> local;
  for(size_t h = 0; h < nhelio; ++h) {
    const ssol_instance* inst = helio[h];
    for(int c = 0; c < 3; ++c) {
      helio_data[6 * h + c] = inst->transform[9 + c];
      helio_data[6 * h + 3 + c] = aims[3 * h + c];
    }
    bool found = false;
    for(const FlatMeta::MeshRange& m : f.meta.meshes) {
      if(m.inst != inst) continue;
      found = true;
      for(int t = 0; t < m.ntris; ++t) {
        tri_helio.push_back((int32_t)h);
        tri_index.push_back(m.tri_first + t);
        tri_samp.push_back(m.samp_first >= 0 ? m.samp_first + t : -1);
        for(int k = 0; k < 3; ++k) {
          const uint32_t id = m.shape->ids[(size_t)t * 3 + k];
          for(int c = 0; c < 3; ++c) local.push_back(m.shape->pos[(size_t)id * 3 + c]);
        }
      }
    }
    if(!found) {
      dev->log_error("tracking: heliostat %zu is not a mesh instance of the scene.\n", h);
      return RES_BAD_ARG;
    }
  }
  /* BVH nodes grouped by depth, deepest first */
  const size_t nnodes = f.nodes.size();
  std::vector<int> depth(nnodes, 0);
  int maxd = 0;
  for(size_t i = 0; i < nnodes; ++i)
    for(int k = 0; k < 2; ++k)
      if(f.nodes[i].count[k] == 0) {
        const int c = f.nodes[i].child[k];
        depth[c] = depth[i] + 1;
        maxd = std::max(maxd, depth[c]);
      }
  std::vector<int32_t> level_first(1, 0), level_nodes;
  for(int d = maxd; d >= 0; --d) {
    for(size_t i = 0; i < nnodes; ++i) if(depth[i] == d) level_nodes.push_back((int32_t)i);
    level_first.push_back((int32_t)level_nodes.size());
  }

  /* One device block: the snapshot, the items' copies, the DScene array and
   * the inputs of the tracking kernels */
  Blob blob;
  add_scene(blob, f);
  const size_t ntri = f.tris.size(), nsamp = f.samp.size();
  size_t total = (blob.host.size() + 255) & ~size_t(255);
  auto take = [&](size_t bytes) { const size_t o = total; total = (total + bytes + 255) & ~size_t(255); return o; };
  const size_t o_tris = take(nitems * ntri * sizeof(DTri<R>));
  const size_t o_samp = take(nitems * nsamp * sizeof(DSampTri<R>));
  const size_t o_nodes = take(nitems * nnodes * sizeof(DNode<R>));
  const size_t o_scenes = take(nitems * sizeof(DScene<R>));
  const size_t o_helio = take(helio_data.size() * sizeof(double));
  const size_t o_sun = take(3 * nitems * sizeof(double));
  const size_t o_th = take(tri_helio.size() * sizeof(int32_t));
  const size_t o_ti = take(tri_index.size() * sizeof(int32_t));
  const size_t o_ts = take(tri_samp.size() * sizeof(int32_t));
  const size_t o_loc = take(local.size() * sizeof(double));
  const size_t o_ln = take(level_nodes.size() * sizeof(int32_t));
  const size_t o_lf = take(level_first.size() * sizeof(int32_t));
  if(dev_alloc(dev, &b->d_scene, total + 256) != cudaSuccess) {
    b->d_scene = nullptr;
    return RES_MEM_ERR;
  }
  b->scene_alloc = total + 256;
  unsigned char* base = (unsigned char*)b->d_scene;
  const cudaStream_t st = (cudaStream_t)dev->stream;
  std::vector<double> to_sun(3 * nitems);
  for(size_t i = 0; i < nitems; ++i)
    for(int c = 0; c < 3; ++c) to_sun[3 * i + c] = -dirs[3 * i + c];
  auto up = [&](size_t off, const void* src, size_t bytes) {
    return !bytes || cudaMemcpyAsync(base + off, src, bytes, cudaMemcpyHostToDevice, st)
                       == cudaSuccess;
  };
  bool ok = up(0, blob.host.data(), blob.host.size())
    && up(o_helio, helio_data.data(), helio_data.size() * sizeof(double))
    && up(o_sun, to_sun.data(), to_sun.size() * sizeof(double))
    && up(o_th, tri_helio.data(), tri_helio.size() * sizeof(int32_t))
    && up(o_ti, tri_index.data(), tri_index.size() * sizeof(int32_t))
    && up(o_ts, tri_samp.data(), tri_samp.size() * sizeof(int32_t))
    && up(o_loc, local.data(), local.size() * sizeof(double))
    && up(o_ln, level_nodes.data(), level_nodes.size() * sizeof(int32_t))
    && up(o_lf, level_first.data(), level_first.size() * sizeof(int32_t));
  DScene<R> S0;
  bind_scene(S0, f, blob, base);
  /* Each item starts from the snapshot's arrays */
  for(size_t i = 0; i < nitems && ok; ++i) {
    ok = cudaMemcpyAsync(base + o_tris + i * ntri * sizeof(DTri<R>), S0.tris,
                         ntri * sizeof(DTri<R>), cudaMemcpyDeviceToDevice, st) == cudaSuccess
      && (!nsamp || cudaMemcpyAsync(base + o_samp + i * nsamp * sizeof(DSampTri<R>), S0.samp,
                                    nsamp * sizeof(DSampTri<R>), cudaMemcpyDeviceToDevice, st)
                    == cudaSuccess)
      && cudaMemcpyAsync(base + o_nodes + i * nnodes * sizeof(DNode<R>), S0.nodes,
                         nnodes * sizeof(DNode<R>), cudaMemcpyDeviceToDevice, st) == cudaSuccess;
  }
  if(!ok) return RES_UNKNOWN_ERR;
  TrackArgs A;
  A.nitems = (int)nitems;
  A.ntracked = (int)tri_helio.size();
  A.nlevels = (int)level_first.size() - 1;
  A.helio = (const double*)(base + o_helio);
  A.to_sun = (const double*)(base + o_sun);
  A.tri_helio = (const int32_t*)(base + o_th);
  A.tri_index = (const int32_t*)(base + o_ti);
  A.tri_samp = (const int32_t*)(base + o_ts);
  A.local = (const double*)(base + o_loc);
  A.tris = base + o_tris; A.tri_stride = ntri;
  A.samp = base + o_samp; A.samp_stride = nsamp;
  A.nodes = base + o_nodes; A.node_stride = nnodes;
  A.primrefs = S0.primrefs;
  A.level_nodes = (const int32_t*)(base + o_ln);
  A.level_first = (const int32_t*)(base + o_lf);
  const int err = sizeof(R) == sizeof(float) ? launch_track_f32(A, st) : launch_track_f64(A, st);
  if(err) {
    dev->log_error("tracking kernels: %s\n", cudaGetErrorString((cudaError_t)err));
    return RES_UNKNOWN_ERR;
  }
  /* The items' records: the snapshot's, with their own triangles, sampled
   * triangles, nodes and sun */
  std::vector<DScene<R>> S(nitems, S0);
  for(size_t i = 0; i < nitems; ++i) {
    S[i].tris = (const DTri<R>*)(base + o_tris) + i * ntri;
    S[i].samp = (const DSampTri<R>*)(base + o_samp) + i * nsamp;
    S[i].nodes = (const DNode<R>*)(base + o_nodes) + i * nnodes;
    double B[9];
    sun_frame(&dirs[3 * i], B);
    for(int c = 0; c < 3; ++c) S[i].sun_dir[c] = (R)dirs[3 * i + c];
    for(int c = 0; c < 9; ++c) S[i].sun_basis[c] = (R)B[c];
    S[i].dni = suns[i].dni;
  }
  if(!up(o_scenes, S.data(), nitems * sizeof(DScene<R>))
  || cudaStreamSynchronize(st) != cudaSuccess)
    return RES_UNKNOWN_ERR;
  b->scene_bytes = blob.host.size() + local.size() * sizeof(double);
  b->d_scenes = base + o_scenes;
  return RES_OK;
}

extern "C" res_T ssol_b200_batch_create_tracking
  (ssol_scene* scn, ssol_instance* const* heliostats, const size_t nhelio,
   const double* aims, const ssol_b200_sun_position* suns, const size_t nsuns,
   const ssol_b200_options* options, ssol_b200_batch** out)
{
  if(!scn || (nhelio && (!heliostats || !aims)) || !suns || !nsuns || !out
  || nsuns > (size_t)INT32_MAX)
    return RES_BAD_ARG;
  ssol_b200_options opt = options ? *options : SSOL_B200_OPTIONS_DEFAULT;
  if(opt.precision != SSOL_B200_FP32 && opt.precision != SSOL_B200_FP64)
    return RES_BAD_ARG;
  if(opt.block_size < 0 || opt.block_size > 256 || opt.grid_blocks < 0
  || opt.waves < 0 || opt.bvh_leaf_size < 0 || opt.min_blocks_per_sm < 0
  || opt.min_blocks_per_sm > 3 || !builder_ok(opt.bvh_builder))
    return RES_BAD_ARG;
  if(opt.block_size == 0) opt.block_size = 256;
  if(opt.block_size % 32) return RES_BAD_ARG;
  if(opt.bvh_leaf_size == 0) opt.bvh_leaf_size = 1;
  if(opt.max_segments == 0) opt.max_segments = 1000000ull;
  if(opt.min_blocks_per_sm == 0) opt.min_blocks_per_sm = default_min_blocks(opt.precision);
  /* Sun directions normalised as ssol_sun_set_direction does */
  std::vector<double> dirs(3 * nsuns);
  for(size_t i = 0; i < nsuns; ++i) {
    const double* d = suns[i].direction;
    const double len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if(!(len > 0) || !(suns[i].dni > 0)) return RES_BAD_ARG;
    for(int c = 0; c < 3; ++c) dirs[3 * i + c] = d[c] / len;
  }
  for(size_t h = 0; h < nhelio; ++h) {
    if(!heliostats[h]) return RES_BAD_ARG;
    for(const ShadedShape& ss : heliostats[h]->object->shaded)
      if(ss.shape->kind != SHAPE_MESH) {
        scn->dev->log_error("tracking: heliostat %zu has a punched surface; only "
                            "meshes are re-aimed on the device.\n", h);
        return RES_BAD_ARG;
      }
  }

  ssol_device* dev = scn->dev;
  ssol_b200_batch* b = new (std::nothrow) ssol_b200_batch();
  if(!b) return RES_MEM_ERR;
  ssol_device_ref_get(dev);
  b->dev = dev;
  for(size_t i = 0; i < nsuns; ++i) {
    ssol_scene_ref_get(scn);
    b->scenes.push_back(scn);
  }
  b->opt = opt;
  BvhBuildParams bp;
  bp.max_leaf = opt.bvh_leaf_size;
  bp.threads = host_threads();
  res_T res;
  FlatScene<float> f32;
  FlatScene<double> f64;
  if(opt.precision == SSOL_B200_FP32) {
    res = flatten_scene(scn, bp, f32);
    if(res == RES_OK && !validate(f32)) res = RES_UNKNOWN_ERR;
  } else {
    res = flatten_scene(scn, bp, f64);
    if(res == RES_OK && !validate(f64)) res = RES_UNKNOWN_ERR;
  }
  if(res != RES_OK) { batch_release(b); return res; }
  const FlatMeta& meta = opt.precision == SSOL_B200_FP32 ? f32.meta : f64.meta;
  if(meta.features & FEAT_ATTRIBUTES) {
    dev->log_error("tracking: scenes with vertex normals or shaders baked per "
                   "vertex are not re-aimed on the device.\n");
    batch_release(b);
    return RES_BAD_ARG;
  }
  for(size_t h = 0; h < nhelio; ++h) {
    bool found = false;
    for(const FlatMeta::MeshRange& m : meta.meshes) found = found || m.inst == heliostats[h];
    if(!found) {
      dev->log_error("tracking: heliostat %zu is not an instance of the scene.\n", h);
      batch_release(b);
      return RES_BAD_ARG;
    }
  }
  b->meta.assign(nsuns, meta);
  b->nsamp.assign(nsuns, (uint32_t)(opt.precision == SSOL_B200_FP32 ? f32.samp.size()
                                                                     : f64.samp.size()));
  res = device_bind(dev);
  if(res == RES_OK)
    res = opt.precision == SSOL_B200_FP32
      ? tracking_upload(b, f32, heliostats, nhelio, aims, dirs, suns)
      : tracking_upload(b, f64, heliostats, nhelio, aims, dirs, suns);
  if(res == RES_OK) res = batch_tallies(b);
  if(res != RES_OK) { batch_release(b); return res; }
  *out = b;
  return ssol_b200_batch_reset(b, nullptr);
}

extern "C" res_T ssol_b200_batch_reset(ssol_b200_batch* b, void* stream)
{
  if(!b) return RES_BAD_ARG;
  const cudaStream_t s = stream ? (cudaStream_t)stream : (cudaStream_t)b->dev->stream;
  if(cudaMemsetAsync(b->d_tally, 0, b->tally_total, s) != cudaSuccess
  || cudaMemsetAsync(b->d_stats, 0, sizeof(DStats), s) != cudaSuccess)
    return RES_UNKNOWN_ERR;
  std::fill(b->done.begin(), b->done.end(), 0ull);
  b->kernel_ms = 0;
  b->timing_valid = false;
  return RES_OK;
}

/* The captured graph: work-counter reset + the persistent batch kernel. Its
 * parameters are device pointers only, so one capture serves every launch */
/* Launch shape of a batch; receiver sums are gathered per warp in shared
 * memory when two slots of the largest item fit in 16 KB per block */
static LaunchConfig batch_config(const ssol_b200_batch* b)
{
  LaunchConfig cfg;
  cfg.block_size = b->opt.block_size;
  cfg.grid_blocks = b->opt.grid_blocks;
  cfg.waves = b->opt.waves;
  cfg.max_segments = b->opt.max_segments;
  cfg.min_blocks = b->opt.min_blocks_per_sm;
  cfg.count_work = b->opt.count_work != 0;
  size_t nrcv = 0;
  cfg.features = 0;
  for(const FlatMeta& m : b->meta) {
    nrcv = std::max(nrcv, m.rcv.size());
    cfg.features |= m.features;
  }
  const size_t rcvd = nrcv * NRCV_Q * 2;
  const size_t warps = (size_t)(cfg.block_size > 0 ? cfg.block_size : 256) / 32;
  cfg.rcv_doubles = warps * 2 * rcvd * sizeof(double) <= 16 * 1024 ? (int)rcvd : 0;
  return cfg;
}

/* The launch's coherent order over the sort scratch (b->sort_cap
 * realisations), or none */
static BatchOrder batch_order(const ssol_b200_batch* b, bool sorted)
{
  BatchOrder o;
  if(!sorted) return o;
  const unsigned long long cap = b->sort_cap;
  unsigned char* p = (unsigned char*)b->d_sort;
  o.sorted_draw = (uint32_t*)p;
  o.sorted_off = (uint32_t*)(p + cap * 16);
  o.hist = b->d_hist;
  o.bin_off = b->d_bin_off;
  o.bin_base = b->d_bin_base;
  o.seg_mul = b->d_mul;
  o.nbins = b->nbins;
  return o;
}

static res_T batch_graph(ssol_b200_batch* b, const ssp_rng* rng, cudaStream_t s,
                         bool sorted)
{
  if(b->graph_exec && b->graph_stream == s && b->graph_sorted == sorted) return RES_OK;
  if(b->graph_exec) { cudaGraphExecDestroy(b->graph_exec); b->graph_exec = nullptr; }
  if(b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
  const LaunchConfig cfg = batch_config(b);
  if(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return RES_UNKNOWN_ERR;
  int err;
  if(b->opt.precision == SSOL_B200_FP32) {
    BatchLaunch<float> L = {(const DScene<float>*)b->d_scenes, b->d_tallies,
      b->d_prefix, b->d_firsts, (int)b->scenes.size(), rng->seed, b->d_next,
      b->d_stats, batch_order(b, sorted)};
    err = launch_batch_f32(L, cfg, s);
  } else {
    BatchLaunch<double> L = {(const DScene<double>*)b->d_scenes, b->d_tallies,
      b->d_prefix, b->d_firsts, (int)b->scenes.size(), rng->seed, b->d_next,
      b->d_stats, batch_order(b, sorted)};
    err = launch_batch_f64(L, cfg, s);
  }
  const cudaError_t e2 = cudaStreamEndCapture(s, &b->graph);
  if(err != 0 || e2 != cudaSuccess) return RES_UNKNOWN_ERR;
  if(cudaGraphInstantiate(&b->graph_exec, b->graph, 0) != cudaSuccess)
    return RES_UNKNOWN_ERR;
  b->graph_stream = s;
  b->graph_sorted = sorted;
  return RES_OK;
}

/* Launches of at least BATCH_SORT_MIN realisations run in the coherent order
 * (up to BATCH_SORT_MAX: the scratch takes 20 B per realisation, and the
 * sorted offsets are 32-bit) */
constexpr unsigned long long BATCH_SORT_MIN = 1ull << 22;
constexpr unsigned long long BATCH_SORT_MAX = 1ull << 29;

/* Whether this launch runs in the coherent order; grows the scratch (and
 * drops the captured graph, which holds its address) as needed */
static bool batch_prepare_order(ssol_b200_batch* b, unsigned long long total)
{
  if(!b->nbins || total < BATCH_SORT_MIN || total > BATCH_SORT_MAX) return false;
  for(const uint32_t n : b->nsamp) if(n < 2) return false;
  if(total > b->sort_cap) {
    /* one allocation for several launches: a quarter more than asked */
    unsigned long long cap = total + total / 4;
    if(cap > BATCH_SORT_MAX) cap = BATCH_SORT_MAX;
    /* a multiple of 256: the offsets after the draws start on 256 bytes */
    cap = (cap + 255) & ~255ull;
    void* p = nullptr;
    if(dev_alloc(b->dev, &p, (size_t)cap * 20) != cudaSuccess) return false;
    if(b->graph_exec) { cudaGraphExecDestroy(b->graph_exec); b->graph_exec = nullptr; }
    dev_free(b->dev, b->d_sort, b->sort_alloc);
    b->d_sort = p;
    b->sort_alloc = (size_t)cap * 20;
    b->sort_cap = cap;
  }
  /* Per item, the stride of its full segments' order: near n / golden
   * ratio, coprime with n, below n */
  const size_t n = b->scenes.size();
  for(size_t i = 0; i < n; ++i) {
    const unsigned long long nfull = (b->h_prefix[i + 1] - b->h_prefix[i]) / SORT_SEGMENT;
    unsigned long long mul = 1;
    if(nfull > 1) {
      mul = (unsigned long long)(0.6180339887 * (double)nfull) | 1ull;
      while(std::gcd(mul, nfull) != 1ull) mul += 2;
      mul %= nfull;
    }
    b->h_mul[i] = (uint32_t)mul;
  }
  return true;
}

extern "C" res_T ssol_b200_batch_launch
  (ssol_b200_batch* b, const ssp_rng* rng, const uint64_t* budgets, void* stream)
{
  if(!b || !rng || !budgets) return RES_BAD_ARG;
  const size_t n = b->scenes.size();
  unsigned long long total = 0;
  for(size_t i = 0; i < n; ++i) {
    b->h_prefix[i] = total;
    b->h_firsts[i] = rng->position + b->done[i];
    total += budgets[i];
  }
  b->h_prefix[n] = total;
  if(!total) return RES_OK;
  const cudaStream_t s = stream ? (cudaStream_t)stream : (cudaStream_t)b->dev->stream;
  /* The seed is a kernel argument baked into the graph */
  if(b->graph_exec && b->graph_stream == s && rng->seed != b->h_seed) {
    cudaGraphExecDestroy(b->graph_exec);
    b->graph_exec = nullptr;
  }
  b->h_seed = rng->seed;
  const bool sorted = batch_prepare_order(b, total);
  res_T res = batch_graph(b, rng, s, sorted);
  if(res != RES_OK) return res;
  if(cudaMemcpyAsync(b->d_prefix, b->h_prefix.data(), (n + 1) * sizeof(unsigned long long),
                     cudaMemcpyHostToDevice, s) != cudaSuccess
  || cudaMemcpyAsync(b->d_firsts, b->h_firsts.data(), n * sizeof(unsigned long long),
                     cudaMemcpyHostToDevice, s) != cudaSuccess
  || (sorted && cudaMemcpyAsync(b->d_mul, b->h_mul.data(), n * sizeof(uint32_t),
                                cudaMemcpyHostToDevice, s) != cudaSuccess))
    return RES_UNKNOWN_ERR;
  cudaEventRecord(b->ev0, s);
  if(cudaGraphLaunch(b->graph_exec, s) != cudaSuccess) return RES_UNKNOWN_ERR;
  cudaEventRecord(b->ev1, s);
  /* Host arrays must stay untouched until the copies ran */
  if(cudaStreamSynchronize(s) != cudaSuccess) return RES_UNKNOWN_ERR;
  float ms = 0;
  if(cudaEventElapsedTime(&ms, b->ev0, b->ev1) == cudaSuccess) b->kernel_ms += ms;
  for(size_t i = 0; i < n; ++i) b->done[i] += budgets[i];
  return RES_OK;
}

/* The no-allocation launch (declared in ssol_b200.h): same kernel and
 * results as ssol_b200_batch_launch, without the graph and with the
 * launch's scratch in a static device array (kernels_batch.cu) */
extern "C" res_T ssol_b200_batch_launch_noalloc
  (ssol_b200_batch* b, const ssp_rng* rng, const uint64_t* budgets, void* stream)
{
  if(!b || !rng || !budgets) return RES_BAD_ARG;
  const size_t n = b->scenes.size();
  if(n > (size_t)NOALLOC_MAX_ITEMS) {
    b->dev->log_error("ssol_b200_batch_launch_noalloc: %zu items, at most %d "
                      "fit its static scratch.\n", n, NOALLOC_MAX_ITEMS);
    return RES_BAD_ARG;
  }
  unsigned long long total = 0;
  for(size_t i = 0; i < n; ++i) {
    b->h_prefix[i] = total;
    b->h_firsts[i] = rng->position + b->done[i];
    total += budgets[i];
  }
  b->h_prefix[n] = total;
  if(!total) return RES_OK;
  const cudaStream_t s = stream ? (cudaStream_t)stream : (cudaStream_t)b->dev->stream;
  /* The call copies the budgets from host memory and waits for `stream`
   * before it returns; on a stream that is recording a capture, the wait
   * would end the capture with an error and the copies would read host
   * arrays that later calls overwrite */
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if(cudaStreamIsCapturing(s, &cap) != cudaSuccess
  || cap != cudaStreamCaptureStatusNone) {
    b->dev->log_error("ssol_b200_batch_launch_noalloc: the stream is being "
                      "captured; this call waits for its launch and must be "
                      "made outside a capture.\n");
    return RES_BAD_ARG;
  }
  const LaunchConfig cfg = batch_config(b);
  const int err = b->opt.precision == SSOL_B200_FP32
    ? launch_batch_noalloc_f32((const DScene<float>*)b->d_scenes, b->d_tallies,
                               (int)n, rng->seed, b->h_prefix.data(),
                               b->h_firsts.data(), cfg, s)
    : launch_batch_noalloc_f64((const DScene<double>*)b->d_scenes, b->d_tallies,
                               (int)n, rng->seed, b->h_prefix.data(),
                               b->h_firsts.data(), cfg, s);
  if(err != 0) {
    b->dev->log_error("ssol_b200_batch_launch_noalloc: %s\n",
                      cudaGetErrorString((cudaError_t)err));
    return RES_UNKNOWN_ERR;
  }
  /* The host budget arrays are read by the copies: wait for them */
  if(cudaStreamSynchronize(s) != cudaSuccess) return RES_UNKNOWN_ERR;
  for(size_t i = 0; i < n; ++i) b->done[i] += budgets[i];
  return RES_OK;
}

extern "C" res_T ssol_b200_batch_get_mc_global
  (ssol_b200_batch* b, void* stream, ssol_mc_global* out)
{
  if(!b || !out) return RES_BAD_ARG;
  const cudaStream_t s = stream ? (cudaStream_t)stream : (cudaStream_t)b->dev->stream;
  const size_t n = b->scenes.size();
  std::vector<double> h(13 * n);
  if(launch_gather_globals(b->d_tallies, (int)n, b->d_gather, s) != 0
  || cudaMemcpyAsync(h.data(), b->d_gather, h.size() * sizeof(double),
                     cudaMemcpyDeviceToHost, s) != cudaSuccess
  || cudaStreamSynchronize(s) != cudaSuccess)
    return RES_UNKNOWN_ERR;
  /* As ssol_estimator_get_mc_global on the item's estimator: realisations
   * launched minus failed ones */
  auto mc = [](const double* w, double nr) {
    ssol_mc_result r;
    if(nr <= 0) { r.E = r.V = r.SE = 0; return r; }
    r.E = w[0] / nr;
    r.V = w[1] / nr - r.E * r.E;
    r.V = r.V > 0 ? r.V : 0;
    r.SE = std::sqrt(r.V / nr);
    return r;
  };
  for(size_t i = 0; i < n; ++i) {
    const double* g = h.data() + 13 * i;
    const double failed = std::min(g[12], (double)b->done[i]);
    const double nr = (double)b->done[i] - failed;
    out[i].cos_factor = mc(g + 0, nr);
    out[i].absorbed_by_receivers = mc(g + 2, nr);
    out[i].shadowed = mc(g + 4, nr);
    out[i].missing = mc(g + 6, nr);
    out[i].extinguished_by_atmosphere = mc(g + 8, nr);
    out[i].other_absorbed = mc(g + 10, nr);
  }
  return RES_OK;
}

extern "C" res_T ssol_b200_batch_finish
  (ssol_b200_batch* b, const ssp_rng* rng, const size_t max_failed,
   void* stream, ssol_estimator** out)
{
  if(!b || !rng || !out) return RES_BAD_ARG;
  const cudaStream_t s = stream ? (cudaStream_t)stream : (cudaStream_t)b->dev->stream;
  /* Pinned read-back buffer, kept with the batch */
  if(!b->h_tally && host_alloc(b->dev, &b->h_tally, b->tally_total) != cudaSuccess) {
    b->h_tally = nullptr;
    return RES_MEM_ERR;
  }
  unsigned char* h = static_cast<unsigned char*>(b->h_tally);
  DStats st;
  if(cudaMemcpyAsync(h, b->d_tally, b->tally_total, cudaMemcpyDeviceToHost, s)
     != cudaSuccess
  || cudaMemcpyAsync(&st, b->d_stats, sizeof(DStats), cudaMemcpyDeviceToHost, s)
     != cudaSuccess)
    return RES_UNKNOWN_ERR;
  const cudaError_t err = cudaStreamSynchronize(s);
  if(err != cudaSuccess) {
    b->dev->log_error("device error: %s\n", cudaGetErrorString(err));
    return RES_UNKNOWN_ERR;
  }
  const size_t n = b->scenes.size();
  std::vector<res_T> item_res(n, RES_OK);
  for(size_t i = 0; i < n; ++i) out[i] = nullptr;
  parallel_for(n, [&](size_t i) {
    item_res[i] = make_estimator(b->dev, b->scenes[i], b->meta[i], b->tl[i],
      h + b->tally_off[i], b->done[i], rng, b->done[i], &st, b->kernel_ms,
      b->scene_bytes, max_failed, &out[i]);
  });
  res_T worst = RES_OK;
  for(size_t i = 0; i < n; ++i) {
    if(item_res[i] != RES_OK && item_res[i] != RES_BAD_OP) {
      for(size_t k = 0; k < n; ++k)
        if(out[k]) { ssol_estimator_ref_put(out[k]); out[k] = nullptr; }
      return item_res[i];
    }
    if(item_res[i] == RES_BAD_OP) worst = RES_BAD_OP;
  }
  return worst;
}

/*******************************************************************************
 * ssol_solve
 ******************************************************************************/
extern "C" res_T ssol_solve_ex
  (ssol_scene* scn, const ssp_rng* rng, const size_t n,
   const size_t max_failed, const ssol_path_tracker* tracker,
   const ssol_b200_options* options, ssol_estimator** out)
{
  if(!scn || !rng || !n || !out) return RES_BAD_ARG;
  *out = nullptr;
  if(n > (size_t)INT64_MAX || max_failed > (size_t)INT64_MAX)
    return RES_BAD_ARG;
  /* The default builder by solve size: below the threshold, building the
   * tree on the device saves more (2 ms on the 1000-heliostat field) than
   * its slightly slower traversal costs */
  ssol_b200_options opt = options ? *options : SSOL_B200_OPTIONS_DEFAULT;
  /* The default builder by solve size. Larger solves start on the device's
   * tree and switch to the host SAH tree, built meanwhile on the host
   * threads, after their first 6e6 realisations (the smallest launch that
   * runs in the coherent order, 8.5 ms on the 1000-heliostat field): the
   * host build (2-3 ms there) no longer delays the first launch, and only
   * that first part traces on the slower tree */
  const bool hybrid = opt.bvh_builder == SSOL_B200_BVH_AUTO && !tracker
    && (unsigned long long)n > SSOL_B200_BVH_AUTO_MAX_PATHS;
  if(opt.bvh_builder == SSOL_B200_BVH_AUTO)
    opt.bvh_builder = (unsigned long long)n <= SSOL_B200_BVH_AUTO_MAX_PATHS || hybrid
      ? SSOL_B200_BVH_LBVH : SSOL_B200_BVH_SAH;
  ssol_b200_plan* plan = nullptr;
  res_T res = plan_create_impl(scn, &opt, &plan, hybrid);
  if(res != RES_OK) return res;
  if(!tracker) {
    const unsigned long long mf = (unsigned long long)max_failed;
    if(hybrid && (plan->keep32 || plan->keep64)) {
      const uint64_t n0 = 6000000;
      res = plan_launch(plan, rng, 0, n0, nullptr, nullptr, mf);
      if(res == RES_OK) res = plan_swap_sah(plan);
      if(res == RES_OK) res = plan_launch(plan, rng, n0, n - n0, nullptr, nullptr, mf, true);
    } else {
      res = plan_launch(plan, rng, 0, n, nullptr, nullptr, mf);
    }
    if(res == RES_OK)
      res = ssol_b200_plan_finish(plan, rng, n, max_failed, nullptr, out);
    ssol_b200_plan_ref_put(plan);
    return res;
  }

  /* Path tracking (src/ssol_solver.c:1211-1220, 898-1126): the first
   * min(N, 2^20) realisations record their paths on the device; negative
   * lengths default to 0.75 x the largest extent of the scene's box */
  double ext = 0;
  for(int c = 0; c < 3; ++c)
    ext = std::max(ext, plan->meta.aabb_hi[c] - plan->meta.aabb_lo[c]);
  ext *= 0.75;
  DTrack tr = {};
  tr.npaths = std::min<unsigned long long>(n, 1ull << 20);
  tr.cap = std::min<unsigned long long>(tr.npaths * 16 + 64, 1ull << 22);
  tr.sun_len = tracker->sun_ray_length < 0 ? ext : tracker->sun_ray_length;
  tr.inf_len = tracker->infinite_ray_length < 0 ? ext : tracker->infinite_ray_length;
  const size_t vbytes = (size_t)tr.cap * sizeof(TrackVertex);
  const size_t bytes = vbytes + 256 + (size_t)tr.npaths * 2 * sizeof(int32_t);
  char* d = nullptr;
  if(cudaMalloc((void**)&d, bytes) != cudaSuccess) {
    ssol_b200_plan_ref_put(plan);
    return RES_MEM_ERR;
  }
  tr.verts = reinterpret_cast<TrackVertex*>(d);
  tr.nverts = reinterpret_cast<unsigned long long*>(d + vbytes);
  tr.path_type = reinterpret_cast<int32_t*>(d + vbytes + 256);
  tr.path_nv = tr.path_type + tr.npaths;
  const cudaStream_t s = plan_stream(plan, nullptr);
  if(cudaMemsetAsync(tr.nverts, 0, sizeof(unsigned long long), s) != cudaSuccess
  || cudaMemsetAsync(tr.path_type, 0xff, (size_t)tr.npaths * sizeof(int32_t), s)
       != cudaSuccess)
    res = RES_UNKNOWN_ERR;
  if(res == RES_OK) res = plan_launch(plan, rng, 0, n, s, &tr, (unsigned long long)max_failed);
  if(res == RES_OK) res = ssol_b200_plan_finish(plan, rng, n, max_failed, s, out);
  if(*out) {
    unsigned long long nv = 0;
    std::vector<int32_t> types(tr.npaths), counts(tr.npaths);
    bool ok = cudaMemcpy(&nv, tr.nverts, sizeof(nv), cudaMemcpyDeviceToHost) == cudaSuccess
      && cudaMemcpy(types.data(), tr.path_type, tr.npaths * sizeof(int32_t),
                    cudaMemcpyDeviceToHost) == cudaSuccess
      && cudaMemcpy(counts.data(), tr.path_nv, tr.npaths * sizeof(int32_t),
                    cudaMemcpyDeviceToHost) == cudaSuccess;
    std::vector<TrackVertex> hv(ok ? (size_t)std::min(nv, tr.cap) : 0);
    ok = ok && (hv.empty() || cudaMemcpy(hv.data(), tr.verts, hv.size() * sizeof(TrackVertex),
                                         cudaMemcpyDeviceToHost) == cudaSuccess);
    if(!ok) {
      res = RES_UNKNOWN_ERR;
    } else {
      std::vector<TrackedPath> paths(tr.npaths);
      std::vector<int32_t> got(tr.npaths, 0);
      for(size_t k = 0; k < tr.npaths; ++k)
        if(types[k] >= 0) paths[k].vertices.resize((size_t)counts[k]);
      for(const TrackVertex& v : hv) {
        if(v.slot >= tr.npaths || types[v.slot] < 0 || (int32_t)v.seq >= counts[v.slot])
          continue;
        ssol_path_vertex& pv = paths[v.slot].vertices[v.seq];
        pv.pos[0] = v.pos[0]; pv.pos[1] = v.pos[1]; pv.pos[2] = v.pos[2];
        pv.weight = v.weight;
        ++got[v.slot];
      }
      size_t dropped = 0;
      for(size_t k = 0; k < tr.npaths; ++k) {
        if(types[k] < 0) continue;
        if(got[k] != counts[k]) { ++dropped; continue; }
        paths[k].type = (ssol_path_type)types[k];
        (*out)->paths.push_back(std::move(paths[k]));
      }
      if(dropped)
        scn->dev->log_warning("path tracking: %zu paths dropped, the vertex buffer "
                              "holds %llu vertices.\n", dropped, tr.cap);
    }
  }
  cudaFree(d);
  ssol_b200_plan_ref_put(plan);
  return res;
}

extern "C" res_T ssol_solve
  (ssol_scene* scn, const ssp_rng* rng, const size_t n,
   const size_t max_failed, const ssol_path_tracker* tracker,
   ssol_estimator** out)
{
  return ssol_solve_ex(scn, rng, n, max_failed, tracker, nullptr, out);
}

extern "C" res_T ssol_estimator_get_b200_stats
  (const ssol_estimator* e, ssol_b200_stats* s)
{
  if(!e || !s) return RES_BAD_ARG;
  std::memset(s, 0, sizeof(*s));
  s->kernel_ms = e->kernel_ms;
  s->rays = e->stats[0];
  s->node_visits = e->stats[1];
  s->triangle_tests = e->stats[2];
  s->quadric_tests = e->stats[3];
  s->bounces = e->stats[4];
  s->paths = e->stats[5];
  s->killed = e->killed;
  s->scene_bytes = e->scene_bytes;
  s->tally_bytes = e->tally_bytes;
  s->bvh_nodes = e->bvh_nodes;
  s->bvh_depth = e->bvh_depth;
  s->bvh_device = e->bvh_device;
  return RES_OK;
}
