// C ABI of edgeMap / vertexMap / vertexFilter with the built-in functors, and
// the applications' Compute() loops (app/*.C) run on the device.
#include <algorithm>
#include <cmath>
#include <vector>

#include "gg_runtime.cuh"

namespace gg {

// ------------------------------------------------------------- helpers
template <class T>
__global__ void k_fill(T* a, uint64_t n, T v) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    a[i] = v;
}

template <class T>
static int fill(gg_graph_s* g, T* a, uint64_t n, T v) {
  k_fill<T><<<generic_grid(g, n), kGenericThreads, 0, g->stream>>>(a, n, v);
  GG_CUDA(cudaGetLastError());
  g->kernels++;
  return GG_OK;
}

template <class T>
static int set_one(gg_graph_s* g, T* a, uint32_t i, T v) {
  return write_small(g, a + i, v);
}

struct FrontierHold {
  gg_frontier_s* f = nullptr;
  ~FrontierHold() { frontier_free(f); }
  void reset(gg_frontier_s* x) {
    frontier_free(f);
    f = x;
  }
  gg_frontier_s* release() {
    gg_frontier_s* x = f;
    f = nullptr;
    return x;
  }
};

// Runs of dense COO rounds of BellmanFord, Components and PageRankDelta as
// one CUDA graph (defined with the PageRank graph below).
enum { kRoundLoopBf = 0, kRoundLoopCc = 1, kRoundLoopPrd = 2 };
static RoundLoop* round_loop_get(gg_graph_s* g, int app);
static void* round_loop_array(RoundLoop* L, int i);
static bool round_takes_coo(const gg_graph_s* g, const gg_frontier_s* f);
static int round_loop_run(gg_graph_s* g, RoundLoop* L, FrontierHold& F, uint32_t max_rounds, int64_t* round,
                          uint64_t* trav, double eps = 0, double* l1 = nullptr);

// contrib[s] = val[s] / outdeg(s)   (0 for out-degree 0, never gathered)
__global__ void k_div_outdeg(uint32_t n, const float* val, const uint32_t* off, float* contrib) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t d = off[i + 1] - off[i];
    contrib[i] = d ? val[i] / (float)d : 0.0f;
  }
}

__device__ __forceinline__ void block_add_double(double v, double* out) {
  __shared__ double s[32];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double x = threadIdx.x < (blockDim.x >> 5) ? s[threadIdx.x] : 0.0;
    x = warp_sum(x);
    if (threadIdx.x == 0 && x != 0.0) atomicAdd(out, x);
  }
}

// PageRank iteration epilogue (app/PageRank.C:133-142), fused:
//   vertexMap(F, PR_Vertex_F)            p_next[i] = d*p_next[i] + (1-d)/n, i in F
//   p_curr[j] = |p_curr[j] - p_next[j]|  for every j, L1 = sum
//   vertexMap(F, PR_Vertex_Reset)        p_curr[i] = 0, i in F
// plus the next iteration's contrib[j] = p_next[j]/outdeg(j).  When the next
// frontier's bitmap is given, sources outside it get -1 (contributions are
// > 0), so the next pull reads membership from the gathered value itself.
__device__ __forceinline__ float pr_vertex(bool in, float pc, float& pn, uint32_t d, bool next_in, float damping,
                                           float added, float& contrib, float& pc_out) {
  if (in) pn = damping * pn + added;
  const float diff = fabsf(pc - pn);
  pc_out = in ? 0.0f : diff;
  contrib = d ? (next_in ? pn / (float)d : -1.0f) : 0.0f;
  return diff;
}

// PageRank round epilogue, four vertices per thread with 16-byte accesses:
// for frontier members p_next = damping * p_next + (1-damping)/n (PR_Vertex_F,
// app/PageRank.C:84-100), L1 += |p_curr - p_next|, p_curr reset, and the next
// iteration's contributions p_next/outdeg (-1 for sources outside the next
// frontier when the frontier is carried in the values).
__global__ void k_pr_epilogue(uint32_t n, int all, const uint32_t* fbits, float* p_curr, float* p_next,
                              const uint32_t* off, float damping, float added, float* contrib, double* l1,
                              const uint32_t* next_bits) {
  double acc = 0;
  const uint64_t n4 = n / 4;
  for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t j = 4 * q;
    const float4 pc = reinterpret_cast<const float4*>(p_curr)[q];
    float4 pn = reinterpret_cast<const float4*>(p_next)[q];
    const uint32_t o0 = off[j], o1 = off[j + 1], o2 = off[j + 2], o3 = off[j + 3], o4 = off[j + 4];
    const uint32_t fw = all ? 0xfu : (fbits[j >> 5] >> (j & 31)) & 0xfu;
    const uint32_t nw = next_bits ? (next_bits[j >> 5] >> (j & 31)) & 0xfu : 0xfu;
    float4 c, po;
    acc += pr_vertex(fw & 1u, pc.x, pn.x, o1 - o0, nw & 1u, damping, added, c.x, po.x);
    acc += pr_vertex(fw & 2u, pc.y, pn.y, o2 - o1, nw & 2u, damping, added, c.y, po.y);
    acc += pr_vertex(fw & 4u, pc.z, pn.z, o3 - o2, nw & 4u, damping, added, c.z, po.z);
    acc += pr_vertex(fw & 8u, pc.w, pn.w, o4 - o3, nw & 8u, damping, added, c.w, po.w);
    reinterpret_cast<float4*>(p_next)[q] = pn;
    reinterpret_cast<float4*>(p_curr)[q] = po;
    reinterpret_cast<float4*>(contrib)[q] = c;
  }
  for (uint64_t j = 4 * n4 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
       j += (uint64_t)gridDim.x * blockDim.x) {
    float pn = p_next[j], c, po;
    acc += pr_vertex(all || test_bit(fbits, (uint32_t)j), p_curr[j], pn, off[j + 1] - off[j],
                     !next_bits || test_bit(next_bits, (uint32_t)j), damping, added, c, po);
    p_next[j] = pn;
    p_curr[j] = po;
    contrib[j] = c;
  }
  block_add_double(acc, l1);
}

// PageRankDelta round epilogue (app/PageRankDelta.C:158-165): L1 = sum|Delta|,
// nghSum reset to 0, next round's contrib = Delta/outdeg.
__global__ void k_prd_epilogue(uint32_t n, const float* delta, float* ngh, const uint32_t* off, float* contrib,
                               double* l1) {
  double acc = 0;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
    const float dl = delta[j];
    acc += fabsf(dl);
    ngh[j] = 0.0f;
    const uint32_t d = off[j + 1] - off[j];
    contrib[j] = d ? dl / (float)d : 0.0f;
  }
  block_add_double(acc, l1);
}

__global__ void k_invert(uint32_t n, float* a) {
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x)
    a[j] = 1.0f / a[j];
}
__global__ void k_bc_final(uint32_t n, float* dep, const float* inv) {
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x)
    dep[j] = (dep[j] - inv[j]) / inv[j];
}

static int read_red(gg_graph_s* g, double* v) { return read_small(g, v, g->ws.d_red); }

static void fill_stats(gg_run_stats* st, double ms, int rounds, uint64_t trav, int kernels) {
  if (!st) return;
  st->ms = ms;
  st->rounds = rounds;
  st->edges_traversed = trav;
  st->kernels = kernels;
}

template <class T>
static int to_host(gg_graph_s* g, T* host, const T* dev, uint64_t n) {
  if (!host) return GG_OK;
  // asynchronous results: a result staged in a given-order array leaves on
  // the copy stream into pinned memory, and the call does not wait for it
  int slot = -1;
  for (int k = 0; k < 3; ++k)
    if (g->ws.d_order[k] && reinterpret_cast<const void*>(dev) == g->ws.d_order[k]) slot = k;
  cudaPointerAttributes pa{};
  if (g->async_results && slot >= 0 && cudaPointerGetAttributes(&pa, host) == cudaSuccess &&
      pa.type == cudaMemoryTypeHost) {
    GG_CUDA(cudaEventRecord(g->result_ready, g->stream));
    GG_CUDA(cudaStreamWaitEvent(g->copy_stream, g->result_ready, 0));
    GG_CUDA(cudaMemcpyAsync(host, dev, sizeof(T) * n, cudaMemcpyDeviceToHost, g->copy_stream));
    GG_CUDA(cudaEventRecord(g->slot_copied[slot], g->copy_stream));
    return GG_OK;
  }
  cudaGetLastError();  // a pageable pointer is not an error
  GG_CUDA(cudaMemcpyAsync(host, dev, sizeof(T) * n, cudaMemcpyDeviceToHost, g->stream));
  GG_CUDA(cudaStreamSynchronize(g->stream));
  return GG_OK;
}

// ================================================================== apps
// app/BFS.C:77-101
static int run_bfs(gg_graph_s* g, uint32_t start, int32_t* parents, int32_t* levels, gg_run_stats* st) {
  const uint32_t n = g->n;
  g->kernels = 0;
  DevBuf<int32_t> par, lev;
  // every level in one cooperative launch (its dense levels pull over the CSC;
  // a graph told to pull over the COO keeps the host loop for them), which
  // writes levels only when they are asked for
  const bool full = g->device_loop == 2 && !g->transposed && g->dense_policy != 2;
  const bool want_lev = levels || !full;
  GG_TRY(par.alloc(g, n));
  if (want_lev) GG_TRY(lev.alloc(g, n));
  EventTimer tm(g->stream);
  GG_TRY(fill<int32_t>(g, par.p, n, -1));
  GG_TRY(set_one<int32_t>(g, par.p, start, (int32_t)start));
  if (want_lev) {
    GG_TRY(fill<int32_t>(g, lev.p, n, -1));
    GG_TRY(set_one<int32_t>(g, lev.p, start, 0));
  }
  FrontierHold F;
  int32_t round = 0;
  uint64_t trav = 0;
  const int64_t thr = app_threshold(g);
  if (full)
    GG_TRY(bfs_device_full(g, start, par.p, lev.p, (uint64_t)thr));
  else
    GG_TRY(gg_frontier_single(g, start, &F.f));
  while (F.f && F.f->dm > 0) {
    if (g->device_loop && (int64_t)(F.f->dm + F.f->out_edges) <= thr && F.f->out_edges > 0) {
      // sparse levels run on the device until the frontier empties or turns dense
      int32_t levels_run = 0;
      uint64_t t = 0;
      gg_frontier_s* cur = F.release();
      const int rc = bfs_device_levels(g, &cur, par.p, lev.p, round + 1, (uint64_t)thr, &levels_run, &t);
      F.f = cur;
      if (rc) return rc;
      round += levels_run;
      trav += t;
      continue;
    }
    ++round;
    BfsF f;
    f.parents = par.p;
    f.levels = lev.p;
    f.round = round;
    trav += F.f->out_edges;
    gg_frontier_s* out = nullptr;
    GG_TRY(edge_map(g, F.f, f, thr, 0, &out));
    F.reset(out);
  }
  const int32_t* par_out = par.p;
  const int32_t* lev_out = lev.p;
  const int pslot = g->async_results && g->ws.d_order[2] ? 2 : 0;  // the given-order array of the parents
  if (g->relabeled && parents) {
    int32_t* tp = reinterpret_cast<int32_t*>(g->ws.d_order[pslot]);
    GG_TRY(slot_write_wait(g, pslot));
    k_ids_to_given<<<generic_grid(g, n), kGenericThreads, 0, g->stream>>>(n, g->d_new_of_old, g->d_old_of_new,
                                                                          par.p, tp);
    g->kernels++;
    par_out = tp;
  }
  if (parents && !g->relabeled) GG_TRY(given_order<int32_t>(g, par.p, pslot, &par_out));
  if (levels) GG_TRY(given_order<int32_t>(g, lev.p, 1, &lev_out));
  const double ms = tm.stop();
  // the all-levels launch is read back after the device work it feeds was
  // queued behind it, so that the stream does not idle for the host
  if (full) GG_TRY(bfs_device_full_result(g, &round, &trav));
  GG_TRY(to_host(g, parents, par_out, n));
  GG_TRY(to_host(g, levels, lev_out, n));
  fill_stats(st, ms, round, trav, g->kernels);
  return GG_OK;
}

// ------------------------------------------------ union-find components
// On a symmetric graph the fixed point of app/Components.C's label
// propagation is the smallest id of each connected component.  Union-find
// reaches it in one pass over the edges: every parent pointer goes to a
// smaller id, so a tree's root is its smallest vertex, and hooking always
// puts the larger of two roots under the smaller one (a CAS on the root's
// own pointer; a failed CAS continues from the root's new parent).
__device__ __forceinline__ uint32_t uf_find(uint32_t* par, uint32_t v) {
  uint32_t cur = __ldcg(par + v);
  if (cur == v) return v;
  uint32_t prev = v;
  for (;;) {
    const uint32_t next = __ldcg(par + cur);
    if (next == cur) return cur;
    par[prev] = next;  // path halving: any ancestor is a valid parent
    prev = cur;
    cur = next;
  }
}

__global__ void k_uf_init(uint32_t n, uint32_t* par, uint32_t* minid) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    par[v] = (uint32_t)v;
    if (minid) minid[v] = 0xffffffffu;
  }
}

__device__ __forceinline__ void uf_union(uint32_t* par, uint32_t u, uint32_t v) {
  uint32_t ru = uf_find(par, u), rv = uf_find(par, v);
  while (ru != rv) {
    if (ru < rv) {
      const uint32_t t = ru;
      ru = rv;
      rv = t;
    }
    const uint32_t old = atomicCAS(par + ru, ru, rv);  // hook the larger root under the smaller
    if (old == ru) break;
    ru = uf_find(par, old);
    rv = uf_find(par, rv);
  }
}

constexpr uint32_t kUfSmallDegree = 32;

// Each undirected edge is taken once, from its larger end.  One thread per
// vertex of degree <= 32; larger vertices are listed for k_uf_hook_big.
__global__ void k_uf_hook_small(uint32_t n, const uint32_t* off, const uint32_t* idx, uint32_t* par, uint32_t* big,
                                uint32_t* nbig) {
  for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t u = (uint32_t)x, e0 = off[u], e1 = off[u + 1];
    if (e1 - e0 > kUfSmallDegree) {
      big[atomicAdd(nbig, 1u)] = u;
      continue;
    }
    for (uint32_t e = e0; e < e1; ++e) {
      const uint32_t v = idx[e];
      if (v < u) uf_union(par, u, v);
    }
  }
}

// One warp per listed vertex, lanes over its edges.
__global__ void k_uf_hook_big(const uint32_t* big, const uint32_t* nbig, const uint32_t* off, const uint32_t* idx,
                              uint32_t* par) {
  const int lane = threadIdx.x & 31;
  const uint64_t w0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t cnt = *nbig;
  for (uint64_t i = w0; i < cnt; i += nw) {
    const uint32_t u = big[i];
    for (uint32_t e = off[u] + lane; e < off[u + 1]; e += 32) {
      const uint32_t v = idx[e];
      if (v < u) uf_union(par, u, v);
    }
  }
}

// minid[root] = the smallest given id of the root's component (renumbered graphs).
__global__ void k_uf_min_given(uint32_t n, uint32_t* par, const uint32_t* old_of_new, uint32_t* minid) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
    atomicMin(minid + uf_find(par, (uint32_t)v), old_of_new[v]);
}

__global__ void k_uf_label(uint32_t n, uint32_t* par, const uint32_t* minid, int32_t* ids) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t r = uf_find(par, (uint32_t)v);
    ids[v] = (int32_t)(minid ? minid[r] : r);
  }
}

static int run_cc_union_find(gg_graph_s* g, int32_t* ids_out, gg_run_stats* st) {
  const uint32_t n = g->n;
  g->kernels = 0;
  DevBuf<uint32_t> par, minid, big;
  DevBuf<int32_t> ids;
  GG_TRY(par.alloc(g, n));
  GG_TRY(ids.alloc(g, n));
  GG_TRY(big.alloc(g, n));  // n + 4 entries: the list, then its length at [n]
  if (g->relabeled) GG_TRY(minid.alloc(g, n));
  EventTimer tm(g->stream);
  const int grid = generic_grid(g, n);
  k_uf_init<<<grid, kGenericThreads, 0, g->stream>>>(n, par.p, g->relabeled ? minid.p : nullptr);
  g->kernels++;
  if (g->m) {
    uint32_t* nbig = big.p + n;
    GG_CUDA(cudaMemsetAsync(nbig, 0, sizeof(uint32_t), g->stream));
    k_uf_hook_small<<<grid, kGenericThreads, 0, g->stream>>>(n, g->out_off(), g->out_idx(), par.p, big.p, nbig);
    k_uf_hook_big<<<(int)g->num_sms * 8, kGenericThreads, 0, g->stream>>>(big.p, nbig, g->out_off(), g->out_idx(),
                                                                           par.p);
    g->kernels += 2;
  }
  if (g->relabeled) {
    k_uf_min_given<<<grid, kGenericThreads, 0, g->stream>>>(n, par.p, g->d_old_of_new, minid.p);
    g->kernels++;
  }
  k_uf_label<<<grid, kGenericThreads, 0, g->stream>>>(n, par.p, g->relabeled ? minid.p : nullptr, ids.p);
  g->kernels++;
  GG_CUDA(cudaGetLastError());
  const int32_t* res = ids.p;
  GG_TRY(given_order<int32_t>(g, ids.p, 0, &res));
  const double ms = tm.stop();
  GG_TRY(to_host(g, ids_out, res, n));
  fill_stats(st, ms, 1, g->m, g->kernels);
  return GG_OK;
}

// app/Components.C:101-126
static int run_cc(gg_graph_s* g, int32_t* ids_out, gg_run_stats* st) {
  if (g->cc_algo == 1 && g->symmetric) return run_cc_union_find(g, ids_out, st);
  const uint32_t n = g->n;
  RoundLoop* L = round_loop_get(g, kRoundLoopCc);  // its arrays, when its graph runs the dense rounds
  g->kernels = 0;
  DevBuf<int32_t> idsb, prevb;
  int32_t *ids = nullptr, *prev = nullptr;
  if (L) {
    ids = static_cast<int32_t*>(round_loop_array(L, 0));
    prev = static_cast<int32_t*>(round_loop_array(L, 1));
  } else {
    GG_TRY(idsb.alloc(g, n));
    GG_TRY(prevb.alloc(g, n));
    ids = idsb.p;
    prev = prevb.p;
  }
  EventTimer tm(g->stream);
  // IDs[i] = i (app/Components.C:112): the given id, also on a renumbered graph
  if (g->relabeled)
    GG_CUDA(cudaMemcpyAsync(ids, g->d_old_of_new, 4ull * n, cudaMemcpyDeviceToDevice, g->stream));
  else
    k_iota<<<generic_grid(g, n), kGenericThreads, 0, g->stream>>>((uint32_t*)ids, n);
  FrontierHold F;
  GG_TRY(gg_frontier_all(g, &F.f));
  int64_t rounds = 0;
  uint64_t trav = 0;
  while (F.f->dm > 0) {
    if (L && round_takes_coo(g, F.f)) {  // dense COO rounds on the device
      GG_TRY(round_loop_run(g, L, F, n, &rounds, &trav));  // labels only fall: at most n rounds
      continue;
    }
    VCcCopy vc{ids, prev};
    GG_TRY(vertex_map(g, F.f, vc));
    CcF f;
    f.ids = ids;
    f.prev = prev;
    // A vertex outside the frontier has prevIDs == IDs, unchanged since the
    // round it last was in the frontier, when every out-neighbour took a
    // label <= it; so its value cannot lower any destination, and the dense
    // pull may gather every source without testing the frontier bitmap
    // (same labels, outputs and rounds).
    f.outside_inert = true;
    trav += F.f->out_edges;
    gg_frontier_s* out = nullptr;
    GG_TRY(edge_map(g, F.f, f, app_threshold(g), 0, &out));
    F.reset(out);
    ++rounds;
  }
  const int32_t* ids_res = ids;
  GG_TRY(given_order<int32_t>(g, ids, 0, &ids_res));
  const double ms = tm.stop();
  GG_TRY(to_host(g, ids_out, ids_res, n));
  fill_stats(st, ms, (int)rounds, trav, g->kernels);
  return GG_OK;
}

// ---------------------------------------------- PageRank as a CUDA graph
// The iteration loop of app/PageRank.C:129-146 captured once per graph handle
// and knob setting, then replayed per call.  The top graph holds the
// initialisation and the first iteration, then a while node whose body runs
// the next iteration with the rank buffers one way round and, under an if
// node, the one after with them the other way round, so that the swap needs
// no host work.  After every iteration a one-thread check kernel decides on
// the device what the host loop decides after its read-back: stop when
// L1 < eps (:371) or after max_iter iterations, and hand the loop back to
// the host when the next edgeMap would not take the dense COO pull that the
// graph holds (ligra-numa.h:953-960 evaluated on the output's count and
// out-degree sum).  One read-back per call replaces two per iteration.
struct PrLoopCtl {
  unsigned long long trav;       // out-degree sums of the input frontiers so far
  unsigned long long dm;         // last output frontier: active vertices
  unsigned long long out_edges;  //   and their out-degree sum
  unsigned long long in_dm;      // input frontier of the last iteration
  unsigned long long in_edges;
  unsigned long long err;        // device error word seen by a check
  double l1;                     // L1 of the last iteration
  double eps;
  long long threshold;           // edgeMap's threshold (m / div)
  long long dense_threshold;     // m / 2
  uint32_t count;                // iterations done
  uint32_t max_iter;
  uint32_t reason;               // 0 running, 1 converged, 2 max_iter, 3 handed back, 4 device error
  uint32_t coo_always;           // the dense policy pins the COO pull (else the m/2 rule)
};

struct PrLoop {
  float* buf[4] = {nullptr, nullptr, nullptr, nullptr};  // ranks (two) and contributions (two), n + 4 each
  uint32_t* bits[2] = {nullptr, nullptr};       // output bitmaps of odd / even iterations
  PrLoopCtl* d_ctl = nullptr;
  PrLoopCtl* h_ctl = nullptr;  // pinned
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int key[3] = {-1, -1, -1};   // bit_all, COO kernel, transposed of the captured graph
  uint64_t bytes = 0;
};

void pr_loop_free(gg_graph_s* g) {
  PrLoop* L = g->pr_loop;
  if (!L) return;
  if (L->exec) cudaGraphExecDestroy(L->exec);
  if (L->graph) cudaGraphDestroy(L->graph);
  for (float* b : L->buf) cudaFree(b);
  for (uint32_t* b : L->bits) cudaFree(b);
  cudaFree(L->d_ctl);
  if (L->h_ctl) cudaFreeHost(L->h_ctl);
  g->device_bytes -= L->bytes;
  delete L;
  g->pr_loop = nullptr;
}

// The graph's first pass: ranks 1/n, accumulators 0, first contributions
// (k_div_outdeg's quotient) and the first output bitmap cleared.
__global__ void k_pr_loop_init(uint32_t n, float* p, float* acc, const uint32_t* off, float* contrib, uint32_t* bits,
                               uint32_t words) {
  const float p0 = (float)(1 / (double)n);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint32_t d = off[i + 1] - off[i];
    p[i] = p0;
    acc[i] = 0.0f;
    contrib[i] = d ? p0 / (float)d : 0.0f;
  }
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += stride) bits[i] = 0;
}

// After iteration i: thread 0 decides (below); every thread clears the
// iteration's input bitmap, read by nothing after its pull and uncovered-range
// pass, which the next iteration writes as its output.
__global__ void k_pr_loop_check(PrLoopCtl* c, unsigned long long* stats, double* red, cudaGraphConditionalHandle h_loop,
                                cudaGraphConditionalHandle h_odd, int set_odd, uint32_t* clear_bits,
                                uint32_t clear_words) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < clear_words;
       i += (uint64_t)gridDim.x * blockDim.x)
    clear_bits[i] = 0;
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const double l1 = red[0];
  const unsigned long long dm = stats[0], oe = stats[1], err = stats[3];
  red[0] = 0;  // the next epilogue's L1 and the next pull's counters start from zero
  for (int i = 0; i < 8; ++i) stats[i] = 0;
  const uint32_t count = c->count + 1;
  c->count = count;
  c->l1 = l1;
  c->dm = dm;
  c->out_edges = oe;
  uint32_t reason = 0;
  if (err) {
    c->err = err;
    reason = 4;
  } else if (l1 < c->eps) {
    reason = 1;
  } else if (count >= c->max_iter) {
    reason = 2;
  } else {
    const long long fm = (long long)dm, tot = (long long)oe;
    const bool pull = tot > 0 && fm + tot > c->threshold && (c->coo_always || fm + tot > c->dense_threshold);
    if (pull) {
      c->trav += oe;
      c->in_dm = dm;
      c->in_edges = oe;
    } else {
      reason = 3;
    }
  }
  c->reason = reason;
  cudaGraphSetConditional(h_loop, reason == 0 ? 1u : 0u);
  if (set_odd) cudaGraphSetConditional(h_odd, reason == 0 ? 1u : 0u);
}

// The per-warp COO pull applies PrFinishF's vertex step at its commits (the
// CTA-ring and source-partition kernels commit with PrT's sum alone).
static bool pr_fused(const gg_graph_s* g) { return g->coo_kernel > 0 && !g->coo_by_source; }

static PrFinishF pr_functor(gg_graph_s* g, const float* contrib, float* contrib_next, float* p_curr, float* p_next,
                            const uint32_t* fbits, bool frontier_in_values, bool masked) {
  PrFinishF f;
  f.contrib = contrib;
  f.acc_out = p_next;
  f.frontier_in_values = frontier_in_values;
  f.p_prev = p_curr;
  f.fbits = fbits;
  f.contrib_next = contrib_next;
  f.l1 = g->ws.d_red;
  f.damping = 0.85f;
  f.added = (float)((1 - 0.85) * (1 / (double)g->n));
  f.masked = masked ? 1 : 0;
  return f;
}

// The vertex step for the destination ranges no COO tile covers (no in-edges).
__global__ void k_pr_finish_gaps(const uint2* gaps, uint32_t ngaps, const PrFinishF f, const uint32_t* off) {
  double acc = 0;
  for (uint32_t r = blockIdx.x; r < ngaps; r += gridDim.x) {
    const uint2 gr = gaps[r];
    for (uint32_t v = gr.x + threadIdx.x; v < gr.x + gr.y; v += blockDim.x)
      acc += f.finish(v, false, 0.0f, off[v + 1] - off[v]);
  }
  block_add_double(acc, f.l1);
}

static int pr_finish_gaps(gg_graph_s* g, const PrFinishF& f) {
  if (!g->coo_gap_count) return GG_OK;
  const int grid = (int)std::min<uint32_t>(g->coo_gap_count, (uint32_t)g->num_sms * 4);
  k_pr_finish_gaps<<<grid, kGenericThreads, 0, g->stream>>>(g->d_coo_gaps, g->coo_gap_count, f, g->out_off());
  GG_CUDA(cudaGetLastError());
  g->kernels++;
  return GG_OK;
}

// One PageRank iteration's launches (the COO pull, as edgeMap picks it for a
// dense frontier, with the vertex step at its commits or as the epilogue)
// into buffers of the loop.
static int pr_iteration(gg_graph_s* g, bool first, bool bit_all, float* p_curr, float* p_next, const float* contrib,
                        float* contrib_next, uint32_t* in_bits, uint32_t* out_bits) {
  const uint32_t n = g->n;  // out_bits arrives cleared (initial pass, or the previous check)
  gg_frontier_s in{}, out{};
  in.g = out.g = g;
  in.n = out.n = n;
  in.bit = first || bit_all;  // the first input is all vertices; PageRankBit keeps output.bit set
  in.has_dense = !in.bit;
  in.d_bits = in_bits;
  out.d_bits = out_bits;
  const bool masked = !bit_all;  // the dense output marks the next contributions
  const PrFinishF f = pr_functor(g, contrib, contrib_next, p_curr, p_next, in.bit ? nullptr : in_bits,
                                 !first && masked, masked);
  GG_TRY((pull_launch<PrFinishF, false>(g, &in, &out, f, true, false)));
  if (pr_fused(g)) return pr_finish_gaps(g, f);
  k_pr_epilogue<<<generic_grid(g, n), kGenericThreads, 0, g->stream>>>(
      n, in.bit ? 1 : 0, in_bits, p_curr, p_next, g->out_off(), f.damping, f.added, contrib_next, g->ws.d_red,
      masked ? out_bits : nullptr);
  GG_CUDA(cudaGetLastError());
  return GG_OK;
}

// Captures the launches of fn into graph (after nothing) and returns the last
// captured node.
template <class Fn>
static int capture_into(gg_graph_s* g, cudaGraph_t graph, Fn fn, cudaGraphNode_t* last) {
  cudaStream_t s = g->stream;
  GG_CUDA(cudaStreamBeginCaptureToGraph(s, graph, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  int rc = fn();
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  if (!rc) {
    if (cudaStreamGetCaptureInfo(s, &cs, nullptr, nullptr, &deps, &nd) != cudaSuccess || nd != 1)
      rc = fail(GG_ERR_CUDA, "PageRank graph: capture did not end in one node");
    else
      *last = deps[0];
  }
  cudaGraph_t out = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s, &out);
  if (!rc && e != cudaSuccess) rc = fail(GG_ERR_CUDA, "PageRank graph: capture failed (%s)", cudaGetErrorString(e));
  return rc;
}

static int add_conditional(cudaGraph_t graph, cudaGraphNode_t dep, cudaGraphConditionalHandle h,
                           cudaGraphConditionalNodeType type, cudaGraph_t* body) {
  cudaGraphNodeParams np{};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = type;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  GG_CUDA(cudaGraphAddNode(&node, graph, dep ? &dep : nullptr, dep ? 1 : 0, &np));
  *body = np.conditional.phGraph_out[0];
  return GG_OK;
}

static int pr_loop_capture(gg_graph_s* g, PrLoop* L, bool bit_all) {
  const uint32_t n = g->n;
  cudaGraph_t graph = nullptr;
  GG_CUDA(cudaGraphCreate(&graph, 0));
  float *A = L->buf[0], *B = L->buf[1], *C0 = L->buf[2], *C1 = L->buf[3];
  uint32_t *X = L->bits[0], *Y = L->bits[1];
  cudaGraphConditionalHandle h_loop = 0, h_odd = 0;
  cudaGraph_t body = nullptr, odd = nullptr;
  cudaGraphNode_t last = nullptr;
  const uint32_t words = g->words() + 4;
  auto check = [&](int set_odd, uint32_t* in_bits) -> int {
    k_pr_loop_check<<<generic_grid(g, words), kGenericThreads, 0, g->stream>>>(
        L->d_ctl, g->ws.d_stats, g->ws.d_red, h_loop, h_odd, set_odd, in_bits, words);
    GG_CUDA(cudaGetLastError());
    return GG_OK;
  };
  int rc = cudaGraphConditionalHandleCreate(&h_loop, graph, 0, cudaGraphCondAssignDefault) == cudaSuccess
               ? GG_OK
               : fail(GG_ERR_CUDA, "PageRank graph: no conditional handle");
  // initialisation and iteration 1 (ranks into B, output bits into X)
  if (!rc)
    rc = capture_into(g, graph, [&]() -> int {
      GG_CUDA(cudaMemsetAsync(g->ws.d_stats, 0, sizeof(unsigned long long) * 8, g->stream));
      GG_CUDA(cudaMemsetAsync(g->ws.d_red, 0, sizeof(double), g->stream));
      k_pr_loop_init<<<generic_grid(g, n), kGenericThreads, 0, g->stream>>>(n, A, B, g->out_off(), C0, X, words);
      GG_CUDA(cudaGetLastError());
      GG_TRY(pr_iteration(g, true, bit_all, A, B, C0, C1, Y, X));
      return check(0, Y);
    }, &last);
  if (!rc) rc = add_conditional(graph, last, h_loop, cudaGraphCondTypeWhile, &body);
  if (!rc && cudaGraphConditionalHandleCreate(&h_odd, body, 0, cudaGraphCondAssignDefault) != cudaSuccess)
    rc = fail(GG_ERR_CUDA, "PageRank graph: no conditional handle");
  // even iterations: ranks into A, contributions into C0, output bits into Y
  if (!rc)
    rc = capture_into(g, body, [&]() -> int {
      GG_TRY(pr_iteration(g, false, bit_all, B, A, C1, C0, X, Y));
      return check(1, X);
    }, &last);
  if (!rc) rc = add_conditional(body, last, h_odd, cudaGraphCondTypeIf, &odd);
  // odd iterations: ranks into B, contributions into C1, output bits into X
  if (!rc)
    rc = capture_into(g, odd, [&]() -> int {
      GG_TRY(pr_iteration(g, false, bit_all, A, B, C0, C1, Y, X));
      return check(0, Y);
    }, &last);
  cudaGraphExec_t exec = nullptr;
  if (!rc && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess)
    rc = fail(GG_ERR_CUDA, "PageRank graph: instantiation refused");
  if (rc) {
    cudaGetLastError();
    cudaGraphDestroy(graph);
    return rc;
  }
  if (L->exec) cudaGraphExecDestroy(L->exec);
  if (L->graph) cudaGraphDestroy(L->graph);
  L->graph = graph;
  L->exec = exec;
  return GG_OK;
}

// The loop of this graph handle for bit_all, captured (again) when a knob it
// depends on changed since.
static int pr_loop_get(gg_graph_s* g, bool bit_all, PrLoop** out) {
  if (!g->pr_loop) {
    PrLoop* L = new (std::nothrow) PrLoop;
    if (!L) return fail(GG_ERR_OOM, "PageRank graph: out of host memory");
    g->pr_loop = L;
    const uint64_t fb = 4ull * ((uint64_t)g->n + 4), bb = 4ull * ((uint64_t)g->words() + 4);
    int rc = GG_OK;
    for (float*& b : L->buf)
      if (!rc && cudaMalloc((void**)&b, fb) != cudaSuccess) rc = fail(GG_ERR_OOM, "PageRank graph: buffers");
    for (uint32_t*& b : L->bits)
      if (!rc && cudaMalloc((void**)&b, bb) != cudaSuccess) rc = fail(GG_ERR_OOM, "PageRank graph: bitmaps");
    if (!rc && cudaMalloc((void**)&L->d_ctl, sizeof(PrLoopCtl)) != cudaSuccess)
      rc = fail(GG_ERR_OOM, "PageRank graph: control block");
    if (!rc && cudaMallocHost((void**)&L->h_ctl, sizeof(PrLoopCtl)) != cudaSuccess)
      rc = fail(GG_ERR_OOM, "PageRank graph: pinned control block");
    if (rc) {
      cudaGetLastError();
      pr_loop_free(g);
      return rc;
    }
    L->bytes = 4 * fb + 2 * bb + sizeof(PrLoopCtl);
    g->device_bytes += L->bytes;
  }
  PrLoop* L = g->pr_loop;
  const int key[3] = {bit_all ? 1 : 0, g->coo_kernel, g->transposed ? 1 : 0};
  if (!L->exec || !std::equal(key, key + 3, L->key)) {
    L->key[0] = -1;
    GG_TRY(pr_loop_capture(g, L, bit_all));
    std::copy(key, key + 3, L->key);
  }
  *out = L;
  return GG_OK;
}

// ------------------- dense rounds of BellmanFord, Components, PageRankDelta
// The round loops of app/BellmanFord.C:119-140, app/Components.C:113-124 and
// app/PageRankDelta.C:141-170 hand each run of rounds whose edgeMap takes the
// dense COO pull to one CUDA graph, like PageRank's iterations: a while node
// whose body runs a round from bitmap 0 into bitmap 1 and, under an if node,
// the next from 1 into 0.  A round is the application's edgeMap (the COO
// pull, with its output count and out-degree sum) and its vertex step
// (BellmanFord: Visited reset over the output; Components: prevIDs = IDs over
// the input, before the pull; PageRankDelta: the vertexFilter over all
// vertices, whose output is the next frontier, and the epilogue with the L1
// norm; its pull's own output goes to a third bitmap nobody reads).  After
// each round a check kernel counts it, clears the round's input bitmap (the
// next output) and applies the host loop's tests: stop on an empty frontier,
// at the round cap (BellmanFord's n rounds) or when L1 < eps
// (PageRankDelta), and hand back to the host when the next edgeMap would not
// take the dense COO pull (sparse push, CSC pull, or a frontier without
// out-edges).  The graph, the bitmaps and the application's vertex arrays
// stay with the graph handle.
struct RoundLoopCtl {
  unsigned long long trav;       // out-degree sums of the inputs of the rounds after the first
  unsigned long long dm;         // next frontier: members
  unsigned long long out_edges;  //   and their out-degree sum
  unsigned long long err;        // device error word seen by a check
  double l1;                     // PageRankDelta: L1 of the last round
  double eps;                    //   and its stop threshold
  long long threshold;           // edgeMap's threshold (m / div)
  long long dense_threshold;     // m / 2
  uint32_t count;                // rounds run
  uint32_t max_rounds;
  uint32_t reason;               // 0 running, 1 empty frontier or L1 < eps, 2 round cap, 3 handed back, 4 device error
  uint32_t coo_always;           // the dense policy pins the COO pull (else the m/2 rule)
  uint32_t use_l1;               // stop on L1 < eps
  uint32_t pad;
};

struct RoundLoop {
  // BellmanFord: distances, Visited; Components: IDs, prevIDs; PageRankDelta:
  // p, Delta, nghSum, contributions (n + 4 entries of 4 bytes each)
  void* arr[4] = {nullptr, nullptr, nullptr, nullptr};
  uint32_t* bits[3] = {nullptr, nullptr, nullptr};  // frontiers of the rounds (0, 1); PageRankDelta's pull output (2)
  unsigned long long* d_fstats = nullptr;  // PageRankDelta: the vertexFilter's count and out-degree sum
  RoundLoopCtl* d_ctl = nullptr;
  RoundLoopCtl* h_ctl = nullptr;  // pinned
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int key[3] = {-1, -1, -1};  // COO kernel, transposed, -P source of the captured graph
  int per_round = 0;          // kernels per round
  uint64_t bytes = 0;
};

void round_loops_free(gg_graph_s* g) {
  for (RoundLoop*& L : g->round_loop) {
    if (!L) continue;
    if (L->exec) cudaGraphExecDestroy(L->exec);
    if (L->graph) cudaGraphDestroy(L->graph);
    for (void* a : L->arr) cudaFree(a);
    for (uint32_t* b : L->bits) cudaFree(b);
    cudaFree(L->d_fstats);
    cudaFree(L->d_ctl);
    if (L->h_ctl) cudaFreeHost(L->h_ctl);
    g->device_bytes -= L->bytes;
    delete L;
    L = nullptr;
  }
}

// fstats: where the round's next frontier was counted (PageRankDelta's
// vertexFilter), else the pull's own counters in stats; red: the round's L1.
__global__ void k_round_check(RoundLoopCtl* c, unsigned long long* stats, unsigned long long* fstats,
                              const double* red, cudaGraphConditionalHandle h_loop,
                              cudaGraphConditionalHandle h_odd, int set_odd, uint32_t* clear_bits,
                              uint32_t clear_words) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < clear_words;
       i += (uint64_t)gridDim.x * blockDim.x)
    clear_bits[i] = 0;
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const unsigned long long dm = fstats ? fstats[0] : stats[0], oe = fstats ? fstats[1] : stats[1], err = stats[3];
  for (int i = 0; i < 8; ++i) stats[i] = 0;  // the next pull's counters and tile counter
  if (fstats) fstats[0] = fstats[1] = 0;
  const uint32_t count = c->count + 1;
  c->count = count;
  c->dm = dm;
  c->out_edges = oe;
  if (c->use_l1) c->l1 = red[0];
  uint32_t reason = 0;
  if (err) {
    c->err = err;
    reason = 4;
  } else if (c->use_l1 ? c->l1 < c->eps : dm == 0) {
    reason = 1;
  } else if (count >= c->max_rounds) {
    reason = 2;
  } else {
    const long long fm = (long long)dm, tot = (long long)oe;
    const bool pull = tot > 0 && fm + tot > c->threshold && (c->coo_always || fm + tot > c->dense_threshold);
    if (pull)
      c->trav += oe;
    else
      reason = 3;
  }
  c->reason = reason;
  cudaGraphSetConditional(h_loop, reason == 0 ? 1u : 0u);
  if (set_odd) cudaGraphSetConditional(h_odd, reason == 0 ? 1u : 0u);
}

// The next edgeMap of a round loop takes the dense COO pull (edge_map's rule
// for flags 0 and a functor without early exit).
static bool round_takes_coo(const gg_graph_s* g, const gg_frontier_s* f) {
  const int64_t fm = (int64_t)f->dm, tot = (int64_t)f->out_edges, m = (int64_t)g->m;
  if (f->bit || tot == 0 || !g->has_coo || fm + tot <= app_threshold(g)) return false;
  const bool ref_rule = g->dense_policy == 0 || g->transposed;
  return ref_rule ? fm + tot > m / 2 : g->dense_policy == 2;
}

static void* round_loop_array(RoundLoop* L, int i) { return L->arr[i]; }

// One round's launches, from bitmap in_bits into out_bits.
static int round_launches(gg_graph_s* g, RoundLoop* L, int app, uint32_t* in_bits, uint32_t* out_bits) {
  gg_frontier_s in{}, out{};
  in.g = out.g = g;
  in.n = out.n = g->n;
  in.has_dense = out.has_dense = true;
  in.d_bits = in_bits;
  out.d_bits = out_bits;
  const bool hw = g->wtype != GG_W_NONE;
  if (app == kRoundLoopBf) {
    BfF f;
    f.sp = static_cast<int32_t*>(L->arr[0]);
    f.visited = static_cast<int32_t*>(L->arr[1]);
    GG_TRY(hw ? (pull_launch<BfF, true>(g, &in, &out, f, true)) : (pull_launch<BfF, false>(g, &in, &out, f, true)));
    VFill<int32_t> vf{f.visited, 0};
    return vertex_map(g, &out, vf);
  }
  if (app == kRoundLoopCc) {
    int32_t* ids = static_cast<int32_t*>(L->arr[0]);
    int32_t* prev = static_cast<int32_t*>(L->arr[1]);
    VCcCopy vc{ids, prev};
    GG_TRY(vertex_map(g, &in, vc));
    CcF f;
    f.ids = ids;
    f.prev = prev;
    f.outside_inert = true;  // as run_cc's rounds
    return pull_launch<CcF, false>(g, &in, &out, f, true);
  }
  // PageRankDelta: the pull's output (discarded by the application) into the
  // third bitmap, the vertexFilter over all vertices into out_bits
  float* p = static_cast<float*>(L->arr[0]);
  float* delta = static_cast<float*>(L->arr[1]);
  float* ngh = static_cast<float*>(L->arr[2]);
  float* contrib = static_cast<float*>(L->arr[3]);
  out.d_bits = L->bits[2];
  PrF f;
  f.contrib = contrib;
  f.acc_out = ngh;
  GG_TRY((pull_launch<PrF, false>(g, &in, &out, f, true)));
  const VPrd vf{p, delta, ngh, 0.85f, 0.01f};
  k_vertex_filter<VPrd, true><<<generic_grid(g, g->n), kGenericThreads, 0, g->stream>>>(
      g->n, nullptr, out_bits, g->out_off(), L->d_fstats, vf);
  GG_CUDA(cudaGetLastError());
  GG_CUDA(cudaMemsetAsync(g->ws.d_red, 0, sizeof(double), g->stream));
  k_prd_epilogue<<<generic_grid(g, g->n), kGenericThreads, 0, g->stream>>>(g->n, delta, ngh, g->out_off(), contrib,
                                                                           g->ws.d_red);
  GG_CUDA(cudaGetLastError());
  g->kernels += 2;
  return GG_OK;
}

static int round_loop_capture(gg_graph_s* g, RoundLoop* L, int app) {
  unsigned long long* fstats = app == kRoundLoopPrd ? L->d_fstats : nullptr;
  cudaGraph_t graph = nullptr;
  GG_CUDA(cudaGraphCreate(&graph, 0));
  uint32_t *X = L->bits[0], *Y = L->bits[1];
  cudaGraphConditionalHandle h_loop = 0, h_odd = 0;
  cudaGraph_t body = nullptr, odd = nullptr;
  cudaGraphNode_t last = nullptr;
  const uint32_t words = g->words() + 4;
  const int k0 = g->kernels;
  auto check = [&](int set_odd, uint32_t* in_bits) -> int {
    k_round_check<<<generic_grid(g, words), kGenericThreads, 0, g->stream>>>(
        L->d_ctl, g->ws.d_stats, fstats, g->ws.d_red, h_loop, h_odd, set_odd, in_bits, words);
    GG_CUDA(cudaGetLastError());
    g->kernels++;
    return GG_OK;
  };
  int rc = cudaGraphConditionalHandleCreate(&h_loop, graph, 1, cudaGraphCondAssignDefault) == cudaSuccess
               ? GG_OK
               : fail(GG_ERR_CUDA, "round graph: no conditional handle");
  if (!rc) rc = add_conditional(graph, nullptr, h_loop, cudaGraphCondTypeWhile, &body);
  if (!rc && cudaGraphConditionalHandleCreate(&h_odd, body, 0, cudaGraphCondAssignDefault) != cudaSuccess)
    rc = fail(GG_ERR_CUDA, "round graph: no conditional handle");
  // odd rounds: bitmap 0 into bitmap 1
  if (!rc)
    rc = capture_into(g, body, [&]() -> int {
      GG_TRY(round_launches(g, L, app, X, Y));
      return check(1, X);
    }, &last);
  const int per_round = g->kernels - k0;
  if (!rc) rc = add_conditional(body, last, h_odd, cudaGraphCondTypeIf, &odd);
  // even rounds: bitmap 1 into bitmap 0
  if (!rc)
    rc = capture_into(g, odd, [&]() -> int {
      GG_TRY(round_launches(g, L, app, Y, X));
      return check(0, Y);
    }, &last);
  cudaGraphExec_t exec = nullptr;
  if (!rc && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess)
    rc = fail(GG_ERR_CUDA, "round graph: instantiation refused");
  if (rc) {
    cudaGetLastError();
    cudaGraphDestroy(graph);
    return rc;
  }
  if (L->exec) cudaGraphExecDestroy(L->exec);
  if (L->graph) cudaGraphDestroy(L->graph);
  L->graph = graph;
  L->exec = exec;
  L->per_round = per_round;
  return GG_OK;
}

// The round loop of app for this graph handle, captured (again) when a knob
// it depends on changed since; nullptr when rounds stay on the host (switch
// off, profiling, no COO, or the driver refused the graph: the switch then
// turns off).
static RoundLoop* round_loop_get(gg_graph_s* g, int app) {
  if (!g->round_graph || g->profiling || !g->has_coo || g->m == 0) return nullptr;
  RoundLoop*& L = g->round_loop[app];
  if (!L) {
    L = new (std::nothrow) RoundLoop;
    if (!L) return nullptr;
    const uint64_t ab = 4ull * ((uint64_t)g->n + 4), bb = 4ull * ((uint64_t)g->words() + 4);
    const int na = app == kRoundLoopPrd ? 4 : 2, nb = app == kRoundLoopPrd ? 3 : 2;
    bool ok = true;
    for (int i = 0; i < na; ++i) ok = ok && cudaMalloc(&L->arr[i], ab) == cudaSuccess;
    for (int i = 0; i < nb; ++i) ok = ok && cudaMalloc((void**)&L->bits[i], bb) == cudaSuccess;
    if (app == kRoundLoopPrd) {
      ok = ok && cudaMalloc((void**)&L->d_fstats, 4 * sizeof(unsigned long long)) == cudaSuccess;
      ok = ok && cudaMemset(L->d_fstats, 0, 4 * sizeof(unsigned long long)) == cudaSuccess;
    }
    ok = ok && cudaMalloc((void**)&L->d_ctl, sizeof(RoundLoopCtl)) == cudaSuccess;
    ok = ok && cudaMallocHost((void**)&L->h_ctl, sizeof(RoundLoopCtl)) == cudaSuccess;
    L->bytes = na * ab + nb * bb + sizeof(RoundLoopCtl) + (app == kRoundLoopPrd ? 32 : 0);
    g->device_bytes += L->bytes;
    if (!ok) {
      cudaGetLastError();
      round_loops_free(g);
      return nullptr;
    }
  }
  const int key[3] = {g->coo_kernel, g->transposed ? 1 : 0, g->coo_by_source ? 1 : 0};
  if (!L->exec || !std::equal(key, key + 3, L->key)) {
    L->key[0] = -1;
    const int k = g->kernels;
    const int rc = round_loop_capture(g, L, app);
    g->kernels = k;
    if (rc) {
      g->round_graph = 0;  // refused by the driver: the host loop from now on
      return nullptr;
    }
    std::copy(key, key + 3, L->key);
  }
  return L;
}

// Runs dense COO rounds from frontier F (which takes the COO pull) on the
// device; afterwards F is the last round's output, *round and *trav count
// the rounds run and their inputs' out-degree sums.
static int round_loop_run(gg_graph_s* g, RoundLoop* L, FrontierHold& F, uint32_t max_rounds, int64_t* round,
                          uint64_t* trav, double eps, double* l1) {
  gg_frontier_s* in = F.f;
  if (!in->has_dense) GG_TRY(frontier_to_dense(in));
  const size_t bb = 4ull * (g->words() + 4);
  GG_CUDA(cudaMemcpyAsync(L->bits[0], in->d_bits, bb, cudaMemcpyDeviceToDevice, g->stream));
  GG_CUDA(cudaMemsetAsync(L->bits[1], 0, bb, g->stream));
  GG_TRY(reset_stats(g));
  RoundLoopCtl& c = *L->h_ctl;
  c = RoundLoopCtl{};
  c.threshold = app_threshold(g);
  c.dense_threshold = (long long)g->m / 2;
  c.max_rounds = max_rounds;
  c.coo_always = (g->dense_policy == 0 || g->transposed) ? 0u : 1u;
  c.use_l1 = l1 ? 1u : 0u;
  c.eps = eps;
  GG_TRY(write_small(g, L->d_ctl, c));
  GG_CUDA(cudaGraphLaunch(L->exec, g->stream));
  GG_TRY(read_small(g, L->h_ctl, L->d_ctl));
  if (c.reason == 4) return fail(GG_ERR_TIMEOUT, "device wait budget exhausted (error word %llu)", c.err);
  if (c.reason < 1 || c.reason > 3 || c.count < 1 || c.count > max_rounds)
    return fail(GG_ERR_CUDA, "round graph: bad loop state");
  *round += c.count;
  *trav += in->out_edges + c.trav;
  if (l1) *l1 = c.l1;
  g->kernels += L->per_round * (int)c.count;
  g->last = gg_edge_map_stats{};
  g->last.kind = 3;
  g->last.output_active = c.dm;
  g->last.output_out_edges = c.out_edges;
  gg_frontier_s* o = nullptr;
  GG_TRY(frontier_new(g, &o));
  F.reset(o);
  GG_TRY(frontier_ensure_bits(o, false));
  GG_CUDA(cudaMemcpyAsync(o->d_bits, L->bits[(c.count & 1) ? 1 : 0], bb, cudaMemcpyDeviceToDevice, g->stream));
  o->has_dense = true;
  o->dm = c.dm;
  o->out_edges = c.out_edges;
  return GG_OK;
}

// app/PageRank.C:102-150 (bit_all: app/PageRankBit.C:145)
static int run_pagerank(gg_graph_s* g, int max_iter, int bit_all, float* ranks, gg_run_stats* st) {
  const uint32_t n = g->n;
  g->kernels = 0;
  const float damping = 0.85f;
  const float added = (float)((1 - 0.85) * (1 / (double)n));
  const double eps = 0.0000001;
  const int64_t m = (int64_t)g->m, threshold = app_threshold(g);
  // the graph holds the COO pull: only where edgeMap picks it for all vertices
  const bool ref_rule = g->dense_policy == 0 || g->transposed;
  const bool coo_first = m > 0 && (int64_t)n + m > threshold && g->has_coo &&
                         (ref_rule ? (int64_t)n + m > m / 2 : g->dense_policy == 2);
  PrLoop* L = nullptr;
  if (g->pr_graph && !g->profiling && coo_first && pr_loop_get(g, bit_all != 0, &L) != GG_OK) {
    g->pr_graph = 0;  // refused by the driver: the host loop from now on
    L = nullptr;
  }
  g->kernels = 0;  // launches captured above are not this call's
  // contributions are double-buffered: the vertex step at the COO pull's
  // commits writes the next ones while other tiles still gather these
  DevBuf<float> a, b, c0, c1;
  float *A, *B, *Cb[2];
  if (L) {
    A = L->buf[0];
    B = L->buf[1];
    Cb[0] = L->buf[2];
    Cb[1] = L->buf[3];
  } else {
    GG_TRY(a.alloc(g, n));
    GG_TRY(b.alloc(g, n));
    GG_TRY(c0.alloc(g, n));
    GG_TRY(c1.alloc(g, n));
    A = a.p;
    B = b.p;
    Cb[0] = c0.p;
    Cb[1] = c1.p;
  }
  EventTimer tm(g->stream);
  float* p_curr = A;
  float* p_next = B;
  float* last = p_next;
  int cur = 0;  // the contributions the next pull gathers
  int count = 0;
  uint64_t trav = 0;
  bool masked = false;  // contrib marks the frontier (sources outside hold -1)
  bool done = false;
  FrontierHold F;
  if (L) {
    PrLoopCtl& c = *L->h_ctl;
    c = PrLoopCtl{};
    c.trav = g->m;  // the first input: all vertices (bits(part, n, m))
    c.in_dm = n;
    c.in_edges = g->m;
    c.eps = eps;
    c.threshold = threshold;
    c.dense_threshold = m / 2;
    c.max_iter = (uint32_t)max_iter;
    c.coo_always = ref_rule ? 0u : 1u;
    GG_TRY(write_small(g, L->d_ctl, c));
    GG_CUDA(cudaGraphLaunch(L->exec, g->stream));
    GG_TRY(read_small(g, L->h_ctl, L->d_ctl));
    if (c.reason == 4) return fail(GG_ERR_TIMEOUT, "device wait budget exhausted (error word %llu)", c.err);
    if (c.reason < 1 || c.reason > 3 || c.count < 1) return fail(GG_ERR_CUDA, "PageRank graph: bad loop state");
    count = (int)c.count;
    trav = c.trav;
    // the initial pass, then per iteration the pull, the vertex step's pass
    // (uncovered ranges or the epilogue) and the check; the control block's
    // write before the graph and read-back after it
    const int per_iter = 2 + (pr_fused(g) && g->coo_gap_count == 0 ? 0 : 1);
    g->kernels = 1 + per_iter * count + 2;
    g->last = gg_edge_map_stats{};
    g->last.kind = 3;
    g->last.frontier_active = c.in_dm;
    g->last.frontier_out_edges = c.in_edges;
    g->last.output_active = c.dm;
    g->last.output_out_edges = c.out_edges;
    last = (count & 1) ? B : A;
    cur = count & 1;
    if (c.reason == 3) {  // the next edgeMap leaves the COO pull: continue on the host
      p_curr = last;
      p_next = last == A ? B : A;
      gg_frontier_s* o = nullptr;
      GG_TRY(frontier_new(g, &o));
      F.reset(o);
      GG_TRY(frontier_ensure_bits(o, false));
      GG_CUDA(cudaMemcpyAsync(o->d_bits, L->bits[(count & 1) ? 0 : 1], 4ull * (g->words() + 4),
                              cudaMemcpyDeviceToDevice, g->stream));
      o->has_dense = true;
      o->dm = c.dm;
      o->out_edges = c.out_edges;
      if (bit_all) o->bit = true;
      masked = !bit_all;
    } else {
      done = true;
    }
  } else {
    GG_TRY(fill<float>(g, p_curr, n, (float)(1 / (double)n)));
    GG_TRY(fill<float>(g, p_next, n, 0.0f));
    k_div_outdeg<<<generic_grid(g, n), kGenericThreads, 0, g->stream>>>(n, p_curr, g->out_off(), Cb[0]);
    g->kernels++;
    GG_TRY(gg_frontier_all(g, &F.f));
  }
  while (!done && count < max_iter) {
    ++count;
    trav += F.f->out_edges;
    // the vertex step reads the input frontier's bitmap during the pull
    if (!F.f->bit && !F.f->has_dense) GG_TRY(frontier_to_dense(F.f));
    GG_CUDA(cudaMemsetAsync(g->ws.d_red, 0, sizeof(double), g->stream));
    // frontier sources have p > 0; a COO pull's output is dense, so it marks
    // the next contributions unless PageRankBit keeps every vertex active
    const PrFinishF f = pr_functor(g, Cb[cur], Cb[cur ^ 1], p_curr, p_next, F.f->bit ? nullptr : F.f->d_bits,
                                   masked, !bit_all);
    gg_frontier_s* out = nullptr;
    GG_TRY(edge_map(g, F.f, f, threshold, 0, &out));
    FrontierHold O;
    O.f = out;
    // the output becomes the next frontier: mark it in the next contributions
    masked = !bit_all && out->n == n && out->has_dense;
    if (g->last.kind == 3 && pr_fused(g)) {  // the pull's commits ran the vertex step
      GG_TRY(pr_finish_gaps(g, f));
    } else {
      k_pr_epilogue<<<generic_grid(g, n), kGenericThreads, 0, g->stream>>>(
          n, F.f->bit ? 1 : 0, F.f->d_bits, p_curr, p_next, g->out_off(), damping, added, Cb[cur ^ 1],
          g->ws.d_red, masked ? out->d_bits : nullptr);
      GG_CUDA(cudaGetLastError());
      g->kernels++;
    }
    last = p_next;
    double l1;
    GG_TRY(read_red(g, &l1));
    if (l1 < eps) break;
    std::swap(p_curr, p_next);
    cur ^= 1;
    gg_frontier_s* o = O.release();
    if (bit_all) o->bit = true;  // output.bit = true
    F.reset(o);
  }
  const float* res = last;
  GG_TRY(given_order<float>(g, last, 0, &res));
  const double ms = tm.stop();
  GG_TRY(to_host(g, ranks, res, n));
  fill_stats(st, ms, count, trav, g->kernels);
  return GG_OK;
}

// PageRankConverage (app/PageRankConverage.C:235-315) kernels.  Sums are
// accumulated in FP64 like the reference's sum()/normdiff().
// Next contributions: add_factor = (0.85 / outdeg) * p (sinks are never gathered).
__global__ void k_prc_contrib(uint32_t n, const float* p, const uint32_t* off, float* contrib) {
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t d = off[j + 1] - off[j];
    contrib[j] = d ? (0.85f / (float)d) * p[j] : 0.0f;
  }
}
__global__ void k_prc_sum(uint32_t n, const float* a, double* out) {
  double acc = 0;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x)
    acc += a[j];
  block_add_double(acc, out);
}
// p_next += (1 - sum)/n (PR_Vertex_Csum), L1 = sum |p_curr - p_next| (normdiff), and the new sum.
__global__ void k_prc_fix(uint32_t n, const float* p_curr, float* p_next, const double* red, double* l1,
                          double* sum2) {
  const float c = (float)((1.0 - red[0]) / (double)n);
  double a = 0, b = 0;
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
    const float pn = p_next[j] + c;
    p_next[j] = pn;
    a += fabsf(p_curr[j] - pn);
    b += pn;
  }
  block_add_double(a, l1);
  __syncthreads();
  block_add_double(b, sum2);
}
// p_next /= sum (PR_Vertex_norm), p_curr = 0 (PR_Vertex_Reset), next contributions from p_next.
__global__ void k_prc_norm(uint32_t n, float* p_curr, float* p_next, const double* sum2, const uint32_t* off,
                           float* contrib) {
  const float inv = (float)(1.0 / sum2[0]);
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
    const float pn = p_next[j] * inv;
    p_next[j] = pn;
    p_curr[j] = 0.0f;
    const uint32_t d = off[j + 1] - off[j];
    contrib[j] = d ? (0.85f / (float)d) * pn : 0.0f;
  }
}

static int run_pagerank_converge(gg_graph_s* g, int32_t max_iter, double eps, float* ranks, gg_run_stats* st) {
  const uint32_t n = g->n;
  g->kernels = 0;
  DevBuf<float> a, b, contrib;
  GG_TRY(a.alloc(g, n));
  GG_TRY(b.alloc(g, n));
  GG_TRY(contrib.alloc(g, n));
  double* red = g->ws.d_red;  // [0] sum after the edgeMap, [1] L1, [2] sum after the correction
  EventTimer tm(g->stream);
  float* p_curr = a.p;
  float* p_next = b.p;
  const int grid = generic_grid(g, n);
  GG_TRY(fill<float>(g, p_curr, n, (float)(1 / (double)n)));
  GG_TRY(fill<float>(g, p_next, n, 0.0f));
  k_prc_contrib<<<grid, kGenericThreads, 0, g->stream>>>(n, p_curr, g->out_off(), contrib.p);
  g->kernels++;
  FrontierHold F;
  GG_TRY(gg_frontier_all(g, &F.f));  // partitioned_vertices::bits
  int count = 0;
  double L1 = 2;
  while (count < max_iter && L1 > eps) {
    PrPosF f;
    f.contrib = contrib.p;
    f.acc_out = p_next;
    gg_frontier_s* out = nullptr;
    GG_TRY(edge_map(g, F.f, f, app_threshold(g), GG_EM_NO_OUTPUT | kEmNoWait, &out));  // output.del(); read_small waits
    frontier_free(out);
    GG_CUDA(cudaMemsetAsync(red, 0, 3 * sizeof(double), g->stream));
    k_prc_sum<<<grid, kGenericThreads, 0, g->stream>>>(n, p_next, red);
    k_prc_fix<<<grid, kGenericThreads, 0, g->stream>>>(n, p_curr, p_next, red, red + 1, red + 2);
    k_prc_norm<<<grid, kGenericThreads, 0, g->stream>>>(n, p_curr, p_next, red + 2, g->out_off(), contrib.p);
    GG_CUDA(cudaGetLastError());
    g->kernels += 3;
    GG_TRY(read_small(g, g->ws.h_red, red, 3));
    L1 = g->ws.h_red[1];
    ++count;
    std::swap(p_curr, p_next);
  }
  const float* res = p_curr;
  GG_TRY(given_order<float>(g, p_curr, 0, &res));
  const double ms = tm.stop();
  GG_TRY(to_host(g, ranks, res, n));
  fill_stats(st, ms, count, (uint64_t)count * g->m, g->kernels);
  return GG_OK;
}

// app/PageRankDelta.C:120-174
static int run_pagerank_delta(gg_graph_s* g, float* ranks, gg_run_stats* st) {
  const uint32_t n = g->n;
  RoundLoop* L = round_loop_get(g, kRoundLoopPrd);  // its arrays, when its graph runs the dense rounds
  g->kernels = 0;
  DevBuf<float> pb, deltab, nghb, contribb;
  float *p = nullptr, *delta = nullptr, *ngh = nullptr, *contrib = nullptr;
  if (L) {
    p = static_cast<float*>(round_loop_array(L, 0));
    delta = static_cast<float*>(round_loop_array(L, 1));
    ngh = static_cast<float*>(round_loop_array(L, 2));
    contrib = static_cast<float*>(round_loop_array(L, 3));
  } else {
    GG_TRY(pb.alloc(g, n));
    GG_TRY(deltab.alloc(g, n));
    GG_TRY(nghb.alloc(g, n));
    GG_TRY(contribb.alloc(g, n));
    p = pb.p;
    delta = deltab.p;
    ngh = nghb.p;
    contrib = contribb.p;
  }
  const float damping = 0.85f, eps2 = 0.01f;  // the round graph's vertexFilter uses the same constants
  const double eps = 0.0000001;
  const float one_over_n = (float)(1 / (double)n);
  const float added = (float)((1 - 0.85) * (1 / (double)n));
  EventTimer tm(g->stream);
  GG_TRY(fill<float>(g, p, n, 0.0f));
  GG_TRY(fill<float>(g, delta, n, one_over_n));
  GG_TRY(fill<float>(g, ngh, n, 0.0f));
  k_div_outdeg<<<generic_grid(g, n), kGenericThreads, 0, g->stream>>>(n, delta, g->out_off(), contrib);
  g->kernels++;
  FrontierHold F, All;
  GG_TRY(gg_frontier_all(g, &F.f));
  GG_TRY(gg_frontier_all(g, &All.f));
  int64_t round = 0;
  uint64_t trav = 0;
  for (;;) {
    if (L && round_takes_coo(g, F.f)) {  // dense COO rounds on the device, each with its L1 test
      double l1 = 0;
      GG_TRY(round_loop_run(g, L, F, 0xffffffffu, &round, &trav, eps, &l1));
      if (l1 < eps) break;
      continue;
    }
    ++round;
    PrF f;
    f.contrib = contrib;
    f.acc_out = ngh;
    trav += F.f->out_edges;
    gg_frontier_s* out = nullptr;
    GG_TRY(edge_map(g, F.f, f, app_threshold(g), 0, &out));
    frontier_free(out);
    gg_frontier_s* active = nullptr;
    if (round == 1) {
      VPrdFirst vf{p, delta, ngh, damping, added, one_over_n, eps2};
      GG_TRY(vertex_filter(g, All.f, vf, &active));
    } else {
      VPrd vf{p, delta, ngh, damping, eps2};
      GG_TRY(vertex_filter(g, All.f, vf, &active));
    }
    FrontierHold A;
    A.f = active;
    GG_CUDA(cudaMemsetAsync(g->ws.d_red, 0, sizeof(double), g->stream));
    k_prd_epilogue<<<generic_grid(g, n), kGenericThreads, 0, g->stream>>>(n, delta, ngh, g->out_off(), contrib,
                                                                          g->ws.d_red);
    GG_CUDA(cudaGetLastError());
    g->kernels++;
    double l1;
    GG_TRY(read_red(g, &l1));
    if (l1 < eps) break;
    F.reset(A.release());
  }
  const float* res = p;
  GG_TRY(given_order<float>(g, p, 0, &res));
  const double ms = tm.stop();
  GG_TRY(to_host(g, ranks, res, n));
  fill_stats(st, ms, (int)round, trav, g->kernels);
  return GG_OK;
}

// An SpMV input uploaded ahead of its gg_spmv_staged call, on the copy
// stream into given-order array 1, so that the upload overlaps whatever the
// stream still runs (the previous application).  The copy starts after the
// work already queued on the stream (which may still read that array) and
// after the copies already leaving from it (same copy stream).
static int stage_spmv_input(gg_graph_s* g, const float* x_host) {
  if (!g->async_results || !g->ws.d_order[1] || !g->copy_stream)
    return fail(GG_ERR_UNSUPPORTED, "gg_spmv_stage_input needs GG_TUNE_ASYNC_RESULTS 1");
  if (!g->input_ready) GG_CUDA(cudaEventCreateWithFlags(&g->input_ready, cudaEventDisableTiming));
  GG_CUDA(cudaEventRecord(g->result_ready, g->stream));
  GG_CUDA(cudaStreamWaitEvent(g->copy_stream, g->result_ready, 0));
  GG_CUDA(cudaMemcpyAsync(g->ws.d_order[1], x_host, 4ull * g->n, cudaMemcpyHostToDevice, g->copy_stream));
  GG_CUDA(cudaEventRecord(g->input_ready, g->copy_stream));
  g->input_staged = true;
  return GG_OK;
}

// app/SPMV.C:64-92.  x_in: host input, or NULL for x = 1/n; staged: the
// input was uploaded by stage_spmv_input (x_in is then ignored).
static int run_spmv(gg_graph_s* g, const float* x_in, float* y_out, gg_run_stats* st, bool staged = false) {
  const uint32_t n = g->n;
  g->kernels = 0;
  DevBuf<float> x, y;
  GG_TRY(x.alloc(g, n));
  GG_TRY(y.alloc(g, n));
  // the input vector is uploaded before the timed Compute loop (like the
  // graph); a renumbered graph takes it through its given-order array 1,
  // which the result uses after it (array 0 may still be leaving for the
  // host with an earlier result)
  float* xg = g->relabeled ? reinterpret_cast<float*>(g->ws.d_order[1]) : x.p;
  if (staged) {
    GG_CUDA(cudaStreamWaitEvent(g->stream, g->input_ready, 0));
    g->input_staged = false;
    x_in = nullptr;
    xg = reinterpret_cast<float*>(g->ws.d_order[1]);
  }
  if (x_in && g->relabeled) GG_TRY(slot_write_wait(g, 1));
  if (x_in) GG_CUDA(cudaMemcpyAsync(xg, x_in, 4ull * n, cudaMemcpyHostToDevice, g->stream));
  EventTimer tm(g->stream);
  if ((x_in || staged) && g->relabeled) GG_TRY(device_order<float>(g, xg, 1, x.p));
  if (staged && !g->relabeled)
    GG_CUDA(cudaMemcpyAsync(x.p, xg, 4ull * n, cudaMemcpyDeviceToDevice, g->stream));
  if (!x_in && !staged) GG_TRY(fill<float>(g, x.p, n, (float)(1 / (double)n)));
  // a renumbered graph's sums go straight to the given ids, in array 1 (the
  // input staged there was consumed above)
  float* yd = g->relabeled ? reinterpret_cast<float*>(g->ws.d_order[1]) : y.p;
  if (g->relabeled && !x_in) GG_TRY(slot_write_wait(g, 1));
  GG_TRY(fill<float>(g, yd, n, 0.0f));
  FrontierHold F;
  GG_TRY(gg_frontier_all(g, &F.f));
  SpmvF f;
  f.x = x.p;
  f.y = yd;
  f.float_w = g->wtype == GG_W_FLOAT32;
  f.y_map = g->relabeled ? g->d_old_of_new : nullptr;
  gg_frontier_s* out = nullptr;
  GG_TRY(edge_map(g, F.f, f, app_threshold(g), GG_EM_NO_OUTPUT | kEmNoWait, &out));  // output.del(); tm.stop() waits
  frontier_free(out);
  const float* res = yd;
  if (!g->relabeled) GG_TRY(given_order<float>(g, y.p, 1, &res));
  const double ms = tm.stop();
  GG_TRY(to_host(g, y_out, res, n));
  fill_stats(st, ms, 1, g->m, g->kernels);
  return GG_OK;
}

// app/BellmanFord.C:106-145
static int run_bf(gg_graph_s* g, uint32_t start, int32_t* dist, gg_run_stats* st) {
  const uint32_t n = g->n;
  RoundLoop* L = round_loop_get(g, kRoundLoopBf);  // its arrays, when its graph runs the dense rounds
  g->kernels = 0;
  DevBuf<int32_t> spb, visb;
  int32_t *sp = nullptr, *vis = nullptr;
  if (L) {
    sp = static_cast<int32_t*>(round_loop_array(L, 0));
    vis = static_cast<int32_t*>(round_loop_array(L, 1));
  } else {
    GG_TRY(spb.alloc(g, n));
    GG_TRY(visb.alloc(g, n));
    sp = spb.p;
    vis = visb.p;
  }
  const int32_t inf = 2147483647 / 2;
  EventTimer tm(g->stream);
  GG_TRY(fill<int32_t>(g, sp, n, inf));
  GG_TRY(set_one<int32_t>(g, sp, start, 0));
  GG_TRY(fill<int32_t>(g, vis, n, 0));
  FrontierHold F;
  GG_TRY(gg_frontier_single(g, start, &F.f));
  int64_t round = 0;
  uint64_t trav = 0;
  while (F.f->dm > 0) {
    if (round == (int64_t)n) {  // negative weight cycle
      GG_TRY(fill<int32_t>(g, sp, n, -inf));
      break;
    }
    if (L && round_takes_coo(g, F.f)) {  // dense COO rounds on the device
      GG_TRY(round_loop_run(g, L, F, (uint32_t)((int64_t)n - round), &round, &trav));
      continue;
    }
    BfF f;
    f.sp = sp;
    f.visited = vis;
    trav += F.f->out_edges;
    gg_frontier_s* out = nullptr;
    GG_TRY(edge_map(g, F.f, f, app_threshold(g), 0, &out));
    VFill<int32_t> vf{vis, 0};
    GG_TRY(vertex_map(g, out, vf));
    F.reset(out);
    ++round;
  }
  const int32_t* res = sp;
  GG_TRY(given_order<int32_t>(g, sp, 0, &res));
  const double ms = tm.stop();
  GG_TRY(to_host(g, dist, res, n));
  fill_stats(st, ms, (int)round, trav, g->kernels);
  return GG_OK;
}

// app/BC.C:156-226 (single source, FP32 like fType)
static int run_bc(gg_graph_s* g, uint32_t start, float* dep_out, float* np_out, gg_run_stats* st) {
  const uint32_t n = g->n;
  g->kernels = 0;
  DevBuf<float> np, dep;
  DevBuf<uint8_t> vis;
  GG_TRY(np.alloc(g, n));
  GG_TRY(dep.alloc(g, n));
  GG_TRY(vis.alloc(g, n));
  EventTimer tm(g->stream);
  GG_TRY(fill<float>(g, np.p, n, 0.0f));
  GG_TRY(fill<uint8_t>(g, vis.p, n, 0));
  GG_TRY(set_one<float>(g, np.p, start, 1.0f));
  GG_TRY(set_one<uint8_t>(g, vis.p, start, 1));
  std::vector<gg_frontier_s*> levels;
  struct LevelsHold {
    std::vector<gg_frontier_s*>* v;
    ~LevelsHold() {
      for (auto* f : *v) frontier_free(f);
    }
  } lh{&levels};
  gg_frontier_s* F0 = nullptr;
  GG_TRY(gg_frontier_single(g, start, &F0));
  levels.push_back(F0);
  int round = 0;
  uint64_t trav = 0;
  gg_frontier_s* F = F0;
  while (F->dm > 0) {
    ++round;
    BcF f;
    f.values = np.p;
    f.visited = vis.p;
    trav += F->out_edges;
    gg_frontier_s* out = nullptr;
    GG_TRY(edge_map(g, F, f, app_threshold(g), 0, &out));
    VBcMark vm{vis.p};
    GG_TRY(vertex_map(g, out, vm));
    levels.push_back(out);
    F = out;
  }
  if (np_out) {
    const float* res = np.p;
    GG_TRY(given_order<float>(g, np.p, 0, &res));
    GG_TRY(to_host(g, np_out, res, n));
  }
  GG_TRY(fill<float>(g, dep.p, n, 0.0f));
  k_invert<<<generic_grid(g, n), kGenericThreads, 0, g->stream>>>(n, np.p);  // inverseNumPaths aliases NumPaths
  g->kernels++;
  GG_TRY(fill<uint8_t>(g, vis.p, n, 0));
  F = levels[round - 1];
  VBcBack vb{vis.p, dep.p, np.p};
  GG_TRY(vertex_map(g, F, vb));
  GG_TRY(gg_graph_transpose(g));
  int rc = GG_OK;
  for (int r = round - 2; r >= 0 && !rc; --r) {
    BcF f;
    f.values = dep.p;
    f.visited = vis.p;
    trav += F->out_edges;
    gg_frontier_s* out = nullptr;
    rc = edge_map(g, F, f, app_threshold(g), 0, &out);
    if (rc) break;
    frontier_free(out);
    F = levels[r];
    rc = vertex_map(g, F, vb);
  }
  gg_graph_transpose(g);
  if (rc) return rc;
  k_bc_final<<<generic_grid(g, n), kGenericThreads, 0, g->stream>>>(n, dep.p, np.p);
  g->kernels++;
  const float* res = dep.p;
  GG_TRY(given_order<float>(g, dep.p, 1, &res));
  const double ms = tm.stop();
  GG_TRY(to_host(g, dep_out, res, n));
  fill_stats(st, ms, round, trav, g->kernels);
  return GG_OK;
}

}  // namespace gg

using namespace gg;

extern "C" {

int gg_edge_map(gg_graph_t g, gg_frontier_t in, int32_t fid, const void* args, int64_t threshold, uint32_t flags,
                gg_frontier_t* out) {
  if (!graph_live(g) || !frontier_live(in) || !out || !args || in->g != g)
    return fail(GG_ERR_INVALID_ARG, "gg_edge_map: bad arguments");
  flags &= GG_EM_FORCE_SPARSE | GG_EM_FORCE_CSC | GG_EM_FORCE_COO | GG_EM_NO_OUTPUT;  // the C ABI's bits
  switch (fid) {
    case GG_F_BFS: {
      const gg_bfs_args* a = (const gg_bfs_args*)args;
      BfsF f;
      f.parents = a->parents;
      f.levels = a->levels;
      f.round = a->round;
      return edge_map(g, in, f, threshold, flags, out);
    }
    case GG_F_CC: {
      const gg_cc_args* a = (const gg_cc_args*)args;
      CcF f;
      f.ids = a->ids;
      f.prev = a->prev_ids;
      return edge_map(g, in, f, threshold, flags, out);
    }
    case GG_F_PR:
    case GG_F_PRDELTA: {
      const float* src;
      float* acc;
      if (fid == GG_F_PR) {
        src = ((const gg_pr_args*)args)->p_curr;
        acc = ((const gg_pr_args*)args)->p_next;
      } else {
        src = ((const gg_prdelta_args*)args)->delta;
        acc = ((const gg_prdelta_args*)args)->ngh_sum;
      }
      DevBuf<float> contrib;
      GG_TRY(contrib.alloc(g, g->n));
      k_div_outdeg<<<generic_grid(g, g->n), kGenericThreads, 0, g->stream>>>(g->n, src, g->out_off(), contrib.p);
      PrF f;
      f.contrib = contrib.p;
      f.acc_out = acc;
      return edge_map(g, in, f, threshold, flags, out);
    }
    case GG_F_SPMV: {
      const gg_spmv_args* a = (const gg_spmv_args*)args;
      SpmvF f;
      f.x = a->p_curr;
      f.y = a->p_next;
      f.float_w = g->wtype == GG_W_FLOAT32;
      return edge_map(g, in, f, threshold, flags, out);
    }
    case GG_F_BF: {
      const gg_bf_args* a = (const gg_bf_args*)args;
      BfF f;
      f.sp = a->sp_len;
      f.visited = a->visited;
      return edge_map(g, in, f, threshold, flags, out);
    }
    case GG_F_BC:
    case GG_F_BC_BACK: {
      const gg_bc_args* a = (const gg_bc_args*)args;
      BcF f;
      f.values = a->values;
      f.visited = a->visited;
      return edge_map(g, in, f, threshold, flags, out);
    }
    default:
      return fail(GG_ERR_UNSUPPORTED, "gg_edge_map: unknown functor id %d", fid);
  }
}

int gg_last_edge_map_stats(gg_graph_t g, gg_edge_map_stats* st) {
  if (!g || !st) return fail(GG_ERR_INVALID_ARG, "gg_last_edge_map_stats: bad arguments");
  *st = g->last;
  return GG_OK;
}

int gg_vertex_map(gg_graph_t g, gg_frontier_t f, int32_t vid, const void* args) {
  if (!graph_live(g) || !frontier_live(f) || !args || f->g != g)
    return fail(GG_ERR_INVALID_ARG, "gg_vertex_map: bad arguments");
  int rc;
  switch (vid) {
    case GG_V_CC_COPY: {
      const gg_cc_args* a = (const gg_cc_args*)args;
      rc = vertex_map(g, f, VCcCopy{a->ids, a->prev_ids});
      break;
    }
    case GG_V_PR_UPDATE: {
      const gg_pr_vertex_args* a = (const gg_pr_vertex_args*)args;
      const float added = (float)((1 - (double)a->damping) * (1 / (double)a->n));
      rc = vertex_map(g, f, VPrUpdate{a->p_next, a->damping, added});
      break;
    }
    case GG_V_FILL_F32: {
      const gg_fill_args* a = (const gg_fill_args*)args;
      rc = vertex_map(g, f, VFill<float>{(float*)a->array, (float)a->value});
      break;
    }
    case GG_V_FILL_I32: {
      const gg_fill_args* a = (const gg_fill_args*)args;
      rc = vertex_map(g, f, VFill<int32_t>{(int32_t*)a->array, (int32_t)a->value});
      break;
    }
    case GG_V_FILL_U8: {
      const gg_fill_args* a = (const gg_fill_args*)args;
      rc = vertex_map(g, f, VFill<uint8_t>{(uint8_t*)a->array, (uint8_t)a->value});
      break;
    }
    case GG_V_BC_MARK: {
      const gg_bc_args* a = (const gg_bc_args*)args;
      rc = vertex_map(g, f, VBcMark{a->visited});
      break;
    }
    case GG_V_BC_BACK: {
      const gg_bc_back_vertex_args* a = (const gg_bc_back_vertex_args*)args;
      rc = vertex_map(g, f, VBcBack{a->visited, a->dependencies, a->inv_num_paths});
      break;
    }
    default:
      return fail(GG_ERR_UNSUPPORTED, "gg_vertex_map: unknown vertex functor id %d", vid);
  }
  if (rc) return rc;
  GG_CUDA(cudaStreamSynchronize(g->stream));
  return GG_OK;
}

int gg_vertex_filter(gg_graph_t g, gg_frontier_t f, int32_t vid, const void* args, gg_frontier_t* out) {
  if (!graph_live(g) || !frontier_live(f) || !args || !out || f->g != g)
    return fail(GG_ERR_INVALID_ARG, "gg_vertex_filter: bad arguments");
  const gg_prdelta_vertex_args* a = (const gg_prdelta_vertex_args*)args;
  switch (vid) {
    case GG_V_PRDELTA_FIRST: {
      const float added = (float)((1 - (double)a->damping) * (double)a->one_over_n);
      return vertex_filter(g, f, VPrdFirst{a->p, a->delta, a->ngh_sum, a->damping, added, a->one_over_n, a->epsilon2},
                           out);
    }
    case GG_V_PRDELTA:
      return vertex_filter(g, f, VPrd{a->p, a->delta, a->ngh_sum, a->damping, a->epsilon2}, out);
    default:
      return fail(GG_ERR_UNSUPPORTED, "gg_vertex_filter: unknown filter id %d", vid);
  }
}

int gg_bfs(gg_graph_t g, uint32_t start, int32_t* parents, int32_t* levels, gg_run_stats* st) {
  if (!g || start >= g->n) return fail(GG_ERR_INVALID_ARG, "gg_bfs: bad arguments");
  return run_bfs(g, g->device_id(start), parents, levels, st);
}
int gg_components(gg_graph_t g, int32_t* ids, gg_run_stats* st) {
  if (!g) return fail(GG_ERR_INVALID_ARG, "gg_components: null graph");
  return run_cc(g, ids, st);
}
int gg_pagerank(gg_graph_t g, int32_t max_iter, int32_t bit_all, float* ranks, gg_run_stats* st) {
  if (!g || max_iter < 1) return fail(GG_ERR_INVALID_ARG, "gg_pagerank: bad arguments");
  return run_pagerank(g, max_iter, bit_all, ranks, st);
}
int gg_pagerank_delta(gg_graph_t g, float* ranks, gg_run_stats* st) {
  if (!g) return fail(GG_ERR_INVALID_ARG, "gg_pagerank_delta: null graph");
  return run_pagerank_delta(g, ranks, st);
}
int gg_pagerank_converge(gg_graph_t g, int32_t max_iter, double eps, float* ranks, gg_run_stats* st) {
  if (!graph_live(g) || max_iter < 0 || !ranks) return fail(GG_ERR_INVALID_ARG, "gg_pagerank_converge: bad arguments");
  return run_pagerank_converge(g, max_iter, eps, ranks, st);
}
int gg_spmv(gg_graph_t g, const float* x, float* y, gg_run_stats* st) {
  if (!g) return fail(GG_ERR_INVALID_ARG, "gg_spmv: null graph");
  return run_spmv(g, x, y, st);
}
int gg_spmv_stage_input(gg_graph_t g, const float* x) {
  if (!graph_live(g) || !x) return fail(GG_ERR_INVALID_ARG, "gg_spmv_stage_input: bad arguments");
  return stage_spmv_input(g, x);
}
int gg_spmv_staged(gg_graph_t g, float* y, gg_run_stats* st) {
  if (!graph_live(g)) return fail(GG_ERR_INVALID_ARG, "gg_spmv_staged: not a live graph");
  if (!g->input_staged) return fail(GG_ERR_INVALID_ARG, "gg_spmv_staged: no input staged (gg_spmv_stage_input)");
  return run_spmv(g, nullptr, y, st, true);
}
int gg_bellman_ford(gg_graph_t g, uint32_t start, int32_t* dist, gg_run_stats* st) {
  if (!g || start >= g->n) return fail(GG_ERR_INVALID_ARG, "gg_bellman_ford: bad arguments");
  return run_bf(g, g->device_id(start), dist, st);
}
int gg_bc(gg_graph_t g, uint32_t start, float* dep, float* np, gg_run_stats* st) {
  if (!g || start >= g->n) return fail(GG_ERR_INVALID_ARG, "gg_bc: bad arguments");
  return run_bc(g, g->device_id(start), dep, np, st);
}

}  // extern "C"
