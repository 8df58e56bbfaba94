// Many graphs in one launch: BFS over a batch of independent graphs of uneven
// size.  All graphs live in one device arena; a persistent kernel's CTAs take
// whole graphs from a device work queue (largest first) and run the
// level-synchronous top-down traversal of app/BFS.C:77-101 inside the CTA,
// with the frontier's edges load-balanced across the CTA's threads by a
// block prefix sum over the frontier's degrees.  The launch sequence is
// captured once as a CUDA graph and replayed.
#include <algorithm>
#include <mutex>
#include <numeric>
#include <unordered_set>
#include <vector>

#include "gg_runtime.cuh"

struct BatchDesc {
  uint64_t off_base;  // first offset of the graph in the offsets arena (n+1 entries)
  uint64_t idx_base;  // first edge of the graph in the index arena
  uint64_t lev_base;  // first level slot of the graph
  uint32_t n;
  uint32_t pad;
};

struct gg_graph_batch_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  int32_t count = 0;
  uint64_t total_n = 0, total_m = 0;
  uint32_t max_n = 0;
  std::vector<uint64_t> firsts;
  uint32_t *d_off = nullptr, *d_idx = nullptr, *d_order = nullptr, *d_src = nullptr, *d_scratch = nullptr;
  BatchDesc* d_desc = nullptr;
  int32_t* d_levels = nullptr;
  unsigned long long* d_ctr = nullptr;  // [0] work ticket, [1] edges traversed
  uint32_t* h_src = nullptr;            // pinned
  int32_t* h_levels = nullptr;          // pinned
  unsigned long long* h_ctr = nullptr;  // pinned
  int grid = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace gg {

static std::mutex g_batch_mu;
static std::unordered_set<const gg_graph_batch_s*> g_batches;

static bool batch_live(const gg_graph_batch_s* b) {
  std::lock_guard<std::mutex> lk(g_batch_mu);
  return b && g_batches.count(b);
}

constexpr int kBatchThreads = 256;

__global__ void __launch_bounds__(kBatchThreads) k_batch_bfs(const BatchDesc* __restrict__ desc,
                                                              const uint32_t* __restrict__ order, int32_t count,
                                                              const uint32_t* __restrict__ off,
                                                              const uint32_t* __restrict__ idx, int32_t* levels,
                                                              const uint32_t* __restrict__ src,
                                                              unsigned long long* ctr, uint32_t* scratch,
                                                              uint64_t stride) {
  __shared__ int32_t s_graph;
  __shared__ uint32_t s_scan[kBatchThreads + 1];
  __shared__ uint32_t s_beg[kBatchThreads];
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_nq;
  const int tid = threadIdx.x, lane = tid & 31;
  const uint32_t lanemask_lt = (1u << lane) - 1u;
  uint32_t* qa = scratch + (uint64_t)blockIdx.x * 2 * stride;
  uint32_t* qb = qa + stride;
  unsigned long long trav = 0;
  for (;;) {
    if (tid == 0) {
      const unsigned long long t = atomicAdd(ctr, 1ull);
      s_graph = t < (unsigned long long)count ? (int32_t)order[t] : -1;
    }
    __syncthreads();
    const int32_t gi = s_graph;
    if (gi < 0) break;
    const BatchDesc d = desc[gi];
    const uint32_t* go = off + d.off_base;
    const uint32_t* gx = idx + d.idx_base;
    int32_t* lev = levels + d.lev_base;
    for (uint32_t v = tid; v < d.n; v += kBatchThreads) lev[v] = -1;
    __syncthreads();
    const uint32_t s = src[gi];
    if (tid == 0) {
      lev[s] = 0;
      qa[0] = s;
    }
    uint32_t qn = 1;
    int32_t r = 0;
    __syncthreads();
    while (qn > 0) {
      ++r;
      if (tid == 0) s_nq = 0;
      for (uint32_t c0 = 0; c0 < qn; c0 += kBatchThreads) {
        const uint32_t i = c0 + tid;
        uint32_t beg = 0, deg = 0;
        if (i < qn) {
          const uint32_t v = qa[i];
          beg = go[v];
          deg = go[v + 1] - beg;
        }
        uint32_t total;
        const uint32_t excl = block_excl_scan(deg, s_warp, &total);
        s_scan[tid] = excl;
        s_beg[tid] = beg;
        if (tid == 0) s_scan[kBatchThreads] = total;
        __syncthreads();
        trav += (tid == 0) ? total : 0u;
        for (uint32_t t0 = 0; t0 < total; t0 += kBatchThreads) {
          const uint32_t t = t0 + tid;
          bool add = false;
          uint32_t u = 0;
          if (t < total) {
            // owner: the last slot whose exclusive start is <= t
            int lo = 0, hi = kBatchThreads - 1;
            while (lo < hi) {
              const int mid = (lo + hi + 1) >> 1;
              if (s_scan[mid] <= t)
                lo = mid;
              else
                hi = mid - 1;
            }
            u = gx[s_beg[lo] + (t - s_scan[lo])];
            if (__ldcg(lev + u) < 0) add = atomicCAS(lev + u, -1, r) == -1;
          }
          const uint32_t bal = __ballot_sync(0xffffffffu, add);
          if (bal) {
            const int leader = __ffs(bal) - 1;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(&s_nq, (uint32_t)__popc(bal));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (add) qb[base + __popc(bal & lanemask_lt)] = u;
          }
        }
        __syncthreads();
      }
      qn = s_nq;
      uint32_t* t = qa;
      qa = qb;
      qb = t;
      __syncthreads();
    }
  }
  if (tid == 0 && trav) atomicAdd(ctr + 1, trav);
}

static void batch_release(gg_graph_batch_s* b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  cudaFree(b->d_off);
  cudaFree(b->d_idx);
  cudaFree(b->d_order);
  cudaFree(b->d_src);
  cudaFree(b->d_scratch);
  cudaFree(b->d_desc);
  cudaFree(b->d_levels);
  cudaFree(b->d_ctr);
  if (b->h_src) cudaFreeHost(b->h_src);
  if (b->h_levels) cudaFreeHost(b->h_levels);
  if (b->h_ctr) cudaFreeHost(b->h_ctr);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

static int batch_build(int32_t count, const gg_host_graph* graphs, gg_graph_batch_s* b) {
  b->count = count;
  std::vector<BatchDesc> desc(count);
  uint64_t offs = 0;
  for (int32_t i = 0; i < count; ++i) {
    const gg_host_graph& h = graphs[i];
    if (h.n == 0 || !h.offsets || (h.m && !h.indices) || h.offsets[h.n] != h.m)
      return fail(GG_ERR_INVALID_ARG, "gg_batch_create: graph %d is malformed", i);
    desc[i] = BatchDesc{offs, b->total_m, b->total_n, h.n, 0};
    b->firsts.push_back(b->total_n);
    offs += (uint64_t)h.n + 1;
    b->total_m += h.m;
    b->total_n += h.n;
    b->max_n = std::max(b->max_n, h.n);
  }
  GG_CUDA(cudaGetDevice(&b->device));
  GG_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  GG_CUDA(cudaMalloc(&b->d_off, 4 * offs));
  GG_CUDA(cudaMalloc(&b->d_idx, 4 * std::max<uint64_t>(b->total_m, 1)));
  GG_CUDA(cudaMalloc(&b->d_levels, 4 * b->total_n));
  GG_CUDA(cudaMalloc(&b->d_desc, sizeof(BatchDesc) * count));
  GG_CUDA(cudaMalloc(&b->d_order, 4 * count));
  GG_CUDA(cudaMalloc(&b->d_src, 4 * count));
  GG_CUDA(cudaMalloc(&b->d_ctr, 16));
  for (int32_t i = 0; i < count; ++i) {
    const gg_host_graph& h = graphs[i];
    GG_CUDA(cudaMemcpy(b->d_off + desc[i].off_base, h.offsets, 4 * ((uint64_t)h.n + 1), cudaMemcpyHostToDevice));
    if (h.m) GG_CUDA(cudaMemcpy(b->d_idx + desc[i].idx_base, h.indices, 4 * h.m, cudaMemcpyHostToDevice));
  }
  std::vector<uint32_t> order(count);
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return graphs[x].m > graphs[y].m; });
  GG_CUDA(cudaMemcpy(b->d_desc, desc.data(), sizeof(BatchDesc) * count, cudaMemcpyHostToDevice));
  GG_CUDA(cudaMemcpy(b->d_order, order.data(), 4 * count, cudaMemcpyHostToDevice));
  int sms = 0, per_sm = 0;
  GG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
  GG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_bfs, kBatchThreads, 0));
  b->grid = std::max(1, std::min(count, sms * std::max(per_sm, 1)));
  GG_CUDA(cudaMalloc(&b->d_scratch, 8ull * b->max_n * b->grid));
  GG_CUDA(cudaMallocHost(&b->h_src, 4 * count));
  GG_CUDA(cudaMallocHost(&b->h_levels, 4 * b->total_n));
  GG_CUDA(cudaMallocHost(&b->h_ctr, 16));
  // the replayed sequence: sources up, counters reset, persistent traversal, levels and counters down
  GG_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  cudaMemcpyAsync(b->d_src, b->h_src, 4 * count, cudaMemcpyHostToDevice, b->stream);
  cudaMemsetAsync(b->d_ctr, 0, 16, b->stream);
  k_batch_bfs<<<b->grid, kBatchThreads, 0, b->stream>>>(b->d_desc, b->d_order, count, b->d_off, b->d_idx,
                                                          b->d_levels, b->d_src, b->d_ctr, b->d_scratch, b->max_n);
  cudaMemcpyAsync(b->h_levels, b->d_levels, 4 * b->total_n, cudaMemcpyDeviceToHost, b->stream);
  cudaMemcpyAsync(b->h_ctr, b->d_ctr, 16, cudaMemcpyDeviceToHost, b->stream);
  GG_CUDA(cudaStreamEndCapture(b->stream, &b->graph));
  GG_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
  return GG_OK;
}

}  // namespace gg

using namespace gg;

extern "C" {

int gg_batch_create(int32_t count, const gg_host_graph* graphs, gg_graph_batch_t* out) {
  if (count <= 0 || !graphs || !out) return fail(GG_ERR_INVALID_ARG, "gg_batch_create: bad arguments");
  int devs = 0;
  if (cudaGetDeviceCount(&devs) != cudaSuccess || devs == 0) {
    cudaGetLastError();
    return fail(GG_ERR_NO_DEVICE, "no CUDA device is visible");
  }
  gg_graph_batch_s* b = new (std::nothrow) gg_graph_batch_s;
  if (!b) return fail(GG_ERR_OOM, "batch: out of host memory");
  const int rc = batch_build(count, graphs, b);
  if (rc) {
    const std::string keep = last_error();
    cudaStreamEndCapture(b->stream, &b->graph);  // leaves no capture open on a failed build
    cudaGetLastError();
    batch_release(b);
    set_error("%s", keep.c_str());
    return rc;
  }
  {
    std::lock_guard<std::mutex> lk(g_batch_mu);
    g_batches.insert(b);
  }
  *out = b;
  return GG_OK;
}

int gg_batch_destroy(gg_graph_batch_t b) {
  {
    std::lock_guard<std::mutex> lk(g_batch_mu);
    if (!b || !g_batches.erase(b)) return fail(GG_ERR_INVALID_ARG, "gg_batch_destroy: unknown batch");
  }
  cudaStreamSynchronize(b->stream);
  batch_release(b);
  return GG_OK;
}

int gg_batch_info(gg_graph_batch_t b, uint64_t* total_vertices, uint64_t* total_edges, uint64_t* firsts) {
  if (!batch_live(b)) return fail(GG_ERR_INVALID_ARG, "gg_batch_info: unknown batch");
  if (total_vertices) *total_vertices = b->total_n;
  if (total_edges) *total_edges = b->total_m;
  if (firsts) std::copy(b->firsts.begin(), b->firsts.end(), firsts);
  return GG_OK;
}

int gg_batch_bfs(gg_graph_batch_t b, const uint32_t* sources, int32_t* levels, gg_run_stats* st) {
  if (!batch_live(b) || !sources) return fail(GG_ERR_INVALID_ARG, "gg_batch_bfs: bad arguments");
  for (int32_t i = 0; i < b->count; ++i) {
    const uint64_t n = (i + 1 < b->count ? b->firsts[i + 1] : b->total_n) - b->firsts[i];
    if (sources[i] >= n) return fail(GG_ERR_INVALID_ARG, "gg_batch_bfs: source %u of graph %d out of range", sources[i], i);
  }
  std::copy(sources, sources + b->count, b->h_src);
  EventTimer tm(b->stream);
  GG_CUDA(cudaGraphLaunch(b->exec, b->stream));
  const double ms = tm.stop();
  GG_CUDA(cudaStreamSynchronize(b->stream));
  GG_CUDA(cudaGetLastError());
  if (levels) std::copy(b->h_levels, b->h_levels + b->total_n, levels);
  if (st) {
    st->ms = ms;
    st->rounds = 1;
    st->edges_traversed = b->h_ctr[1];
    st->kernels = 1;
  }
  return GG_OK;
}

}  // extern "C"
