// Device graph construction (partitioned_graph, graphgrind/graph-numa.h:642-685)
// and the vertexSubset C API (partitioned_vertices, graphgrind/ligra-numa.h:91-272).
//
// Layout in HBM (uint32 ids and offsets):
//   CSR  out_off[n+1], out_idx[m(+16 pad)], out_w[m]      (forward push)
//   CSC  in_off[n+1],  in_idx[m(+16 pad)],  in_w[m]       (dense pull); shared with
//        the CSR arrays when the graph is symmetric
//   COO  per destination tile, Hilbert (or source-major) ordered inside the
//        reference partition, padded to 8 edges: src[], dloc[] (u16 offset of
//        the destination inside its tile), w[]
//   tiles {v0, nv, e0, ne} per CTA work item, largest first.
#include <cub/cub.cuh>

#include <algorithm>
#include <mutex>
#include <numeric>
#include <unordered_set>
#include <vector>

#include "gg_hilbert.h"
#include "gg_runtime.cuh"

namespace gg {

// ------------------------------------------------------------ memory pools
constexpr int kPoolDevices = 16;
static std::mutex g_pool_mu;
static cudaMemPool_t g_pools[kPoolDevices];
static bool g_pool_failed[kPoolDevices];

static cudaMemPool_t lib_pool(int device) {
  if (device < 0 || device >= kPoolDevices) return nullptr;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pools[device] && !g_pool_failed[device]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
      cudaGetLastError();
      g_pool_failed[device] = true;
      return nullptr;
    }
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    g_pools[device] = pool;
  }
  return g_pools[device];
}

__global__ void k_get_words(uint32_t* dst, const uint32_t* src, uint32_t words) {
  for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) dst[i] = __ldcg(src + i);
}

cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t s, int device) {
  cudaMemPool_t pool = lib_pool(device);
  return pool ? cudaMallocFromPoolAsync(p, bytes, pool, s) : cudaMallocAsync(p, bytes, s);
}

void pool_trim(int device) {
  if (device < 0 || device >= kPoolDevices) return;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (g_pools[device]) cudaMemPoolTrimTo(g_pools[device], 0);
}

static std::mutex g_reg_mu;
static std::unordered_set<const gg_graph_s*> g_graphs;
static std::unordered_set<const gg_frontier_s*> g_frontiers;

bool graph_live(const gg_graph_s* g) {
  std::lock_guard<std::mutex> lk(g_reg_mu);
  return g && g_graphs.count(g);
}
bool frontier_live(const gg_frontier_s* f) {
  std::lock_guard<std::mutex> lk(g_reg_mu);
  return f && g_frontiers.count(f);
}

template <class T>
static int dev_alloc(gg_graph_s* g, T** p, size_t count) {
  size_t bytes = sizeof(T) * std::max<size_t>(count, 1);
  cudaError_t e = cudaMalloc((void**)p, bytes);
  if (e != cudaSuccess) return fail(GG_ERR_OOM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
  g->device_bytes += bytes;
  return GG_OK;
}

// ------------------------------------------------------------- frontiers
int frontier_new(gg_graph_s* g, gg_frontier_s** out) {
  gg_frontier_s* f = new (std::nothrow) gg_frontier_s;
  if (!f) return fail(GG_ERR_OOM, "frontier: out of host memory");
  f->g = g;
  f->n = g->n;
  {
    std::lock_guard<std::mutex> lk(g_reg_mu);
    g_frontiers.insert(f);
  }
  g->frontiers.insert(f);
  *out = f;
  return GG_OK;
}

int frontier_ensure_bits(gg_frontier_s* f, bool zero) {
  gg_graph_s* g = f->g;
  const size_t bytes = sizeof(uint32_t) * ((size_t)g->words() + 4);
  if (!f->d_bits) GG_CUDA(pool_alloc((void**)&f->d_bits, bytes, g->stream, g->device));
  if (zero) GG_CUDA(cudaMemsetAsync(f->d_bits, 0, bytes, g->stream));
  return GG_OK;
}

int frontier_ensure_queue(gg_frontier_s* f) {
  gg_graph_s* g = f->g;
  if (!f->d_queue)
    GG_CUDA(pool_alloc((void**)&f->d_queue, sizeof(uint32_t) * ((size_t)g->n + 4), g->stream, g->device));
  return GG_OK;
}

void frontier_free(gg_frontier_s* f) {
  if (!f) return;
  gg_graph_s* g = f->g;
  {
    std::lock_guard<std::mutex> lk(g_reg_mu);
    g_frontiers.erase(f);
  }
  g->frontiers.erase(f);
  if (f->d_bits) cudaFreeAsync(f->d_bits, g->stream);
  if (f->d_queue) cudaFreeAsync(f->d_queue, g->stream);
  delete f;
}

__global__ void k_all_bits(uint32_t* bits, uint32_t n) {
  const uint32_t words = (n + 31) / 32;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t rem = n - (uint32_t)i * 32;
    bits[i] = rem >= 32 ? 0xffffffffu : ((1u << rem) - 1u);
  }
}

// toDense, graphgrind/ligra-numa.h:228-244
int frontier_to_dense(gg_frontier_s* f) {
  gg_graph_s* g = f->g;
  if (f->has_dense) return GG_OK;
  GG_TRY(frontier_ensure_bits(f, true));
  if (f->bit) {
    k_all_bits<<<generic_grid(g, g->words()), kGenericThreads, 0, g->stream>>>(f->d_bits, g->n);
  } else if (f->has_sparse && f->dm) {
    k_queue_to_bits<<<generic_grid(g, f->dm), kGenericThreads, 0, g->stream>>>(f->d_queue, f->dm, f->d_bits);
  }
  GG_CUDA(cudaGetLastError());
  g->kernels++;
  f->has_dense = true;
  return GG_OK;
}

// toSparse, graphgrind/ligra-numa.h:246-260 (packIndex -> ballot compaction)
int frontier_to_sparse(gg_frontier_s* f) {
  gg_graph_s* g = f->g;
  if (f->has_sparse) return GG_OK;
  GG_TRY(frontier_ensure_queue(f));
  if (f->bit) {
    k_iota<<<generic_grid(g, g->n), kGenericThreads, 0, g->stream>>>(f->d_queue, g->n);
    GG_CUDA(cudaGetLastError());
    g->kernels++;
    f->has_sparse = true;
    return GG_OK;
  }
  if (!f->has_dense || f->dm == 0) {
    f->has_sparse = true;
    return GG_OK;
  }
  GG_TRY(reset_stats(g));
  k_bits_to_queue<<<generic_grid(g, g->words()), kGenericThreads, 0, g->stream>>>(f->d_bits, g->words(), f->d_queue,
                                                                                g->ws.d_stats + 2);
  GG_CUDA(cudaGetLastError());
  g->kernels++;
  GG_TRY(read_stats(g));
  if (g->ws.h_stats[2] != f->dm)
    return fail(GG_ERR_INVALID_ARG, "bad stored value of m: frontier holds %llu vertices, stats say %llu",
                (unsigned long long)g->ws.h_stats[2], (unsigned long long)f->dm);
  f->has_sparse = true;
  return GG_OK;
}

int reset_stats(gg_graph_s* g) {
  GG_CUDA(cudaMemsetAsync(g->ws.d_stats, 0, sizeof(unsigned long long) * 8, g->stream));
  return GG_OK;
}

int read_stats(gg_graph_s* g) {
  GG_TRY(read_small(g, g->ws.h_stats, g->ws.d_stats, 8));
  if (g->ws.h_stats[3])
    return fail(GG_ERR_TIMEOUT, "device wait budget exhausted (error word %llu)", (unsigned long long)g->ws.h_stats[3]);
  return GG_OK;
}

// ------------------------------------------------------------------ tiles
// Greedy destination tiles over [vbeg, vend): at most tv vertices and about
// te edges (a single vertex above te gets its own tile); edge-less ranges
// are dropped (their vertices can never be updated by a pull).
static void make_tiles(const uint32_t* off, uint32_t vbeg, uint32_t vend, uint32_t tv, uint64_t te,
                       std::vector<uint4>& out) {
  uint32_t v = vbeg;
  while (v < vend) {
    const uint32_t t0 = v;
    uint64_t ne = 0;
    while (v < vend && v - t0 < tv) {
      const uint64_t d = off[v + 1] - off[v];
      if (v > t0 && ne + d > te) break;
      ne += d;
      ++v;
    }
    if (ne > 0) out.push_back(make_uint4(t0, v - t0, off[t0], (uint32_t)ne));
  }
}

// Head bits, per-block head counts and the compressed row list of the edge
// stream described by host offsets `off` (n+1 entries), see SegIndex.
static int build_seg(gg_graph_s* g, const uint32_t* off, SegIndex& si) {
  const uint32_t n = g->n;
  const uint64_t nwords = g->m_pad / 32;
  const uint64_t nblk = g->m_pad / kSegBlock;
  std::vector<uint32_t> head(nwords, 0), blk(nblk + 1, 0), rows;
  rows.reserve(n);
  for (uint32_t v = 0; v < n; ++v) {
    if (off[v + 1] == off[v]) continue;
    const uint32_t e = off[v];
    head[e >> 5] |= 1u << (e & 31);
    blk[e / kSegBlock + 1]++;
    rows.push_back(v);
  }
  for (uint64_t b = 0; b < nblk; ++b) blk[b + 1] += blk[b];
  si.nrows = rows.size();
  rows.resize(rows.size() + 8, 0);
  GG_TRY(dev_alloc(g, &si.d_head, nwords));
  GG_TRY(dev_alloc(g, &si.d_blk, nblk + 1));
  GG_TRY(dev_alloc(g, &si.d_rows, rows.size()));
  GG_CUDA(cudaMemcpy(si.d_head, head.data(), 4 * nwords, cudaMemcpyHostToDevice));
  GG_CUDA(cudaMemcpy(si.d_blk, blk.data(), 4 * (nblk + 1), cudaMemcpyHostToDevice));
  GG_CUDA(cudaMemcpy(si.d_rows, rows.data(), 4 * rows.size(), cudaMemcpyHostToDevice));
  return GG_OK;
}

static int upload_tiles(gg_graph_s* g, TileSet& ts, std::vector<uint4>& tiles) {
  std::stable_sort(tiles.begin(), tiles.end(), [](const uint4& a, const uint4& b) { return a.w > b.w; });
  ts.host = tiles;
  ts.count = (uint32_t)tiles.size();
  GG_TRY(dev_alloc(g, &ts.d_tiles, tiles.size()));
  if (!tiles.empty())
    GG_CUDA(cudaMemcpy(ts.d_tiles, tiles.data(), sizeof(uint4) * tiles.size(), cudaMemcpyHostToDevice));
  return GG_OK;
}

// ------------------------------------------------------- COO construction
__global__ void k_edge_dst(const uint32_t* off, uint32_t n, uint32_t* dst) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
    for (uint32_t j = off[v]; j < off[v + 1]; ++j) dst[j] = (uint32_t)v;
}

// sort key of every CSC edge inside its partition: Hilbert (EDGES_HILBERT=1,
// graphgrind/graph-numa.h:482-490) or (src, dst) (CSRDestSort, :338-350)
__global__ void k_coo_keys(const uint32_t* src, const uint32_t* dst, uint64_t m, const int64_t* starts, int P,
                           const int64_t* part_side, int hilbert, uint64_t* keys, uint32_t* vals) {
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t d = dst[j], s = src[j];
    uint64_t key;
    if (hilbert) {
      int lo = 0, hi = P;  // partition p with starts[p] <= d < starts[p+1]
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (starts[mid] <= (int64_t)d) lo = mid; else hi = mid;
      }
      key = (uint64_t)hilbert_xy2d(part_side[lo], (int64_t)s, (int64_t)d);
    } else {
      key = ((uint64_t)s << 32) | d;
    }
    keys[j] = key;
    vals[j] = (uint32_t)j;
  }
}

// Second-level order inside a tile: positions keep their 256-edge window of
// the Hilbert order, and inside a window edges go by destination, so that a
// thread's 8 consecutive edges form destination runs while the window keeps
// the Hilbert locality of its sources.  key = window << dbits | local
// destination (dbits covers the tile width).
__global__ void k_coo_window_keys(const uint4* seg, uint32_t ntiles, const uint32_t* perm, const uint32_t* dst,
                                  uint32_t window, uint32_t dbits, uint32_t* keys) {
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint4 s = seg[t];  // {v0, nv, e0 (CSC), ne}
    for (uint32_t i = threadIdx.x; i < s.w; i += blockDim.x)
      keys[s.z + i] = ((i / window) << dbits) | (dst[perm[s.z + i]] - s.x);
  }
}

// Alternative second-level order: windows of W edges of the Hilbert order,
// sources ascending inside a window, so that 32 consecutive edges gather from
// few cache lines.  key = window << 32 | source.
__global__ void k_coo_window_src_keys(const uint4* seg, uint32_t ntiles, const uint32_t* perm, const uint32_t* src,
                                      uint32_t window, uint64_t* keys) {
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint4 s = seg[t];  // {v0, nv, e0 (CSC), ne}
    for (uint32_t i = threadIdx.x; i < s.w; i += blockDim.x)
      keys[s.z + i] = ((uint64_t)(i / window) << 32) | src[perm[s.z + i]];
  }
}

// scatter sorted tile segments into their padded COO slots
__global__ void k_coo_scatter(const uint4* seg, const uint32_t* pad_start, uint32_t ntiles, const uint32_t* perm,
                              const uint32_t* src, const uint32_t* dst, const uint32_t* w, uint32_t* coo_src,
                              uint16_t* coo_dloc, uint32_t* coo_w) {
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint4 s = seg[t];  // {v0, nv, e0 (CSC), ne}
    const uint32_t base = pad_start[t];
    for (uint32_t i = threadIdx.x; i < s.w; i += blockDim.x) {
      const uint32_t j = perm[s.z + i];
      coo_src[base + i] = src[j];
      coo_dloc[base + i] = (uint16_t)(dst[j] - s.x);
      if (w) coo_w[base + i] = w[j];
    }
  }
}

// ---------------------------------------- in-lists for the bottom-up BFS
// key of a CSC edge: the complement of its source's out-degree, so that an
// ascending sort puts the sources with the most out-edges first
__global__ void k_bu_keys(const uint32_t* src, uint64_t m, const uint32_t* out_off, uint32_t* keys) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = src[e];
    keys[e] = ~(out_off[s + 1] - out_off[s]);
  }
}

int build_bu_index(gg_graph_s* g) {
  if (g->d_bu_idx) return GG_OK;
  const uint64_t m = g->m;
  const uint32_t n = g->n;
  if (m >= (1ull << 31)) return fail(GG_ERR_UNSUPPORTED, "bottom-up in-lists: more than 2^31 edges");
  uint32_t* out = nullptr;
  GG_TRY(dev_alloc(g, &out, g->m_pad));
  // the copy is kept only once it is complete
  auto build = [&]() -> int {
    GG_CUDA(cudaMemsetAsync(out + m, 0, 4ull * (g->m_pad - m), g->stream));
    if (m == 0) return GG_OK;
    DevBuf<uint32_t> keys, keys_out;
    GG_TRY(keys.alloc(g, m));
    GG_TRY(keys_out.alloc(g, m));
    k_bu_keys<<<generic_grid(g, m), kGenericThreads, 0, g->stream>>>(g->d_csc_idx, m, g->d_csr_off, keys.p);
    GG_CUDA(cudaGetLastError());
    size_t temp = 0;
    GG_CUDA(cub::DeviceSegmentedSort::StableSortPairs(nullptr, temp, keys.p, keys_out.p, g->d_csc_idx, out, (int)m,
                                                       (int)n, g->d_csc_off, g->d_csc_off + 1, g->stream));
    DevBuf<unsigned char> tmp;
    GG_TRY(tmp.alloc(g, temp));
    GG_CUDA(cub::DeviceSegmentedSort::StableSortPairs(tmp.p, temp, keys.p, keys_out.p, g->d_csc_idx, out, (int)m,
                                                       (int)n, g->d_csc_off, g->d_csc_off + 1, g->stream));
    return GG_OK;
  };
  const int rc = build();
  if (rc) {
    cudaStreamSynchronize(g->stream);
    cudaFree(out);
    g->device_bytes -= 4ull * g->m_pad;
    return rc;
  }
  g->d_bu_idx = out;
  return GG_OK;
}

static int build_coo(gg_graph_s* g, const uint32_t* h_in_off) {
  const uint32_t n = g->n;
  const uint64_t m = g->m;
  const int P = (int)g->coo_sizes.size();
  const uint32_t tv = (uint32_t)g->opts.coo_tile_vertices;
  const uint64_t te = (uint64_t)g->opts.tile_edges;
  std::vector<uint4> segs;  // in vertex order
  for (int p = 0; p < P; ++p)
    make_tiles(h_in_off, (uint32_t)g->coo_starts[p], (uint32_t)g->coo_starts[p + 1], tv, te, segs);
  // padded placement
  std::vector<uint32_t> pad_start(segs.size());
  uint64_t pos = 0;
  for (size_t t = 0; t < segs.size(); ++t) {
    pad_start[t] = (uint32_t)pos;
    pos += (segs[t].w + 7u) & ~7u;
  }
  if (pos + 16 >= (1ull << 31)) return fail(GG_ERR_SIZE, "padded COO exceeds the 2^31-edge sort limit");
  // 32-bit window keys: the local destination in dbits bits, the window above
  uint32_t dbits = 1;
  while ((1u << dbits) < tv) ++dbits;
  for (const uint4& sg : segs)
    if (g->opts.coo_window == 0 && (uint64_t)sg.w / (uint64_t)g->opts.coo_dst_window >= (1ull << (32 - dbits)))
      return fail(GG_ERR_SIZE, "a COO tile of %u edges exceeds the window-key range", sg.w);
  g->coo_len = pos;
  GG_TRY(dev_alloc(g, &g->d_coo_src, pos + 16));
  GG_TRY(dev_alloc(g, &g->d_coo_dloc, pos + 16));
  if (g->wtype != GG_W_NONE) GG_TRY(dev_alloc(g, &g->d_coo_w, pos + 16));
  GG_CUDA(cudaMemset(g->d_coo_src, 0xff, sizeof(uint32_t) * (pos + 16)));
  GG_CUDA(cudaMemset(g->d_coo_dloc, 0, sizeof(uint16_t) * (pos + 16)));
  if (g->d_coo_w) GG_CUDA(cudaMemset(g->d_coo_w, 0, sizeof(uint32_t) * (pos + 16)));
  // partition grid sides: roundUpPow2(edges of partition p)
  std::vector<int64_t> side(P);
  for (int p = 0; p < P; ++p) {
    const int64_t ne = (int64_t)h_in_off[g->coo_starts[p + 1]] - (int64_t)h_in_off[g->coo_starts[p]];
    side[p] = hilbert_side(ne);
  }
  uint32_t *d_dst = nullptr, *d_vals = nullptr, *d_perm = nullptr, *d_pad = nullptr;
  uint64_t *d_keys = nullptr, *d_keys_out = nullptr;
  int64_t *d_starts = nullptr, *d_side = nullptr;
  uint4* d_segs = nullptr;
  int* d_seg_begin = nullptr;
  void* d_temp = nullptr;
  size_t temp_bytes = 0;
  int rc = GG_OK;
  auto cleanup = [&]() {
    cudaFree(d_dst); cudaFree(d_vals); cudaFree(d_perm); cudaFree(d_pad); cudaFree(d_keys);
    cudaFree(d_keys_out); cudaFree(d_starts); cudaFree(d_side); cudaFree(d_segs); cudaFree(d_seg_begin);
    cudaFree(d_temp);
  };
#define GG_BUILD(call)                                                                      \
  do {                                                                                      \
    cudaError_t e__ = (call);                                                               \
    if (e__ != cudaSuccess) {                                                               \
      rc = fail(GG_ERR_CUDA, "COO build: %s: %s", #call, cudaGetErrorString(e__));          \
      cleanup();                                                                            \
      return rc;                                                                            \
    }                                                                                       \
  } while (0)
  const uint64_t mm = std::max<uint64_t>(m, 1);
  GG_BUILD(cudaMalloc(&d_dst, 4 * mm));
  GG_BUILD(cudaMalloc(&d_vals, 4 * mm));
  GG_BUILD(cudaMalloc(&d_perm, 4 * mm));
  GG_BUILD(cudaMalloc(&d_keys, 8 * mm));
  GG_BUILD(cudaMalloc(&d_keys_out, 8 * mm));
  GG_BUILD(cudaMalloc(&d_starts, 8 * (P + 1)));
  GG_BUILD(cudaMalloc(&d_side, 8 * P));
  GG_BUILD(cudaMalloc(&d_segs, sizeof(uint4) * std::max<size_t>(segs.size(), 1)));
  GG_BUILD(cudaMalloc(&d_pad, 4 * std::max<size_t>(segs.size(), 1)));
  GG_BUILD(cudaMalloc(&d_seg_begin, sizeof(int) * (segs.size() + 1)));
  GG_BUILD(cudaMemcpy(d_starts, g->coo_starts.data(), 8 * (P + 1), cudaMemcpyHostToDevice));
  GG_BUILD(cudaMemcpy(d_side, side.data(), 8 * P, cudaMemcpyHostToDevice));
  if (!segs.empty()) {
    GG_BUILD(cudaMemcpy(d_segs, segs.data(), sizeof(uint4) * segs.size(), cudaMemcpyHostToDevice));
    GG_BUILD(cudaMemcpy(d_pad, pad_start.data(), 4 * segs.size(), cudaMemcpyHostToDevice));
  }
  // segment boundaries: tile edge ranges are contiguous and cover [0, m)
  std::vector<int> seg_begin(segs.size() + 1);
  for (size_t t = 0; t < segs.size(); ++t) seg_begin[t] = (int)segs[t].z;
  seg_begin[segs.size()] = (int)m;
  GG_BUILD(cudaMemcpy(d_seg_begin, seg_begin.data(), sizeof(int) * seg_begin.size(), cudaMemcpyHostToDevice));
  const int grid = g->num_sms * 8;
  k_edge_dst<<<grid, 256>>>(g->d_csc_off, n, d_dst);
  k_coo_keys<<<grid, 256>>>(g->d_csc_idx, d_dst, m, d_starts, P, d_side, g->opts.order == GG_ORDER_HILBERT ? 1 : 0,
                            d_keys, d_vals);
  GG_BUILD(cudaGetLastError());
  if (!segs.empty()) {
    GG_BUILD(cub::DeviceSegmentedRadixSort::SortPairs(nullptr, temp_bytes, d_keys, d_keys_out, d_vals, d_perm, (int)m,
                                                      (int)segs.size(), d_seg_begin, d_seg_begin + 1));
    GG_BUILD(cudaMalloc(&d_temp, temp_bytes));
    GG_BUILD(cub::DeviceSegmentedRadixSort::SortPairs(d_temp, temp_bytes, d_keys, d_keys_out, d_vals, d_perm, (int)m,
                                                      (int)segs.size(), d_seg_begin, d_seg_begin + 1));
    if (g->opts.coo_window > 0) {
      // source order inside windows of coo_window edges (64-bit keys)
      k_coo_window_src_keys<<<grid, 256>>>(d_segs, (uint32_t)segs.size(), d_perm, g->d_csc_idx,
                                           (uint32_t)g->opts.coo_window, d_keys);
      GG_BUILD(cudaGetLastError());
      size_t temp2 = 0;
      GG_BUILD(cub::DeviceSegmentedRadixSort::SortPairs(nullptr, temp2, d_keys, d_keys_out, d_perm, d_vals, (int)m,
                                                        (int)segs.size(), d_seg_begin, d_seg_begin + 1));
      if (temp2 > temp_bytes) {
        cudaFree(d_temp);
        d_temp = nullptr;
        GG_BUILD(cudaMalloc(&d_temp, temp2));
        temp_bytes = temp2;
      }
      GG_BUILD(cub::DeviceSegmentedRadixSort::SortPairs(d_temp, temp2, d_keys, d_keys_out, d_perm, d_vals, (int)m,
                                                        (int)segs.size(), d_seg_begin, d_seg_begin + 1));
    } else {
      // destination order inside 256-edge windows (the u64 key buffers are reused as u32)
      uint32_t* k32 = reinterpret_cast<uint32_t*>(d_keys);
      uint32_t* k32_out = reinterpret_cast<uint32_t*>(d_keys_out);
      k_coo_window_keys<<<grid, 256>>>(d_segs, (uint32_t)segs.size(), d_perm, d_dst,
                                       (uint32_t)g->opts.coo_dst_window, dbits, k32);
      GG_BUILD(cudaGetLastError());
      size_t temp2 = 0;
      GG_BUILD(cub::DeviceSegmentedRadixSort::SortPairs(nullptr, temp2, k32, k32_out, d_perm, d_vals, (int)m,
                                                        (int)segs.size(), d_seg_begin, d_seg_begin + 1));
      if (temp2 > temp_bytes) {
        cudaFree(d_temp);
        d_temp = nullptr;
        GG_BUILD(cudaMalloc(&d_temp, temp2));
        temp_bytes = temp2;
      }
      GG_BUILD(cub::DeviceSegmentedRadixSort::SortPairs(d_temp, temp2, k32, k32_out, d_perm, d_vals, (int)m,
                                                        (int)segs.size(), d_seg_begin, d_seg_begin + 1));
    }
    k_coo_scatter<<<grid, 256>>>(d_segs, d_pad, (uint32_t)segs.size(), d_vals, g->d_csc_idx, d_dst, g->d_csc_w,
                                 g->d_coo_src, g->d_coo_dloc, g->d_coo_w);
    GG_BUILD(cudaGetLastError());
  }
  GG_BUILD(cudaDeviceSynchronize());
#undef GG_BUILD
  cleanup();
  // work items: padded segments
  std::vector<uint4> tiles(segs.size());
  for (size_t t = 0; t < segs.size(); ++t)
    tiles[t] = make_uint4(segs[t].x, segs[t].y, pad_start[t], (segs[t].w + 7u) & ~7u);
  GG_TRY(upload_tiles(g, g->coo_tiles, tiles));
  // destination ranges that no tile covers (no in-edges at all): a vertex
  // step run at the tiles' commits visits them separately
  std::vector<uint2> gaps;
  uint32_t covered = 0;
  for (const uint4& sg : segs) {
    if (sg.x > covered) gaps.push_back(make_uint2(covered, sg.x - covered));
    covered = sg.x + sg.y;
  }
  if (covered < n) gaps.push_back(make_uint2(covered, n - covered));
  g->coo_gap_count = (uint32_t)gaps.size();
  if (!gaps.empty()) {
    GG_TRY(dev_alloc(g, &g->d_coo_gaps, gaps.size()));
    GG_CUDA(cudaMemcpy(g->d_coo_gaps, gaps.data(), sizeof(uint2) * gaps.size(), cudaMemcpyHostToDevice));
  }
  g->has_coo = true;
  if (g->opts.coo_window > 0) g->coo_kernel = 4;  // the lane-contiguous pull matches source-ordered windows
  return GG_OK;
}

// -P source (COOPartitionBySour, graphgrind/graph-numa.h:1145-1171): partition
// p holds the out-edges of the sources in [coo_starts[p], coo_starts[p+1]),
// which are contiguous in the CSR; they are Hilbert-ordered inside the
// partition with the same key as the destination form (or left in CSR order).
__global__ void k_coo_src_keys(const uint32_t* src, const uint32_t* dst, uint64_t m, const int64_t* starts, int P,
                               const int64_t* part_side, int hilbert, uint64_t* keys, uint32_t* vals) {
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < m; j += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = src[j], d = dst[j];
    uint64_t key;
    if (hilbert) {
      int lo = 0, hi = P;  // partition p with starts[p] <= s < starts[p+1]
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (starts[mid] <= (int64_t)s) lo = mid; else hi = mid;
      }
      key = (uint64_t)hilbert_xy2d(part_side[lo], (int64_t)s, (int64_t)d);
    } else {
      key = ((uint64_t)s << 32) | d;
    }
    keys[j] = key;
    vals[j] = (uint32_t)j;
  }
}

__global__ void k_coo_src_scatter(uint64_t m, const uint32_t* perm, const uint32_t* src, const uint32_t* dst,
                                  const uint32_t* w, uint32_t* coo_src, uint32_t* coo_dst, uint32_t* coo_w) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t j = perm[i];
    coo_src[i] = src[j];
    coo_dst[i] = dst[j];
    if (w) coo_w[i] = w[j];
  }
}

static int build_coo_src(gg_graph_s* g) {
  const uint32_t n = g->n;
  const uint64_t m = g->m;
  const int P = (int)g->coo_sizes.size();
  const uint32_t* off = g->h_csr_off.data();
  if (m >= (1ull << 31)) return fail(GG_ERR_SIZE, "source-partitioned COO exceeds the 2^31-edge sort limit");
  std::vector<int64_t> side(P);
  std::vector<int> seg_begin(P + 1);
  for (int p = 0; p < P; ++p) {
    seg_begin[p] = (int)off[g->coo_starts[p]];
    side[p] = hilbert_side((int64_t)off[g->coo_starts[p + 1]] - (int64_t)off[g->coo_starts[p]]);
  }
  seg_begin[P] = (int)m;
  GG_TRY(dev_alloc(g, &g->d_coo_src, m + 16));
  GG_TRY(dev_alloc(g, &g->d_coo_dst, m + 16));
  if (g->wtype != GG_W_NONE) GG_TRY(dev_alloc(g, &g->d_coo_w, m + 16));
  uint32_t *d_src = nullptr, *d_vals = nullptr, *d_perm = nullptr;
  uint64_t *d_keys = nullptr, *d_keys_out = nullptr;
  int64_t *d_starts = nullptr, *d_side = nullptr;
  int* d_seg = nullptr;
  void* d_temp = nullptr;
  size_t temp_bytes = 0;
  int rc = GG_OK;
  auto cleanup = [&]() {
    cudaFree(d_src); cudaFree(d_vals); cudaFree(d_perm); cudaFree(d_keys); cudaFree(d_keys_out);
    cudaFree(d_starts); cudaFree(d_side); cudaFree(d_seg); cudaFree(d_temp);
  };
#define GG_BUILD(call)                                                                      \
  do {                                                                                      \
    cudaError_t e__ = (call);                                                               \
    if (e__ != cudaSuccess) {                                                               \
      rc = fail(GG_ERR_CUDA, "COO build: %s: %s", #call, cudaGetErrorString(e__));          \
      cleanup();                                                                            \
      return rc;                                                                            \
    }                                                                                       \
  } while (0)
  GG_BUILD(cudaMalloc(&d_src, 4 * m));
  GG_BUILD(cudaMalloc(&d_vals, 4 * m));
  GG_BUILD(cudaMalloc(&d_perm, 4 * m));
  GG_BUILD(cudaMalloc(&d_keys, 8 * m));
  GG_BUILD(cudaMalloc(&d_keys_out, 8 * m));
  GG_BUILD(cudaMalloc(&d_starts, 8 * (P + 1)));
  GG_BUILD(cudaMalloc(&d_side, 8 * P));
  GG_BUILD(cudaMalloc(&d_seg, sizeof(int) * (P + 1)));
  GG_BUILD(cudaMemcpy(d_starts, g->coo_starts.data(), 8 * (P + 1), cudaMemcpyHostToDevice));
  GG_BUILD(cudaMemcpy(d_side, side.data(), 8 * P, cudaMemcpyHostToDevice));
  GG_BUILD(cudaMemcpy(d_seg, seg_begin.data(), sizeof(int) * (P + 1), cudaMemcpyHostToDevice));
  const int grid = g->num_sms * 8;
  k_edge_dst<<<grid, 256>>>(g->d_csr_off, n, d_src);  // the row (source) of every CSR edge
  k_coo_src_keys<<<grid, 256>>>(d_src, g->d_csr_idx, m, d_starts, P, d_side,
                                g->opts.order == GG_ORDER_HILBERT ? 1 : 0, d_keys, d_vals);
  GG_BUILD(cudaGetLastError());
  GG_BUILD(cub::DeviceSegmentedRadixSort::SortPairs(nullptr, temp_bytes, d_keys, d_keys_out, d_vals, d_perm, (int)m,
                                                    P, d_seg, d_seg + 1));
  GG_BUILD(cudaMalloc(&d_temp, temp_bytes));
  GG_BUILD(cub::DeviceSegmentedRadixSort::SortPairs(d_temp, temp_bytes, d_keys, d_keys_out, d_vals, d_perm, (int)m,
                                                    P, d_seg, d_seg + 1));
  k_coo_src_scatter<<<grid, 256>>>(m, d_perm, d_src, g->d_csr_idx, g->d_csr_w, g->d_coo_src, g->d_coo_dst,
                                   g->d_coo_w);
  GG_BUILD(cudaGetLastError());
  GG_BUILD(cudaDeviceSynchronize());
#undef GG_BUILD
  cleanup();
  g->coo_len = m;
  g->coo_by_source = true;
  g->has_coo = true;
  return GG_OK;
}

static void graph_release(gg_graph_s* g) {
  if (!g) return;
  {
    std::lock_guard<std::mutex> lk(g_reg_mu);
    g_graphs.erase(g);
  }
  // frontiers and vertex arrays still alive die with their graph
  const std::vector<gg_frontier_s*> fl(g->frontiers.begin(), g->frontiers.end());
  for (gg_frontier_s* f : fl) frontier_free(f);
  if (g->stream) cudaStreamSynchronize(g->stream);
  if (g->copy_stream) cudaStreamSynchronize(g->copy_stream);
  pr_loop_free(g);
  round_loops_free(g);
  for (void* a : g->arrays) cudaFree(a);
  g->arrays.clear();
  cudaFree(g->d_csr_off);
  cudaFree(g->d_csr_idx);
  cudaFree(g->d_csr_w);
  if (!g->symmetric) {
    cudaFree(g->d_csc_off);
    cudaFree(g->d_csc_idx);
    cudaFree(g->d_csc_w);
  }
  for (auto& t : g->csc_tiles) cudaFree(t.d_tiles);
  for (auto& s : g->seg) {
    cudaFree(s.d_head);
    cudaFree(s.d_blk);
    cudaFree(s.d_rows);
  }
  cudaFree(g->coo_tiles.d_tiles);
  cudaFree(g->d_coo_gaps);
  cudaFree(g->d_coo_src);
  cudaFree(g->d_coo_dloc);
  cudaFree(g->d_coo_dst);
  cudaFree(g->d_coo_w);
  cudaFree(g->ws.d_stats);
  cudaFree(g->ws.d_dedup);
  cudaFree(g->ws.d_scan);
  cudaFree(g->ws.d_bsum);
  cudaFree(g->ws.d_red);
  cudaFree(g->ws.d_loop);
  cudaFree(g->d_bu_idx);
  cudaFree(g->d_new_of_old);
  cudaFree(g->d_old_of_new);
  for (auto* a : g->ws.d_order) cudaFree(a);
  if (g->ws.h_stats) cudaFreeHost(g->ws.h_stats);
  if (g->ws.h_red) cudaFreeHost(g->ws.h_red);
  if (g->ws.h_map) cudaFreeHost(g->ws.h_map);
  for (auto& e : g->prof_ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : g->slot_copied)
    if (e) cudaEventDestroy(e);
  if (g->result_ready) cudaEventDestroy(g->result_ready);
  if (g->input_ready) cudaEventDestroy(g->input_ready);
  if (g->copy_stream) cudaStreamDestroy(g->copy_stream);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
}

static int graph_build(const gg_host_graph* hg_given, const gg_build_opts* opts_in, gg_graph_s* g) {
  const gg_host_graph* hg = hg_given;
  const uint32_t n = hg->n;
  const uint64_t m = hg->m;
  gg_build_opts o{};
  if (opts_in) o = *opts_in;
  if (o.vertex_order != GG_VORDER_GIVEN && o.vertex_order != GG_VORDER_HOT_FIRST)
    return fail(GG_ERR_INVALID_ARG, "gg_graph_build: unknown vertex_order %d", o.vertex_order);
  if (o.num_partitions <= 0) o.num_partitions = 384;
  if (o.tile_vertices <= 0 || o.tile_vertices > kMaxTileVertices) o.tile_vertices = kMaxTileVertices;
  if (o.coo_tile_vertices <= 0) o.coo_tile_vertices = o.tile_vertices;
  if (o.coo_tile_vertices > kMaxCooTileVertices) o.coo_tile_vertices = kMaxCooTileVertices;
  if (o.tile_edges <= 0) o.tile_edges = 1 << 16;
  if (o.coo_window < 0) o.coo_window = 0;
  if (o.coo_window > 0) o.coo_window = (o.coo_window + kSegBlock - 1) / kSegBlock * kSegBlock;
  if (o.coo_dst_window <= 0) o.coo_dst_window = kSegBlock;
  o.coo_dst_window = std::min((o.coo_dst_window + kSegBlock - 1) / kSegBlock * kSegBlock, 1 << 16);
  if (o.order != GG_ORDER_CSR) o.order = GG_ORDER_HILBERT;
  g->opts = o;
  g->n = n;
  g->m = m;
  g->symmetric = hg->symmetric != 0;
  g->wtype = hg->weights ? hg->weight_type : GG_W_NONE;
  GG_CUDA(cudaGetDevice(&g->device));
  GG_CUDA(cudaDeviceGetAttribute(&g->num_sms, cudaDevAttrMultiProcessorCount, g->device));
  GG_CUDA(cudaStreamCreate(&g->stream));
  // CSC on the host: deterministic in-lists ordered by source id
  gg_host_graph csc{};
  const gg_host_graph* in = hg;
  if (!g->symmetric) {
    GG_TRY(gg_host_graph_transpose(hg, &csc));
    in = &csc;
  }
  g->h_csr_off.assign(hg->offsets, hg->offsets + n + 1);
  g->h_csc_off.assign(in->offsets, in->offsets + n + 1);
  std::vector<uint32_t> indeg(n), outdeg(n);
  for (uint32_t v = 0; v < n; ++v) {
    outdeg[v] = hg->offsets[v + 1] - hg->offsets[v];
    indeg[v] = in->offsets[v + 1] - in->offsets[v];
  }
  const int P = o.num_partitions;
  g->coo_sizes.assign(P, 0);
  g->csc_sizes.assign(P, 0);
  int rc = gg_partition_sizes(indeg.data(), outdeg.data(), n, m, P, o.balance, o.part_how, o.relabel,
                              g->coo_sizes.data(), g->csc_sizes.data());
  if (rc) {
    if (!g->symmetric) gg_host_graph_free(&csc);
    return rc;
  }
  g->coo_starts.assign(P + 1, 0);
  g->csc_starts.assign(P + 1, 0);
  for (int p = 0; p < P; ++p) {
    g->coo_starts[p + 1] = g->coo_starts[p] + g->coo_sizes[p];
    g->csc_starts[p + 1] = g->csc_starts[p] + g->csc_sizes[p];
  }
  // vertex_order: the device graph is the given graph renumbered inside every
  // COO partition; the partitions (computed above on the given ids) keep
  // their vertex sets and sizes
  struct HostHold {
    gg_host_graph h{};
    ~HostHold() { gg_host_graph_free(&h); }
  } renum;
  if (o.vertex_order == GG_VORDER_HOT_FIRST) {
    if (g->coo_starts[P] != (int64_t)n) {
      if (!g->symmetric) gg_host_graph_free(&csc);
      return fail(GG_ERR_PARTITION, "partition sizes sum to %lld, not n=%u", (long long)g->coo_starts[P], n);
    }
    g->relabeled = true;
    g->h_old_of_new.resize(n);
    g->h_new_of_old.resize(n);
    hot_first_order(hg, g->coo_starts.data(), P, g->h_old_of_new.data(), g->h_new_of_old.data());
    if (!g->symmetric) gg_host_graph_free(&csc);
    GG_TRY(relabel_host_graph(hg, g->h_old_of_new.data(), g->h_new_of_old.data(), &renum.h));
    hg = &renum.h;
    in = hg;
    if (!g->symmetric) {
      GG_TRY(gg_host_graph_transpose(hg, &csc));
      in = &csc;
    }
    g->h_csr_off.assign(hg->offsets, hg->offsets + n + 1);
    g->h_csc_off.assign(in->offsets, in->offsets + n + 1);
    rc = dev_alloc(g, &g->d_new_of_old, n);
    if (!rc) rc = dev_alloc(g, &g->d_old_of_new, n);
    if (!rc && cudaMemcpy(g->d_new_of_old, g->h_new_of_old.data(), 4ull * n, cudaMemcpyHostToDevice) != cudaSuccess)
      rc = fail(GG_ERR_CUDA, "vertex order upload failed");
    if (!rc && cudaMemcpy(g->d_old_of_new, g->h_old_of_new.data(), 4ull * n, cudaMemcpyHostToDevice) != cudaSuccess)
      rc = fail(GG_ERR_CUDA, "vertex order upload failed");
    if (rc) {
      if (!g->symmetric) gg_host_graph_free(&csc);
      return rc;
    }
  }
  auto up = [&](uint32_t** d, const void* h, size_t count, size_t pad) -> int {
    GG_TRY(dev_alloc(g, d, count + pad));
    if (pad) GG_CUDA(cudaMemset(*d + count, 0, sizeof(uint32_t) * pad));
    if (count) GG_CUDA(cudaMemcpy(*d, h, sizeof(uint32_t) * count, cudaMemcpyHostToDevice));
    return GG_OK;
  };
  // edge arrays padded (with zeros) to whole 256-edge blocks plus one block,
  // so that the segmented pull may copy any block that holds a tile edge
  g->m_pad = (m + kSegBlock - 1) / kSegBlock * kSegBlock + kSegBlock;
  const size_t epad = (size_t)(g->m_pad - m);
  rc = up(&g->d_csr_off, hg->offsets, (size_t)n + 1, 4);
  if (!rc) rc = up(&g->d_csr_idx, hg->indices, m, epad);
  if (!rc && g->wtype != GG_W_NONE) rc = up(&g->d_csr_w, hg->weights, m, epad);
  if (!rc) {
    if (g->symmetric) {
      g->d_csc_off = g->d_csr_off;
      g->d_csc_idx = g->d_csr_idx;
      g->d_csc_w = g->d_csr_w;
    } else {
      rc = up(&g->d_csc_off, in->offsets, (size_t)n + 1, 4);
      if (!rc) rc = up(&g->d_csc_idx, in->indices, m, epad);
      if (!rc && g->wtype != GG_W_NONE) rc = up(&g->d_csc_w, in->weights, m, epad);
    }
  }
  // row structure of the pulled streams: CSC, and CSR for the transposed pull
  if (!rc) rc = build_seg(g, in->offsets, g->seg[0]);
  if (!rc && !g->symmetric) rc = build_seg(g, hg->offsets, g->seg[1]);
  else if (!rc) {
    g->seg[1] = g->seg[0];
    g->seg[1].d_head = g->seg[1].d_blk = g->seg[1].d_rows = nullptr;  // shared; never used
  }
  // CTA tiles for the CSC pull, both orientations
  if (!rc) {
    std::vector<uint4> t0;
    make_tiles(in->offsets, 0, n, (uint32_t)o.tile_vertices, (uint64_t)o.tile_edges, t0);
    rc = upload_tiles(g, g->csc_tiles[0], t0);
  }
  if (!rc && !g->symmetric) {
    std::vector<uint4> t1;
    make_tiles(hg->offsets, 0, n, (uint32_t)o.tile_vertices, (uint64_t)o.tile_edges, t1);
    rc = upload_tiles(g, g->csc_tiles[1], t1);
  } else if (!rc) {
    g->csc_tiles[1] = g->csc_tiles[0];
    g->csc_tiles[1].d_tiles = nullptr;  // shared; released once
  }
  // partitioned COO: only for -v edge (graphgrind/graph-numa.h:661)
  const bool want_coo = o.balance == GG_BALANCE_EDGE && o.build_coo >= 0;
  if (!rc && want_coo && m > 0)
    rc = o.part_how == GG_PART_SOURCE ? build_coo_src(g) : build_coo(g, in->offsets);
  if (!g->symmetric) gg_host_graph_free(&csc);
  if (rc) return rc;
  // workspace
  GG_TRY(dev_alloc(g, &g->ws.d_stats, 8));
  GG_CUDA(cudaMemset(g->ws.d_stats, 0, 64));
  GG_CUDA(cudaMallocHost((void**)&g->ws.h_stats, 64));
  GG_TRY(dev_alloc(g, &g->ws.d_dedup, (size_t)g->words() + 4));
  GG_CUDA(cudaMemset(g->ws.d_dedup, 0, sizeof(uint32_t) * ((size_t)g->words() + 4)));
  GG_TRY(dev_alloc(g, &g->ws.d_scan, (size_t)n + 4));
  GG_TRY(dev_alloc(g, &g->ws.d_red, 64));
  GG_TRY(dev_alloc(g, &g->ws.d_loop, 64));
  if (g->relabeled)
    for (int k = 0; k < 2; ++k) GG_TRY(dev_alloc(g, &g->ws.d_order[k], (size_t)n + 4));
  GG_CUDA(cudaMallocHost((void**)&g->ws.h_red, 64 * sizeof(double)));
  GG_CUDA(cudaHostAlloc((void**)&g->ws.h_map, kMapBytes, cudaHostAllocMapped));
  GG_CUDA(cudaHostGetDevicePointer((void**)&g->ws.d_map, g->ws.h_map, 0));
  GG_CUDA(cudaDeviceSynchronize());
  return GG_OK;
}

}  // namespace gg

using namespace gg;

extern "C" {

const char* gg_version(void) { return "graphgrind_b200 0.1 (sm_100a)"; }

int gg_graph_build(const gg_host_graph* hg, const gg_build_opts* opts, gg_graph_t* out) {
  if (!hg || !out || !hg->offsets || (hg->m && !hg->indices) || hg->n == 0)
    return fail(GG_ERR_INVALID_ARG, "gg_graph_build: bad arguments");
  if (hg->m >= (1ull << 32) - 64) return fail(GG_ERR_SIZE, "m=%llu exceeds uint32 offsets", (unsigned long long)hg->m);
  if (hg->n > (1u << 31)) return fail(GG_ERR_SIZE, "n=%u exceeds the supported vertex range", hg->n);
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(GG_ERR_NO_DEVICE, "no CUDA device is visible");
  }
  gg_graph_s* g = new (std::nothrow) gg_graph_s;
  if (!g) return fail(GG_ERR_OOM, "graph: out of host memory");
  int rc = graph_build(hg, opts, g);
  if (rc) {
    std::string keep = last_error();
    graph_release(g);
    set_error("%s", keep.c_str());
    return rc;
  }
  {
    std::lock_guard<std::mutex> lk(g_reg_mu);
    g_graphs.insert(g);
  }
  *out = g;
  return GG_OK;
}

int gg_graph_synchronize(gg_graph_t g) {
  if (!graph_live(g)) return fail(GG_ERR_INVALID_ARG, "gg_graph_synchronize: not a live graph");
  if (g->copy_stream) GG_CUDA(cudaStreamSynchronize(g->copy_stream));
  GG_CUDA(cudaStreamSynchronize(g->stream));
  return GG_OK;
}

int gg_graph_destroy(gg_graph_t g) {
  if (!graph_live(g)) return fail(GG_ERR_INVALID_ARG, "gg_graph_destroy: not a live graph");
  cudaStreamSynchronize(g->stream);
  const int device = g->device;
  graph_release(g);
  pool_trim(device);  // only memory no graph holds goes back
  return GG_OK;
}

int gg_graph_get_info(gg_graph_t g, gg_graph_info* info) {
  if (!g || !info) return fail(GG_ERR_INVALID_ARG, "gg_graph_get_info: bad arguments");
  info->n = g->n;
  info->m = g->m;
  info->symmetric = g->symmetric;
  info->weight_type = g->wtype;
  info->num_partitions = (int32_t)g->coo_sizes.size();
  info->has_coo = g->has_coo;
  info->transposed = g->transposed;
  info->num_csc_tiles = (int32_t)g->csc_tiles[0].count;
  info->num_coo_tiles = (int32_t)g->coo_tiles.count;
  info->device_bytes = g->device_bytes;
  info->num_coo_gaps = (int32_t)g->coo_gap_count;
  return GG_OK;
}

int gg_graph_partition_starts(gg_graph_t g, int64_t* starts) {
  if (!g || !starts) return fail(GG_ERR_INVALID_ARG, "gg_graph_partition_starts: bad arguments");
  std::copy(g->coo_starts.begin(), g->coo_starts.end(), starts);
  return GG_OK;
}

namespace gg {
__global__ void k_coo_unpack(const uint4* tiles, uint32_t ntiles, const uint32_t* src, const uint16_t* dloc,
                             uint32_t* out_src, uint32_t* out_dst) {
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint4 tl = tiles[t];  // {v0, nv, first slot, padded edge count}
    for (uint32_t i = threadIdx.x; i < tl.w; i += blockDim.x) {
      const uint32_t s = src[tl.z + i];
      out_src[tl.z + i] = s;
      out_dst[tl.z + i] = s == 0xffffffffu ? 0xffffffffu : tl.x + dloc[tl.z + i];
    }
  }
}
}  // namespace gg

int gg_graph_coo_layout(gg_graph_t g, uint64_t* num_tiles, uint32_t* tiles, uint64_t* coo_len, uint32_t* src,
                        uint32_t* dst) {
  if (!graph_live(g) || !num_tiles || !coo_len)
    return fail(GG_ERR_INVALID_ARG, "gg_graph_coo_layout: bad arguments");
  if (!g->has_coo) return fail(GG_ERR_UNSUPPORTED, "gg_graph_coo_layout: the graph has no partitioned COO");
  std::vector<uint4> tl;
  if (g->coo_by_source) {
    const int P = (int)g->coo_sizes.size();
    for (int p = 0; p < P; ++p) {
      const uint32_t a = (uint32_t)g->coo_starts[p], b = (uint32_t)g->coo_starts[p + 1];
      tl.push_back(make_uint4(a, b - a, g->h_csr_off[a], g->h_csr_off[b] - g->h_csr_off[a]));
    }
  } else {
    tl = g->coo_tiles.host;
  }
  *num_tiles = tl.size();
  *coo_len = g->coo_len;
  if (tiles) memcpy(tiles, tl.data(), sizeof(uint4) * tl.size());
  if (!src && !dst) return GG_OK;
  if (!src || !dst) return fail(GG_ERR_INVALID_ARG, "gg_graph_coo_layout: give both src and dst");
  if (g->coo_by_source) {
    GG_CUDA(cudaMemcpy(src, g->d_coo_src, 4 * g->coo_len, cudaMemcpyDeviceToHost));
    GG_CUDA(cudaMemcpy(dst, g->d_coo_dst, 4 * g->coo_len, cudaMemcpyDeviceToHost));
    return GG_OK;
  }
  DevBuf<uint32_t> ds, dd;
  GG_TRY(ds.alloc(g, g->coo_len + 1));
  GG_TRY(dd.alloc(g, g->coo_len + 1));
  if (!tl.empty()) {
    k_coo_unpack<<<g->num_sms * 4, 256, 0, g->stream>>>(g->coo_tiles.d_tiles, (uint32_t)tl.size(), g->d_coo_src,
                                                         g->d_coo_dloc, ds.p, dd.p);
    GG_CUDA(cudaGetLastError());
  }
  GG_CUDA(cudaStreamSynchronize(g->stream));
  GG_CUDA(cudaMemcpy(src, ds.p, 4 * g->coo_len, cudaMemcpyDeviceToHost));
  GG_CUDA(cudaMemcpy(dst, dd.p, 4 * g->coo_len, cudaMemcpyDeviceToHost));
  return GG_OK;
}

int gg_graph_set_profiling(gg_graph_t g, int32_t enable) {
  if (!g) return fail(GG_ERR_INVALID_ARG, "gg_graph_set_profiling: null graph");
  if (enable && !g->prof_ev[0]) {
    GG_CUDA(cudaEventCreate(&g->prof_ev[0]));
    GG_CUDA(cudaEventCreate(&g->prof_ev[1]));
  }
  g->profiling = enable != 0;
  return GG_OK;
}

int gg_graph_get_profile(gg_graph_t g, gg_profile* out) {
  if (!g || !out) return fail(GG_ERR_INVALID_ARG, "gg_graph_get_profile: bad arguments");
  *out = g->prof;
  g->prof = gg_profile{};
  return GG_OK;
}

int gg_graph_set_dense_policy(gg_graph_t g, int32_t policy) {
  if (!g || policy < 0 || policy > 2) return fail(GG_ERR_INVALID_ARG, "gg_graph_set_dense_policy: bad arguments");
  g->dense_policy = policy;
  return GG_OK;
}

int gg_graph_set_tuning(gg_graph_t g, int32_t key, int64_t value) {
  if (!graph_live(g)) return fail(GG_ERR_INVALID_ARG, "gg_graph_set_tuning: not a live graph");
  switch (key) {
    case GG_TUNE_DENSE_POLICY:
      return gg_graph_set_dense_policy(g, (int32_t)value);
    case GG_TUNE_COO_KERNEL:
      if (value < 0 || value > 7) return fail(GG_ERR_INVALID_ARG, "COO kernel must be 0..7");
      g->coo_kernel = (int)value;
      return GG_OK;
    case GG_TUNE_SPARSE_DIV:
      if (value < 1 || value > (1 << 20)) return fail(GG_ERR_INVALID_ARG, "threshold divisor must be 1..2^20");
      g->sparse_div = (int)value;
      return GG_OK;
    case GG_TUNE_DEVICE_LOOP:
      if (value < 0 || value > 2) return fail(GG_ERR_INVALID_ARG, "device loop switch must be 0, 1 or 2");
      g->device_loop = (int)value;
      return GG_OK;
    case GG_TUNE_CC_ALGO:
      if (value != 0 && value != 1) return fail(GG_ERR_INVALID_ARG, "components algorithm must be 0 or 1");
      g->cc_algo = (int)value;
      return GG_OK;
    case GG_TUNE_PR_GRAPH:
      if (value != 0 && value != 1) return fail(GG_ERR_INVALID_ARG, "PageRank graph switch must be 0 or 1");
      g->pr_graph = (int)value;
      return GG_OK;
    case GG_TUNE_EARLY_KERNEL:
      if (value < 0 || value > 3) return fail(GG_ERR_INVALID_ARG, "early-exit kernel must be 0..3");
      g->early_kernel = (int)value;
      return GG_OK;
    case GG_TUNE_PUSH_DENSE_DIV:
      if (value < 0 || value > (1ll << 30)) return fail(GG_ERR_INVALID_ARG, "push-dense divisor must be 0..2^30");
      g->push_dense_div = (int)value;
      return GG_OK;
    case GG_TUNE_ROUND_GRAPH:
      if (value != 0 && value != 1) return fail(GG_ERR_INVALID_ARG, "round graph switch must be 0 or 1");
      g->round_graph = (int)value;
      return GG_OK;
    case GG_TUNE_LOOP_CTAS:
      if (value < 0 || value > 16) return fail(GG_ERR_INVALID_ARG, "loop CTAs per SM must be 0..16");
      g->loop_ctas_per_sm = (int)value;
      return GG_OK;
    case GG_TUNE_LOOP_WAIT_BUDGET:
      if (value < 0 || value > (1ll << 22))
        return fail(GG_ERR_INVALID_ARG, "loop wait budget must be 0..2^22 spins");
      g->loop_wait_budget = (uint32_t)value;
      return GG_OK;
    case GG_TUNE_ASYNC_RESULTS:
      if (value != 0 && value != 1) return fail(GG_ERR_INVALID_ARG, "asynchronous results switch must be 0 or 1");
      if (value && !g->copy_stream) {
        GG_CUDA(cudaStreamCreateWithFlags(&g->copy_stream, cudaStreamNonBlocking));
        GG_CUDA(cudaEventCreateWithFlags(&g->result_ready, cudaEventDisableTiming));
        for (auto& e : g->slot_copied) GG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      }
      if (value)  // results of graphs with their given ids are staged there too; BFS's parents in array 2
        for (auto& a : g->ws.d_order)
          if (!a) GG_TRY(dev_alloc(g, &a, (size_t)g->n + 4));
      if (!value && g->copy_stream) GG_CUDA(cudaStreamSynchronize(g->copy_stream));
      g->async_results = (int)value;
      return GG_OK;
    default:
      return fail(GG_ERR_INVALID_ARG, "unknown tuning key %d", key);
  }
}

int gg_graph_get_tuning(gg_graph_t g, int32_t key, int64_t* value) {
  if (!graph_live(g) || !value) return fail(GG_ERR_INVALID_ARG, "gg_graph_get_tuning: bad arguments");
  switch (key) {
    case GG_TUNE_DENSE_POLICY:
      *value = g->dense_policy;
      return GG_OK;
    case GG_TUNE_COO_KERNEL:
      *value = g->coo_kernel;
      return GG_OK;
    case GG_TUNE_SPARSE_DIV:
      *value = g->sparse_div;
      return GG_OK;
    case GG_TUNE_DEVICE_LOOP:
      *value = g->device_loop;
      return GG_OK;
    case GG_TUNE_CC_ALGO:
      *value = g->cc_algo;
      return GG_OK;
    case GG_TUNE_PR_GRAPH:
      *value = g->pr_graph;
      return GG_OK;
    case GG_TUNE_ASYNC_RESULTS:
      *value = g->async_results;
      return GG_OK;
    case GG_TUNE_LOOP_WAIT_BUDGET:
      *value = g->loop_wait_budget;
      return GG_OK;
    case GG_TUNE_EARLY_KERNEL:
      *value = g->early_kernel;
      return GG_OK;
    case GG_TUNE_PUSH_DENSE_DIV:
      *value = g->push_dense_div;
      return GG_OK;
    case GG_TUNE_LOOP_CTAS:
      *value = g->loop_ctas_per_sm;
      return GG_OK;
    case GG_TUNE_ROUND_GRAPH:
      *value = g->round_graph;
      return GG_OK;
    default:
      return fail(GG_ERR_INVALID_ARG, "unknown tuning key %d", key);
  }
}

int gg_graph_transpose(gg_graph_t g) {
  if (!g) return fail(GG_ERR_INVALID_ARG, "gg_graph_transpose: null graph");
  if (!g->symmetric) g->transposed = !g->transposed;  // graphgrind/graph-numa.h:598-611
  return GG_OK;
}

int gg_graph_vertex_order(gg_graph_t g, uint32_t* new_of_old) {
  if (!graph_live(g) || !new_of_old) return fail(GG_ERR_INVALID_ARG, "gg_graph_vertex_order: bad arguments");
  for (uint32_t v = 0; v < g->n; ++v) new_of_old[v] = g->device_id(v);
  return GG_OK;
}

int gg_graph_device_arrays(gg_graph_t g, const uint32_t** oo, const uint32_t** oi, const uint32_t** io,
                           const uint32_t** ii) {
  if (!g) return fail(GG_ERR_INVALID_ARG, "gg_graph_device_arrays: null graph");
  if (oo) *oo = g->out_off();
  if (oi) *oi = g->out_idx();
  if (io) *io = g->in_off();
  if (ii) *ii = g->in_idx();
  return GG_OK;
}

int gg_graph_device_weights(gg_graph_t g, const void** out_w, const void** in_w) {
  if (!graph_live(g)) return fail(GG_ERR_INVALID_ARG, "gg_graph_device_weights: not a live graph");
  if (out_w) *out_w = g->wtype == GG_W_NONE ? nullptr : g->out_w();
  if (in_w) *in_w = g->wtype == GG_W_NONE ? nullptr : g->in_w();
  return GG_OK;
}

// ---------------------------------------------------------- frontier API
int gg_frontier_single(gg_graph_t g, uint32_t v, gg_frontier_t* out) {
  if (!g || !out || v >= g->n) return fail(GG_ERR_INVALID_ARG, "gg_frontier_single: bad arguments");
  gg_frontier_s* f;
  GG_TRY(frontier_new(g, &f));
  int rc = frontier_ensure_queue(f);
  if (!rc) rc = write_small(g, f->d_queue, v);
  if (rc) {
    frontier_free(f);
    return rc;
  }
  f->has_sparse = true;
  f->dm = 1;
  f->out_edges = g->h_out_off()[v + 1] - g->h_out_off()[v];
  *out = f;
  return GG_OK;
}

int gg_frontier_all(gg_graph_t g, gg_frontier_t* out) {
  if (!g || !out) return fail(GG_ERR_INVALID_ARG, "gg_frontier_all: bad arguments");
  gg_frontier_s* f;
  GG_TRY(frontier_new(g, &f));
  f->bit = true;
  f->has_dense = false;
  f->dm = g->n;
  f->out_edges = g->m;  // bits(part, n, m)
  *out = f;
  return GG_OK;
}

int gg_frontier_empty(gg_graph_t g, gg_frontier_t* out) {
  if (!g || !out) return fail(GG_ERR_INVALID_ARG, "gg_frontier_empty: bad arguments");
  return frontier_new(g, out);
}

int gg_frontier_from_mask(gg_graph_t g, const uint8_t* mask, gg_frontier_t* out) {
  if (!g || !mask || !out) return fail(GG_ERR_INVALID_ARG, "gg_frontier_from_mask: bad arguments");
  std::vector<uint32_t> words((size_t)g->words() + 4, 0);
  for (uint32_t v = 0; v < g->n; ++v)
    if (mask[v]) words[v >> 5] |= 1u << (v & 31);
  gg_frontier_s* f;
  GG_TRY(frontier_new(g, &f));
  int rc = frontier_ensure_bits(f, false);
  if (!rc && cudaMemcpyAsync(f->d_bits, words.data(), 4 * words.size(), cudaMemcpyHostToDevice, g->stream) != cudaSuccess)
    rc = fail(GG_ERR_CUDA, "frontier upload failed");
  if (!rc) rc = reset_stats(g);
  if (!rc) {
    k_bits_stats<<<generic_grid(g, g->words()), kGenericThreads, 0, g->stream>>>(f->d_bits, g->n, g->out_off(),
                                                                                g->ws.d_stats);
    rc = read_stats(g);
  }
  if (rc) {
    frontier_free(f);
    return rc;
  }
  f->has_dense = true;
  f->dm = g->ws.h_stats[0];
  f->out_edges = g->ws.h_stats[1];
  *out = f;
  return GG_OK;
}

int gg_frontier_from_list(gg_graph_t g, const uint32_t* verts, uint64_t count, gg_frontier_t* out) {
  if (!g || (!verts && count) || !out || count > g->n)
    return fail(GG_ERR_INVALID_ARG, "gg_frontier_from_list: bad arguments");
  const uint32_t* off = g->h_out_off();
  uint64_t oe = 0;
  for (uint64_t i = 0; i < count; ++i) {
    if (verts[i] >= g->n) return fail(GG_ERR_INVALID_ARG, "vertex %u out of range", verts[i]);
    oe += off[verts[i] + 1] - off[verts[i]];
  }
  gg_frontier_s* f;
  GG_TRY(frontier_new(g, &f));
  int rc = frontier_ensure_queue(f);
  if (!rc && count &&
      cudaMemcpyAsync(f->d_queue, verts, 4 * count, cudaMemcpyHostToDevice, g->stream) != cudaSuccess)
    rc = fail(GG_ERR_CUDA, "frontier upload failed");
  if (!rc && cudaStreamSynchronize(g->stream) != cudaSuccess) rc = fail(GG_ERR_CUDA, "sync failed");
  if (rc) {
    frontier_free(f);
    return rc;
  }
  f->has_sparse = true;
  f->dm = count;
  f->out_edges = oe;
  *out = f;
  return GG_OK;
}

int gg_frontier_destroy(gg_frontier_t f) {
  if (!frontier_live(f)) return fail(GG_ERR_INVALID_ARG, "gg_frontier_destroy: not a live frontier");
  frontier_free(f);
  return GG_OK;
}

int gg_frontier_stats(gg_frontier_t f, uint64_t* active, uint64_t* out_edges) {
  if (!f) return fail(GG_ERR_INVALID_ARG, "gg_frontier_stats: null frontier");
  if (active) *active = f->dm;
  if (out_edges) *out_edges = f->out_edges;
  return GG_OK;
}

int gg_frontier_to_mask(gg_frontier_t f, uint8_t* mask) {
  if (!f || !mask) return fail(GG_ERR_INVALID_ARG, "gg_frontier_to_mask: bad arguments");
  gg_graph_s* g = f->g;
  const uint32_t n = g->n;
  if (f->bit) {
    memset(mask, 1, n);
    return GG_OK;
  }
  memset(mask, 0, n);
  if (f->dm == 0) return GG_OK;
  if (f->has_dense) {
    std::vector<uint32_t> words(g->words());
    GG_CUDA(cudaMemcpyAsync(words.data(), f->d_bits, 4ull * words.size(), cudaMemcpyDeviceToHost, g->stream));
    GG_CUDA(cudaStreamSynchronize(g->stream));
    for (uint32_t v = 0; v < n; ++v) mask[v] = (words[v >> 5] >> (v & 31)) & 1u;
  } else {
    std::vector<uint32_t> q(f->dm);
    GG_CUDA(cudaMemcpyAsync(q.data(), f->d_queue, 4ull * f->dm, cudaMemcpyDeviceToHost, g->stream));
    GG_CUDA(cudaStreamSynchronize(g->stream));
    for (uint32_t v : q) mask[v] = 1;
  }
  return GG_OK;
}

int gg_frontier_to_dense(gg_frontier_t f) {
  if (!f) return fail(GG_ERR_INVALID_ARG, "gg_frontier_to_dense: null frontier");
  int rc = frontier_to_dense(f);
  if (!rc) rc = cudaStreamSynchronize(f->g->stream) == cudaSuccess ? GG_OK : fail(GG_ERR_CUDA, "sync failed");
  return rc;
}

int gg_frontier_to_sparse(gg_frontier_t f) {
  if (!f) return fail(GG_ERR_INVALID_ARG, "gg_frontier_to_sparse: null frontier");
  int rc = frontier_to_sparse(f);
  if (!rc) rc = cudaStreamSynchronize(f->g->stream) == cudaSuccess ? GG_OK : fail(GG_ERR_CUDA, "sync failed");
  return rc;
}

int gg_frontier_repr(gg_frontier_t f) {
  if (!f) return fail(GG_ERR_INVALID_ARG, "gg_frontier_repr: null frontier");
  if (f->bit) return 4;
  return (f->has_dense ? 1 : 0) | (f->has_sparse ? 2 : 0);
}

int gg_vertex_array_alloc(gg_graph_t g, size_t elem_bytes, void** dev_ptr) {
  if (!g || !dev_ptr || !elem_bytes) return fail(GG_ERR_INVALID_ARG, "gg_vertex_array_alloc: bad arguments");
  GG_CUDA(cudaMalloc(dev_ptr, elem_bytes * ((size_t)g->n + 4)));
  g->arrays.insert(*dev_ptr);
  return GG_OK;
}
int gg_vertex_array_free(gg_graph_t g, void* p) {
  if (!graph_live(g)) return fail(GG_ERR_INVALID_ARG, "gg_vertex_array_free: not a live graph");
  if (!g->arrays.erase(p)) return fail(GG_ERR_INVALID_ARG, "gg_vertex_array_free: not an array of this graph");
  cudaStreamSynchronize(g->stream);
  GG_CUDA(cudaFree(p));
  return GG_OK;
}
int gg_memcpy_h2d(void* d, const void* h, size_t bytes) {
  GG_CUDA(cudaMemcpy(d, h, bytes, cudaMemcpyHostToDevice));
  return GG_OK;
}
int gg_memcpy_d2h(void* h, const void* d, size_t bytes) {
  GG_CUDA(cudaMemcpy(h, d, bytes, cudaMemcpyDeviceToHost));
  return GG_OK;
}
int gg_host_alloc_pinned(size_t bytes, void** p) {
  if (!p || !bytes) return fail(GG_ERR_INVALID_ARG, "gg_host_alloc_pinned: bad arguments");
  GG_CUDA(cudaMallocHost(p, bytes));
  return GG_OK;
}
int gg_host_free_pinned(void* p) {
  GG_CUDA(cudaFreeHost(p));
  return GG_OK;
}

}  // extern "C"
