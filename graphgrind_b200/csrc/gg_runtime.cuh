// Host side of the engine: vertexSubset bookkeeping and the templated
// edgeMap / vertexMap / vertexFilter drivers that launch the kernels of
// gg_engine.cuh.  Mirrors graphgrind/ligra-numa.h:91-1082.
#pragma once
#include <algorithm>
#include <atomic>
#include <cstring>

#include "gg_engine.cuh"
#include "gg_functors.cuh"

namespace gg {

constexpr uint32_t kGenericThreads = 256;

// Device time between construction and stop() on one stream.
struct EventTimer {
  cudaEvent_t a = nullptr, b = nullptr;
  cudaStream_t s;
  explicit EventTimer(cudaStream_t st) : s(st) {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s);
  }
  double stop() {
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
  }
  ~EventTimer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
};

// Stream-ordered allocations of the library (temporaries of the
// applications, frontiers) come from one memory pool per device whose release
// threshold is unlimited: memory freed back to it stays mapped across stream
// synchronisations, so the next call reuses it instead of mapping it again
// (the default pool returns it at every synchronisation).  Devices past the
// pool table, or a pool the driver refuses, take cudaMallocAsync.
cudaError_t pool_alloc(void** p, size_t bytes, cudaStream_t s, int device);
// Returns the pool's unused memory of `device` to the system.
void pool_trim(int device);

// ------------------------------------------------ small control transfers
// Loop states, statistics and reductions are read back (and loop control
// blocks written) by one-warp kernels through the graph's mapped pinned block
// instead of cudaMemcpyAsync: a small copy on a copy engine waits behind the
// large result copies that GG_TUNE_ASYNC_RESULTS leaves in flight (a 64 MiB
// copy takes about 1.2 ms over PCIe), while a kernel's stores to mapped host
// memory do not.
__global__ void k_get_words(uint32_t* dst, const uint32_t* src, uint32_t words);
template <class T>
__global__ void k_put(T* dst, const T v) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *dst = v;
}
// Copies `count` values of T from device memory to `host` (any host memory)
// after the graph's stream has reached this point; synchronises the stream.
template <class T>
int read_small(gg_graph_s* g, T* host, const T* dev, size_t count = 1) {
  static_assert(sizeof(T) % 4 == 0, "control values are whole 32-bit words");
  const size_t bytes = sizeof(T) * count;
  if (bytes > kMapBytes) return fail(GG_ERR_INVALID_ARG, "control block of %zu bytes exceeds the mapped block", bytes);
  k_get_words<<<1, 128, 0, g->stream>>>(g->ws.d_map, reinterpret_cast<const uint32_t*>(dev), (uint32_t)(bytes / 4));
  GG_CUDA(cudaGetLastError());
  g->kernels++;
  GG_CUDA(cudaStreamSynchronize(g->stream));
  std::memcpy(host, g->ws.h_map, bytes);
  return GG_OK;
}
// Writes one T to device memory in stream order (the value travels as a
// kernel argument).
template <class T>
int write_small(gg_graph_s* g, T* dev, const T& v) {
  static_assert(sizeof(T) <= 1024, "control blocks travel as kernel arguments");
  k_put<T><<<1, 32, 0, g->stream>>>(dev, v);
  GG_CUDA(cudaGetLastError());
  g->kernels++;
  return GG_OK;
}

// A stream-ordered device allocation released when the holder leaves scope.
template <class T>
struct DevBuf {
  T* p = nullptr;
  gg_graph_s* g = nullptr;
  int alloc(gg_graph_s* gg_, uint64_t n) {
    g = gg_;
    GG_CUDA(pool_alloc((void**)&p, sizeof(T) * (n + 4), g->stream, g->device));
    return GG_OK;
  }
  ~DevBuf() {
    if (p) cudaFreeAsync(p, g->stream);
  }
};

// Kernel attributes (dynamic shared memory opt-in) and occupancy are per
// device: launchers cache them per device index, in atomics so that threads
// driving different graphs may share them.
constexpr int kMaxDevices = 16;
struct DeviceOnce {
  std::atomic<int> v[kMaxDevices];  // 0 = not yet set, else the cached value
  // the cached value of device d, computing it with fn() once (uncached past kMaxDevices)
  template <class Fn>
  int get(int d, Fn fn) {
    if (d < 0 || d >= kMaxDevices) return fn();
    int x = v[d].load(std::memory_order_acquire);
    if (x == 0) {
      x = fn();
      if (x > 0) v[d].store(x, std::memory_order_release);
    }
    return x;
  }
};

// edgeMap threshold of the application loops: m/20 in app/*.C, m/sparse_div when tuned.
inline int64_t app_threshold(const gg_graph_s* g) { return (int64_t)g->m / g->sparse_div; }

inline int generic_grid(const gg_graph_s* g, uint64_t work) {
  uint64_t b = (work + kGenericThreads - 1) / kGenericThreads;
  uint64_t cap = (uint64_t)g->num_sms * 8;
  if (b < 1) b = 1;
  return (int)std::min<uint64_t>(b, cap);
}

// ------------------------------------------ given ids <-> device ids
// Graphs built with a vertex_order hold their vertices renumbered; the
// applications move per-vertex arrays (rows of k entries) between the two
// orders at their boundary.  The renumbering stays inside partitions, so both
// directions read and write within one partition's stretch of the array.
// to_given: out[u] = in[new_of_old[u]];  to_device: out[i] = in[old_of_new[i]].
// Each thread takes kPermIlp entries a grid stride apart per round, their
// loads issued together (the map read, then the gather it feeds).
constexpr int kPermIlp = 4;
template <class T>
__global__ void k_permute_rows(uint32_t n, uint32_t k, const uint32_t* map, const T* in, T* out) {
  const uint64_t total = (uint64_t)n * k;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < total; i0 += kPermIlp * stride) {
    uint64_t src[kPermIlp];
#pragma unroll
    for (int t = 0; t < kPermIlp; ++t) {
      const uint64_t i = i0 + t * stride;
      src[t] = i < total ? (uint64_t)map[i / k] * k + i % k : 0;
    }
    T val[kPermIlp];
#pragma unroll
    for (int t = 0; t < kPermIlp; ++t) val[t] = i0 + t * stride < total ? in[src[t]] : T();
#pragma unroll
    for (int t = 0; t < kPermIlp; ++t)
      if (i0 + t * stride < total) out[i0 + t * stride] = val[t];
  }
}
// vertex ids held as values (BFS parents): the given id of the value, for the
// given vertex u
static __global__ void k_ids_to_given(uint32_t n, const uint32_t* new_of_old, const uint32_t* old_of_new,
                               const int32_t* in, int32_t* out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t u0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u0 < n; u0 += kPermIlp * stride) {
    uint32_t w[kPermIlp];
#pragma unroll
    for (int t = 0; t < kPermIlp; ++t) w[t] = u0 + t * stride < n ? new_of_old[u0 + t * stride] : 0u;
    int32_t v[kPermIlp];
#pragma unroll
    for (int t = 0; t < kPermIlp; ++t) v[t] = u0 + t * stride < n ? in[w[t]] : -1;
    uint32_t gv[kPermIlp];
#pragma unroll
    for (int t = 0; t < kPermIlp; ++t) gv[t] = v[t] >= 0 ? old_of_new[v[t]] : 0u;
#pragma unroll
    for (int t = 0; t < kPermIlp; ++t)
      if (u0 + t * stride < n) out[u0 + t * stride] = v[t] < 0 ? v[t] : (int32_t)gv[t];
  }
}

// `dev` (n rows of k, device order) in the given order: dev itself on a graph
// with its given ids, else a permuted copy in tmp.
template <class T>
int given_order(gg_graph_s* g, const T* dev, uint32_t k, DevBuf<T>& tmp, const T** res) {
  *res = dev;
  if (!g->relabeled) return GG_OK;
  GG_TRY(tmp.alloc(g, (uint64_t)g->n * k));
  k_permute_rows<T><<<generic_grid(g, (uint64_t)g->n * k), kGenericThreads, 0, g->stream>>>(g->n, k, g->d_new_of_old,
                                                                                             dev, tmp.p);
  GG_CUDA(cudaGetLastError());
  g->kernels++;
  *res = tmp.p;
  return GG_OK;
}
// Before the stream writes the given-order array `slot`: wait until a copy to
// the host that still reads it (GG_TUNE_ASYNC_RESULTS) is done.
inline int slot_write_wait(gg_graph_s* g, int slot) {
  if (g->slot_copied[slot]) GG_CUDA(cudaStreamWaitEvent(g->stream, g->slot_copied[slot], 0));
  if (slot == 1 && g->input_staged) {  // a staged SpMV input in the array is given up
    GG_CUDA(cudaStreamWaitEvent(g->stream, g->input_ready, 0));
    g->input_staged = false;
  }
  return GG_OK;
}
// The same for one 4-byte value per vertex, into the graph's given-order
// array `slot` (0 or 1; nothing is allocated on the application's path).
// With asynchronous results the array also stages results of graphs that
// keep their given ids, so that they can leave while the stream goes on.
template <class T>
int given_order(gg_graph_s* g, const T* dev, int slot, const T** res) {
  static_assert(sizeof(T) == 4, "the given-order arrays hold 4-byte values");
  *res = dev;
  if (!g->relabeled && !g->async_results) return GG_OK;
  T* out = reinterpret_cast<T*>(g->ws.d_order[slot]);
  GG_TRY(slot_write_wait(g, slot));
  if (!g->relabeled) {
    GG_CUDA(cudaMemcpyAsync(out, dev, sizeof(T) * (uint64_t)g->n, cudaMemcpyDeviceToDevice, g->stream));
    *res = out;
    return GG_OK;
  }
  k_permute_rows<T><<<generic_grid(g, g->n), kGenericThreads, 0, g->stream>>>(g->n, 1, g->d_new_of_old, dev, out);
  GG_CUDA(cudaGetLastError());
  g->kernels++;
  *res = out;
  return GG_OK;
}
// `given` (n rows of k, given order, device memory) into `dev` in device order
// (a copy when the graph keeps its given ids).
template <class T>
int device_order(gg_graph_s* g, const T* given, uint32_t k, T* dev) {
  if (!g->relabeled) {
    GG_CUDA(cudaMemcpyAsync(dev, given, sizeof(T) * (uint64_t)g->n * k, cudaMemcpyDeviceToDevice, g->stream));
    return GG_OK;
  }
  k_permute_rows<T><<<generic_grid(g, (uint64_t)g->n * k), kGenericThreads, 0, g->stream>>>(g->n, k, g->d_old_of_new,
                                                                                             given, dev);
  GG_CUDA(cudaGetLastError());
  g->kernels++;
  return GG_OK;
}

// ------------------------------------------------------------ frontiers
int frontier_new(gg_graph_s* g, gg_frontier_s** out);
int frontier_ensure_bits(gg_frontier_s* f, bool zero);
int frontier_ensure_queue(gg_frontier_s* f);
int frontier_to_dense(gg_frontier_s* f);
int frontier_to_sparse(gg_frontier_s* f);
void frontier_free(gg_frontier_s* f);
int bfs_device_levels(gg_graph_s* g, gg_frontier_s** F, int32_t* parents, int32_t* levels, int32_t round0,
                      uint64_t threshold, int32_t* rounds, uint64_t* trav);
int bfs_device_full(gg_graph_s* g, uint32_t start, int32_t* parents, int32_t* levels, uint64_t threshold);
// The CSC's in-lists with each one's sources by descending out-degree (ties by
// id), for BFS's bottom-up levels; built once per graph (g->d_bu_idx).
int build_bu_index(gg_graph_s* g);
int bfs_device_full_result(gg_graph_s* g, int32_t* rounds, uint64_t* trav);
int reset_stats(gg_graph_s* g);
void pr_loop_free(gg_graph_s* g);  // releases the captured PageRank loop and its buffers
void round_loops_free(gg_graph_s* g);  // the same for the BellmanFord / Components round loops
int read_stats(gg_graph_s* g);  // blocks; checks the device error word

// -------------------------------------------------------------- edgeMap
// graphgrind/ligra-numa.h:919-1019
template <class F, bool HW>
int pull_launch(gg_graph_s* g, gg_frontier_s* in, gg_frontier_s* out, const F& f, bool coo, bool no_out = false) {
  // a positive functor whose gathered values already mark the frontier needs no bitmap
  const bool all = in->bit || (F::kPositive && f.frontier_in_values) || f.outside_inert;
  if (coo && g->coo_by_source) {  // -P source: atomic updates over the source partitions
    SrcParams sp{g->d_coo_src, g->d_coo_dst, g->d_coo_w, g->coo_len, in->d_bits, out->d_bits, g->out_off(),
                 g->ws.d_stats};
    const int grid = generic_grid(g, g->coo_len) ;
    if (all)
      k_coo_src<F, HW, true><<<grid, 256, 0, g->stream>>>(sp, f);
    else
      k_coo_src<F, HW, false><<<grid, 256, 0, g->stream>>>(sp, f);
    GG_CUDA(cudaGetLastError());
    g->kernels++;
    return GG_OK;
  }
  PullParams p{};
  const int orient = g->transposed ? 1 : 0;
  if (coo) {
    p.tiles = g->coo_tiles.d_tiles;
    p.ntiles = g->coo_tiles.count;
    p.src = g->d_coo_src;
    p.dloc = g->d_coo_dloc;
    p.wts = g->d_coo_w;
    p.off = nullptr;
  } else {
    p.tiles = g->csc_tiles[orient].d_tiles;
    p.ntiles = g->csc_tiles[orient].count;
    p.src = g->in_idx();
    p.dloc = nullptr;
    p.wts = g->in_w();
    p.off = g->in_off();
  }
  p.tile_counter = g->ws.d_stats + 4;
  p.fr_bits = in->d_bits;
  p.next_bits = out->d_bits;
  p.deg_off = g->out_off();
  // compressed-CSC membership (PartitionByDest, graphgrind/graph-numa.h:1098-1107):
  // after transpose the pull still walks only vertices with original in-degree > 0
  p.member_off = (g->transposed && !coo) ? g->d_csc_off : nullptr;
  p.stats = g->ws.d_stats;
  p.err = g->ws.d_stats + 3;
  if (p.ntiles == 0) return GG_OK;
  constexpr bool kHW = HW;
  p.tv = (uint32_t)(coo ? g->opts.coo_tile_vertices : g->opts.tile_vertices);
  const size_t smem_coo = pull_smem_bytes(true, kHW, 4, p.tv);
  const size_t smem_csc = pull_smem_bytes(false, kHW, 4);
  // opt in once per device to the largest dynamic shared memory (widest
  // tiles); the occupancy follows the tile width of this graph
  static DeviceOnce opted_ring[2][2];
  auto launch = [&](auto kern, size_t smem, DeviceOnce& once) -> int {
    const int ok = once.get(g->device, [&]() {
      return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)pull_smem_bytes(true, kHW, 4, kMaxCooTileVertices)) == cudaSuccess ? 1 : -1;
    });
    if (ok < 0) return fail(GG_ERR_CUDA, "cudaFuncSetAttribute failed for the dense pull");
    int blocks = 1;
    GG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, kPullThreads, smem));
    if (blocks < 1) blocks = 1;
    const int grid = (int)std::min<uint64_t>((uint64_t)g->num_sms * blocks, p.ntiles);
    kern<<<grid, kPullThreads, smem, g->stream>>>(p, f);
    GG_CUDA(cudaGetLastError());
    g->kernels++;
    return GG_OK;
  };
  if (coo && g->coo_kernel > 0) {  // per-warp COO pull: 0, 2 or 3 staging stages
    static DeviceOnce opted[2][4];
    static DeviceOnce opted_pf[2];
    static DeviceOnce opted_no[3][2];
    static DeviceOnce opted_mg[2];
    constexpr int kFlags = coo_w_flag_bytes<F, false>(), kFlagsNoOut = coo_w_flag_bytes<F, true>();
    auto launch_w = [&](auto kern, int stages, DeviceOnce& once, int flags) -> int {
      const size_t smem = coo_w_smem_bytes(kHW, stages, 4, p.tv, flags);
      const int ok = once.get(g->device, [&]() {
        return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)coo_w_smem_bytes(kHW, stages, 4, kMaxCooTileVertices, flags)) == cudaSuccess
                   ? 1
                   : -1;
      });
      if (ok < 0) return fail(GG_ERR_CUDA, "cudaFuncSetAttribute failed for the COO pull");
      int blocks = 1;
      GG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, kCooThreads, smem));
      if (blocks < 1) blocks = 1;
      const int grid = (int)std::min<uint64_t>((uint64_t)g->num_sms * blocks, p.ntiles);
      kern<<<grid, kCooThreads, smem, g->stream>>>(p, f);
      GG_CUDA(cudaGetLastError());
      g->kernels++;
      return GG_OK;
    };
    if constexpr (F::kIdentityCommitNoop) {
      if (no_out && g->coo_kernel == 1)
        return all ? launch_w(k_pull_coo_w<F, kHW, true, 0, false, false, true>, 0, opted_no[0][1], kFlagsNoOut)
                   : launch_w(k_pull_coo_w<F, kHW, false, 0, false, false, true>, 0, opted_no[0][0], kFlagsNoOut);
      if (no_out && g->coo_kernel == 6)
        return all ? launch_w(k_pull_coo_w<F, kHW, true, 0, false, false, true, true>, 0, opted_no[1][1], kFlagsNoOut)
                   : launch_w(k_pull_coo_w<F, kHW, false, 0, false, false, true, true>, 0, opted_no[1][0],
                              kFlagsNoOut);
      if (no_out && g->coo_kernel == 7)
        return all ? launch_w(k_pull_coo_w<F, kHW, true, 0, false, false, true, true, 3>, 0, opted_no[2][1],
                              kFlagsNoOut)
                   : launch_w(k_pull_coo_w<F, kHW, false, 0, false, false, true, true, 3>, 0, opted_no[2][0],
                              kFlagsNoOut);
    }
    static DeviceOnce opted_h[2];
    switch (g->coo_kernel) {
      case 7:
        return all ? launch_w(k_pull_coo_w<F, kHW, true, 0, false, false, false, true, 7>, 0, opted_h[1], kFlags)
                   : launch_w(k_pull_coo_w<F, kHW, false, 0, false, false, false, true, 7>, 0, opted_h[0], kFlags);
      case 6:
        return all ? launch_w(k_pull_coo_w<F, kHW, true, 0, false, false, false, true>, 0, opted_mg[1], kFlags)
                   : launch_w(k_pull_coo_w<F, kHW, false, 0, false, false, false, true>, 0, opted_mg[0], kFlags);
      case 5:
        return all ? launch_w(k_pull_coo_w<F, kHW, true, 0, false, true>, 0, opted_pf[1], kFlags)
                   : launch_w(k_pull_coo_w<F, kHW, false, 0, false, true>, 0, opted_pf[0], kFlags);
      case 4:
        return all ? launch_w(k_pull_coo_w<F, kHW, true, 0, true>, 0, opted[1][0], kFlags)
                   : launch_w(k_pull_coo_w<F, kHW, false, 0, true>, 0, opted[0][0], kFlags);
      case 1:
        return all ? launch_w(k_pull_coo_w<F, kHW, true, 0>, 0, opted[1][1], kFlags)
                   : launch_w(k_pull_coo_w<F, kHW, false, 0>, 0, opted[0][1], kFlags);
      case 2:
        return all ? launch_w(k_pull_coo_w<F, kHW, true, 2>, 2, opted[1][2], kFlags)
                   : launch_w(k_pull_coo_w<F, kHW, false, 2>, 2, opted[0][2], kFlags);
      default:
        return all ? launch_w(k_pull_coo_w<F, kHW, true, 3>, 3, opted[1][3], kFlags)
                   : launch_w(k_pull_coo_w<F, kHW, false, 3>, 3, opted[0][3], kFlags);
    }
  }
  if (coo) {
    if (all) return launch(k_pull<F, true, kHW, true>, smem_coo, opted_ring[1][1]);
    return launch(k_pull<F, true, kHW, false>, smem_coo, opted_ring[1][0]);
  }
  (void)smem_csc;
  // CSC: the segmented pull over head bits
  SegParams s{};
  const SegIndex& si = g->seg[orient];
  s.tiles = p.tiles;
  s.ntiles = p.ntiles;
  s.tile_counter = p.tile_counter;
  s.src = p.src;
  s.wts = p.wts;
  s.head = si.d_head;
  s.blk = si.d_blk;
  s.rows = si.d_rows;
  s.fr_bits = p.fr_bits;
  s.next_bits = p.next_bits;
  s.deg_off = p.deg_off;
  s.member_off = p.member_off;
  s.stats = p.stats;
  s.err = p.err;
  const size_t smem_seg = seg_smem_bytes(kHW, 4);
  static DeviceOnce occ_seg[2];
  auto launch_seg = [&](auto kern, DeviceOnce& once) -> int {
    const int o = once.get(g->device, [&]() {
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_seg) != cudaSuccess)
        return -1;
      int b = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, kSegThreads, smem_seg) != cudaSuccess) return -1;
      return b < 1 ? 1 : b;
    });
    if (o < 0) return fail(GG_ERR_CUDA, "kernel set-up failed for the CSC pull");
    const int grid = (int)std::min<uint64_t>((uint64_t)g->num_sms * o, s.ntiles);
    kern<<<grid, kSegThreads, smem_seg, g->stream>>>(s, f);
    GG_CUDA(cudaGetLastError());
    g->kernels++;
    return GG_OK;
  };
  if (all) return launch_seg(k_pull_seg<F, kHW, true>, occ_seg[1]);
  return launch_seg(k_pull_seg<F, kHW, false>, occ_seg[0]);
}

template <class F, bool HW>
int pull_early_launch(gg_graph_s* g, gg_frontier_s* in, gg_frontier_s* out, const F& f) {
  const uint32_t* member = g->transposed ? g->d_csc_off : nullptr;
  const int grid = generic_grid(g, g->n);
  static_assert(kGenericThreads == 256, "k_pull_early_g stages 8 warps of candidates");
  if (g->early_kernel == 1) {
    if (in->bit)
      k_pull_early_g<F, HW, true><<<grid, kGenericThreads, 0, g->stream>>>(
          g->n, g->in_off(), g->in_idx(), g->in_w(), nullptr, out->d_bits, g->out_off(), member, g->ws.d_stats, f);
    else
      k_pull_early_g<F, HW, false><<<grid, kGenericThreads, 0, g->stream>>>(
          g->n, g->in_off(), g->in_idx(), g->in_w(), in->d_bits, out->d_bits, g->out_off(), member, g->ws.d_stats, f);
  } else if (g->early_kernel >= 2) {
    if (in->bit)
      k_pull_early<F, HW, true, true><<<grid, kGenericThreads, 0, g->stream>>>(
          g->n, g->in_off(), g->in_idx(), g->in_w(), nullptr, out->d_bits, g->out_off(), member, g->ws.d_stats, f);
    else
      k_pull_early<F, HW, false, true><<<grid, kGenericThreads, 0, g->stream>>>(
          g->n, g->in_off(), g->in_idx(), g->in_w(), in->d_bits, out->d_bits, g->out_off(), member, g->ws.d_stats, f);
  } else if (in->bit) {
    k_pull_early<F, HW, true><<<grid, kGenericThreads, 0, g->stream>>>(
        g->n, g->in_off(), g->in_idx(), g->in_w(), nullptr, out->d_bits, g->out_off(), member, g->ws.d_stats, f);
  } else {
    k_pull_early<F, HW, false><<<grid, kGenericThreads, 0, g->stream>>>(
        g->n, g->in_off(), g->in_idx(), g->in_w(), in->d_bits, out->d_bits, g->out_off(), member, g->ws.d_stats, f);
  }
  GG_CUDA(cudaGetLastError());
  g->kernels++;
  return GG_OK;
}

template <class F, bool HW>
int push_launch(gg_graph_s* g, gg_frontier_s* in, gg_frontier_s* out, const F& f) {
  const uint32_t k = (uint32_t)in->dm;
  const uint32_t nb = (k + kScanTile - 1) / kScanTile;
  Workspace& ws = g->ws;
  if (nb > ws.bsum_cap) {
    if (ws.d_bsum) cudaFree(ws.d_bsum);
    GG_CUDA(cudaMalloc(&ws.d_bsum, sizeof(uint32_t) * (nb + 32)));
    ws.bsum_cap = nb;
  }
  const uint32_t* off = g->out_off();
  k_scan_sums<<<nb, kScanThreads, 0, g->stream>>>(in->d_queue, k, off, ws.d_bsum);
  k_scan_blocks<<<1, 1024, 0, g->stream>>>(ws.d_bsum, nb, ws.d_stats + 5);
  k_scan_write<<<nb, kScanThreads, 0, g->stream>>>(in->d_queue, k, off, ws.d_bsum, ws.d_scan);
  PushParams p{};
  p.q = in->d_queue;
  p.k = k;
  p.offs = ws.d_scan;
  p.total = ws.d_stats + 5;
  p.off = off;
  p.idx = g->out_idx();
  p.wts = g->out_w();
  p.deg_off = off;
  p.dedup = ws.d_dedup;
  p.out_q = out->d_queue;
  p.stats = ws.d_stats;
  // persistent CTAs: the edge total is read on the device
  const uint64_t work_ub = std::max<uint64_t>(in->out_edges, 1);
  const int grid = (int)std::min<uint64_t>((work_ub + kPushEdgesPerCta - 1) / kPushEdgesPerCta + 1,
                                           (uint64_t)g->num_sms * 8);
  k_push<F, HW><<<std::max(grid, g->num_sms), kPushThreads, 0, g->stream>>>(p, f);
  k_clear_dedup<<<g->num_sms, kGenericThreads, 0, g->stream>>>(out->d_queue, ws.d_stats + 2, ws.d_dedup);
  GG_CUDA(cudaGetLastError());
  g->kernels += 5;
  return GG_OK;
}

// Top-down step into a bitmap (k_push_bits): `out` bits zeroed, stats reset.
template <class F, bool HW>
int push_bits_launch(gg_graph_s* g, gg_frontier_s* in, gg_frontier_s* out, const F& f) {
  const uint32_t k = (uint32_t)in->dm;
  const uint32_t nb = (k + kScanTile - 1) / kScanTile;
  Workspace& ws = g->ws;
  if (nb > ws.bsum_cap) {
    if (ws.d_bsum) cudaFree(ws.d_bsum);
    GG_CUDA(cudaMalloc(&ws.d_bsum, sizeof(uint32_t) * (nb + 32)));
    ws.bsum_cap = nb;
  }
  const uint32_t* off = g->out_off();
  k_scan_sums<<<nb, kScanThreads, 0, g->stream>>>(in->d_queue, k, off, ws.d_bsum);
  k_scan_blocks<<<1, 1024, 0, g->stream>>>(ws.d_bsum, nb, ws.d_stats + 5);
  k_scan_write<<<nb, kScanThreads, 0, g->stream>>>(in->d_queue, k, off, ws.d_bsum, ws.d_scan);
  PushParams p{};
  p.q = in->d_queue;
  p.k = k;
  p.offs = ws.d_scan;
  p.total = ws.d_stats + 5;
  p.off = off;
  p.idx = g->out_idx();
  p.wts = g->out_w();
  p.deg_off = off;
  p.dedup = out->d_bits;
  p.out_q = nullptr;
  p.stats = ws.d_stats;
  const uint64_t work_ub = std::max<uint64_t>(in->out_edges, 1);
  const int grid = (int)std::min<uint64_t>((work_ub + kPushEdgesPerCta - 1) / kPushEdgesPerCta + 1,
                                           (uint64_t)g->num_sms * 8);
  k_push_bits<F, HW><<<std::max(grid, g->num_sms), kPushThreads, 0, g->stream>>>(p, f);
  GG_CUDA(cudaGetLastError());
  g->kernels += 4;
  return GG_OK;
}

// Internal edge_map flag (beside the GG_EM_* bits of the C ABI, which
// gg_edge_map passes on alone): with GG_EM_NO_OUTPUT, the caller waits for the
// stream itself, so the call need not.
constexpr uint32_t kEmNoWait = 0x80000000u;

template <class F>
int edge_map(gg_graph_s* g, gg_frontier_s* in, const F& f, int64_t threshold, uint32_t flags, gg_frontier_s** out) {
  const int64_t m = (int64_t)g->m;
  if (threshold < 0) threshold = m / 20;    // :932
  const int64_t dense_threshold = m / 2;    // :934
  if (in->n != g->n)  // :936-942 (an edgeMap result that was empty() carries 0 rows)
    return fail(GG_ERR_INVALID_ARG, "edgeMap: Sizes Don't match (numVertices %u and rows %u)", g->n, in->n);
  const int64_t fm = (int64_t)in->dm;
  const int64_t tot = (int64_t)in->out_edges;
  g->last = gg_edge_map_stats{};
  g->last.frontier_active = (uint64_t)fm;
  g->last.frontier_out_edges = (uint64_t)tot;
  gg_frontier_s* o = nullptr;
  GG_TRY(frontier_new(g, &o));
  if (tot == 0) {                           // :947 partitioned_vertices::empty()
    o->n = 0;
    *out = o;
    return GG_OK;
  }
  const bool hw = F::kUsesWeight && g->wtype != GG_W_NONE;
  int rc = GG_OK;
  bool dense = fm + tot > threshold;        // :953
  if (flags & GG_EM_FORCE_SPARSE) dense = false;
  if ((flags & (GG_EM_FORCE_CSC | GG_EM_FORCE_COO)) && !(flags & GG_EM_FORCE_SPARSE)) dense = true;
  auto prof_begin = [&]() {
    if (g->profiling) cudaEventRecord(g->prof_ev[0], g->stream);
  };
  auto prof_end = [&](int kind, uint64_t edges) {  // after read_stats (stream synchronised)
    if (!g->profiling) return;
    float ms = 0;
    cudaEventElapsedTime(&ms, g->prof_ev[0], g->prof_ev[1]);
    g->prof.launches[kind]++;
    g->prof.ms[kind] += ms;
    g->prof.edges[kind] += edges;
  };
  if (dense) {
    // :957 (!part_ver).  The GPU policy may pin the dense kernel, which keeps the
    // results only while the graph is not transposed: the reference never
    // transposes its COO partitions (graphgrind/graph-numa.h:721-728), so after
    // transpose() the COO and CSC kernels compute different maps and the
    // reference's rule is followed exactly.
    const bool ref_rule = g->dense_policy == 0 || g->transposed;
    bool coo = g->has_coo && (ref_rule ? fm + tot > dense_threshold : g->dense_policy == 2);
    if (flags & GG_EM_FORCE_CSC) coo = false;
    if ((flags & GG_EM_FORCE_COO) && g->has_coo) coo = true;
    const bool early = !coo && F::kEarlyExit;
    // a dense step of an early-exit functor from few frontier vertices (a
    // hub level): push the frontier's out-edges into the output bitmap
    // instead of walking every unvisited in-list
    const bool push_bits = early && !in->bit && g->push_dense_div > 0 && !(flags & GG_EM_FORCE_CSC) &&
                           (uint64_t)fm * (uint64_t)g->push_dense_div <= (uint64_t)g->n;
    // GG_EM_NO_OUTPUT: the caller discards the output, which the COO pull of a
    // sum functor then does not build
    const bool no_out = (flags & GG_EM_NO_OUTPUT) && coo && F::kIdentityCommitNoop;
    if (push_bits) {
      if (!in->has_sparse) rc = frontier_to_sparse(in);
    } else if (!in->bit && !in->has_dense) {
      rc = frontier_to_dense(in);
    }
    if (!rc) rc = frontier_ensure_bits(o, true);
    if (!rc) rc = reset_stats(g);
    if (!rc) {
      prof_begin();
      if (push_bits)
        rc = hw ? push_bits_launch<F, true>(g, in, o, f) : push_bits_launch<F, false>(g, in, o, f);
      else if (early)
        rc = hw ? pull_early_launch<F, true>(g, in, o, f) : pull_early_launch<F, false>(g, in, o, f);
      else
        rc = hw ? pull_launch<F, true>(g, in, o, f, coo, no_out) : pull_launch<F, false>(g, in, o, f, coo, no_out);
      if (g->profiling) cudaEventRecord(g->prof_ev[1], g->stream);
    }
    // an output nobody reads from a pull without waits (the direct-load COO
    // kernels; only the bulk-copy rings, 0/2/3, can set the error word), for
    // an application that synchronises later itself (kEmNoWait): no
    // statistics to read, and the stream goes on without a host round trip
    const bool skip_stats = no_out && (flags & kEmNoWait) && g->coo_kernel != 0 && g->coo_kernel != 2 &&
                            g->coo_kernel != 3;
    if (!rc && skip_stats && g->profiling) {
      if (cudaEventSynchronize(g->prof_ev[1]) != cudaSuccess) rc = fail(GG_ERR_CUDA, "edgeMap: profiling event");
    } else if (!rc && !skip_stats) {
      rc = read_stats(g);
    }
    if (!rc && no_out) {  // an output nobody reads: empty
      o->dm = 0;
      o->out_edges = 0;
      g->last.kind = 3;
      prof_end(2, g->coo_len);
    } else if (!rc) {
      o->has_dense = true;
      o->dm = g->ws.h_stats[0];
      o->out_edges = g->ws.h_stats[1];
      g->last.kind = coo ? 3 : 2;
      prof_end(push_bits ? 0 : (early ? 3 : (coo ? 2 : 1)), push_bits ? (uint64_t)tot : (coo ? g->coo_len : g->m));
    }
  } else {
    if (!in->has_sparse) rc = frontier_to_sparse(in);
    if (!rc) rc = frontier_ensure_queue(o);
    if (!rc) rc = reset_stats(g);
    if (!rc && in->dm > 0) {
      prof_begin();
      rc = hw ? push_launch<F, true>(g, in, o, f) : push_launch<F, false>(g, in, o, f);
      if (g->profiling) cudaEventRecord(g->prof_ev[1], g->stream);
    }
    if (!rc) rc = read_stats(g);
    if (!rc) {
      o->has_sparse = true;
      o->dm = g->ws.h_stats[2];
      o->out_edges = g->ws.h_stats[1];
      g->last.kind = 1;
      if (in->dm > 0) prof_end(0, g->ws.h_stats[5]);
    }
  }
  if (rc) {
    frontier_free(o);
    return rc;
  }
  g->last.output_active = o->dm;
  g->last.output_out_edges = o->out_edges;
  *out = o;
  return GG_OK;
}

// ------------------------------------------------------------ vertexMap
// graphgrind/ligra-numa.h:1023-1049
template <class VF>
int vertex_map(gg_graph_s* g, gg_frontier_s* f, const VF& vf) {
  const int grid = generic_grid(g, f->has_dense || f->bit ? g->n : std::max<uint64_t>(f->dm, 1));
  if (f->bit) {
    k_vertex_map<VF, 0><<<generic_grid(g, g->n), kGenericThreads, 0, g->stream>>>(g->n, nullptr, nullptr, 0, vf);
  } else if (f->has_dense) {
    k_vertex_map<VF, 1><<<grid, kGenericThreads, 0, g->stream>>>(g->n, f->d_bits, nullptr, 0, vf);
  } else if (f->has_sparse) {
    if (f->dm == 0) return GG_OK;
    k_vertex_map<VF, 2><<<grid, kGenericThreads, 0, g->stream>>>(g->n, nullptr, f->d_queue, f->dm, vf);
  } else {
    return GG_OK;  // empty
  }
  GG_CUDA(cudaGetLastError());
  g->kernels++;
  return GG_OK;
}

// ---------------------------------------------------------- vertexFilter
// graphgrind/ligra-numa.h:1053-1082: dense output plus (count, out-degree)
template <class VF>
int vertex_filter(gg_graph_s* g, gg_frontier_s* f, const VF& vf, gg_frontier_s** out) {
  gg_frontier_s* o = nullptr;
  GG_TRY(frontier_new(g, &o));
  int rc = GG_OK;
  if (!f->bit && !f->has_dense && f->dm > 0) rc = frontier_to_dense(f);
  if (!rc) rc = frontier_ensure_bits(o, true);
  if (!rc) rc = reset_stats(g);
  if (!rc) {
    const int grid = generic_grid(g, g->n);
    if (f->bit)
      k_vertex_filter<VF, true><<<grid, kGenericThreads, 0, g->stream>>>(g->n, nullptr, o->d_bits, g->out_off(),
                                                                        g->ws.d_stats, vf);
    else if (f->has_dense)
      k_vertex_filter<VF, false><<<grid, kGenericThreads, 0, g->stream>>>(g->n, f->d_bits, o->d_bits,
                                                                         g->out_off(), g->ws.d_stats, vf);
    if (cudaGetLastError() != cudaSuccess) rc = fail(GG_ERR_CUDA, "vertex_filter launch failed");
    g->kernels++;
  }
  if (!rc) rc = read_stats(g);
  if (rc) {
    frontier_free(o);
    return rc;
  }
  o->has_dense = true;
  o->dm = g->ws.h_stats[0];
  o->out_edges = g->ws.h_stats[1];
  *out = o;
  return GG_OK;
}

}  // namespace gg
