// Traversal engine for B200 (sm_100a): graph / vertexSubset state and the
// kernels behind edgeMap, vertexMap and vertexFilter.
//
//   k_pull      dense pull over CTA-owned destination tiles (CSC or the
//               partitioned COO): edges stream into shared memory by bulk
//               copies (cp.async.bulk + mbarrier ring), contributions reduce
//               into per-tile shared-memory accumulators, each destination is
//               committed once.  No global atomics on vertex values: the GPU
//               form of PART96's "one owner per destination range"
//               (graphgrind/ligra-numa.h:558-562, 810-832).
//   k_pull_early  dense pull for functors whose cond() turns false after one
//               successful update (BFS): one thread per destination stops at
//               the first frontier in-neighbour, as edgeMapDenseCSC's break
//               (graphgrind/ligra-numa.h:621-626).
//   k_push      sparse push over CSR (edgeMapSparseWithG, :868-916): the
//               frontier's degrees are prefix-summed, every thread takes
//               edges of the scanned range (load-balanced search), applies
//               cond && updateAtomic, and appends winners to a bitmap-
//               de-duplicated queue with warp-aggregated atomics.
//   k_bits_to_queue / k_queue_to_bits  vertexSubset conversion (toSparse
//               :246 by ballot/popc compaction, toDense :228).
//   k_vertex_map / k_vertex_filter      vertexMap :1023, vertexFilter :1053.
//
// Device functor protocol (the reference's update/updateAtomic/cond and
// functor-cache protocol, :364-543, in reduction form):
//   using value_t;                       32-bit contribution type
//   static constexpr bool kEarlyExit;    cond(d) is false after one update
//   bool    cond(d)                      = F::cond
//   value_t gather(s, w)                 contribution of source s (the read
//                                        half of update(cache, s[, w]))
//   static value_t identity(), combine(a, b), atomic_combine(smem*, v)
//   bool    commit(d, acc)               create_cache + updates + commit_cache:
//                                        applies the reduced contribution,
//                                        returns "d joins the output"
//   bool    update_atomic(s, d, w)       = F::updateAtomic (push)
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>
#include <utility>

#include <unordered_set>
#include <vector>

#include "gg_common.h"
#include "gg_device.cuh"

#define GG_CUDA(call)                                                                       \
  do {                                                                                      \
    cudaError_t e__ = (call);                                                               \
    if (e__ != cudaSuccess)                                                                 \
      return ::gg::fail(GG_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,            \
                        cudaGetErrorString(e__));                                           \
  } while (0)

#define GG_TRY(expr)          \
  do {                        \
    int r__ = (expr);         \
    if (r__ != GG_OK) return r__; \
  } while (0)

namespace gg {

// ------------------------------------------------------------ constants
constexpr int kPullThreads = 256;
constexpr int kPullK = 8;                                   // edges per thread per chunk
constexpr int kPullSlots = kPullThreads * kPullK;           // 2048 stage slots
constexpr int kPullChunk = kPullSlots - 8;                  // edges per chunk (8-aligned slack)
constexpr int kPullStages = 3;
constexpr int kMaxTileVertices = 4096;
constexpr int kMaxCooTileVertices = 16384;  // COO tiles (16-bit destination offsets)
constexpr uint32_t kPad = 0xffffffffu;                      // COO padding source id

constexpr int kPushThreads = 256;
constexpr int kPushEdgesPerCta = 4096;
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;        // 2048 queue entries per block

// -------------------------------------------------------- graph state
struct TileSet {
  uint4* d_tiles = nullptr;   // {v0, nv, e0, ne}, ordered by ne descending
  uint32_t count = 0;
  std::vector<uint4> host;
};

// Row structure of a CSC (or, transposed, CSR) edge stream for the
// segmented pull: bit j of `head` is set iff edge j is the first in-edge of
// its destination; blk[b] = number of heads in edges [0, 256 b); rows[r] =
// the vertex of the r-th non-empty row (the compressed CSC vertex list of
// the reference, PartitionByDest, graphgrind/graph-numa.h:1098-1107).
constexpr int kSegBlock = 256;  // edges per warp block
struct SegIndex {
  uint32_t* d_head = nullptr;
  uint32_t* d_blk = nullptr;
  uint32_t* d_rows = nullptr;
  uint64_t nrows = 0;
};

// Size of Workspace::h_map, the largest control block read back through it.
constexpr size_t kMapBytes = 4096;

struct Workspace {
  unsigned long long* d_stats = nullptr;  // [0] count [1] outdeg [2] queue len [3] err [4] tile ctr [5] total edges
  unsigned long long* h_stats = nullptr;  // pinned mirror
  uint32_t* d_dedup = nullptr;            // n bits, zero between calls
  uint32_t* d_scan = nullptr;             // n+1 offsets of the push scan
  uint32_t* d_bsum = nullptr;             // per-block sums of the scan
  uint32_t bsum_cap = 0;
  double* d_red = nullptr;                // reduction scratch (double)
  double* h_red = nullptr;                // pinned
  unsigned long long* d_loop = nullptr;   // state of the device-driven level loops (64 words)
  uint32_t* h_map = nullptr;              // pinned host block (kMapBytes) that kernels write directly
  uint32_t* d_map = nullptr;              //   and its device address
  // renumbered graphs: n-entry arrays for the given-order copies (0, 1); with
  // GG_TUNE_ASYNC_RESULTS also BFS's parents (2), so that they need not wait
  // for the copy out of array 0 of the application before
  uint32_t* d_order[3] = {nullptr, nullptr, nullptr};
};

struct PrLoop;  // PageRank iterations captured as a CUDA graph (buffers, graph, control block)
struct RoundLoop;  // dense COO rounds of BellmanFord / Components captured as a CUDA graph

}  // namespace gg

struct gg_graph_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 148;
  uint32_t n = 0;
  uint64_t m = 0;
  bool symmetric = false;
  int wtype = GG_W_NONE;
  gg_build_opts opts{};
  std::vector<int64_t> coo_sizes, coo_starts, csc_sizes, csc_starts;
  // device CSR / CSC of the ORIGINAL orientation
  uint32_t *d_csr_off = nullptr, *d_csr_idx = nullptr, *d_csr_w = nullptr;
  uint32_t *d_csc_off = nullptr, *d_csc_idx = nullptr, *d_csc_w = nullptr;
  std::vector<uint32_t> h_csr_off, h_csc_off;  // host copies of the offsets
  gg::TileSet csc_tiles[2];  // [0]: pull over CSC (in-edges); [1]: transposed (pull over CSR)
  gg::SegIndex seg[2];       // row structure of the pulled stream, same indexing
  uint64_t m_pad = 0;        // edge arrays hold m_pad entries (zero padded)
  gg::TileSet coo_tiles;
  uint2* d_coo_gaps = nullptr;  // {first, count} of the destination ranges outside every COO tile
  uint32_t coo_gap_count = 0;
  bool has_coo = false;
  bool coo_by_source = false;       // -P source: partitions of sources, destinations in d_coo_dst
  uint32_t* d_coo_dst = nullptr;
  uint32_t *d_coo_src = nullptr, *d_coo_w = nullptr;
  uint16_t* d_coo_dloc = nullptr;
  uint64_t coo_len = 0;
  bool transposed = false;
  gg::Workspace ws;
  gg_edge_map_stats last{};
  bool profiling = false;
  gg_profile prof{};
  cudaEvent_t prof_ev[2] = {nullptr, nullptr};
  int dense_policy = 0;
  int sparse_div = 20;  // the apps' edgeMap threshold is m / sparse_div (app/*.C pass m/20)
  int device_loop = 2;  // 2: the whole BFS in one cooperative launch; 1: runs of sparse levels; 0: none
  int cc_algo = 0;      // Components on symmetric graphs: 0 label propagation, 1 union-find
  int loop_ctas_per_sm = 0;  // CTAs per SM of the device BFS loops (capped by occupancy); 0: 4 / 8 by loop
  uint32_t loop_wait_budget = 1u << 22;  // spins of the BFS level loop's grid-barrier wait
  int early_kernel = 3;  // early-exit dense pull: 0 one lane per destination, 1 8-lane groups, 2 one lane per
                         // destination reading 4 in-edges per load, 3 the same over in-lists with hub sources
                         // first (fastest on R-MAT)
  int push_dense_div = 0;  // a dense edgeMap of an early-exit functor pushes into a bitmap when
                           // the frontier has at most n / push_dense_div vertices (0: never)
  int pr_graph = 1;     // PageRank iterations replayed as one CUDA graph (0: one host round trip per iteration)
  // GG_TUNE_ASYNC_RESULTS: results bound for pinned host memory leave from the
  // given-order arrays on copy_stream, and the call returns without waiting
  int async_results = 0;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t result_ready = nullptr;                // on stream: the result to copy is complete
  cudaEvent_t input_ready = nullptr;                 // on copy_stream: a staged SpMV input has arrived
  bool input_staged = false;                         // given-order array 1 holds a staged SpMV input
  cudaEvent_t slot_copied[3] = {nullptr, nullptr, nullptr};  // on copy_stream: the last copy out of ws.d_order[k]
  gg::PrLoop* pr_loop = nullptr;  // created by the first graph-driven PageRank call
  gg::RoundLoop* round_loop[3] = {nullptr, nullptr, nullptr};  // BellmanFord, Components, PageRankDelta: created by their first call
  int round_graph = 1;  // dense COO rounds of BellmanFord / Components / PageRankDelta as a CUDA graph
  // GG_TUNE_EARLY_KERNEL 3's in-lists (the CSC's, each by descending source
  // out-degree), built by the first all-levels BFS (m_pad entries)
  uint32_t* d_bu_idx = nullptr;
  int coo_kernel = 7;  // 0 CTA ring (k_pull), 1 per-warp direct loads, 2/3 per-warp bulk-copy rings, 6 direct loads
                       // with cross-lane run merging, 7 the same with cache hints (fastest measured)
  // gg_build_opts.vertex_order: device ids differ from the given ids
  bool relabeled = false;
  std::vector<uint32_t> h_new_of_old, h_old_of_new;
  uint32_t *d_new_of_old = nullptr, *d_old_of_new = nullptr;
  uint32_t device_id(uint32_t v) const { return relabeled ? h_new_of_old[v] : v; }
  uint64_t device_bytes = 0;
  int kernels = 0;  // kernels launched since the counter was last reset
  std::unordered_set<gg_frontier_s*> frontiers;  // live frontiers (freed with the graph)
  std::unordered_set<void*> arrays;             // live vertex arrays
  // current orientation views
  const uint32_t* out_off() const { return transposed ? d_csc_off : d_csr_off; }
  const uint32_t* out_idx() const { return transposed ? d_csc_idx : d_csr_idx; }
  const uint32_t* out_w() const { return transposed ? d_csc_w : d_csr_w; }
  const uint32_t* in_off() const { return transposed ? d_csr_off : d_csc_off; }
  const uint32_t* in_idx() const { return transposed ? d_csr_idx : d_csc_idx; }
  const uint32_t* in_w() const { return transposed ? d_csr_w : d_csc_w; }
  const uint32_t* h_out_off() const { return transposed ? h_csc_off.data() : h_csr_off.data(); }
  uint32_t words() const { return (n + 31) / 32; }
};

struct gg_frontier_s {
  gg_graph_s* g = nullptr;
  uint32_t n = 0;
  bool bit = false;         // "all vertices active" (partitioned_vertices::bit)
  bool has_dense = false;
  bool has_sparse = false;
  uint32_t* d_bits = nullptr;   // words()+4
  uint32_t* d_queue = nullptr;  // n+4
  uint64_t dm = 0;              // d_m
  uint64_t out_edges = 0;       // num_out_edges
};

namespace gg {

// Handle registry: C-ABI calls on a destroyed graph or frontier fail with
// GG_ERR_INVALID_ARG instead of touching freed memory.
bool graph_live(const gg_graph_s* g);
bool frontier_live(const gg_frontier_s* f);

// ===================================================== kernel parameters
struct PullParams {
  const uint4* tiles;
  uint32_t ntiles;
  unsigned long long* tile_counter;
  const uint32_t* src;      // CSC in-neighbour ids or COO sources
  const uint16_t* dloc;     // COO destination offsets inside the tile
  const uint32_t* wts;      // weights aligned with src (raw 32-bit)
  const uint32_t* off;      // CSC offsets (absolute), CSC layout only
  const uint32_t* fr_bits;  // frontier bitmap (unused when all active)
  uint32_t* next_bits;      // output bitmap, zeroed by the caller
  const uint32_t* deg_off;  // out-offsets of the current orientation (stats)
  const uint32_t* member_off;  // original in-offsets: compressed-CSC membership, or null
  unsigned long long* stats;   // [0] count [1] out-degree sum
  unsigned long long* err;
  uint32_t tv;                 // widest tile of the tile set
};

// tv: the widest tile of the tile set (its accumulators and flags are sized by it)
__host__ __device__ constexpr size_t pull_smem_bytes(bool coo, bool hw, int vbytes, uint32_t tv = kMaxTileVertices) {
  return 128                                                       // mbarriers
         + (size_t)kPullStages * kPullSlots * 4                     // src
         + (hw ? (size_t)kPullStages * kPullSlots * 4 : 0)          // weights
         + (coo ? (size_t)kPullStages * kPullSlots * 2 : 0)         // dloc
         + (size_t)((tv + 3) & ~3u) * vbytes                         // accumulators
         + (coo ? 0 : (size_t)(tv + 4) * 4)                         // tile offsets
         + (size_t)((tv + 3) & ~3u) * 2;                             // touched + cond flags
}

// One CTA per tile at a time; CTAs pull tiles from a global ticket counter
// (tiles are ordered by edge count, largest first).
template <class F, bool COO, bool HW, bool ALL>
__global__ void __launch_bounds__(kPullThreads, 2) k_pull(const PullParams p, const F f) {
  using V = typename F::value_t;
  extern __shared__ __align__(128) unsigned char smem[];
  const uint32_t tv4 = (p.tv + 3) & ~3u;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
  uint32_t* s_src = reinterpret_cast<uint32_t*>(smem + 128);
  uint32_t* s_w = s_src + kPullStages * kPullSlots;
  uint16_t* s_dl = reinterpret_cast<uint16_t*>(s_w + (HW ? kPullStages * kPullSlots : 0));
  V* s_acc = reinterpret_cast<V*>(s_dl + (COO ? kPullStages * kPullSlots : 0));
  uint32_t* s_off = reinterpret_cast<uint32_t*>(s_acc + tv4);
  uint8_t* s_touch = reinterpret_cast<uint8_t*>(s_off + (COO ? 0 : p.tv + 4));
  uint8_t* s_cond = s_touch + tv4;
  __shared__ uint32_t s_tile;
  __shared__ unsigned long long s_red[2][kPullThreads / 32];
  __shared__ int s_fail;

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    for (int s = 0; s < kPullStages; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
    s_fail = 0;
  }
  __syncthreads();
  uint32_t parity = 0;  // bit s: parity of the next wait on stage s
  unsigned long long my_cnt = 0, my_deg = 0;

  for (;;) {
    if (tid == 0) s_tile = (uint32_t)atomicAdd(p.tile_counter, 1ull);
    __syncthreads();
    const uint32_t t = s_tile;
    if (t >= p.ntiles || s_fail) break;
    const uint4 td = p.tiles[t];
    const uint32_t v0 = td.x, nv = td.y, e0 = td.z, ne = td.w;
    const uint32_t nchunks = (ne + kPullChunk - 1) / kPullChunk;

    auto issue = [&](uint32_t c, int st) {
      const uint32_t cs = e0 + c * kPullChunk;
      const uint32_t ce = min(e0 + ne, cs + kPullChunk);
      const uint32_t ca = cs & ~7u, cb = (ce + 7u) & ~7u;
      const uint32_t nel = cb - ca;
      const uint32_t bytes = nel * 4u * (HW ? 2u : 1u) + (COO ? nel * 2u : 0u);
      mbar_arrive_expect_tx(&bars[st], bytes);
      bulk_g2s(s_src + st * kPullSlots, p.src + ca, nel * 4u, &bars[st]);
      if (HW) bulk_g2s(s_w + st * kPullSlots, p.wts + ca, nel * 4u, &bars[st]);
      if (COO) bulk_g2s(s_dl + st * kPullSlots, p.dloc + ca, nel * 2u, &bars[st]);
    };
    if (tid == 0) {
      for (uint32_t c = 0; c < nchunks && c < (uint32_t)kPullStages; ++c) issue(c, (int)c);
    }
    for (uint32_t i = tid; i < nv; i += kPullThreads) {
      const uint32_t v = v0 + i;
      s_acc[i] = F::identity();
      s_touch[i] = 0;
      bool c = f.cond(v);
      if (p.member_off) c = c && (__ldg(p.member_off + v + 1) > __ldg(p.member_off + v));
      s_cond[i] = c ? 1 : 0;
      if (!COO) s_off[i] = __ldg(p.off + v);
    }
    if (!COO && tid == 0) s_off[nv] = __ldg(p.off + v0 + nv);
    __syncthreads();

    uint32_t issued = nchunks < (uint32_t)kPullStages ? nchunks : (uint32_t)kPullStages;
    for (uint32_t c = 0; c < nchunks; ++c) {
      const int st = (int)(c % kPullStages);
      // a timed-out wait skips this chunk's edges (the stage may hold stale data)
      const bool ok = mbar_wait_bounded(&bars[st], (parity >> st) & 1u);
      if (!ok) {
        atomicOr(p.err, (unsigned long long)DEV_ERR_TIMEOUT);
        s_fail = 1;
      }
      parity ^= 1u << st;
      const uint32_t cs = e0 + c * kPullChunk;
      const uint32_t ce = min(e0 + ne, cs + kPullChunk);
      const uint32_t ca = cs & ~7u;
      // this thread's 8 stage slots: positions ca + 8*tid .. +7
      const uint32_t pos0 = ca + (uint32_t)tid * kPullK;
      const uint32_t* ssrc = s_src + st * kPullSlots + tid * kPullK;
      uint32_t sv[kPullK], wv[kPullK];
      uint16_t dv[kPullK];
      {
        const uint4 a = reinterpret_cast<const uint4*>(ssrc)[0];
        const uint4 b = reinterpret_cast<const uint4*>(ssrc)[1];
        sv[0] = a.x; sv[1] = a.y; sv[2] = a.z; sv[3] = a.w;
        sv[4] = b.x; sv[5] = b.y; sv[6] = b.z; sv[7] = b.w;
      }
      if (HW) {
        const uint32_t* sw = s_w + st * kPullSlots + tid * kPullK;
        const uint4 a = reinterpret_cast<const uint4*>(sw)[0];
        const uint4 b = reinterpret_cast<const uint4*>(sw)[1];
        wv[0] = a.x; wv[1] = a.y; wv[2] = a.z; wv[3] = a.w;
        wv[4] = b.x; wv[5] = b.y; wv[6] = b.z; wv[7] = b.w;
      } else {
#pragma unroll
        for (int k = 0; k < kPullK; ++k) wv[k] = 1u;
      }
      if (COO) {
        const uint4 a = reinterpret_cast<const uint4*>(s_dl + st * kPullSlots + tid * kPullK)[0];
        dv[0] = a.x & 0xffff; dv[1] = a.x >> 16; dv[2] = a.y & 0xffff; dv[3] = a.y >> 16;
        dv[4] = a.z & 0xffff; dv[5] = a.z >> 16; dv[6] = a.w & 0xffff; dv[7] = a.w >> 16;
      }
      // The slots are processed in phases so that each thread keeps all of
      // its frontier-bit loads, then all of its gathers, in flight at once.
      // phase 1: tile-local destination and validity of every slot
      uint32_t lv[kPullK];
      bool vld[kPullK];
      uint32_t li = 0;
      if (!COO && ok && pos0 + kPullK > cs && pos0 < ce) {
        // last tile-local vertex whose offset is <= max(pos0, cs)
        const uint32_t key = max(pos0, cs);
        uint32_t lo = 0, hi = nv;  // invariant: s_off[lo] <= key < s_off[hi]
        while (hi - lo > 1) {
          const uint32_t mid = (lo + hi) >> 1;
          if (s_off[mid] <= key) lo = mid; else hi = mid;
        }
        li = lo;
      }
#pragma unroll
      for (int k = 0; k < kPullK; ++k) {
        const uint32_t pos = pos0 + k;
        bool v = ok && pos >= cs && pos < ce;
        uint32_t l = 0;
        if (COO) {
          v = v && sv[k] != kPad;
          l = dv[k];
        } else if (v) {
          while (s_off[li + 1] <= pos) ++li;
          l = li;
        }
        lv[k] = l;
        vld[k] = v && (F::kCondTrue || s_cond[l]);
      }
      // phase 2: frontier membership of the sources (independent loads)
      if (!ALL) {
#pragma unroll
        for (int k = 0; k < kPullK; ++k)
          if (vld[k]) vld[k] = test_bit(p.fr_bits, sv[k]);
      }
      // phase 3: contributions (independent gathers)
      V val[kPullK];
#pragma unroll
      for (int k = 0; k < kPullK; ++k) {
        val[k] = vld[k] ? f.gather(sv[k], wv[k]) : F::identity();
        // positive functors mark sources outside the frontier with a negative value
        if (F::kPositive) vld[k] = vld[k] && !(val[k] < F::identity());
      }
      // phase 4: run accumulation into the tile's shared-memory accumulators
      int cur = -1;
      V acc = F::identity();
#pragma unroll
      for (int k = 0; k < kPullK; ++k) {
        if (!vld[k]) continue;
        const int l = (int)lv[k];
        if (l != cur) {
          if (cur >= 0) {
            F::atomic_combine(&s_acc[cur], acc);
            if (!F::kPositive) s_touch[cur] = 1;
          }
          cur = l;
          acc = val[k];
        } else {
          acc = F::combine(acc, val[k]);
        }
      }
      // final run: warp-aggregate when the whole warp ends on one destination
      const int c0 = __shfl_sync(0xffffffffu, cur, 0);
      if (__all_sync(0xffffffffu, cur == c0) && c0 >= 0) {
        V r = acc;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r = F::combine(r, __shfl_xor_sync(0xffffffffu, r, o));
        if (lane == 0) {
          F::atomic_combine(&s_acc[c0], r);
          if (!F::kPositive) s_touch[c0] = 1;
        }
      } else if (cur >= 0) {
        F::atomic_combine(&s_acc[cur], acc);
        if (!F::kPositive) s_touch[cur] = 1;
      }
      __syncthreads();  // stage st fully consumed
      if (s_fail) {
        // drain the copies still in flight (bounded), then leave
        for (uint32_t cc = c + 1; cc < issued; ++cc) {
          const int s2 = (int)(cc % kPullStages);
          mbar_wait_bounded(&bars[s2], (parity >> s2) & 1u);
          parity ^= 1u << s2;
        }
        break;
      }
      if (c + kPullStages < nchunks) {
        if (tid == 0) {
          fence_proxy_async_smem();
          issue(c + kPullStages, st);
        }
        ++issued;
      }
    }
    if (s_fail) break;
    // commit: one thread per destination, warp-aligned on global vertex ids
    const uint32_t base0 = v0 & ~31u;
    for (uint32_t b = base0 + (uint32_t)warp * 32u; b < v0 + nv; b += kPullThreads) {
      const uint32_t v = b + (uint32_t)lane;
      bool act = false;
      if (v >= v0 && v < v0 + nv) {
        const uint32_t l = v - v0;
        const bool touched = F::kPositive ? (s_acc[l] != F::identity()) : (s_touch[l] != 0);
        if (touched && s_cond[l]) act = f.commit(v, s_acc[l]);
      }
      const uint32_t word = __ballot_sync(0xffffffffu, act);
      if (act) my_deg += __ldg(p.deg_off + v + 1) - __ldg(p.deg_off + v);
      if (lane == 0 && word) {
        atomicOr(p.next_bits + (b >> 5), word);
        my_cnt += __popc(word);
      }
    }
    __syncthreads();
  }
  // block reduction of the output statistics
  my_deg = warp_sum(my_deg);
  my_cnt = warp_sum(my_cnt);
  if (lane == 0) {
    s_red[0][warp] = my_cnt;
    s_red[1][warp] = my_deg;
  }
  __syncthreads();
  if (tid == 0) {
    unsigned long long a = 0, b = 0;
    for (int w = 0; w < kPullThreads / 32; ++w) {
      a += s_red[0][w];
      b += s_red[1][w];
    }
    if (a) atomicAdd(p.stats + 0, a);
    if (b) atomicAdd(p.stats + 1, b);
  }
}

// ------------------------------------------ per-warp partitioned-COO pull
// Same tile ownership as k_pull (shared-memory accumulators, one commit per
// destination), but every warp streams its own 256-edge blocks of the tile:
// STAGES > 0 through a private bulk-copy ring in shared memory, STAGES == 0
// with direct 16-byte loads (no staging; all of L1 left to the source
// gathers).  No CTA-wide barrier per block.
// F::kFinish when the functor declares it (a vertex step the per-warp COO
// pull applies to every destination of a tile at its commit), else false
template <class F, class = void>
struct finishes {
  static constexpr bool value = false;
};
template <class F>
struct finishes<F, decltype((void)F::kFinish)> {
  static constexpr bool value = F::kFinish;
};

constexpr int kCooWarps = 8;
constexpr int kCooThreads = kCooWarps * 32;

__host__ __device__ constexpr size_t coo_w_stage_bytes(bool hw) {
  return (size_t)kSegBlock * 4 + (size_t)kSegBlock * 2 + (hw ? (size_t)kSegBlock * 4 : 0);
}
// Per tile destination: the accumulator plus a "touched" byte (functors whose
// identity does not mark untouched destinations, when the output is kept)
// and a "cond" byte (functors with a condition on the destination).
template <class F, bool NOOUT>
__host__ __device__ constexpr int coo_w_flag_bytes() {
  return (!F::kPositive && !NOOUT ? 1 : 0) + (F::kCondTrue ? 0 : 1);
}
__host__ __device__ constexpr size_t coo_w_smem_bytes(bool hw, int stages, int vbytes, uint32_t tv, int flag_bytes = 2) {
  return (stages > 0 ? 256 : 0) + (size_t)kCooWarps * stages * coo_w_stage_bytes(hw) +
         (size_t)((tv + 3) & ~3u) * (vbytes + flag_bytes);
}

#ifndef GG_COO_MIN_BLOCKS
#define GG_COO_MIN_BLOCKS 4  // resident CTAs per SM the register allocation must allow
#endif
// NOOUT: the caller discards edgeMap's output (GG_EM_NO_OUTPUT) and F's
// commit of the identity is a no-op (sums): no touched flags, no next-frontier
// bits, no stats; destinations with a non-identity sum are committed.
// MERGE: destination runs that continue across lanes are combined with warp
// shuffles before the shared-memory accumulation, so a destination appears in
// at most one accumulation per block (instead of one per lane it spans, all
// on one address).
// The pull as a device function, so that a persistent loop kernel can run it
// once per iteration (k_pull_coo_w is one call of it).
// F::gather_pol (a gather that takes an L2 eviction policy), when declared
template <class F, class = void>
struct has_gather_pol : std::false_type {};
template <class F>
struct has_gather_pol<F, decltype((void)std::declval<const F&>().gather_pol(0u, 0u, 0ull))> : std::true_type {};

// HINT bits of the direct-load pull: 1 the edge stream bypasses L1 and is
// marked evict-first in L2; 2 the source gathers (functors with gather_pol)
// are marked evict-last in L1 and L2; 4 a vertex step at the commits
// (PrFinishF) issues the loads of four 32-vertex groups before it uses them.
template <class F, bool HW, bool ALL, int STAGES, bool CONTIG, bool PF, bool NOOUT, bool MERGE, int HINT = 0>
__device__ __forceinline__ void pull_coo_w_run(const PullParams& p, const F& f) {
  static_assert(!NOOUT || F::kIdentityCommitNoop, "discarding the output needs a no-op identity commit");
  constexpr bool kFin = finishes<F>::value;  // the vertex step runs at the commit (PrFinishF)
  static_assert(!kFin || (!NOOUT && F::kPositive && F::kCondTrue), "the vertex step needs the output");
  static_assert(!CONTIG || STAGES == 0, "lane-contiguous edges use direct loads");
  static_assert(!PF || (STAGES == 0 && !CONTIG), "register prefetch applies to direct loads");
  using V = typename F::value_t;
  extern __shared__ __align__(128) unsigned char smem[];
  constexpr uint32_t SB = (uint32_t)coo_w_stage_bytes(HW);
  const uint32_t tv4 = (p.tv + 3) & ~3u;
  constexpr bool kTouch = !F::kPositive && !NOOUT;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
  unsigned char* stages = smem + (STAGES > 0 ? 256 : 0);
  V* s_acc = reinterpret_cast<V*>(stages + (size_t)kCooWarps * STAGES * SB);
  uint8_t* s_touch = reinterpret_cast<uint8_t*>(s_acc + tv4);  // kTouch only
  uint8_t* s_cond = s_touch + (kTouch ? tv4 : 0);              // !F::kCondTrue only
  __shared__ uint32_t s_tile;
  __shared__ unsigned long long s_red[2][kCooWarps];
  __shared__ double s_l1[kFin ? kCooWarps : 1];
  __shared__ int s_fail;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint64_t* wbar = bars + warp * (STAGES > 0 ? STAGES : 1);
  unsigned char* wst = stages + (size_t)warp * STAGES * SB;
  if (STAGES > 0 && lane == 0)
    for (int s = 0; s < STAGES; ++s) mbar_init(&wbar[s], 1);
  if (tid == 0) s_fail = 0;
  if (STAGES > 0) fence_mbar_init();
  __syncthreads();
  uint32_t parity = 0;
  unsigned long long my_cnt = 0, my_deg = 0;
  double my_l1 = 0;
  constexpr bool kStreamHint = (HINT & 1) != 0 && STAGES == 0 && !CONTIG && !PF;
  constexpr bool kGatherHint = (HINT & 2) != 0 && has_gather_pol<F>::value;
  const uint64_t pol_stream = kStreamHint ? l2_policy_evict_first() : 0ull;
  const uint64_t pol_keep = kGatherHint ? l2_policy_evict_last() : 0ull;
  auto gather = [&](uint32_t s, uint32_t w) -> V {
    if constexpr (kGatherHint)
      return f.gather_pol(s, w, pol_keep);
    else
      return f.gather(s, w);
  };
  auto ld16 = [&](const void* ptr) -> uint4 {
    if constexpr (kStreamHint)
      return ld_stream_v4(ptr, pol_stream);
    else
      return __ldg(reinterpret_cast<const uint4*>(ptr));
  };

  for (;;) {
    if (tid == 0) s_tile = (uint32_t)atomicAdd(p.tile_counter, 1ull);
    __syncthreads();
    const uint32_t t = s_tile;
    if (t >= p.ntiles || s_fail) break;
    const uint4 td = p.tiles[t];
    const uint32_t v0 = td.x, nv = td.y, e0 = td.z, ne = td.w;  // e0, ne multiples of 8
    for (uint32_t i = tid; i < nv; i += kCooThreads) {
      s_acc[i] = F::identity();
      if (kTouch) s_touch[i] = 0;
      if (!F::kCondTrue) s_cond[i] = f.cond(v0 + i) ? 1 : 0;
    }
    __syncthreads();
    const uint32_t nb = (ne + kSegBlock - 1) / kSegBlock;
    const uint32_t nbw = (uint32_t)warp < nb ? (nb - (uint32_t)warp + kCooWarps - 1) / kCooWarps : 0;
    auto blk_len = [&](uint32_t j) { return min((uint32_t)kSegBlock, ne - j * kSegBlock); };
    auto issue = [&](uint32_t i, int st) {
      const uint32_t j = (uint32_t)warp + i * kCooWarps;
      const uint32_t b0 = e0 + j * kSegBlock, nel = blk_len(j);
      unsigned char* d = wst + st * SB;
      mbar_arrive_expect_tx(&wbar[st], nel * (HW ? 10u : 6u));
      bulk_g2s(d, p.src + b0, nel * 4, &wbar[st]);
      bulk_g2s(d + kSegBlock * 4, p.dloc + b0, nel * 2, &wbar[st]);
      if (HW) bulk_g2s(d + kSegBlock * 6, p.wts + b0, nel * 4, &wbar[st]);
    };
    uint32_t issued = 0;
    if constexpr (STAGES > 0) {
      if (lane == 0)
        for (uint32_t i = 0; i < nbw && i < (uint32_t)STAGES; ++i) issue(i, (int)i);
      issued = nbw < (uint32_t)STAGES ? nbw : (uint32_t)STAGES;
    }
    // PF: the next block's edge stream is loaded into registers while the
    // current block's gathers are in flight
    uint4 pa = make_uint4(0, 0, 0, 0), pc = pa, pq = pa, pu = pa, pw = pa;
    auto pload = [&](uint32_t i2) {
      const uint32_t j2 = (uint32_t)warp + i2 * kCooWarps;
      if ((uint32_t)lane * 8 < blk_len(j2)) {
        const size_t b = (size_t)e0 + (size_t)j2 * kSegBlock + (size_t)lane * 8;
        pa = __ldg(reinterpret_cast<const uint4*>(p.src + b));
        pc = __ldg(reinterpret_cast<const uint4*>(p.src + b) + 1);
        pq = __ldg(reinterpret_cast<const uint4*>(p.dloc + b));
        if (HW) {
          pu = __ldg(reinterpret_cast<const uint4*>(p.wts + b));
          pw = __ldg(reinterpret_cast<const uint4*>(p.wts + b) + 1);
        }
      }
    };
    if constexpr (PF) {
      if (nbw > 0) pload(0);
    }
    for (uint32_t i = 0; i < nbw; ++i) {
      const uint32_t j = (uint32_t)warp + i * kCooWarps;
      const uint32_t nel = blk_len(j);
      const bool in = (uint32_t)lane * 8 < nel;  // 8-slot groups are wholly in or out
      uint32_t sv[8], wv[8];
      uint16_t dv[8];
      if constexpr (STAGES > 0) {
        const int st = (int)(i % STAGES);
        const bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(&wbar[st], (parity >> st) & 1u));
        parity ^= 1u << st;
        if (!ok) {
          if (lane == 0) atomicOr(p.err, (unsigned long long)DEV_ERR_TIMEOUT);
          s_fail = 1;
          for (uint32_t cc = i + 1; cc < issued; ++cc) {
            const int s2 = (int)(cc % STAGES);
            mbar_wait_bounded(&wbar[s2], (parity >> s2) & 1u);
            parity ^= 1u << s2;
          }
          break;
        }
        const unsigned char* d = wst + st * SB;
        if (in) {
          const uint4 a = reinterpret_cast<const uint4*>(d)[lane * 2];
          const uint4 c = reinterpret_cast<const uint4*>(d)[lane * 2 + 1];
          sv[0] = a.x; sv[1] = a.y; sv[2] = a.z; sv[3] = a.w;
          sv[4] = c.x; sv[5] = c.y; sv[6] = c.z; sv[7] = c.w;
          const uint4 q = reinterpret_cast<const uint4*>(d + kSegBlock * 4)[lane];
          dv[0] = q.x & 0xffff; dv[1] = q.x >> 16; dv[2] = q.y & 0xffff; dv[3] = q.y >> 16;
          dv[4] = q.z & 0xffff; dv[5] = q.z >> 16; dv[6] = q.w & 0xffff; dv[7] = q.w >> 16;
          if (HW) {
            const uint4 u = reinterpret_cast<const uint4*>(d + kSegBlock * 6)[lane * 2];
            const uint4 v = reinterpret_cast<const uint4*>(d + kSegBlock * 6)[lane * 2 + 1];
            wv[0] = u.x; wv[1] = u.y; wv[2] = u.z; wv[3] = u.w;
            wv[4] = v.x; wv[5] = v.y; wv[6] = v.z; wv[7] = v.w;
          }
        }
        __syncwarp();
        if (lane == 0 && i + STAGES < nbw) {
          fence_proxy_async_smem();
          issue(i + STAGES, st);
        }
        if (i + STAGES < nbw) ++issued;
      } else if (CONTIG) {
        // lane l takes edges 32 k + l of the block: each gather instruction
        // covers 32 consecutive (source-ordered) edges
        const size_t b0 = (size_t)e0 + (size_t)j * kSegBlock + (size_t)lane;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const bool ink = (uint32_t)(32 * k + lane) < nel;
          sv[k] = ink ? __ldg(p.src + b0 + 32 * k) : kPad;
          dv[k] = ink ? __ldg(p.dloc + b0 + 32 * k) : (uint16_t)0;
          if (HW) wv[k] = ink ? __ldg(p.wts + b0 + 32 * k) : 0u;
        }
      } else if (PF) {
        const uint4 a = pa, c = pc, q = pq, u = pu, w = pw;
        if (i + 1 < nbw) pload(i + 1);
        if (in) {
          sv[0] = a.x; sv[1] = a.y; sv[2] = a.z; sv[3] = a.w;
          sv[4] = c.x; sv[5] = c.y; sv[6] = c.z; sv[7] = c.w;
          dv[0] = q.x & 0xffff; dv[1] = q.x >> 16; dv[2] = q.y & 0xffff; dv[3] = q.y >> 16;
          dv[4] = q.z & 0xffff; dv[5] = q.z >> 16; dv[6] = q.w & 0xffff; dv[7] = q.w >> 16;
          if (HW) {
            wv[0] = u.x; wv[1] = u.y; wv[2] = u.z; wv[3] = u.w;
            wv[4] = w.x; wv[5] = w.y; wv[6] = w.z; wv[7] = w.w;
          }
        }
      } else if (in) {
        const size_t b0 = (size_t)e0 + (size_t)j * kSegBlock + (size_t)lane * 8;
        const uint4 a = ld16(p.src + b0);
        const uint4 c = ld16(p.src + b0 + 4);
        sv[0] = a.x; sv[1] = a.y; sv[2] = a.z; sv[3] = a.w;
        sv[4] = c.x; sv[5] = c.y; sv[6] = c.z; sv[7] = c.w;
        const uint4 q = ld16(p.dloc + b0);
        dv[0] = q.x & 0xffff; dv[1] = q.x >> 16; dv[2] = q.y & 0xffff; dv[3] = q.y >> 16;
        dv[4] = q.z & 0xffff; dv[5] = q.z >> 16; dv[6] = q.w & 0xffff; dv[7] = q.w >> 16;
        if (HW) {
          const uint4 u = ld16(p.wts + b0);
          const uint4 v = ld16(p.wts + b0 + 4);
          wv[0] = u.x; wv[1] = u.y; wv[2] = u.z; wv[3] = u.w;
          wv[4] = v.x; wv[5] = v.y; wv[6] = v.z; wv[7] = v.w;
        }
      }
      if (!HW) {
#pragma unroll
        for (int k = 0; k < 8; ++k) wv[k] = 1u;
      }
      bool vld[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) vld[k] = (CONTIG || in) && sv[k] != kPad && (F::kCondTrue || s_cond[dv[k]]);
      if (!ALL) {
#pragma unroll
        for (int k = 0; k < 8; ++k)
          if (vld[k]) vld[k] = test_bit(p.fr_bits, sv[k]);
      }
      V val[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        val[k] = vld[k] ? gather(sv[k], wv[k]) : F::identity();
        if (F::kPositive) vld[k] = vld[k] && !(val[k] < F::identity());
      }
      if constexpr (CONTIG) {
        // destinations of consecutive source-ordered edges are scattered:
        // one shared-memory accumulation per edge
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          if (!vld[k]) continue;
          F::atomic_combine(&s_acc[dv[k]], val[k]);
          if (kTouch) s_touch[dv[k]] = 1;
        }
        continue;
      }
      auto flush = [&](int l, V v) {
        F::atomic_combine(&s_acc[l], v);
        if (kTouch) s_touch[l] = 1;
      };
      if constexpr (MERGE) {
        // The block is sorted by destination, so a lane's middle runs are
        // complete and go straight to shared memory, while its first run
        // (held back when the lane has two or more) and its last run may
        // continue in the neighbouring lanes.
        int cur = -1, hd = -1;
        V acc = F::identity(), ha = F::identity();
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          if (!vld[k]) continue;
          const int l = (int)dv[k];
          if (l != cur) {
            if (cur >= 0) {
              if (hd < 0) {
                hd = cur;
                ha = acc;
              } else {
                flush(cur, acc);
              }
            }
            cur = l;
            acc = val[k];
          } else {
            acc = F::combine(acc, val[k]);
          }
        }
        // a held-back first run joins the previous lane's last run
        const int nhd = __shfl_down_sync(0xffffffffu, hd, 1);
        const V nha = __shfl_down_sync(0xffffffffu, ha, 1);
        const int ptl = __shfl_up_sync(0xffffffffu, cur, 1);
        if (lane < 31 && nhd >= 0 && nhd == cur) acc = F::combine(acc, nha);
        if (hd >= 0 && !(lane > 0 && ptl == hd)) flush(hd, ha);
        // last runs: equal destinations sit in consecutive lanes; a segmented
        // reduction leaves each segment's total in its last lane
        const uint32_t heads = __ballot_sync(0xffffffffu, lane == 0 || cur != ptl);
        const int s0 = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const V t = __shfl_up_sync(0xffffffffu, acc, d);
          if (lane - d >= s0) acc = F::combine(t, acc);
        }
        const bool seg_end = lane == 31 || ((heads >> (lane + 1)) & 1u);
        if (seg_end && cur >= 0) flush(cur, acc);
        continue;
      }
      int cur = -1;
      V acc = F::identity();
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        if (!vld[k]) continue;
        const int l = (int)dv[k];
        if (l != cur) {
          if (cur >= 0) flush(cur, acc);
          cur = l;
          acc = val[k];
        } else {
          acc = F::combine(acc, val[k]);
        }
      }
      const int c0 = __shfl_sync(0xffffffffu, cur, 0);
      if (__all_sync(0xffffffffu, cur == c0) && c0 >= 0) {
        V r = acc;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r = F::combine(r, __shfl_xor_sync(0xffffffffu, r, o));
        if (lane == 0) {
          F::atomic_combine(&s_acc[c0], r);
          if (kTouch) s_touch[c0] = 1;
        }
      } else if (cur >= 0) {
        F::atomic_combine(&s_acc[cur], acc);
        if (kTouch) s_touch[cur] = 1;
      }
    }
    __syncthreads();
    if (s_fail) break;
    if constexpr (NOOUT) {
      for (uint32_t l = tid; l < nv; l += kCooThreads)
        if (s_acc[l] != F::identity() && (F::kCondTrue || s_cond[l])) f.commit(v0 + l, s_acc[l]);
      __syncthreads();
      continue;
    }
    const uint32_t base0 = v0 & ~31u;
    if constexpr (kFin && (HINT & 4)) {
      // the vertex step of kCommitAhead 32-vertex groups per round: every
      // group's loads (degree bounds, rank, previous rank, frontier word)
      // are issued before the first group's arithmetic and stores
      constexpr int kCommitAhead = 4;
      for (uint32_t b0 = base0 + (uint32_t)warp * 32u; b0 < v0 + nv; b0 += kCommitAhead * kCooThreads) {
        typename F::FinishIn x[kCommitAhead];
        uint32_t dg[kCommitAhead];
        bool inr[kCommitAhead];
#pragma unroll
        for (int u = 0; u < kCommitAhead; ++u) {
          const uint32_t v = b0 + (uint32_t)u * kCooThreads + (uint32_t)lane;
          inr[u] = v >= v0 && v < v0 + nv;
          dg[u] = 0;
          if (inr[u]) {
            dg[u] = __ldg(p.deg_off + v + 1) - __ldg(p.deg_off + v);
            x[u] = f.finish_load(v);
          }
        }
#pragma unroll
        for (int u = 0; u < kCommitAhead; ++u) {
          const uint32_t bb = b0 + (uint32_t)u * kCooThreads;
          if (bb >= v0 + nv) break;  // warp-uniform
          const uint32_t v = bb + (uint32_t)lane;
          bool act = false;
          if (inr[u]) {
            const uint32_t l = v - v0;
            const bool touched = s_acc[l] != F::identity();
            my_l1 += f.finish_apply(v, x[u], touched, s_acc[l], dg[u]);
            act = touched;
          }
          const uint32_t word = __ballot_sync(0xffffffffu, act);
          if (act) my_deg += dg[u];
          if (lane == 0 && word) {
            atomicOr(p.next_bits + (bb >> 5), word);
            my_cnt += __popc(word);
          }
        }
      }
      __syncthreads();
      continue;
    }
    for (uint32_t bb = base0 + (uint32_t)warp * 32u; bb < v0 + nv; bb += kCooThreads) {
      const uint32_t v = bb + (uint32_t)lane;
      bool act = false;
      uint32_t dg = 0;
      if (v >= v0 && v < v0 + nv) {
        const uint32_t l = v - v0;
        const bool touched = F::kPositive ? (s_acc[l] != F::identity()) : (s_touch[l] != 0);
        if constexpr (kFin) {
          dg = __ldg(p.deg_off + v + 1) - __ldg(p.deg_off + v);
          my_l1 += f.finish(v, touched, s_acc[l], dg);
          act = touched;
        } else if (touched && (F::kCondTrue || s_cond[l])) {
          act = f.commit(v, s_acc[l]);
        }
      }
      const uint32_t word = __ballot_sync(0xffffffffu, act);
      if (kFin) {
        if (act) my_deg += dg;
      } else if (act) {
        my_deg += __ldg(p.deg_off + v + 1) - __ldg(p.deg_off + v);
      }
      if (lane == 0 && word) {
        atomicOr(p.next_bits + (bb >> 5), word);
        my_cnt += __popc(word);
      }
    }
    __syncthreads();
  }
  my_deg = warp_sum(my_deg);
  my_cnt = warp_sum(my_cnt);
  if (kFin) my_l1 = warp_sum(my_l1);
  if (lane == 0) {
    s_red[0][warp] = my_cnt;
    s_red[1][warp] = my_deg;
    if (kFin) s_l1[warp] = my_l1;
  }
  __syncthreads();
  if (tid == 0) {
    unsigned long long a = 0, b2 = 0;
    double l1 = 0;
    for (int w = 0; w < kCooWarps; ++w) {
      a += s_red[0][w];
      b2 += s_red[1][w];
      if (kFin) l1 += s_l1[w];
    }
    if (a) atomicAdd(p.stats + 0, a);
    if (b2) atomicAdd(p.stats + 1, b2);
    if constexpr (kFin) {
      if (l1 != 0) atomicAdd(f.l1, l1);
    }
  }
}

template <class F, bool HW, bool ALL, int STAGES, bool CONTIG = false, bool PF = false, bool NOOUT = false,
          bool MERGE = false, int HINT = 0>
__global__ void __launch_bounds__(kCooThreads, GG_COO_MIN_BLOCKS) k_pull_coo_w(const PullParams p, const F f) {
  pull_coo_w_run<F, HW, ALL, STAGES, CONTIG, PF, NOOUT, MERGE, HINT>(p, f);
}

// ------------------------------------------ source-partitioned COO (-P source)
// edgeMapDense over partitions of sources (graphgrind/graph-numa.h:1145-1171,
// graphgrind/ligra-numa.h:803-866): a partition's edges reach destinations
// anywhere, so every edge applies F's atomic update (edgeOpInAtomic) and the
// output bit of a destination is counted once, by the thread that sets it.
struct SrcParams {
  const uint32_t* src;
  const uint32_t* dst;
  const uint32_t* wts;
  uint64_t len;
  const uint32_t* fr_bits;
  uint32_t* next_bits;
  const uint32_t* deg_off;
  unsigned long long* stats;
};

template <class F, bool HW, bool ALL>
__global__ void __launch_bounds__(256) k_coo_src(const SrcParams p, const F f) {
  using V = typename F::value_t;
  unsigned long long cnt = 0, deg = 0;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < p.len;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = __ldg(p.src + e), d = __ldg(p.dst + e);
    if (!ALL && !test_bit(p.fr_bits, s)) continue;
    if (!F::kCondTrue && !f.cond(d)) continue;
    const uint32_t w = HW ? __ldg(p.wts + e) : 1u;
    if (F::kPositive) {  // sources outside the frontier carry negative values
      const V v = f.gather(s, w);
      if (v < F::identity()) continue;
    }
    if (f.update_atomic(s, d, w)) {
      const uint32_t bit = 1u << (d & 31);
      uint32_t* word = p.next_bits + (d >> 5);
      if (!(__ldcg(word) & bit) && !(atomicOr(word, bit) & bit)) {
        ++cnt;
        deg += __ldg(p.deg_off + d + 1) - __ldg(p.deg_off + d);
      }
    }
  }
  cnt = warp_sum(cnt);
  deg = warp_sum(deg);
  if ((threadIdx.x & 31) == 0 && (cnt | deg)) {
    atomicAdd(p.stats + 0, cnt);
    atomicAdd(p.stats + 1, deg);
  }
}

// ------------------------------------------------ segmented CSC pull
// The CTA owns a destination tile (accumulators in shared memory, one
// commit per destination, no global atomics).  Inside the tile each warp
// streams its own 256-edge blocks through a private 3-stage bulk-copy ring
// (no CTA-wide barrier per block); lane l takes 8 consecutive edges.
// Destinations come from the head-bit stream: a warp prefix count of head
// bits plus the block's head count gives every edge's row ordinal, and the
// compressed row list gives the vertex.  Contributions reduce in registers
// along rows; only rows that cross a lane boundary touch shared memory.
constexpr int kSegWarps = 8;
constexpr int kSegThreads = kSegWarps * 32;
constexpr int kSegStages = 3;

struct SegParams {
  const uint4* tiles;
  uint32_t ntiles;
  unsigned long long* tile_counter;
  const uint32_t* src;      // in-neighbour ids, padded to whole 256-edge blocks
  const uint32_t* wts;      // weights, same padding, or null
  const uint32_t* head;     // head bits
  const uint32_t* blk;      // heads before each 256-edge block
  const uint32_t* rows;     // vertex of every non-empty row
  const uint32_t* fr_bits;
  uint32_t* next_bits;
  const uint32_t* deg_off;
  const uint32_t* member_off;
  unsigned long long* stats;
  unsigned long long* err;
};

__host__ __device__ constexpr size_t seg_stage_bytes(bool hw) {
  return (size_t)kSegBlock * 4 + 32 + (hw ? (size_t)kSegBlock * 4 : 0);
}
__host__ __device__ constexpr size_t seg_smem_bytes(bool hw, int vbytes) {
  return 256 + (size_t)kSegWarps * kSegStages * seg_stage_bytes(hw) + (size_t)kMaxTileVertices * vbytes +
         (size_t)kMaxTileVertices * 2;
}

template <class F, bool HW, bool ALL>
__global__ void __launch_bounds__(kSegThreads, 3) k_pull_seg(const SegParams p, const F f) {
  using V = typename F::value_t;
  extern __shared__ __align__(128) unsigned char smem[];
  constexpr uint32_t SB = (uint32_t)seg_stage_bytes(HW);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem);  // [warp][stage]
  unsigned char* stages = smem + 256;
  V* s_acc = reinterpret_cast<V*>(stages + (size_t)kSegWarps * kSegStages * SB);
  uint8_t* s_touch = reinterpret_cast<uint8_t*>(s_acc + kMaxTileVertices);
  uint8_t* s_cond = s_touch + kMaxTileVertices;
  __shared__ uint32_t s_tile;
  __shared__ unsigned long long s_red[2][kSegWarps];
  __shared__ int s_fail;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint64_t* wbar = bars + warp * kSegStages;
  unsigned char* wst = stages + (size_t)warp * kSegStages * SB;
  if (lane == 0)
    for (int s = 0; s < kSegStages; ++s) mbar_init(&wbar[s], 1);
  if (tid == 0) s_fail = 0;
  fence_mbar_init();
  __syncthreads();
  uint32_t parity = 0;
  unsigned long long my_cnt = 0, my_deg = 0;

  for (;;) {
    if (tid == 0) s_tile = (uint32_t)atomicAdd(p.tile_counter, 1ull);
    __syncthreads();
    const uint32_t t = s_tile;
    if (t >= p.ntiles || s_fail) break;
    const uint4 td = p.tiles[t];
    const uint32_t v0 = td.x, nv = td.y, e0 = td.z, ne = td.w;
    for (uint32_t i = tid; i < nv; i += kSegThreads) {
      const uint32_t v = v0 + i;
      s_acc[i] = F::identity();
      s_touch[i] = 0;
      bool c = F::kCondTrue ? true : f.cond(v);
      if (p.member_off) c = c && (__ldg(p.member_off + v + 1) > __ldg(p.member_off + v));
      s_cond[i] = c ? 1 : 0;
    }
    __syncthreads();
    const bool need_cond = !F::kCondTrue || p.member_off != nullptr;
    const uint32_t e1 = e0 + ne;
    const uint32_t b_first = e0 / kSegBlock;
    const uint32_t nb = (e1 - 1) / kSegBlock - b_first + 1;
    const uint32_t nbw = (uint32_t)warp < nb ? (nb - (uint32_t)warp + kSegWarps - 1) / kSegWarps : 0;
    auto issue = [&](uint32_t i, int st) {
      const uint32_t b = b_first + (uint32_t)warp + i * kSegWarps;
      unsigned char* d = wst + st * SB;
      mbar_arrive_expect_tx(&wbar[st], SB);
      bulk_g2s(d, p.src + (size_t)b * kSegBlock, kSegBlock * 4, &wbar[st]);
      bulk_g2s(d + kSegBlock * 4, p.head + (size_t)b * (kSegBlock / 32), 32, &wbar[st]);
      if (HW) bulk_g2s(d + kSegBlock * 4 + 32, p.wts + (size_t)b * kSegBlock, kSegBlock * 4, &wbar[st]);
    };
    if (lane == 0)
      for (uint32_t i = 0; i < nbw && i < (uint32_t)kSegStages; ++i) issue(i, (int)i);
    uint32_t issued = nbw < (uint32_t)kSegStages ? nbw : (uint32_t)kSegStages;
    bool fail = false;
    for (uint32_t i = 0; i < nbw; ++i) {
      const int st = (int)(i % kSegStages);
      const uint32_t b = b_first + (uint32_t)warp + i * kSegWarps;
      const uint32_t hb = __ldg(p.blk + b);  // heads before this block
      // warp-uniform outcome: the lanes leave the loop together
      const bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(&wbar[st], (parity >> st) & 1u));
      parity ^= 1u << st;
      if (!ok) {
        if (lane == 0) atomicOr(p.err, (unsigned long long)DEV_ERR_TIMEOUT);
        s_fail = 1;
        fail = true;
        for (uint32_t cc = i + 1; cc < issued; ++cc) {  // drain (bounded)
          const int s2 = (int)(cc % kSegStages);
          mbar_wait_bounded(&wbar[s2], (parity >> s2) & 1u);
          parity ^= 1u << s2;
        }
        break;
      }
      const unsigned char* d = wst + st * SB;
      const uint32_t* ssrc = reinterpret_cast<const uint32_t*>(d) + lane * 8;
      uint32_t sv[8], wv[8];
      {
        const uint4 a = reinterpret_cast<const uint4*>(ssrc)[0];
        const uint4 c = reinterpret_cast<const uint4*>(ssrc)[1];
        sv[0] = a.x; sv[1] = a.y; sv[2] = a.z; sv[3] = a.w;
        sv[4] = c.x; sv[5] = c.y; sv[6] = c.z; sv[7] = c.w;
      }
      if (HW) {
        const uint32_t* sw = reinterpret_cast<const uint32_t*>(d + kSegBlock * 4 + 32) + lane * 8;
        const uint4 a = reinterpret_cast<const uint4*>(sw)[0];
        const uint4 c = reinterpret_cast<const uint4*>(sw)[1];
        wv[0] = a.x; wv[1] = a.y; wv[2] = a.z; wv[3] = a.w;
        wv[4] = c.x; wv[5] = c.y; wv[6] = c.z; wv[7] = c.w;
      } else {
#pragma unroll
        for (int k = 0; k < 8; ++k) wv[k] = 1u;
      }
      const uint32_t hw32 = reinterpret_cast<const uint32_t*>(d + kSegBlock * 4)[lane >> 2];
      const uint32_t bits = (hw32 >> ((lane & 3) * 8)) & 0xffu;
      // heads strictly before this lane's first edge
      const uint32_t cnt = __popc(bits);
      uint32_t incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      const uint32_t before = hb + incl - cnt;
      __syncwarp();
      if (lane == 0 && i + kSegStages < nbw) {  // refill this stage: the warp has read it
        fence_proxy_async_smem();
        issue(i + kSegStages, st);
      }
      if (i + kSegStages < nbw) ++issued;
      const uint32_t pos0 = b * kSegBlock + (uint32_t)lane * 8;
      // destinations: row ordinal of slot k = before + heads in slots [0, k] - 1
      uint32_t lv[8];
      bool vld[8];
      uint32_t cur_ord = 0xffffffffu, cur_l = 0;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t pos = pos0 + k;
        const bool in = pos >= e0 && pos < e1;
        const uint32_t ord = before + __popc(bits & ((2u << k) - 1u)) - 1u;
        if (in && ord != cur_ord) {
          cur_ord = ord;
          cur_l = __ldg(p.rows + ord) - v0;
        }
        lv[k] = cur_l;
        vld[k] = in;
      }
      if (need_cond) {
#pragma unroll
        for (int k = 0; k < 8; ++k) vld[k] = vld[k] && s_cond[lv[k]];
      }
      if (!ALL) {
#pragma unroll
        for (int k = 0; k < 8; ++k)
          if (vld[k]) vld[k] = test_bit(p.fr_bits, sv[k]);
      }
      V val[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        val[k] = vld[k] ? f.gather(sv[k], wv[k]) : F::identity();
        if (F::kPositive) vld[k] = vld[k] && !(val[k] < F::identity());
      }
      int cur = -1;
      V acc = F::identity();
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        if (!vld[k]) continue;
        const int l = (int)lv[k];
        if (l != cur) {
          if (cur >= 0) {
            F::atomic_combine(&s_acc[cur], acc);
            if (!F::kPositive) s_touch[cur] = 1;
          }
          cur = l;
          acc = val[k];
        } else {
          acc = F::combine(acc, val[k]);
        }
      }
      const int c0 = __shfl_sync(0xffffffffu, cur, 0);
      if (__all_sync(0xffffffffu, cur == c0) && c0 >= 0) {  // whole warp on one row (hubs)
        V r = acc;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r = F::combine(r, __shfl_xor_sync(0xffffffffu, r, o));
        if (lane == 0) {
          F::atomic_combine(&s_acc[c0], r);
          if (!F::kPositive) s_touch[c0] = 1;
        }
      } else if (cur >= 0) {
        F::atomic_combine(&s_acc[cur], acc);
        if (!F::kPositive) s_touch[cur] = 1;
      }
    }
    (void)fail;
    __syncthreads();
    if (s_fail) break;
    const uint32_t base0 = v0 & ~31u;
    for (uint32_t bb = base0 + (uint32_t)warp * 32u; bb < v0 + nv; bb += kSegThreads) {
      const uint32_t v = bb + (uint32_t)lane;
      bool act = false;
      if (v >= v0 && v < v0 + nv) {
        const uint32_t l = v - v0;
        const bool touched = F::kPositive ? (s_acc[l] != F::identity()) : (s_touch[l] != 0);
        if (touched && s_cond[l]) act = f.commit(v, s_acc[l]);
      }
      const uint32_t word = __ballot_sync(0xffffffffu, act);
      if (act) my_deg += __ldg(p.deg_off + v + 1) - __ldg(p.deg_off + v);
      if (lane == 0 && word) {
        atomicOr(p.next_bits + (bb >> 5), word);
        my_cnt += __popc(word);
      }
    }
    __syncthreads();
  }
  my_deg = warp_sum(my_deg);
  my_cnt = warp_sum(my_cnt);
  if (lane == 0) {
    s_red[0][warp] = my_cnt;
    s_red[1][warp] = my_deg;
  }
  __syncthreads();
  if (tid == 0) {
    unsigned long long a = 0, b2 = 0;
    for (int w = 0; w < kSegWarps; ++w) {
      a += s_red[0][w];
      b2 += s_red[1][w];
    }
    if (a) atomicAdd(p.stats + 0, a);
    if (b2) atomicAdd(p.stats + 1, b2);
  }
}

// Dense pull with early exit (kEarlyExit functors): one lane per destination.
// VEC: the in-list is read in 16-byte aligned groups of 4 edges (edge arrays
// are 16-byte aligned and padded past their end) whose frontier tests issue
// together; the edges are still taken in list order.
template <class F, bool HW, bool ALL, bool VEC = false>
__global__ void __launch_bounds__(256) k_pull_early(uint32_t n, const uint32_t* off, const uint32_t* idx,
                                                    const uint32_t* wts, const uint32_t* fr_bits,
                                                    uint32_t* next_bits, const uint32_t* deg_off,
                                                    const uint32_t* member_off, unsigned long long* stats,
                                                    const F f) {
  unsigned long long my_cnt = 0, my_deg = 0;
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); b < n; b += stride) {
    const uint32_t v = (uint32_t)b + lane;
    bool act = false;
    if (v < n && f.cond(v) && (!member_off || member_off[v + 1] > member_off[v])) {
      const uint32_t j0 = off[v], e1 = off[v + 1];
      if constexpr (VEC) {
        bool done = false;
        for (uint32_t a = j0 & ~3u; a < e1 && !done; a += 4) {
          const uint4 q = __ldg(reinterpret_cast<const uint4*>(idx + a));
          const uint32_t ss[4] = {q.x, q.y, q.z, q.w};
          bool hit[4];
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const uint32_t e = a + (uint32_t)t;
            hit[t] = e >= j0 && e < e1 && (ALL || test_bit(fr_bits, ss[t]));
          }
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            if (!done && hit[t]) {
              act = f.commit(v, f.gather(ss[t], HW ? wts[a + t] : 1u));
              if (act || !f.cond(v)) done = true;
            }
          }
        }
      } else {
        for (uint32_t j = j0; j < e1; ++j) {
          const uint32_t s = idx[j];
          if (ALL || test_bit(fr_bits, s)) {
            act = f.commit(v, f.gather(s, HW ? wts[j] : 1u));
            if (act || !f.cond(v)) break;
          }
        }
      }
    }
    const uint32_t word = __ballot_sync(0xffffffffu, act);
    if (act) my_deg += deg_off[v + 1] - deg_off[v];
    if (lane == 0 && word) {
      atomicOr(next_bits + (b >> 5), word);
      my_cnt += __popc(word);
    }
  }
  my_cnt = warp_sum(my_cnt);
  my_deg = warp_sum(my_deg);
  if (lane == 0) {
    if (my_cnt) atomicAdd(stats + 0, my_cnt);
    if (my_deg) atomicAdd(stats + 1, my_deg);
  }
}

// Dense pull with early exit, cooperative form: a warp takes 32 consecutive
// destinations, keeps those that pass cond (and have in-edges), and walks
// their in-lists 4 at a time with 8 lanes each, 8 consecutive in-edges per
// step (one 32-byte read per group).  A destination stops at the first step
// holding a frontier in-neighbour and takes the first one of that step, so
// it still takes its first frontier in-neighbour in list order, as the
// one-lane form does; a hub row is walked 8 edges per step instead of 1.
template <class F, bool HW, bool ALL>
__global__ void __launch_bounds__(256) k_pull_early_g(uint32_t n, const uint32_t* off, const uint32_t* idx,
                                                      const uint32_t* wts, const uint32_t* fr_bits,
                                                      uint32_t* next_bits, const uint32_t* deg_off,
                                                      const uint32_t* member_off, unsigned long long* stats,
                                                      const F f) {
  __shared__ uint32_t s_cand[8][32];
  unsigned long long my_cnt = 0, my_deg = 0;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t grp = lane >> 3, sub = lane & 7;
  const uint32_t gmask = 0xffu << (grp * 8);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); b < n; b += stride) {
    const uint32_t v = (uint32_t)b + lane;
    bool cand = false;
    if (v < n && (!member_off || member_off[v + 1] > member_off[v]))
      cand = off[v + 1] > off[v] && f.cond(v);
    const uint32_t cm = __ballot_sync(0xffffffffu, cand);
    if (cand) s_cand[warp][__popc(cm & ((1u << lane) - 1u))] = lane;
    __syncwarp();
    const uint32_t nc = __popc(cm);
    uint32_t found = 0;  // lanes (vertex offsets in the warp's 32) that took a parent
    for (uint32_t c0 = 0; c0 < nc; c0 += 4) {
      const uint32_t c = c0 + grp;
      const bool mine = c < nc;
      const uint32_t lv = mine ? s_cand[warp][c] : 0u;
      const uint32_t vv = (uint32_t)b + lv;
      uint32_t j = mine ? off[vv] + sub : 0u;
      const uint32_t e1 = mine ? off[vv + 1] : 0u;
      bool live = mine;
      while (__any_sync(0xffffffffu, live)) {
        bool hit = false;
        uint32_t s = 0;
        if (live && j < e1) {
          s = idx[j];
          hit = ALL || test_bit(fr_bits, s);
        }
        const uint32_t hm = __ballot_sync(0xffffffffu, hit) & gmask;
        if (live) {
          if (hm) {
            const uint32_t first = __ffs(hm) - 1;
            if (lane == first) {
              if (f.commit(vv, f.gather(s, HW ? wts[j] : 1u))) found |= 1u << lv;
            }
            live = false;
          } else {
            j += 8;
            if (j - sub >= e1) live = false;  // the group's next step starts past the row
          }
        }
      }
    }
    // every lane's found bits of this warp's 32 destinations
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) found |= __shfl_xor_sync(0xffffffffu, found, o);
    const bool act = (found >> lane) & 1u;
    if (act) my_deg += deg_off[v + 1] - deg_off[v];
    if (lane == 0 && found) {
      atomicOr(next_bits + (b >> 5), found);
      my_cnt += __popc(found);
    }
    __syncwarp();
  }
  my_cnt = warp_sum(my_cnt);
  my_deg = warp_sum(my_deg);
  if (lane == 0) {
    if (my_cnt) atomicAdd(stats + 0, my_cnt);
    if (my_deg) atomicAdd(stats + 1, my_deg);
  }
}

// ------------------------------------------------------------ push path
// Block-level exclusive scan of up to kScanTile degrees (deg of queue[i]).
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* s_warp, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    s_warp[lane] = w;  // inclusive warp totals
  }
  __syncthreads();
  const uint32_t before = warp ? s_warp[warp - 1] : 0;
  *total = s_warp[(blockDim.x >> 5) - 1];
  __syncthreads();
  return before + x - v;
}

// pass 1: per-block degree sums
static __global__ void __launch_bounds__(kScanThreads) k_scan_sums(const uint32_t* q, uint32_t k, const uint32_t* off,
                                                            uint32_t* bsum) {
  __shared__ uint32_t s_warp[32];
  const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  uint32_t t = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const uint32_t j = base + i;
    if (j < k) {
      const uint32_t v = q[j];
      t += off[v + 1] - off[v];
    }
  }
  uint32_t tot;
  block_excl_scan(t, s_warp, &tot);
  if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}
// pass 2: exclusive scan of the block sums (one block, serial over chunks);
// writes the grand total to *total.
static __global__ void __launch_bounds__(1024) k_scan_blocks(uint32_t* bsum, uint32_t nb, unsigned long long* total) {
  __shared__ uint32_t s_warp[32];
  uint32_t carry = 0;
  for (uint32_t b0 = 0; b0 < nb; b0 += blockDim.x) {
    const uint32_t j = b0 + threadIdx.x;
    const uint32_t v = j < nb ? bsum[j] : 0;
    uint32_t tot;
    const uint32_t ex = block_excl_scan(v, s_warp, &tot);
    if (j < nb) bsum[j] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) *total = carry;
}
// pass 3: exclusive offsets of every queue entry; offs[k] = total
static __global__ void __launch_bounds__(kScanThreads) k_scan_write(const uint32_t* q, uint32_t k, const uint32_t* off,
                                                             const uint32_t* bsum, uint32_t* offs) {
  __shared__ uint32_t s_warp[32];
  const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  uint32_t d[kScanItems];
  uint32_t t = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const uint32_t j = base + i;
    d[i] = 0;
    if (j < k) {
      const uint32_t v = q[j];
      d[i] = off[v + 1] - off[v];
    }
    t += d[i];
  }
  uint32_t tot;
  uint32_t run = block_excl_scan(t, s_warp, &tot) + bsum[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const uint32_t j = base + i;
    if (j < k) offs[j] = run;
    run += d[i];
    if (j + 1 == k) offs[k] = run;
  }
}

struct PushParams {
  const uint32_t* q;        // frontier queue
  uint32_t k;               // queue length
  const uint32_t* offs;     // k+1 scanned degrees
  const unsigned long long* total;
  const uint32_t* off;      // out-offsets (current orientation)
  const uint32_t* idx;      // out-neighbours
  const uint32_t* wts;      // weights or null
  const uint32_t* deg_off;  // out-offsets for output statistics
  uint32_t* dedup;          // n-bit scratch, zero on entry and exit
  uint32_t* out_q;          // output queue
  unsigned long long* stats;  // [0] -, [1] out-degree sum, [2] queue length
};

// Push whose output is a bitmap: the dense edgeMap of a frontier with few
// vertices but many out-edges (the level after a hub level), where the
// bottom-up pull would walk every unvisited in-list.  The same per-edge work
// as k_push (cond && update_atomic); the first winner of a destination sets
// its bit in p.dedup (here the zeroed output bitmap), and the output's size
// and out-degree sum are counted per warp, with no queue and no per-warp
// atomic on one shared counter.
template <class F, bool HW>
__global__ void __launch_bounds__(kPushThreads) k_push_bits(const PushParams p, const F f) {
  __shared__ uint32_t s_q[2];
  const uint64_t E = *p.total;
  const int lane = threadIdx.x & 31;
  unsigned long long my_deg = 0, my_cnt = 0;
  for (uint64_t c = blockIdx.x; c * kPushEdgesPerCta < E; c += gridDim.x) {
    const uint32_t e_lo = (uint32_t)(c * kPushEdgesPerCta);
    const uint64_t e_end = (uint64_t)e_lo + kPushEdgesPerCta;
    const uint32_t e_hi = (uint32_t)(E < e_end ? E : e_end);
    if (threadIdx.x < 2) {
      const uint32_t key = threadIdx.x == 0 ? e_lo : e_hi - 1;
      uint32_t lo = 0, hi = p.k;  // largest i with offs[i] <= key
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (p.offs[mid] <= key) lo = mid; else hi = mid;
      }
      s_q[threadIdx.x] = lo;
    }
    __syncthreads();
    const uint32_t qlo = s_q[0], qhi = s_q[1];
    const uint32_t iters = (e_hi - e_lo + kPushThreads - 1) / kPushThreads;
    for (uint32_t it = 0; it < iters; ++it) {
      const uint32_t e = e_lo + it * kPushThreads + threadIdx.x;
      if (e < e_hi) {
        uint32_t lo = qlo, hi = qhi + 1;
        while (hi - lo > 1) {
          const uint32_t mid = (lo + hi) >> 1;
          if (p.offs[mid] <= e) lo = mid; else hi = mid;
        }
        const uint32_t s = p.q[lo];
        const uint32_t ei = p.off[s] + (e - p.offs[lo]);
        const uint32_t d = p.idx[ei];
        const uint32_t w = HW ? p.wts[ei] : 1u;
        if (f.cond(d) && f.update_atomic(s, d, w)) {
          const uint32_t bit = 1u << (d & 31);
          if (!(atomicOr(p.dedup + (d >> 5), bit) & bit)) {
            ++my_cnt;
            my_deg += p.deg_off[d + 1] - p.deg_off[d];
          }
        }
      }
    }
    __syncthreads();
  }
  my_deg = warp_sum(my_deg);
  my_cnt = warp_sum(my_cnt);
  if (lane == 0) {
    if (my_cnt) atomicAdd(p.stats + 0, my_cnt);
    if (my_deg) atomicAdd(p.stats + 1, my_deg);
  }
}

template <class F, bool HW>
__global__ void __launch_bounds__(kPushThreads) k_push(const PushParams p, const F f) {
  __shared__ uint32_t s_q[2];
  const uint64_t E = *p.total;
  const int lane = threadIdx.x & 31;
  unsigned long long my_deg = 0;
  for (uint64_t c = blockIdx.x; c * kPushEdgesPerCta < E; c += gridDim.x) {
    const uint32_t e_lo = (uint32_t)(c * kPushEdgesPerCta);
    const uint64_t e_end = (uint64_t)e_lo + kPushEdgesPerCta;
    const uint32_t e_hi = (uint32_t)(E < e_end ? E : e_end);
    if (threadIdx.x < 2) {
      const uint32_t key = threadIdx.x == 0 ? e_lo : e_hi - 1;
      uint32_t lo = 0, hi = p.k;  // largest i with offs[i] <= key
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (p.offs[mid] <= key) lo = mid; else hi = mid;
      }
      s_q[threadIdx.x] = lo;
    }
    __syncthreads();
    const uint32_t qlo = s_q[0], qhi = s_q[1];
    const uint32_t iters = (e_hi - e_lo + kPushThreads - 1) / kPushThreads;
    for (uint32_t it = 0; it < iters; ++it) {
      const uint32_t e = e_lo + it * kPushThreads + threadIdx.x;
      bool take = false;
      uint32_t d = 0;
      if (e < e_hi) {
        uint32_t lo = qlo, hi = qhi + 1;
        while (hi - lo > 1) {
          const uint32_t mid = (lo + hi) >> 1;
          if (p.offs[mid] <= e) lo = mid; else hi = mid;
        }
        const uint32_t s = p.q[lo];
        const uint32_t ei = p.off[s] + (e - p.offs[lo]);
        d = p.idx[ei];
        const uint32_t w = HW ? p.wts[ei] : 1u;
        if (f.cond(d) && f.update_atomic(s, d, w)) {
          const uint32_t bit = 1u << (d & 31);
          take = !(atomicOr(p.dedup + (d >> 5), bit) & bit);
        }
      }
      const uint32_t ball = __ballot_sync(0xffffffffu, take);
      if (ball) {
        uint32_t base = 0;
        if (lane == 0) base = (uint32_t)atomicAdd(p.stats + 2, (unsigned long long)__popc(ball));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (take) {
          p.out_q[base + __popc(ball & ((1u << lane) - 1u))] = d;
          my_deg += p.deg_off[d + 1] - p.deg_off[d];
        }
      }
    }
    __syncthreads();
  }
  my_deg = warp_sum(my_deg);
  if (lane == 0 && my_deg) atomicAdd(p.stats + 1, my_deg);
}

// zero the dedup words touched by a queue
static __global__ void k_clear_dedup(const uint32_t* q, const unsigned long long* len, uint32_t* dedup) {
  const uint64_t k = *len;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < k; i += (uint64_t)gridDim.x * blockDim.x)
    dedup[q[i] >> 5] = 0u;
}

// ------------------------------------------------------- vertexSubset ops
static __global__ void k_queue_to_bits(const uint32_t* q, uint64_t k, uint32_t* bits) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < k; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = q[i];
    atomicOr(bits + (v >> 5), 1u << (v & 31));
  }
}

// ballot/popc compaction of a bitmap into a queue (one word per lane)
static __global__ void k_bits_to_queue(const uint32_t* bits, uint32_t words, uint32_t* q, unsigned long long* len) {
  const int lane = threadIdx.x & 31;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); b < words; b += stride) {
    const uint64_t wi = b + lane;
    const uint32_t w = wi < words ? bits[wi] : 0u;
    const uint32_t c = __popc(w);
    uint32_t x = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    const uint32_t tot = __shfl_sync(0xffffffffu, x, 31);
    uint32_t base = 0;
    if (lane == 31 && tot) base = (uint32_t)atomicAdd(len, (unsigned long long)tot);
    base = __shfl_sync(0xffffffffu, base, 31);
    uint32_t pos = base + x - c;
    uint32_t ww = w;
    while (ww) {
      const int bpos = __ffs(ww) - 1;
      ww &= ww - 1;
      q[pos++] = (uint32_t)(wi * 32 + bpos);
    }
  }
}

// count and out-degree sum of a bitmap's members
static __global__ void k_bits_stats(const uint32_t* bits, uint32_t n, const uint32_t* deg_off, unsigned long long* stats) {
  unsigned long long c = 0, d = 0;
  const uint32_t words = (n + 31) / 32;
  for (uint64_t wi = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; wi < words; wi += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t w = bits[wi];
    c += __popc(w);
    while (w) {
      const int b = __ffs(w) - 1;
      w &= w - 1;
      const uint32_t v = (uint32_t)(wi * 32 + b);
      d += deg_off[v + 1] - deg_off[v];
    }
  }
  c = warp_sum(c);
  d = warp_sum(d);
  if ((threadIdx.x & 31) == 0) {
    if (c) atomicAdd(stats + 0, c);
    if (d) atomicAdd(stats + 1, d);
  }
}

// vertexMap: mode 0 all vertices, 1 dense members, 2 sparse list
template <class VF, int MODE>
__global__ void k_vertex_map(uint32_t n, const uint32_t* bits, const uint32_t* q, uint64_t k, const VF vf) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  if (MODE == 2) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < k; i += stride) vf(q[i]);
  } else {
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride)
      if (MODE == 0 || test_bit(bits, (uint32_t)v)) vf((uint32_t)v);
  }
}

// vertexFilter over a dense (or all-active) subset: output bitmap + stats
template <class VF, bool ALL>
__global__ void k_vertex_filter(uint32_t n, const uint32_t* bits, uint32_t* out_bits, const uint32_t* deg_off,
                                unsigned long long* stats, const VF vf) {
  unsigned long long c = 0, d = 0;
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); b < n; b += stride) {
    const uint32_t v = (uint32_t)b + lane;
    bool act = false;
    if (v < n && (ALL || test_bit(bits, v))) act = vf(v);
    const uint32_t word = __ballot_sync(0xffffffffu, act);
    if (act) d += deg_off[v + 1] - deg_off[v];
    if (lane == 0) {
      out_bits[b >> 5] = word;
      c += __popc(word);
    }
  }
  c = warp_sum(c);
  d = warp_sum(d);
  if (lane == 0) {
    if (c) atomicAdd(stats + 0, c);
    if (d) atomicAdd(stats + 1, d);
  }
}

}  // namespace gg

namespace gg {
static __global__ void k_iota(uint32_t* q, uint32_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    q[i] = (uint32_t)i;
}
}  // namespace gg
