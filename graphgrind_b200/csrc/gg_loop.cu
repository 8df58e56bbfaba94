// Device-driven BFS levels: one cooperative launch runs consecutive
// sparse-push levels of app/BFS.C:77-101 (edgeMap's sparse branch,
// graphgrind/ligra-numa.h:868-916, with BFS_F::updateAtomic) without
// returning to the host between levels.  All CTAs are co-resident
// (cooperative launch); a level ends at a grid barrier, after which every CTA
// reads the next frontier's size and out-degree and applies edgeMap's
// direction rule (size + out-degree > threshold means a dense level): the
// launch returns when the frontier is empty, needs a dense level, or a level
// cap is reached, and the host continues with edgeMap.  Each level's queue
// chunks of 256 frontier vertices are spread over the CTAs; inside a CTA a
// block prefix sum over the chunk's degrees balances its edges over the
// threads.  The barrier wait is bounded: on expiry the kernel records an error
// and returns.
#include "gg_runtime.cuh"

namespace gg {

// One frontier's counters; the loops keep three, by level mod 3.
struct LoopSlot {
  // queue form: (slots << 32) | out-edges; vertices with out-edges fill the
  // queue from the front in edge-offset order
  unsigned long long packed;
  unsigned long long zeros;  // queue form: members without out-edges (not among the slots)
  unsigned long long dcnt;   // bitmap form: members
  unsigned long long ddeg;   // bitmap form: their out-degree sum
  int32_t rep;               // 0 queue (and bitmap), 1 bitmap only
  int32_t pad;
};

// State of a device level loop.  The counters are read after each grid
// barrier by one thread per CTA (into shared memory); the barrier's arrival
// word sits on a cache line of its own.
struct LoopState {
  LoopSlot slot[3];
  unsigned long long trav;  // out-edges of the frontiers processed
  alignas(128) unsigned int bar;  // barrier arrivals
  int32_t levels_done;
  int32_t exit_reason;  // 1 empty, 2 next level is dense (sparse loop), 3 level cap, -1 barrier timeout
};
static_assert(sizeof(LoopState) <= 64 * sizeof(unsigned long long), "loop state exceeds its workspace");

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int ld_relaxed_i32(const int32_t* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// A slot's counters into shared memory: packed, zeros, dcnt, ddeg, rep.
__device__ __forceinline__ void read_slot(const LoopSlot* sl, unsigned long long* s_rd) {
  s_rd[0] = ld_relaxed_u64(&sl->packed);
  s_rd[1] = ld_relaxed_u64(&sl->zeros);
  s_rd[2] = ld_relaxed_u64(&sl->dcnt);
  s_rd[3] = ld_relaxed_u64(&sl->ddeg);
  s_rd[4] = (unsigned long long)(uint32_t)ld_relaxed_i32(&sl->rep);
}

// All CTAs of the (co-resident) grid arrive; returns false if the wait ran out
// (more than `budget` probes of the arrival count, each followed by a short
// sleep).  The arrival is a release and the wait an acquire by thread 0, so
// with the block barriers around them every write of the grid before the
// barrier is visible to every thread after it.  With `rd`, thread 0 then
// reads that slot's counters into s_rd for the whole CTA.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned target, unsigned budget, int* s_ok,
                                             const LoopSlot* rd = nullptr, unsigned long long* s_rd = nullptr) {
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(bar) : "memory");
    int ok = 1;
    for (unsigned it = 0; (int)(ld_acquire_u32(bar) - target) < 0; ++it) {
      if (it >= budget) {
        ok = 0;
        break;
      }
      __nanosleep(32);
    }
    if (ok && rd) read_slot(rd, s_rd);
    *s_ok = ok;
  }
  __syncthreads();
  return *s_ok != 0;
}

// Warp-cooperative append to the next frontier (every lane calls it).  A
// vertex with out-edges gets its queue slot and its first edge offset from one
// 64-bit atomic (slots in the high half, edges in the low half), so slot order
// is edge-offset order; a vertex without out-edges goes to the far end.
__device__ __forceinline__ void loop_append(bool add, uint32_t u, uint32_t deg, uint32_t* nq, uint32_t* neo,
                                            uint32_t n, unsigned long long* packed, unsigned long long* zeros,
                                            uint32_t* nbits = nullptr) {
  const int lane = threadIdx.x & 31;
  if (nbits && add) atomicOr(nbits + (u >> 5), 1u << (u & 31));
  const uint32_t lanemask_lt = (1u << lane) - 1u;
  const bool pos = add && deg > 0, zer = add && deg == 0;
  uint32_t inc = pos ? deg : 0u;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += t;
  }
  const uint32_t wsum = __shfl_sync(0xffffffffu, inc, 31);
  const uint32_t bal = __ballot_sync(0xffffffffu, pos);
  if (bal) {
    const int leader = __ffs(bal) - 1;
    unsigned long long old = 0;
    if (lane == leader) old = atomicAdd(packed, ((unsigned long long)__popc(bal) << 32) | wsum);
    old = __shfl_sync(0xffffffffu, old, leader);
    if (pos) {
      const uint64_t slot = (old >> 32) + __popc(bal & lanemask_lt);
      nq[slot] = u;
      neo[slot] = (uint32_t)old + inc - deg;
    }
  }
  const uint32_t zb = __ballot_sync(0xffffffffu, zer);
  if (zb) {
    const int leader = __ffs(zb) - 1;
    unsigned long long old = 0;
    if (lane == leader) old = atomicAdd(zeros, (unsigned long long)__popc(zb));
    old = __shfl_sync(0xffffffffu, old, leader);
    if (zer) nq[n - 1 - (old + __popc(zb & lanemask_lt))] = u;
  }
}

// block-wide exclusive scan of two 32-bit counts (blockDim.x == 256)
__device__ __forceinline__ void block_scan2(uint32_t a, uint32_t b, uint32_t* ea, uint32_t* eb, uint32_t* ta,
                                           uint32_t* tb, uint32_t (*s)[8]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = a, y = b;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t u = __shfl_up_sync(0xffffffffu, x, o), w = __shfl_up_sync(0xffffffffu, y, o);
    if (lane >= o) {
      x += u;
      y += w;
    }
  }
  if (lane == 31) {
    s[0][warp] = x;
    s[1][warp] = y;
  }
  __syncthreads();
  uint32_t pa = 0, pb = 0, sa = 0, sb = 0;
  for (int w = 0; w < 8; ++w) {
    if (w < warp) {
      pa += s[0][w];
      pb += s[1][w];
    }
    sa += s[0][w];
    sb += s[1][w];
  }
  *ea = pa + x - a;
  *eb = pb + y - b;
  *ta = sa;
  *tb = sb;
  __syncthreads();
}

// Block-wide append to the next frontier (every thread calls it): one
// 64-bit atomic per CTA for the vertices with out-edges (slots and edge
// offsets, as loop_append) and one for those without.
__device__ __forceinline__ void block_append(bool add, uint32_t u, uint32_t deg, uint32_t* nq, uint32_t* neo,
                                             uint32_t n, unsigned long long* packed, unsigned long long* zeros,
                                             uint32_t* nbits, uint32_t (*s_scan)[8], unsigned long long* s_base) {
  if (nbits && add) atomicOr(nbits + (u >> 5), 1u << (u & 31));
  const bool pos = add && deg > 0, zer = add && deg == 0;
  // counts packed as (with out-edges << 16) | without; at most 256 each
  uint32_t ec, ed, tc, td;
  block_scan2((pos ? 1u << 16 : 0u) | (zer ? 1u : 0u), pos ? deg : 0u, &ec, &ed, &tc, &td, s_scan);
  if (threadIdx.x == 0) {
    s_base[0] = (tc >> 16) ? atomicAdd(packed, ((unsigned long long)(tc >> 16) << 32) | td) : 0ull;
    s_base[1] = (tc & 0xffffu) ? atomicAdd(zeros, (unsigned long long)(tc & 0xffffu)) : 0ull;
  }
  __syncthreads();
  if (pos) {
    const unsigned long long old = s_base[0];
    const uint64_t slot = (old >> 32) + (ec >> 16);
    nq[slot] = u;
    neo[slot] = (uint32_t)old + ed;
  } else if (zer) {
    nq[n - 1 - (s_base[1] + (ec & 0xffffu))] = u;
  }
}

// One sparse (top-down) level, this CTA's contiguous share of its E edges:
// queue q with slot edge offsets eo (k slots, each with >= 1 edge); vertices
// reached for the first time go to nq/neo (and nbits when given).
__device__ __noinline__ void push_level(const uint32_t* __restrict__ off, const uint32_t* __restrict__ idx,
                                           int32_t* parents, int32_t* levels, const uint32_t* q, const uint32_t* eo,
                                           uint32_t* nq, uint32_t* neo, uint64_t k, uint64_t E, uint32_t n, int32_t r,
                                           unsigned long long* packed, unsigned long long* zeros, uint32_t* nbits,
                                           uint32_t* s_eo, uint32_t* s_v, uint32_t* s_beg, uint32_t (*s_scan)[8],
                                           unsigned long long* s_base) {
  const int tid = threadIdx.x;
  // this CTA's contiguous share of the level's edges
  const uint64_t per = (E + gridDim.x - 1) / gridDim.x;
  const uint64_t b0 = (uint64_t)blockIdx.x * per, b1 = b0 + per < E ? b0 + per : E;
  if (b0 < b1) {
    // first slot: the last one whose edge offset is <= b0 (256-way search rounds)
    uint64_t lo = 0, hi = k;
    while (hi - lo > 1) {
      const uint64_t step = (hi - lo + 255) / 256;
      const uint64_t probe = lo + (uint64_t)tid * step;
      const bool le = probe < hi && eo[probe] <= b0;
      const int cnt = __syncthreads_count(le);
      lo = lo + (uint64_t)(cnt - 1) * step;
      hi = lo + step < hi ? lo + step : hi;
    }
    uint64_t scur = lo;
    for (uint64_t base = b0; base < b1; base += 256) {
      const uint64_t last = base + 255 < b1 ? base + 255 : b1 - 1;
      // Stage the slots this window touches.  scur holds the window's first
      // edge and every slot has >= 1 edge, so at most 256 slots start at or
      // before `last`; offset 257 tells whether the next window starts a slot.
      const uint64_t sl = scur + tid;
      const uint32_t e = sl < k ? eo[sl] : 0xffffffffu;
      s_eo[tid] = e;
      if (tid == 0) s_eo[256] = scur + 256 < k ? eo[scur + 256] : 0xffffffffu;
      const int ns = __syncthreads_count(sl < k && e <= last);
      if (tid < ns) {
        const uint32_t v = q[scur + tid];
        s_v[tid] = v;
        s_beg[tid] = off[v];
      }
      __syncthreads();
      const uint64_t t = base + tid;
      bool add = false;
      uint32_t u = 0, deg = 0;
      if (t <= last) {
        int a = 0, b = ns - 1;  // the last staged slot whose offset is <= t
        while (a < b) {
          const int mid = (a + b + 1) >> 1;
          if (s_eo[mid] <= t)
            a = mid;
          else
            b = mid - 1;
        }
        u = idx[s_beg[a] + (uint32_t)(t - s_eo[a])];
        if (__ldcg(parents + u) == -1 && atomicCAS(parents + u, -1, (int32_t)s_v[a]) == -1) {
          add = true;
          if (levels) levels[u] = r;
          deg = off[u + 1] - off[u];
        }
      }
      block_append(add, u, deg, nq, neo, n, packed, zeros, nbits, s_scan, s_base);
      // the slot holding edge last + 1: the next staged one if it starts there,
      // else the last one staged (which runs past `last`)
      scur += (s_eo[ns] == (uint32_t)(last + 1)) ? ns : ns - 1;
      __syncthreads();
    }
  }
}

// Level 0's queue: the input frontier's vertices with out-edges, with offsets.
__global__ void k_loop_seed(const uint32_t* in_q, uint64_t k, const uint32_t* off, uint32_t* q0, uint32_t* eo0,
                            uint32_t n, LoopState* st) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x; i0 < k; i0 += stride) {  // warp-uniform trip count
    const uint64_t i = i0 + threadIdx.x;
    uint32_t v = 0, deg = 0;
    if (i < k) {
      v = in_q[i];
      deg = off[v + 1] - off[v];
    }
    loop_append(i < k && deg > 0, v, deg, q0, eo0, n, &st->slot[0].packed, &st->slot[0].zeros);
  }
}

__global__ void __launch_bounds__(256) k_bfs_push_loop(const uint32_t* __restrict__ off,
                                                       const uint32_t* __restrict__ idx, int32_t* parents,
                                                       int32_t* levels, uint32_t* q0, uint32_t* q1, uint32_t* eo0,
                                                       uint32_t* eo1, uint32_t n, LoopState* st, int32_t round0,
                                                       unsigned long long threshold, int32_t max_levels,
                                                       unsigned wait_budget) {
  __shared__ uint32_t s_eo[257];
  __shared__ uint32_t s_v[256];
  __shared__ uint32_t s_beg[256];
  __shared__ uint32_t s_scan[2][8];
  __shared__ unsigned long long s_base[2];
  __shared__ unsigned long long s_rd[5];
  __shared__ int s_ok;
  const int tid = threadIdx.x;
  if (tid == 0) read_slot(&st->slot[0], s_rd);
  __syncthreads();
  unsigned long long pk = s_rd[0];
  unsigned target = 0;
  for (int32_t i = 0; i < max_levels; ++i) {
    const int nxt = (i + 1) % 3, old = (i + 2) % 3;
    const uint32_t* q = (i & 1) ? q1 : q0;
    const uint32_t* eo = (i & 1) ? eo1 : eo0;
    uint32_t* nq = (i & 1) ? q0 : q1;
    uint32_t* neo = (i & 1) ? eo0 : eo1;
    const uint64_t k = pk >> 32;
    const uint64_t E = pk & 0xffffffffull;
    if (blockIdx.x == 0 && tid == 0) {  // counters of level i+2's frontier; nobody touches them in level i
      st->slot[old].packed = 0;
      st->slot[old].zeros = 0;
      st->trav += E;
    }
    const int32_t r = round0 + i;
    push_level(off, idx, parents, levels, q, eo, nq, neo, k, E, n, r, &st->slot[nxt].packed, &st->slot[nxt].zeros,
               nullptr, s_eo, s_v, s_beg, s_scan, s_base);
    target += gridDim.x;
    if (!grid_barrier(&st->bar, target, wait_budget, &s_ok, &st->slot[nxt], s_rd)) {
      if (tid == 0) atomicExch(&st->exit_reason, -1);
      return;
    }
    pk = s_rd[0];
    const unsigned long long nk = (pk >> 32) + s_rd[1];
    const unsigned long long nE = pk & 0xffffffffull;
    const int reason = nk == 0 ? 1 : (nk + nE > threshold ? 2 : 0);
    if (reason) {
      if (blockIdx.x == 0 && tid == 0) {
        st->levels_done = i + 1;
        atomicCAS(&st->exit_reason, 0, reason);  // a timeout (-1) recorded by any CTA stays
      }
      return;
    }
  }
  if (blockIdx.x == 0 && tid == 0) {
    st->levels_done = max_levels;
    atomicCAS(&st->exit_reason, 0, 3);
  }
}

// Runs sparse BFS levels from frontier *F (its size plus out-degree at most
// `threshold`) on the device.  On return *F holds the next frontier (queue
// form, every vertex of it), *rounds the levels run and *trav their out-degree
// sum.
int bfs_device_levels(gg_graph_s* g, gg_frontier_s** F, int32_t* parents, int32_t* levels, int32_t round0,
                      uint64_t threshold, int32_t* rounds, uint64_t* trav) {
  gg_frontier_s* in = *F;
  const uint32_t n = g->n;
  if (!in->has_sparse) GG_TRY(frontier_to_sparse(in));
  static DeviceOnce occ;
  const int per_sm = occ.get(g->device, [dev = g->device]() {
    int coop = 0, b = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_bfs_push_loop, 256, 0) != cudaSuccess || b < 1)
      return -1;
    return b;
  });
  if (per_sm < 1) return fail(GG_ERR_UNSUPPORTED, "no cooperative launch of the BFS level loop on this device");
  gg_frontier_s *fa = nullptr, *fb = nullptr;
  GG_TRY(frontier_new(g, &fa));
  int rc = frontier_new(g, &fb);
  if (!rc) rc = frontier_ensure_queue(fa);
  if (!rc) rc = frontier_ensure_queue(fb);
  DevBuf<uint32_t> eo0, eo1;
  if (!rc) rc = eo0.alloc(g, n);
  if (!rc) rc = eo1.alloc(g, n);
  if (rc) {
    frontier_free(fa);
    frontier_free(fb);
    return rc;
  }
  LoopState* d_st = reinterpret_cast<LoopState*>(g->ws.d_loop);
  LoopState h{};
  cudaError_t e = cudaMemsetAsync(d_st, 0, sizeof(LoopState), g->stream);
  if (e == cudaSuccess) {
    k_loop_seed<<<generic_grid(g, in->dm), kGenericThreads, 0, g->stream>>>(in->d_queue, in->dm, g->out_off(),
                                                                            fa->d_queue, eo0.p, n, d_st);
    e = cudaGetLastError();
  }
  // a few CTAs per SM (4 unless set): sparse levels are small, and every CTA joins each barrier
  const int grid = g->num_sms * std::min(per_sm, g->loop_ctas_per_sm > 0 ? g->loop_ctas_per_sm : 4);
  const uint32_t* off = g->out_off();
  const uint32_t* idx = g->out_idx();
  uint32_t* q0 = fa->d_queue;
  uint32_t* q1 = fb->d_queue;
  uint32_t* e0 = eo0.p;
  uint32_t* e1 = eo1.p;
  uint32_t nn = n;
  unsigned long long thr = threshold;
  int32_t cap = 1 << 20;
  unsigned budget = g->loop_wait_budget;
  void* args[] = {(void*)&off, (void*)&idx, (void*)&parents, (void*)&levels, (void*)&q0, (void*)&q1, (void*)&e0,
                  (void*)&e1, (void*)&nn, (void*)&d_st, (void*)&round0, (void*)&thr, (void*)&cap, (void*)&budget};
  if (e == cudaSuccess)
    e = cudaLaunchCooperativeKernel((const void*)k_bfs_push_loop, grid, 256, args, 0, g->stream);
  int rr = GG_OK;
  if (e == cudaSuccess) rr = read_small(g, &h, d_st);
  g->kernels += 2;
  if (e != cudaSuccess || rr != GG_OK || h.exit_reason < 0) {
    frontier_free(fa);
    frontier_free(fb);
    if (e != cudaSuccess) return fail(GG_ERR_CUDA, "BFS level loop: %s", cudaGetErrorString(e));
    if (rr != GG_OK) return rr;
    return fail(GG_ERR_TIMEOUT, "BFS level loop: a grid barrier wait ran out");
  }
  const int32_t L = h.levels_done;
  // level L-1 appended into queue (L & 1): fb when L is odd, fa when even
  gg_frontier_s* res = (L & 1) ? fb : fa;
  gg_frontier_s* dead = res == fa ? fb : fa;
  const LoopSlot& last = h.slot[L % 3];
  const uint64_t K = last.packed >> 32, Z = last.zeros;
  if (Z) {  // the vertices without out-edges move from the far end next to the others
    e = cudaMemcpyAsync(res->d_queue + K, res->d_queue + (n - Z), 4 * Z, cudaMemcpyDeviceToDevice, g->stream);
    if (e != cudaSuccess) {
      frontier_free(fa);
      frontier_free(fb);
      return fail(GG_ERR_CUDA, "BFS level loop: %s", cudaGetErrorString(e));
    }
  }
  res->has_sparse = true;
  res->has_dense = false;
  res->bit = false;
  res->dm = K + Z;
  res->out_edges = last.packed & 0xffffffffull;
  frontier_free(dead);
  frontier_free(in);
  *F = res;
  *rounds = L;
  *trav = h.trav;
  return GG_OK;
}

// ===================================================== every level on device
// The whole BFS (app/BFS.C:77-101) in one cooperative launch: after each
// level's grid barrier every CTA reads the next frontier's size and
// out-degree and applies edgeMap's direction rule itself
// (graphgrind/ligra-numa.h:953: size + out-degree > threshold is dense).
// A dense level runs bottom-up over the in-edges with early exit
// (edgeMapDenseCSC with BFS_F, :608-626: a destination takes its first
// frontier in-neighbour), a sparse level runs top-down over the queue
// (push_level).  Every frontier keeps a bitmap (the dense step's input);
// a sparse level also builds its successor's queue, and a dense level whose
// successor is sparse builds that queue from its bitmap in two more grid
// phases (per-CTA counts, then each CTA writes its vertices at the prefix of
// the counts before it, in id order).  Three bitmaps rotate: the one of the
// level before the current is cleared while the current level runs.
// One bottom-up level, this CTA's share (warps over 32-vertex groups, grid
// stride): a vertex without a parent takes its first in-neighbour that is in
// the frontier bitmap bcur and joins bnxt.  *cnt / *deg: this thread's new
// vertices and their out-degree sum.  Not inlined: the loop then keeps its
// registers whatever the rest of the level-loop kernel holds.
// vec: the in-list is read in 16-byte aligned groups of 4 edges (the edge
// arrays are 16-byte aligned and padded past their end), the group's 4
// frontier tests issued together; the first hit in list order still wins.
__device__ __noinline__ void bottom_up_level(const uint32_t* __restrict__ off, const uint32_t* __restrict__ ioff,
                                             const uint32_t* __restrict__ iidx, int32_t* parents, int32_t* levels,
                                             const uint32_t* bcur, uint32_t* bnxt, uint32_t n, int32_t r,
                                             uint32_t* cnt, uint32_t* deg, int vec) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t stride = gridDim.x * blockDim.x;  // <= 2^31 threads
  uint32_t c = 0, dg = 0;
  uint32_t b = blockIdx.x * blockDim.x + (threadIdx.x & ~31u);
  // Loads run ahead of the walk: a lane's parent word and in-list bounds two
  // groups ahead, its first in-neighbour one group ahead, so that they arrive
  // while the current group walks its in-lists (a vertex is this lane's alone
  // during a bottom-up level: nobody else writes its parent).
  auto load = [&](uint32_t bb, int32_t& pv, uint32_t& j0, uint32_t& e1) {
    const uint32_t v = bb + lane;
    pv = 0;
    j0 = e1 = 0;
    if (v < n) {
      pv = __ldcg(parents + v);
      j0 = ioff[v];
      e1 = ioff[v + 1];
    }
  };
  auto first = [&](int32_t pv, uint32_t j0, uint32_t e1) -> uint32_t {
    return (pv == -1 && j0 < e1) ? iidx[j0] : 0u;
  };
  // groups b (pv, j0, e1, s0) and b + stride (pv1, j1, e11)
  int32_t pv = 0, pv1 = 0;
  uint32_t j0 = 0, e1 = 0, j1 = 0, e11 = 0, s0 = 0;
  if (b < n) load(b, pv, j0, e1);
  if ((uint64_t)b + stride < n) load(b + stride, pv1, j1, e11);
  if (b < n) s0 = first(pv, j0, e1);
  for (; b < n; b += stride) {
    const bool last = (uint64_t)b + stride >= n;  // no group after this one
    int32_t pv2 = 0;
    uint32_t j2 = 0, e2 = 0, s1 = 0;
    if ((uint64_t)b + 2ull * stride < n) load(b + 2 * stride, pv2, j2, e2);
    if (!last) s1 = first(pv1, j1, e11);
    const uint32_t v = b + lane;
    bool act = false;
    if (v < n && pv == -1 && j0 < e1) {
      if ((bcur[s0 >> 5] >> (s0 & 31)) & 1u) {
        parents[v] = (int32_t)s0;
        if (levels) levels[v] = r;
        act = true;
      } else if (vec) {
        for (uint32_t a = (j0 + 1) & ~3u; a < e1; a += 4) {
          const uint4 q = __ldg(reinterpret_cast<const uint4*>(iidx + a));
          const uint32_t ss[4] = {q.x, q.y, q.z, q.w};
          int hit = -1;
#pragma unroll
          for (int t = 3; t >= 0; --t) {
            const uint32_t e = a + (uint32_t)t;
            if (e > j0 && e < e1 && ((bcur[ss[t] >> 5] >> (ss[t] & 31)) & 1u)) hit = t;
          }
          if (hit >= 0) {
            parents[v] = (int32_t)ss[hit];
            if (levels) levels[v] = r;
            act = true;
            break;
          }
        }
      } else {
        for (uint32_t j = j0 + 1; j < e1; ++j) {
          const uint32_t s = iidx[j];
          if ((bcur[s >> 5] >> (s & 31)) & 1u) {
            parents[v] = (int32_t)s;
            if (levels) levels[v] = r;
            act = true;
            break;
          }
        }
      }
    }
    const uint32_t word = __ballot_sync(0xffffffffu, act);
    if (act) dg += off[v + 1] - off[v];
    if (lane == 0 && word) {
      atomicOr(bnxt + (b >> 5), word);
      c += __popc(word);
    }
    if (last) break;
    pv = pv1;
    j0 = j1;
    e1 = e11;
    s0 = s1;
    pv1 = pv2;
    j1 = j2;
    e11 = e2;
  }
  *cnt = c;
  *deg = dg;
}

__global__ void k_bfs_full_seed(uint32_t start, const uint32_t* off, uint32_t* q0, uint32_t* eo0, uint32_t* bits0,
                                LoopState* st) {
  if (threadIdx.x == 0) {
    const uint32_t d = off[start + 1] - off[start];
    bits0[start >> 5] = 1u << (start & 31);
    q0[0] = start;
    eo0[0] = 0;
    if (d > 0)
      st->slot[0].packed = (1ull << 32) | d;
    else
      st->slot[0].zeros = 1;
  }
}

// Sums of five values over the CTA (blockDim.x == 256), returned to every thread.
__device__ __forceinline__ void block_sum5(unsigned long long* v, unsigned long long (*s_red)[8]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < 5; ++j) v[j] = warp_sum(v[j]);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int j = 0; j < 5; ++j) s_red[j][warp] = v[j];
  __syncthreads();
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    unsigned long long t = 0;
    for (int w = 0; w < 8; ++w) t += s_red[j][w];
    v[j] = t;
  }
}

__global__ void __launch_bounds__(256, 8) k_bfs_full(const uint32_t* __restrict__ off, const uint32_t* __restrict__ idx,
                                                     const uint32_t* __restrict__ ioff,
                                                     const uint32_t* __restrict__ iidx, int32_t* parents,
                                                     int32_t* levels, uint32_t* q0, uint32_t* q1, uint32_t* eo0,
                                                     uint32_t* eo1, uint32_t* bits, uint32_t wstride,
                                                     unsigned long long* cta, uint32_t n, LoopState* st,
                                                     int32_t round0, unsigned long long threshold,
                                                     int32_t max_levels, unsigned wait_budget, int bu_vec) {
  __shared__ uint32_t s_eo[257];
  __shared__ uint32_t s_v[256];
  __shared__ uint32_t s_beg[256];
  __shared__ uint32_t s_scan[2][8];
  __shared__ unsigned long long s_base[2];
  __shared__ unsigned long long s_red[5][8];
  __shared__ unsigned long long s_rd[5];
  __shared__ int s_ok;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t nw = (n + 31) / 32;
  const uint32_t wper = (nw + gridDim.x - 1) / gridDim.x;
  const uint32_t w0 = min(nw, blockIdx.x * wper), w1 = min(nw, w0 + wper);
  // s_rd holds the current frontier's counters (slot layout), from one level to the next
  if (tid == 0) read_slot(&st->slot[0], s_rd);
  __syncthreads();
  unsigned target = 0;
  for (int32_t i = 0; i < max_levels; ++i) {
    const int cur = i % 3, nxt = (i + 1) % 3, old = (i + 2) % 3;
    const int rep = (int)s_rd[4];
    const unsigned long long pk = s_rd[0];
    const uint32_t* q = (i & 1) ? q1 : q0;
    const uint32_t* eo = (i & 1) ? eo1 : eo0;
    uint32_t* nq = (i & 1) ? q0 : q1;
    uint32_t* neo = (i & 1) ? eo0 : eo1;
    const uint32_t* bcur = bits + (size_t)cur * wstride;
    uint32_t* bnxt = bits + (size_t)nxt * wstride;
    uint32_t* bold = bits + (size_t)old * wstride;
    const uint64_t k = rep == 0 ? pk >> 32 : 0;
    const uint64_t E = rep == 0 ? pk & 0xffffffffull : s_rd[3];
    const uint64_t nk = rep == 0 ? k + s_rd[1] : s_rd[2];
    if (blockIdx.x == 0 && tid == 0) {  // counters of level i+2's frontier; nobody touches them in level i
      LoopSlot& o = st->slot[old];
      o.packed = 0;
      o.zeros = 0;
      o.dcnt = 0;
      o.ddeg = 0;
      st->trav += E;
    }
    for (uint32_t w = w0 + tid; w < w1; w += blockDim.x) bold[w] = 0u;  // level i-1's frontier, done with
    const int32_t r = round0 + i;
    if (nk + E > threshold) {
      // bottom-up: one lane per destination, the first frontier in-neighbour wins
      uint32_t c32 = 0, dg32 = 0;
      bottom_up_level(off, ioff, iidx, parents, levels, bcur, bnxt, n, r, &c32, &dg32, bu_vec);
      unsigned long long c = warp_sum((unsigned long long)c32), dg = warp_sum((unsigned long long)dg32);
      if (lane == 0) {
        s_red[0][warp] = c;
        s_red[1][warp] = dg;
      }
      __syncthreads();
      if (tid == 0) {
        unsigned long long tc = 0, td = 0;
        for (int w = 0; w < 8; ++w) {
          tc += s_red[0][w];
          td += s_red[1][w];
        }
        if (tc) atomicAdd(&st->slot[nxt].dcnt, tc);
        if (td) atomicAdd(&st->slot[nxt].ddeg, td);
        if (blockIdx.x == 0) st->slot[nxt].rep = 1;
      }
    } else {
      push_level(off, idx, parents, levels, q, eo, nq, neo, k, E, n, r, &st->slot[nxt].packed,
                 &st->slot[nxt].zeros, bnxt, s_eo, s_v, s_beg, s_scan, s_base);
      if (blockIdx.x == 0 && tid == 0) st->slot[nxt].rep = 0;
    }
    target += gridDim.x;
    if (!grid_barrier(&st->bar, target, wait_budget, &s_ok, &st->slot[nxt], s_rd)) {
      if (tid == 0) atomicExch(&st->exit_reason, -1);
      return;
    }
    const int nrep = (int)s_rd[4];
    const unsigned long long npk = s_rd[0];
    const unsigned long long nk2 = nrep == 0 ? (npk >> 32) + s_rd[1] : s_rd[2];
    const unsigned long long nE = nrep == 0 ? npk & 0xffffffffull : s_rd[3];
    if (nk2 == 0) {
      if (blockIdx.x == 0 && tid == 0) {
        st->levels_done = i + 1;
        atomicCAS(&st->exit_reason, 0, 1);  // a timeout (-1) recorded by any CTA stays
      }
      return;
    }
    if (nrep == 1 && nk2 + nE <= threshold) {
      // the next level pushes: its queue from the bitmap, vertices with
      // out-edges in id order (phase A: this CTA's counts of its words)
      unsigned long long v5[5] = {0, 0, 0, 0, 0};
      for (uint32_t w = w0 + tid; w < w1; w += blockDim.x) {
        uint32_t x = bnxt[w];
        while (x) {
          const uint32_t v = w * 32 + (__ffs(x) - 1);
          x &= x - 1;
          const uint32_t d = off[v + 1] - off[v];
          if (d) {
            ++v5[0];
            v5[1] += d;
          } else {
            ++v5[2];
          }
        }
      }
      block_sum5(v5, s_red);
      if (tid < 3) cta[(size_t)blockIdx.x * 3 + tid] = v5[tid];
      target += gridDim.x;
      if (!grid_barrier(&st->bar, target, wait_budget, &s_ok)) {
        if (tid == 0) atomicExch(&st->exit_reason, -1);
        return;
      }
      // phase B: the counts of the CTAs before this one and of all, then the writes
      unsigned long long t5[5] = {0, 0, 0, 0, 0};  // before: slots, edges; all: slots, edges, zeros
      for (uint32_t c2 = tid; c2 < gridDim.x; c2 += blockDim.x) {
        const unsigned long long x0 = cta[(size_t)c2 * 3], x1 = cta[(size_t)c2 * 3 + 1],
                                 x2 = cta[(size_t)c2 * 3 + 2];
        if (c2 < blockIdx.x) {
          t5[0] += x0;
          t5[1] += x1;
        }
        t5[2] += x0;
        t5[3] += x1;
        t5[4] += x2;
      }
      block_sum5(t5, s_red);
      unsigned long long base_p = t5[0], base_d = t5[1];
      // words in chunks of 256, one per thread, in order
      for (uint32_t c0 = w0; c0 < w1; c0 += blockDim.x) {
        const uint32_t w = c0 + tid;
        const uint32_t x = w < w1 ? bnxt[w] : 0u;
        uint32_t mp = 0, md = 0;
        uint32_t y = x;
        while (y) {
          const uint32_t v = w * 32 + (__ffs(y) - 1);
          y &= y - 1;
          const uint32_t d = off[v + 1] - off[v];
          if (d) {
            ++mp;
            md += d;
          }
        }
        uint32_t ep, ed, tpc, tdc;
        block_scan2(mp, md, &ep, &ed, &tpc, &tdc, s_scan);
        uint32_t slot = (uint32_t)base_p + ep, eoff = (uint32_t)base_d + ed;
        y = x;
        while (y) {
          const uint32_t v = w * 32 + (__ffs(y) - 1);
          y &= y - 1;
          const uint32_t d = off[v + 1] - off[v];
          if (d) {
            nq[slot] = v;
            neo[slot] = eoff;
            ++slot;
            eoff += d;
          }
        }
        base_p += tpc;
        base_d += tdc;
      }
      // every CTA holds the totals (the next level's counters); the slot records them as well
      if (tid == 0) {
        s_rd[0] = (t5[2] << 32) | t5[3];
        s_rd[1] = t5[4];
        s_rd[4] = 0;
        if (blockIdx.x == 0) {
          st->slot[nxt].packed = s_rd[0];
          st->slot[nxt].zeros = s_rd[1];
          st->slot[nxt].rep = 0;
        }
      }
      target += gridDim.x;
      if (!grid_barrier(&st->bar, target, wait_budget, &s_ok)) {
        if (tid == 0) atomicExch(&st->exit_reason, -1);
        return;
      }
    }
  }
  if (blockIdx.x == 0 && tid == 0) {
    st->levels_done = max_levels;
    atomicCAS(&st->exit_reason, 0, 3);
  }
}

// Enqueues every level of the BFS from `start` as one cooperative launch
// (k_bfs_full) on the graph's stream and returns without waiting;
// parents/levels hold the source's entries already (levels may be null).
// bfs_device_full_result reads the outcome once the stream has passed it.
int bfs_device_full(gg_graph_s* g, uint32_t start, int32_t* parents, int32_t* levels, uint64_t threshold) {
  const uint32_t n = g->n;
  static DeviceOnce occ;
  const int per_sm = occ.get(g->device, [dev = g->device]() {
    int coop = 0, b = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (!coop || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_bfs_full, 256, 0) != cudaSuccess || b < 1)
      return -1;
    return b;
  });
  if (per_sm < 1) return fail(GG_ERR_UNSUPPORTED, "no cooperative launch of the BFS loop on this device");
  // every warp slot unless set: the bottom-up levels are latency-bound
  const int grid = g->num_sms * std::min(per_sm, g->loop_ctas_per_sm > 0 ? g->loop_ctas_per_sm : 8);
  const uint32_t words = (n + 31) / 32;
  const uint32_t wstride = (words + 31) & ~31u;  // 128-byte aligned bitmaps
  DevBuf<uint32_t> q0, q1, eo0, eo1, bits;
  DevBuf<unsigned long long> cta;
  GG_TRY(q0.alloc(g, n));
  GG_TRY(q1.alloc(g, n));
  GG_TRY(eo0.alloc(g, n));
  GG_TRY(eo1.alloc(g, n));
  GG_TRY(bits.alloc(g, 3ull * wstride));
  GG_TRY(cta.alloc(g, 3ull * grid));
  LoopState* d_st = reinterpret_cast<LoopState*>(g->ws.d_loop);
  GG_CUDA(cudaMemsetAsync(bits.p, 0, 4ull * 3 * wstride, g->stream));
  GG_CUDA(cudaMemsetAsync(d_st, 0, sizeof(LoopState), g->stream));
  k_bfs_full_seed<<<1, 32, 0, g->stream>>>(start, g->out_off(), q0.p, eo0.p, bits.p, d_st);
  GG_CUDA(cudaGetLastError());
  const uint32_t* off = g->out_off();
  const uint32_t* idx = g->out_idx();
  const uint32_t* ioff = g->in_off();
  // the bottom-up levels walk the in-lists hub sources first (same edges,
  // other order: a vertex then meets a frontier in-neighbour sooner)
  // (graphs the copy cannot be built for, past 2^31 edges or without the
  // memory, walk the CSC's own in-lists)
  if (g->early_kernel == 3 && !g->d_bu_idx && build_bu_index(g) != GG_OK) cudaGetLastError();
  const uint32_t* iidx = g->early_kernel == 3 && g->d_bu_idx ? g->d_bu_idx : g->in_idx();
  uint32_t* a0 = q0.p;
  uint32_t* a1 = q1.p;
  uint32_t* e0 = eo0.p;
  uint32_t* e1 = eo1.p;
  uint32_t* bp = bits.p;
  uint32_t ws = wstride;
  unsigned long long* cp = cta.p;
  uint32_t nn = n;
  int32_t round0 = 1;
  unsigned long long thr = threshold;
  int32_t cap = n < (uint32_t)INT32_MAX ? (int32_t)n + 1 : INT32_MAX;
  unsigned budget = g->loop_wait_budget;
  int vec = g->early_kernel >= 2 ? 1 : 0;
  void* args[] = {(void*)&off, (void*)&idx, (void*)&ioff, (void*)&iidx, (void*)&parents, (void*)&levels,
                  (void*)&a0,  (void*)&a1,  (void*)&e0,   (void*)&e1,   (void*)&bp,      (void*)&ws,
                  (void*)&cp,  (void*)&nn,  (void*)&d_st, (void*)&round0, (void*)&thr,   (void*)&cap,
                  (void*)&budget, (void*)&vec};
  GG_CUDA(cudaLaunchCooperativeKernel((const void*)k_bfs_full, grid, 256, args, 0, g->stream));
  g->kernels += 2;
  return GG_OK;
}

// The outcome of the BFS bfs_device_full enqueued (synchronises the stream):
// *rounds, the number of edgeMap rounds (the last one finds nothing), *trav,
// the out-degree sum of the frontiers processed.
int bfs_device_full_result(gg_graph_s* g, int32_t* rounds, uint64_t* trav) {
  LoopState h{};
  GG_TRY(read_small(g, &h, reinterpret_cast<const LoopState*>(g->ws.d_loop)));
  if (h.exit_reason < 0) return fail(GG_ERR_TIMEOUT, "BFS loop: a grid barrier wait ran out");
  if (h.exit_reason != 1)
    return fail(GG_ERR_CUDA, "BFS loop: stopped without an empty frontier (reason %d)", h.exit_reason);
  *rounds = h.levels_done;
  *trav = h.trav;
  return GG_OK;
}

}  // namespace gg
