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

struct BfsLoopState {
  // frontier by level mod 3: (queue slots << 32) | out-edges; vertices with out-edges
  // fill the queue from the front in edge-offset order
  unsigned long long packed[3];
  unsigned long long zeros[3];  // vertices without out-edges, kept at the queue's far end
  unsigned long long trav;      // out-edges of the frontiers processed
  unsigned int bar;             // barrier arrivals
  int32_t levels_done;
  int32_t exit_reason;          // 1 empty, 2 next level is dense, 3 level cap, -1 barrier timeout
  int32_t pad;
};


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

// All CTAs of the (co-resident) grid arrive; returns false if the wait ran out
// (more than `budget` probes of the arrival count, each followed by a short sleep).
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned target, unsigned budget, int* s_ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(bar, 1u);
    int ok = 1;
    for (unsigned it = 0; (int)(ld_acquire_u32(bar) - target) < 0; ++it) {
      if (it >= budget) {
        ok = 0;
        break;
      }
      __nanosleep(32);
    }
    __threadfence();
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
                                            uint32_t n, unsigned long long* packed, unsigned long long* zeros) {
  const int lane = threadIdx.x & 31;
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

// Level 0's queue: the input frontier's vertices with out-edges, with offsets.
__global__ void k_loop_seed(const uint32_t* in_q, uint64_t k, const uint32_t* off, uint32_t* q0, uint32_t* eo0,
                            uint32_t n, BfsLoopState* st) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x; i0 < k; i0 += stride) {  // warp-uniform trip count
    const uint64_t i = i0 + threadIdx.x;
    uint32_t v = 0, deg = 0;
    if (i < k) {
      v = in_q[i];
      deg = off[v + 1] - off[v];
    }
    loop_append(i < k && deg > 0, v, deg, q0, eo0, n, &st->packed[0], &st->zeros[0]);
  }
}

__global__ void __launch_bounds__(256) k_bfs_push_loop(const uint32_t* __restrict__ off,
                                                       const uint32_t* __restrict__ idx, int32_t* parents,
                                                       int32_t* levels, uint32_t* q0, uint32_t* q1, uint32_t* eo0,
                                                       uint32_t* eo1, uint32_t n, BfsLoopState* st, int32_t round0,
                                                       unsigned long long threshold, int32_t max_levels,
                                                       unsigned wait_budget) {
  __shared__ uint32_t s_eo[257];
  __shared__ uint32_t s_v[256];
  __shared__ uint32_t s_beg[256];
  __shared__ int s_ok;
  const int tid = threadIdx.x;
  unsigned target = 0;
  for (int32_t i = 0; i < max_levels; ++i) {
    const int cur = i % 3, nxt = (i + 1) % 3, old = (i + 2) % 3;
    const uint32_t* q = (i & 1) ? q1 : q0;
    const uint32_t* eo = (i & 1) ? eo1 : eo0;
    uint32_t* nq = (i & 1) ? q0 : q1;
    uint32_t* neo = (i & 1) ? eo0 : eo1;
    const unsigned long long pk = ld_relaxed_u64(&st->packed[cur]);
    const uint64_t k = pk >> 32;
    const uint64_t E = pk & 0xffffffffull;
    if (blockIdx.x == 0 && tid == 0) {  // counters of level i+2's frontier; nobody touches them in level i
      st->packed[old] = 0;
      st->zeros[old] = 0;
      st->trav += E;
    }
    const int32_t r = round0 + i;
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
        loop_append(add, u, deg, nq, neo, n, &st->packed[nxt], &st->zeros[nxt]);
        // the slot holding edge last + 1: the next staged one if it starts there,
        // else the last one staged (which runs past `last`)
        scur += (s_eo[ns] == (uint32_t)(last + 1)) ? ns : ns - 1;
        __syncthreads();
      }
    }
    target += gridDim.x;
    if (!grid_barrier(&st->bar, target, wait_budget, &s_ok)) {
      if (tid == 0) atomicExch(&st->exit_reason, -1);
      return;
    }
    const unsigned long long npk = ld_relaxed_u64(&st->packed[nxt]);
    const unsigned long long nk = (npk >> 32) + ld_relaxed_u64(&st->zeros[nxt]);
    const unsigned long long nE = npk & 0xffffffffull;
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
  static int per_sm = -1;
  if (per_sm < 0) {
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, g->device);
    if (!coop) return fail(GG_ERR_UNSUPPORTED, "device does not support cooperative launches");
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bfs_push_loop, 256, 0) != cudaSuccess)
      return fail(GG_ERR_CUDA, "occupancy query failed");
  }
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
  BfsLoopState* d_st = reinterpret_cast<BfsLoopState*>(g->ws.d_loop);
  BfsLoopState h{};
  cudaError_t e = cudaMemsetAsync(d_st, 0, sizeof(BfsLoopState), g->stream);
  if (e == cudaSuccess) {
    k_loop_seed<<<generic_grid(g, in->dm), kGenericThreads, 0, g->stream>>>(in->d_queue, in->dm, g->out_off(),
                                                                            fa->d_queue, eo0.p, n, d_st);
    e = cudaGetLastError();
  }
  // a few CTAs per SM: sparse levels are small, and every CTA joins each barrier
  const int grid = g->num_sms * std::min(std::max(per_sm, 1), 4);
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
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d_st, sizeof(h), cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  g->kernels += 2;
  if (e != cudaSuccess || h.exit_reason < 0) {
    frontier_free(fa);
    frontier_free(fb);
    if (e != cudaSuccess) return fail(GG_ERR_CUDA, "BFS level loop: %s", cudaGetErrorString(e));
    return fail(GG_ERR_TIMEOUT, "BFS level loop: a grid barrier wait ran out");
  }
  const int32_t L = h.levels_done;
  // level L-1 appended into queue (L & 1): fb when L is odd, fa when even
  gg_frontier_s* res = (L & 1) ? fb : fa;
  gg_frontier_s* dead = res == fa ? fb : fa;
  const uint64_t K = h.packed[L % 3] >> 32, Z = h.zeros[L % 3];
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
  res->out_edges = h.packed[L % 3] & 0xffffffffull;
  frontier_free(dead);
  frontier_free(in);
  *F = res;
  *rounds = L;
  *trav = h.trav;
  return GG_OK;
}

}  // namespace gg
