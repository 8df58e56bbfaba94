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
  unsigned long long cnt[3];  // frontier sizes, indexed by level mod 3
  unsigned long long od[3];   // their out-degree sums
  unsigned long long trav;    // out-degree sum of the frontiers processed
  unsigned int bar;           // barrier arrivals
  int32_t levels_done;
  int32_t exit_reason;        // 1 empty, 2 next level is dense, 3 level cap, -1 barrier timeout
  int32_t pad;
};

constexpr unsigned kBarrierSpin = 1u << 22;

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

// All CTAs of the (co-resident) grid arrive; returns false if the wait ran out.
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned target, int* s_ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(bar, 1u);
    int ok = 1;
    for (unsigned it = 0; (int)(ld_acquire_u32(bar) - target) < 0; ++it) {
      if (it > kBarrierSpin) {
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

__global__ void __launch_bounds__(256) k_bfs_push_loop(const uint32_t* __restrict__ off,
                                                       const uint32_t* __restrict__ idx, int32_t* parents,
                                                       int32_t* levels, uint32_t* q0, uint32_t* q1,
                                                       BfsLoopState* st, int32_t round0, unsigned long long threshold,
                                                       int32_t max_levels) {
  __shared__ uint32_t s_scan[257];
  __shared__ uint32_t s_beg[256];
  __shared__ uint32_t s_src[256];
  __shared__ uint32_t s_warp[32];
  __shared__ int s_ok;
  const int tid = threadIdx.x, lane = tid & 31;
  const uint32_t lanemask_lt = (1u << lane) - 1u;
  unsigned target = 0;
  for (int32_t i = 0; i < max_levels; ++i) {
    const int cur = i % 3, nxt = (i + 1) % 3, old = (i + 2) % 3;
    const uint32_t* q = (i & 1) ? q1 : q0;
    uint32_t* nq = (i & 1) ? q0 : q1;
    const unsigned long long k = ld_relaxed_u64(&st->cnt[cur]);
    if (blockIdx.x == 0 && tid == 0) {  // the counters level i+1 appends to; nobody reads them in level i
      st->cnt[old] = 0;
      st->od[old] = 0;
    }
    const int32_t r = round0 + i;
    unsigned long long my_od = 0, my_trav = 0;
    for (unsigned long long c0 = (unsigned long long)blockIdx.x * 256; c0 < k;
         c0 += (unsigned long long)gridDim.x * 256) {
      const unsigned long long ii = c0 + tid;
      uint32_t beg = 0, deg = 0, v = 0;
      if (ii < k) {
        v = q[ii];
        beg = off[v];
        deg = off[v + 1] - beg;
      }
      uint32_t total;
      const uint32_t excl = block_excl_scan(deg, s_warp, &total);
      s_scan[tid] = excl;
      s_beg[tid] = beg;
      s_src[tid] = v;
      if (tid == 0) s_scan[256] = total;
      __syncthreads();
      if (tid == 0) my_trav += total;
      for (uint32_t t0 = 0; t0 < total; t0 += 256) {
        const uint32_t t = t0 + tid;
        bool add = false;
        uint32_t u = 0;
        if (t < total) {
          int lo = 0, hi = 255;  // the last slot whose exclusive start is <= t
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (s_scan[mid] <= t)
              lo = mid;
            else
              hi = mid - 1;
          }
          const uint32_t s = s_src[lo];
          u = idx[s_beg[lo] + (t - s_scan[lo])];
          if (__ldcg(parents + u) == -1 && atomicCAS(parents + u, -1, (int32_t)s) == -1) {
            add = true;
            if (levels) levels[u] = r;
            my_od += off[u + 1] - off[u];
          }
        }
        const uint32_t bal = __ballot_sync(0xffffffffu, add);
        if (bal) {
          const int leader = __ffs(bal) - 1;
          unsigned long long base = 0;
          if (lane == leader) base = atomicAdd(&st->cnt[nxt], (unsigned long long)__popc(bal));
          base = __shfl_sync(0xffffffffu, base, leader);
          if (add) nq[base + __popc(bal & lanemask_lt)] = u;
        }
      }
      __syncthreads();
    }
    my_od = warp_sum(my_od);
    if (lane == 0 && my_od) atomicAdd(&st->od[nxt], my_od);
    if (tid == 0 && my_trav) atomicAdd(&st->trav, my_trav);
    target += gridDim.x;
    if (!grid_barrier(&st->bar, target, &s_ok)) {
      if (tid == 0) atomicExch(&st->exit_reason, -1);
      return;
    }
    const unsigned long long nk = ld_relaxed_u64(&st->cnt[nxt]), nod = ld_relaxed_u64(&st->od[nxt]);
    const int reason = nk == 0 ? 1 : (nk + nod > threshold ? 2 : 0);
    if (reason) {
      if (blockIdx.x == 0 && tid == 0) {
        st->levels_done = i + 1;
        st->exit_reason = reason;
      }
      return;
    }
  }
  if (blockIdx.x == 0 && tid == 0) {
    st->levels_done = max_levels;
    st->exit_reason = 3;
  }
}

// Runs sparse BFS levels from frontier *F (a queue of dm vertices whose size
// plus out-degree is at most `threshold`) on the device.  On return *F holds
// the next frontier (queue form), *rounds the levels run and *trav their
// out-degree sum.
int bfs_device_levels(gg_graph_s* g, gg_frontier_s** F, int32_t* parents, int32_t* levels, int32_t round0,
                      uint64_t threshold, int32_t* rounds, uint64_t* trav) {
  gg_frontier_s* in = *F;
  if (!in->has_sparse) GG_TRY(frontier_to_sparse(in));
  gg_frontier_s* other = nullptr;
  GG_TRY(frontier_new(g, &other));
  int rc = frontier_ensure_queue(other);
  static int per_sm = -1;
  if (!rc && per_sm < 0) {
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, g->device);
    if (!coop) rc = fail(GG_ERR_UNSUPPORTED, "device does not support cooperative launches");
    else if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bfs_push_loop, 256, 0) != cudaSuccess)
      rc = fail(GG_ERR_CUDA, "occupancy query failed");
  }
  if (rc) {
    frontier_free(other);
    return rc;
  }
  BfsLoopState h{};
  h.cnt[0] = in->dm;
  h.od[0] = in->out_edges;
  BfsLoopState* d_st = reinterpret_cast<BfsLoopState*>(g->ws.d_loop);
  GG_CUDA(cudaMemcpyAsync(d_st, &h, sizeof(h), cudaMemcpyHostToDevice, g->stream));
  // a few CTAs per SM: sparse levels are small, and every CTA joins each barrier
  const int grid = g->num_sms * std::min(std::max(per_sm, 1), 4);
  const uint32_t* off = g->out_off();
  const uint32_t* idx = g->out_idx();
  uint32_t* q0 = in->d_queue;
  uint32_t* q1 = other->d_queue;
  unsigned long long thr = threshold;
  int32_t cap = 1 << 20;
  void* args[] = {(void*)&off, (void*)&idx, (void*)&parents, (void*)&levels, (void*)&q0, (void*)&q1,
                  (void*)&d_st, (void*)&round0, (void*)&thr, (void*)&cap};
  cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_bfs_push_loop, grid, 256, args, 0, g->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d_st, sizeof(h), cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  g->kernels++;
  if (e != cudaSuccess) {
    frontier_free(other);
    return fail(GG_ERR_CUDA, "BFS level loop: %s", cudaGetErrorString(e));
  }
  if (h.exit_reason < 0) {
    frontier_free(other);
    return fail(GG_ERR_TIMEOUT, "BFS level loop: a grid barrier wait ran out");
  }
  const int32_t L = h.levels_done;
  // level L-1 appended into q1 when L-1 is even, into q0 when odd
  gg_frontier_s* res = ((L - 1) & 1) ? in : other;
  gg_frontier_s* dead = res == in ? other : in;
  res->has_sparse = true;
  res->has_dense = false;
  res->bit = false;
  res->dm = h.cnt[L % 3];
  res->out_edges = h.od[L % 3];
  frontier_free(dead);
  *F = res;
  *rounds = L;
  *trav = h.trav;
  return GG_OK;
}

}  // namespace gg
