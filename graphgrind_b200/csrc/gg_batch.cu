// Batched traversals: k-column personalised PageRank as one SpMM-shaped pull
// per iteration (every edge moves a whole 64- or 32-column row of the source
// contributions instead of one 4-byte value).
//
//   X_0 = T,  X_{t+1} = d * A X_t + (1 - d) * T,  A[v,u] = 1/outdeg(u) for u->v
//
// the personalised form of PR_F / PR_Vertex_F (app/PageRank.C:256-315) with a
// teleport matrix T (n x k, row-major) in place of the uniform 1/n, all
// vertices active (PageRankBit, app/PageRankBit.C:145).
#include <algorithm>
#include <functional>
#include <vector>

#include "gg_runtime.cuh"

namespace gg {

// Sum pull: S[v, c] = sum over in-edges u->v of XS[u, c], for c in one
// 32-column slab per lane pair.  One warp per 256-edge block of the CSC; the
// head-bit row structure tells every edge's row.  Rows that end inside the
// block are stored; rows that cross a block boundary are added atomically
// (those rows were zeroed before the launch).
template <int KW>  // KW = columns per lane (1 -> 32 columns, 2 -> 64 columns)
__global__ void __launch_bounds__(256) k_ppr_pull(const uint32_t* idx, const uint32_t* head, const uint32_t* blk,
                                                   const uint32_t* rows, uint64_t nblocks, uint64_t m,
                                                   const float* xs, float* S, uint32_t k) {
  __shared__ uint32_t s_idx[8][kSegBlock];
  __shared__ uint8_t s_head[8][kSegBlock];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t b = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp; b < nblocks; b += warps) {
    const uint64_t e0 = b * kSegBlock;
    // stage this block's sources and row-head flags (lane l: edges 8l .. 8l+7)
    const uint4 ia = __ldg(reinterpret_cast<const uint4*>(idx + e0) + 2 * lane);
    const uint4 ib = __ldg(reinterpret_cast<const uint4*>(idx + e0) + 2 * lane + 1);
    const uint32_t hw = __ldg(head + b * 8 + (lane >> 2));
    const uint32_t bits = (hw >> ((lane & 3) * 8)) & 0xffu;
    reinterpret_cast<uint4*>(s_idx[warp])[2 * lane] = ia;
    reinterpret_cast<uint4*>(s_idx[warp])[2 * lane + 1] = ib;
#pragma unroll
    for (int q = 0; q < 8; ++q) s_head[warp][lane * 8 + q] = (bits >> q) & 1u;
    __syncwarp();
    const uint32_t blk_end = m - e0 < (uint64_t)kSegBlock ? (uint32_t)(m - e0) : (uint32_t)kSegBlock;
    // the row continuing from the previous block has ordinal blk[b] - 1
    uint32_t cur_ord = __ldg(blk + b) - 1u;
    bool started_here = false;
    int have = 0;
    float acc[KW];
#pragma unroll
    for (int c = 0; c < KW; ++c) acc[c] = 0.f;
    auto flush = [&](bool complete) {
      float* dst = S + (uint64_t)__ldg(rows + cur_ord) * k + lane * KW;
      if (complete) {
#pragma unroll
        for (int c = 0; c < KW; ++c) dst[c] = acc[c];
      } else {
#pragma unroll
        for (int c = 0; c < KW; ++c) atomicAdd(dst + c, acc[c]);
      }
    };
    for (uint32_t g0 = 0; g0 < blk_end; g0 += 8) {
      // issue the group's row gathers before consuming them
      float v[8][KW];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const uint32_t e = g0 + q;
        if (e < blk_end) {
          const float* xr = xs + (uint64_t)s_idx[warp][e] * k + lane * KW;
          if (KW == 2) {
            const float2 t = __ldg(reinterpret_cast<const float2*>(xr));
            v[q][0] = t.x;
            v[q][KW - 1] = t.y;
          } else {
            v[q][0] = __ldg(xr);
          }
        }
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const uint32_t e = g0 + q;
        if (e >= blk_end) break;
        if (s_head[warp][e]) {  // a new row starts: the current one is done
          if (have > 0) flush(started_here);
          ++cur_ord;
          started_here = true;
          have = 0;
#pragma unroll
          for (int c = 0; c < KW; ++c) acc[c] = 0.f;
        }
#pragma unroll
        for (int c = 0; c < KW; ++c) acc[c] += v[q][c];
        ++have;
      }
    }
    if (have > 0) {  // the last row is complete only if the next block starts a new row
      const uint64_t nxt = e0 + blk_end;
      const bool ends_here = nxt >= m || ((__ldg(head + (nxt >> 5)) >> (nxt & 31)) & 1u);
      flush(started_here && ends_here);
    }
    __syncwarp();
  }
}

// Zero the S rows that receive partial sums (rows crossing a block boundary).
__global__ void k_zero_rows(const uint32_t* rows_list, uint32_t count, float* S, uint32_t k) {
  const uint64_t total = (uint64_t)count * k;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x)
    S[(uint64_t)rows_list[i / k] * k + (i % k)] = 0.f;
}

// Vertex pass: Y = d*S + (1-d)*T (S = 0 for vertices without in-edges), and
// the next iteration's per-source rows XS = Y / outdeg.
__global__ void k_ppr_vertex(uint32_t n, uint32_t k, const uint32_t* in_off, const uint32_t* out_off, const float* S,
                             const float* T, float damping, float* Y, float* XS, int write_y) {
  const uint64_t total = (uint64_t)n * k;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = (uint32_t)(i / k);
    const float s = in_off[v + 1] > in_off[v] ? S[i] : 0.f;
    const float y = damping * s + (1.f - damping) * T[i];
    if (write_y) Y[i] = y;
    const uint32_t d = out_off[v + 1] - out_off[v];
    XS[i] = d ? y / (float)d : 0.f;
  }
}

__global__ void k_ppr_onehot(const uint32_t* seeds, uint32_t k, float* T) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < k) T[(uint64_t)seeds[j] * k + j] = 1.f;
}

__global__ void k_ppr_init(uint32_t n, uint32_t k, const float* T, const uint32_t* out_off, float* XS) {
  const uint64_t total = (uint64_t)n * k;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = (uint32_t)(i / k);
    const uint32_t d = out_off[v + 1] - out_off[v];
    XS[i] = d ? T[i] / (float)d : 0.f;
  }
}

// Rows whose in-edges cross a 256-edge block boundary (static per graph).
static int boundary_rows(gg_graph_s* g, std::vector<uint32_t>& out) {
  const uint32_t* off = g->transposed ? g->h_csr_off.data() : g->h_csc_off.data();
  for (uint32_t v = 0; v < g->n; ++v) {
    const uint32_t a = off[v], b = off[v + 1];
    if (b > a && (a / kSegBlock) != ((b - 1) / kSegBlock)) out.push_back(v);
  }
  return GG_OK;
}

static int run_ppr_k(gg_graph_s* g, int32_t k, int32_t iters, float damping, const float* tele_host,
                     const uint32_t* seeds, float* out, gg_run_stats* st) {
  const uint32_t n = g->n;
  const uint64_t nk = (uint64_t)n * (uint64_t)k;
  std::vector<uint32_t> brows;
  boundary_rows(g, brows);
  float *T = nullptr, *XS = nullptr, *S = nullptr, *Y = nullptr;
  uint32_t *d_brows = nullptr, *d_seeds = nullptr;
  auto cleanup = [&]() {
    cudaFreeAsync(d_seeds, g->stream);
    cudaFreeAsync(T, g->stream);
    cudaFreeAsync(XS, g->stream);
    cudaFreeAsync(S, g->stream);
    cudaFreeAsync(Y, g->stream);
    cudaFreeAsync(d_brows, g->stream);
  };
  struct Guard {
    std::function<void()> f;
    ~Guard() { f(); }
  } guard{cleanup};
  GG_CUDA(cudaMallocAsync((void**)&T, 4 * nk, g->stream));
  GG_CUDA(cudaMallocAsync((void**)&XS, 4 * nk, g->stream));
  GG_CUDA(cudaMallocAsync((void**)&S, 4 * nk, g->stream));
  GG_CUDA(cudaMallocAsync((void**)&Y, 4 * nk, g->stream));
  GG_CUDA(cudaMallocAsync((void**)&d_brows, 4 * (brows.size() + 1), g->stream));
  if (!brows.empty())
    GG_CUDA(cudaMemcpyAsync(d_brows, brows.data(), 4 * brows.size(), cudaMemcpyHostToDevice, g->stream));
  g->kernels = 0;
  cudaEvent_t ea, eb;
  cudaEventCreate(&ea);
  cudaEventCreate(&eb);
  cudaEventRecord(ea, g->stream);
  if (tele_host) {
    GG_CUDA(cudaMemcpyAsync(T, tele_host, 4 * nk, cudaMemcpyHostToDevice, g->stream));
  } else {
    GG_CUDA(cudaMallocAsync((void**)&d_seeds, 4 * k, g->stream));
    GG_CUDA(cudaMemcpyAsync(d_seeds, seeds, 4 * k, cudaMemcpyHostToDevice, g->stream));
    GG_CUDA(cudaMemsetAsync(T, 0, 4 * nk, g->stream));
    k_ppr_onehot<<<1, 64, 0, g->stream>>>(d_seeds, (uint32_t)k, T);
    g->kernels++;
  }
  const int grid = generic_grid(g, nk);
  k_ppr_init<<<grid, kGenericThreads, 0, g->stream>>>(n, (uint32_t)k, T, g->out_off(), XS);
  g->kernels++;
  const uint64_t nblocks = (g->m + kSegBlock - 1) / kSegBlock;
  const SegIndex& si = g->seg[g->transposed ? 1 : 0];
  const int pgrid = (int)std::min<uint64_t>((nblocks + 7) / 8, (uint64_t)g->num_sms * 16);
  gg_frontier_s* all = nullptr;
  if (k == 1) GG_TRY(gg_frontier_all(g, &all));
  struct AllGuard {
    gg_frontier_s* f;
    ~AllGuard() { frontier_free(f); }
  } all_guard{all};
  for (int32_t it = 0; it < iters && k == 1; ++it) {
    // one column: the engine's scalar dense pull (edgeMap with every source active)
    GG_CUDA(cudaMemsetAsync(S, 0, 4 * nk, g->stream));
    PrPosF f;
    f.contrib = XS;
    f.acc_out = S;
    gg_frontier_s* o = nullptr;
    GG_TRY(edge_map(g, all, f, (int64_t)g->m / 20, GG_EM_FORCE_CSC | GG_EM_FORCE_COO, &o));
    frontier_free(o);
    k_ppr_vertex<<<grid, kGenericThreads, 0, g->stream>>>(n, 1u, g->in_off(), g->out_off(), S, T, damping, Y, XS,
                                                         it == iters - 1);
    g->kernels++;
  }
  for (int32_t it = 0; it < iters && k > 1; ++it) {
    if (!brows.empty()) {
      k_zero_rows<<<generic_grid(g, (uint64_t)brows.size() * k), kGenericThreads, 0, g->stream>>>(
          d_brows, (uint32_t)brows.size(), S, (uint32_t)k);
      g->kernels++;
    }
    if (nblocks) {
      if (k == 64)
        k_ppr_pull<2><<<std::max(pgrid, 1), 256, 0, g->stream>>>(g->in_idx(), si.d_head, si.d_blk, si.d_rows,
                                                                  nblocks, g->m, XS, S, (uint32_t)k);
      else
        k_ppr_pull<1><<<std::max(pgrid, 1), 256, 0, g->stream>>>(g->in_idx(), si.d_head, si.d_blk, si.d_rows,
                                                                  nblocks, g->m, XS, S, (uint32_t)k);
      g->kernels++;
    }
    k_ppr_vertex<<<grid, kGenericThreads, 0, g->stream>>>(n, (uint32_t)k, g->in_off(), g->out_off(), S, T, damping,
                                                         Y, XS, it == iters - 1);
    g->kernels++;
  }
  if (iters == 0) GG_CUDA(cudaMemcpyAsync(Y, T, 4 * nk, cudaMemcpyDeviceToDevice, g->stream));
  GG_CUDA(cudaGetLastError());
  cudaEventRecord(eb, g->stream);
  GG_CUDA(cudaEventSynchronize(eb));
  float ms = 0;
  cudaEventElapsedTime(&ms, ea, eb);
  cudaEventDestroy(ea);
  cudaEventDestroy(eb);
  if (out) {
    GG_CUDA(cudaMemcpyAsync(out, Y, 4 * nk, cudaMemcpyDeviceToHost, g->stream));
    GG_CUDA(cudaStreamSynchronize(g->stream));
  }
  if (st) {
    st->ms = ms;
    st->rounds = iters;
    st->edges_traversed = g->m * (uint64_t)iters;
    st->kernels = g->kernels;
  }
  return GG_OK;
}

}  // namespace gg

using namespace gg;

extern "C" int gg_ppr_k(gg_graph_t g, int32_t k, int32_t iters, float damping, const float* tele,
                        const uint32_t* seeds, float* out, gg_run_stats* st) {
  if (!graph_live(g) || (k != 1 && k != 32 && k != 64) || iters < 0 || !(damping >= 0.f && damping <= 1.f) ||
      (!tele && !seeds))
    return fail(GG_ERR_INVALID_ARG, "gg_ppr_k: k must be 1, 32 or 64, iters >= 0, 0 <= damping <= 1, tele or seeds");
  if (!tele)
    for (int32_t j = 0; j < k; ++j)
      if (seeds[j] >= g->n) return fail(GG_ERR_INVALID_ARG, "gg_ppr_k: seed %u out of range", seeds[j]);
  return run_ppr_k(g, k, iters, damping, tele, seeds, out, st);
}
