// Batched traversals: k-column personalised PageRank as one SpMM-shaped pull
// per iteration (every edge moves a whole 64- or 32-column row of the source
// contributions instead of one 4-byte value).
//
//   X_0 = T,  X_{t+1} = d * A X_t + (1 - d) * T,  A[v,u] = 1/outdeg(u) for u->v
//
// the personalised form of PR_F / PR_Vertex_F (app/PageRank.C:28-87) with a
// teleport matrix T (n x k, row-major) in place of the uniform 1/n, all
// vertices active (PageRankBit, app/PageRankBit.C:145).
#include <cub/cub.cuh>

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
  GG_CUDA(pool_alloc((void**)&T, 4 * nk, g->stream, g->device));
  GG_CUDA(pool_alloc((void**)&XS, 4 * nk, g->stream, g->device));
  GG_CUDA(pool_alloc((void**)&S, 4 * nk, g->stream, g->device));
  GG_CUDA(pool_alloc((void**)&Y, 4 * nk, g->stream, g->device));
  GG_CUDA(pool_alloc((void**)&d_brows, 4 * (brows.size() + 1), g->stream, g->device));
  if (!brows.empty())
    GG_CUDA(cudaMemcpyAsync(d_brows, brows.data(), 4 * brows.size(), cudaMemcpyHostToDevice, g->stream));
  g->kernels = 0;
  struct EvHold {
    cudaEvent_t a = nullptr, b = nullptr;
    ~EvHold() {
      if (a) cudaEventDestroy(a);
      if (b) cudaEventDestroy(b);
    }
  } ev;
  cudaEventCreate(&ev.a);
  cudaEventCreate(&ev.b);
  cudaEvent_t ea = ev.a, eb = ev.b;
  // inputs are uploaded before the timed region (a renumbered graph's teleport
  // rows go through Y, which is written only later)
  if (tele_host) {
    GG_CUDA(cudaMemcpyAsync(g->relabeled ? Y : T, tele_host, 4 * nk, cudaMemcpyHostToDevice, g->stream));
    cudaEventRecord(ea, g->stream);
    if (g->relabeled) GG_TRY(device_order<float>(g, Y, (uint32_t)k, T));
  } else {
    std::vector<uint32_t> dev_seeds(seeds, seeds + k);
    for (auto& v : dev_seeds) v = g->device_id(v);
    GG_CUDA(pool_alloc((void**)&d_seeds, 4 * k, g->stream, g->device));
    GG_CUDA(cudaMemcpyAsync(d_seeds, dev_seeds.data(), 4 * k, cudaMemcpyHostToDevice, g->stream));
    GG_CUDA(cudaStreamSynchronize(g->stream));  // dev_seeds leaves scope
    cudaEventRecord(ea, g->stream);
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
  DevBuf<float> ty;
  const float* res = Y;
  GG_TRY(given_order<float>(g, Y, (uint32_t)k, ty, &res));
  GG_CUDA(cudaGetLastError());
  cudaEventRecord(eb, g->stream);
  GG_CUDA(cudaEventSynchronize(eb));
  float ms = 0;
  cudaEventElapsedTime(&ms, ea, eb);
  if (out) {
    GG_CUDA(cudaMemcpyAsync(out, res, 4 * nk, cudaMemcpyDeviceToHost, g->stream));
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


// ------------------------------------------------------------------ multi-source
// k <= 64 sources share one level-synchronous traversal.  Per vertex, bit j of
// a 64-bit mask says "reached from sources[j]"; per (vertex, source) values
// (levels, path counts, dependencies) are n x 64 row-major.
//
// Row pull over a segmented edge stream (CSC for the forward levels, CSR for
// the backward dependency pass): for each row x and edge (x, y) of the row,
//   b = filter(x) & edge_mask(y)
//   out[x] |= b                        (the next frontier's masks, forward)
//   vals[x][j] += vals[y][j] for j in b  (path counts or dependencies)
// filter(x) = ~seen[x] forward and the level-r mask backward.  One warp per
// 256-edge block; lane l owns columns 2l, 2l+1.  (x, j) pairs written and
// (y, j) pairs read are disjoint in both passes (unreached vs frontier,
// level r vs level r+1), so the pass updates vals in place.
struct MsPull {
  const uint32_t* idx;
  const uint32_t* head;
  const uint32_t* blk;
  const uint32_t* rows;
  uint64_t nblocks, m;
  const uint64_t* row_mask;
  uint64_t row_xor, kmask;
  const uint64_t* edge_mask;
  float* vals;
  uint64_t* out;
};

#ifndef GG_MS_MIN_BLOCKS
#define GG_MS_MIN_BLOCKS 3  // resident CTAs per SM the register allocation must allow (3: fastest measured)
#endif
// Dynamic shared memory per CTA (8 warps): row filters and rows of the block,
// and for VALS the active edges' masks, sources and row slots.
template <bool VALS>
constexpr size_t ms_pull_smem() {
  return 8 * (kSegBlock + 1) * (8 + 4) + (VALS ? 8 * kSegBlock * (8 + 4 + 2) : 0);
}

template <bool VALS, bool OUT>
__global__ void __launch_bounds__(256, GG_MS_MIN_BLOCKS) k_ms_pull(MsPull p) {
  extern __shared__ __align__(16) unsigned char ms_smem[];
  auto s_filt = reinterpret_cast<uint64_t(*)[kSegBlock + 1]>(ms_smem);
  auto s_em = reinterpret_cast<uint64_t(*)[kSegBlock]>(ms_smem + 8 * (kSegBlock + 1) * 8);
  auto s_row = reinterpret_cast<uint32_t(*)[kSegBlock + 1]>(ms_smem + 8 * (kSegBlock + 1) * 8 +
                                                            (VALS ? 8 * kSegBlock * 8 : 0));
  auto s_src = reinterpret_cast<uint32_t(*)[kSegBlock]>(reinterpret_cast<unsigned char*>(s_row) +
                                                        8 * (kSegBlock + 1) * 4);
  auto s_rel = reinterpret_cast<uint16_t(*)[kSegBlock]>(reinterpret_cast<unsigned char*>(s_src) +
                                                        (VALS ? 8 * kSegBlock * 4 : 0));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lanemask_le = 0xffffffffu >> (31 - lane);
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t b = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp; b < p.nblocks; b += warps) {
    const uint64_t e0 = b * kSegBlock;
    // rows touching the block: slot 0 continues from the previous block, one slot per head
    const uint32_t h0 = __ldg(p.blk + b), nr = __ldg(p.blk + b + 1) - h0 + 1;
    bool live = false;  // some row of the block still takes bits
    for (uint32_t i = lane; i < nr; i += 32) {
      uint64_t f = 0;
      uint32_t x = 0;
      if (i > 0 || h0 > 0) {
        x = __ldg(p.rows + h0 - 1 + i);
        f = (__ldg(p.row_mask + x) ^ p.row_xor) & p.kmask;
      }
      s_row[warp][i] = x;
      s_filt[warp][i] = f;
      live = live || f != 0;
    }
    // every row filtered out (forward: reached from all sources): no edge of
    // the block can set a bit or move a value
    if (!__any_sync(0xffffffffu, live)) continue;
    __syncwarp();
    const uint64_t nb = e0 + kSegBlock;
    const bool ends_block = nb >= p.m || (__ldg(p.head + (nb >> 5)) & 1u);
    // mask phase: lane l takes edge 32 i + l of the block
    uint32_t running = 0, act[8];
    uint64_t carry = 0;
    uint32_t hw = __ldg(p.head + b * 8);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const uint32_t hw_next = i < 7 ? __ldg(p.head + b * 8 + i + 1) : 0u;
      const uint64_t e = e0 + 32 * i + lane;
      const uint32_t rel = running + __popc(hw & lanemask_le);
      const uint64_t f = s_filt[warp][rel];
      const uint32_t y = (e < p.m && f) ? __ldg(p.idx + e) : 0u;  // edges of filtered rows are not read
      uint64_t x = (e < p.m && f) ? (__ldg(p.edge_mask + y) & f) : 0ull;
      if (VALS) {
        s_em[warp][32 * i + lane] = x;
        s_src[warp][32 * i + lane] = y;
        s_rel[warp][32 * i + lane] = (uint16_t)rel;
        act[i] = __ballot_sync(0xffffffffu, x != 0);
      }
      if (OUT) {
        // segmented inclusive OR over the lanes of each row
        const uint32_t hb = hw & lanemask_le;
        const int seg0 = hb ? 31 - __clz(hb) : 0;
        if (lane == 0 && !(hw & 1u)) x |= carry;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const uint64_t t = __shfl_up_sync(0xffffffffu, x, d);
          if (lane >= seg0 + d) x |= t;
        }
        const bool ends = lane < 31 ? ((hw >> (lane + 1)) & 1u) : (i < 7 ? (hw_next & 1u) : ends_block);
        if ((ends || (lane == 31 && i == 7)) && x) {
          const uint32_t row = s_row[warp][rel];
          if (rel > 0 && ends)
            p.out[row] = x;
          else
            atomicOr(reinterpret_cast<unsigned long long*>(p.out + row), (unsigned long long)x);
        }
        const uint64_t x31 = __shfl_sync(0xffffffffu, x, 31);
        carry = (i < 7 && !(hw_next & 1u)) ? x31 : 0ull;
      }
      running += __popc(hw);
      hw = hw_next;
    }
    if (VALS) {
      __syncwarp();
      // column phase over the active edges in edge order; lane l owns columns 2l, 2l+1
      uint32_t cur = 0xffffffffu;
      uint64_t rm = 0;
      float a0 = 0.f, a1 = 0.f;
      auto flush = [&]() {
        if (cur == 0xffffffffu || rm == 0) return;
        const bool complete = cur > 0 && (cur < nr - 1 || ends_block);
        const uint32_t mb = (uint32_t)(rm >> (2 * lane)) & 3u;
        float* dst = p.vals + (uint64_t)s_row[warp][cur] * 64 + 2 * lane;
        if (complete) {
          if (mb & 1u) dst[0] += a0;
          if (mb & 2u) dst[1] += a1;
        } else {
          if (mb & 1u) atomicAdd(dst, a0);
          if (mb & 2u) atomicAdd(dst + 1, a1);
        }
      };
      int i = 0;
      uint32_t bits = act[0];
      while (true) {
        // next batch of up to 8 active edges
        uint32_t el[8];
        int cnt = 0;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          while (bits == 0 && i < 7) bits = act[++i];
          el[q] = 0xffffffffu;
          if (bits) {
            el[q] = 32 * i + __ffs(bits) - 1;
            bits &= bits - 1;
            ++cnt;
          }
        }
        if (cnt == 0) break;
        float2 v[8];
        uint64_t em[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          v[q] = make_float2(0.f, 0.f);
          em[q] = 0;
          if (el[q] != 0xffffffffu) {
            em[q] = s_em[warp][el[q]];
            if ((uint32_t)(em[q] >> (2 * lane)) & 3u)
              v[q] = __ldg(reinterpret_cast<const float2*>(p.vals + (uint64_t)s_src[warp][el[q]] * 64) + lane);
          }
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          if (el[q] == 0xffffffffu) break;
          const uint32_t rel = s_rel[warp][el[q]];
          if (rel != cur) {
            flush();
            cur = rel;
            rm = 0;
            a0 = a1 = 0.f;
          }
          rm |= em[q];
          const uint32_t mb = (uint32_t)(em[q] >> (2 * lane)) & 3u;
          if (mb & 1u) a0 += v[q].x;
          if (mb & 2u) a1 += v[q].y;
        }
      }
      flush();
    }
    __syncwarp();
  }
}

// Sources: seen = visit = bit j at sources[j], level 0, one path.  Levels
// go straight to out_lv (n x k, given rows: old_of_new[v], or v when the
// graph keeps its ids), when given.
__global__ void k_ms_seed(const uint32_t* src, uint32_t k, uint64_t* seen, uint64_t* visit, int32_t* out_lv,
                          const uint32_t* old_of_new, float* sigma) {
  const uint32_t j = threadIdx.x;
  if (j >= k) return;
  const uint32_t s = src[j];
  atomicOr(reinterpret_cast<unsigned long long*>(seen + s), 1ull << j);
  atomicOr(reinterpret_cast<unsigned long long*>(visit + s), 1ull << j);
  if (out_lv) out_lv[(uint64_t)(old_of_new ? old_of_new[s] : s) * k + j] = 0;
  if (sigma) sigma[(uint64_t)s * 64 + j] = 1.f;
}

// After a forward level r: the new frontier masks become visit and join
// seen; the frontier's vertices are appended to queue (with their
// out-degrees in qdeg, and for BC their new masks in qmask) for a push of the
// next level and for the backward pass; the levels of the new
// (vertex, source) pairs are written by the whole warp, one vertex at a time
// with lanes over sources (whole-row stores).  stats[0] = frontier vertices
// (the queue length), stats[1] += sum of out-degree x sources over it,
// stats[2] += sum of out-degree (the edges a push expands).
__global__ void k_ms_fwd_vertex(uint32_t n, int32_t r, uint64_t* seen, uint64_t* visit, uint64_t* next,
                                int32_t* out_lv, uint32_t out_k, const uint32_t* old_of_new, const uint32_t* out_off,
                                uint32_t* queue, uint32_t* qdeg, uint64_t* qmask, unsigned long long* stats) {
  const int lane = threadIdx.x & 31;
  const uint64_t w0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long trav = 0, edges = 0;
  for (uint64_t base = w0 * 32; base < n; base += nw * 32) {
    const uint64_t v = base + lane;
    uint64_t nm = 0;
    uint32_t d = 0;
    if (v < n) {
      nm = next[v];
      visit[v] = nm;
      if (nm) {
        next[v] = 0;
        seen[v] |= nm;
        d = out_off[v + 1] - out_off[v];
        trav += (unsigned long long)d * __popcll(nm);
        edges += d;
      }
    }
    uint32_t act = __ballot_sync(0xffffffffu, nm != 0);
    if (!act) continue;
    uint32_t pos = 0;
    if (lane == 0) pos = (uint32_t)atomicAdd(stats, (unsigned long long)__popc(act));
    pos = __shfl_sync(0xffffffffu, pos, 0) + __popc(act & ((1u << lane) - 1u));
    if (nm) {
      queue[pos] = (uint32_t)v;
      qdeg[pos] = d;
      if (qmask) qmask[pos] = nm;
    }
    while (act) {
      const int b = __ffs(act) - 1;
      act &= act - 1;
      const uint64_t vv = base + b;
      const uint64_t mm = __shfl_sync(0xffffffffu, nm, b);
      const bool lo = (mm >> lane) & 1u, hi = (mm >> (lane + 32)) & 1u;
      if (out_lv) {
        const uint64_t row = (uint64_t)(old_of_new ? old_of_new[vv] : vv) * out_k;
        if (lo) out_lv[row + lane] = r;
        if (hi) out_lv[row + 32 + lane] = r;
      }
    }
  }
  trav = warp_sum(trav);
  edges = warp_sum(edges);
  if (lane == 0 && (trav | edges)) {
    atomicAdd(stats + 1, trav);
    atomicAdd(stats + 2, edges);
  }
}

// Push of a sparse forward level (the frontier's out-edges are few): one
// thread per frontier edge, load-balanced through the exclusive degree sums
// qoff of the frontier queue; each edge (u, v) ORs the sources reaching u
// for the first time at v into next[v], and for BC adds u's path counts of
// those sources to v's.  The pairs (v, j) written are unreached ones, the
// (u, j) read are frontier ones, so sigma is updated in place.
__global__ void k_ms_push(const uint32_t* queue, const uint32_t* qoff, uint32_t nq, uint64_t edges,
                          const uint32_t* out_off, const uint32_t* out_idx, const uint64_t* visit,
                          const uint64_t* seen, uint64_t kmask, uint64_t* next, float* sigma) {
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < edges;
       t += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = nq - 1;  // the last queue entry whose first edge is <= t
    while (lo < hi) {
      const uint32_t mid = lo + (hi - lo + 1) / 2;
      if (qoff[mid] <= t)
        lo = mid;
      else
        hi = mid - 1;
    }
    const uint32_t u = queue[lo];
    const uint32_t v = out_idx[out_off[u] + (uint32_t)(t - qoff[lo])];
    uint64_t m = visit[u] & ~seen[v] & kmask;
    if (!m) continue;
    atomicOr(reinterpret_cast<unsigned long long*>(next + v), (unsigned long long)m);
    if (sigma) {
      while (m) {
        const int j = __ffsll((long long)m) - 1;
        m &= m - 1;
        atomicAdd(sigma + (uint64_t)v * 64 + j, sigma[(uint64_t)u * 64 + j]);
      }
    }
  }
}

// Backward level r from the level's vertex list (recorded by the forward
// pass): mask[v] = the sources with level r at v and dep[v][j] = 1/paths[v][j]
// there (BC_Back_Vertex_F, app/BC.C:142-154).  One warp per listed vertex.
__global__ void k_ms_level_seed(const uint32_t* list, const uint64_t* masks, uint32_t cnt, uint64_t* mask,
                                const float* sigma, float* dep) {
  const int lane = threadIdx.x & 31;
  const uint64_t w0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t i = w0; i < cnt; i += nw) {
    const uint64_t v = list[i];
    const uint64_t mk = masks[i];
    if (lane == 0) mask[v] = mk;
    if ((mk >> lane) & 1u) dep[v * 64 + lane] = 1.f / sigma[v * 64 + lane];
    if ((mk >> (lane + 32)) & 1u) dep[v * 64 + 32 + lane] = 1.f / sigma[v * 64 + 32 + lane];
  }
}

// Backward step of a sparse level: one thread per out-edge (x, y) of the
// level-r vertices (load-balanced through the exclusive degree sums qoff of
// the list); dep[x][j] += dep[y][j] for the sources j at level r at x and
// r + 1 at y.  The pairs written (level r) and read (level r + 1) differ.
__global__ void k_ms_back_edges(const uint32_t* list, const uint32_t* qoff, uint32_t cnt, uint64_t edges,
                                const uint32_t* out_off, const uint32_t* out_idx, const uint64_t* cur,
                                const uint64_t* prev, float* dep) {
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < edges;
       t += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = cnt - 1;  // the last list entry whose first edge is <= t
    while (lo < hi) {
      const uint32_t mid = lo + (hi - lo + 1) / 2;
      if (qoff[mid] <= t)
        lo = mid;
      else
        hi = mid - 1;
    }
    const uint32_t x = list[lo];
    const uint32_t y = out_idx[out_off[x] + (uint32_t)(t - qoff[lo])];
    uint64_t b = cur[x] & prev[y];
    while (b) {
      const int j = __ffsll((long long)b) - 1;
      b &= b - 1;
      atomicAdd(dep + (uint64_t)x * 64 + j, dep[(uint64_t)y * 64 + j]);
    }
  }
}

// (dep - 1/paths) / (1/paths), app/BC.C:220-222, into n x k outputs; NaN where unreached.
// Output rows in the given vertex order: row u of the output is device row
// new_of_old[u] (u itself when the graph keeps its given ids).
__global__ void k_ms_bc_final(uint32_t n, uint32_t k, const uint32_t* new_of_old, const float* dep,
                              const float* sigma, float* dep_out, float* sigma_out) {
  const uint64_t total = (uint64_t)n * k;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t u = i / k, j = i % k;
    const uint64_t v = new_of_old ? new_of_old[u] : u;
    const float inv = 1.0f / sigma[v * 64 + j];
    dep_out[i] = (dep[v * 64 + j] - inv) / inv;
    if (sigma_out) sigma_out[i] = sigma[v * 64 + j];
  }
}

// Device allocations released (stream-ordered) when the holder leaves scope.
struct DevAllocs {
  cudaStream_t st;
  int device;
  std::vector<void*> ptrs;
  DevAllocs(cudaStream_t s, int dev) : st(s), device(dev) {}
  template <class T>
  int get(T** p, uint64_t count) {
    *p = nullptr;
    GG_CUDA(pool_alloc((void**)p, sizeof(T) * count + 64, st, device));
    ptrs.push_back(*p);
    return GG_OK;
  }
  ~DevAllocs() {
    for (void* q : ptrs) cudaFreeAsync(q, st);
  }
};

static int ms_pull(gg_graph_s* g, bool vals, bool out, bool forward, const uint64_t* row_mask, uint64_t row_xor,
                   uint64_t kmask, const uint64_t* edge_mask, float* v, uint64_t* o) {
  if (g->m == 0) return GG_OK;
  MsPull p{};
  // forward pulls in-edges, backward pulls out-edges of the current orientation
  const bool in_edges = forward;
  const int seg = g->symmetric ? 0 : ((in_edges != g->transposed) ? 0 : 1);
  const SegIndex& si = g->seg[seg];
  p.idx = in_edges ? g->in_idx() : g->out_idx();
  p.head = si.d_head;
  p.blk = si.d_blk;
  p.rows = si.d_rows;
  p.nblocks = (g->m + kSegBlock - 1) / kSegBlock;
  p.m = g->m;
  p.row_mask = row_mask;
  p.row_xor = row_xor;
  p.kmask = kmask;
  p.edge_mask = edge_mask;
  p.vals = v;
  p.out = o;
  const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((p.nblocks + 7) / 8, (uint64_t)g->num_sms * 8));
  static DeviceOnce opted;
  const int ok = opted.get(g->device, []() {
    const bool a = cudaFuncSetAttribute(k_ms_pull<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)ms_pull_smem<true>()) == cudaSuccess;
    const bool b = cudaFuncSetAttribute(k_ms_pull<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)ms_pull_smem<true>()) == cudaSuccess;
    return a && b ? 1 : -1;
  });
  if (ok < 0) return fail(GG_ERR_CUDA, "cudaFuncSetAttribute failed for the multi-source pull");
  if (vals && out)
    k_ms_pull<true, true><<<grid, 256, ms_pull_smem<true>(), g->stream>>>(p);
  else if (vals)
    k_ms_pull<true, false><<<grid, 256, ms_pull_smem<true>(), g->stream>>>(p);
  else
    k_ms_pull<false, true><<<grid, 256, ms_pull_smem<false>(), g->stream>>>(p);
  g->kernels++;
  return GG_OK;
}

static int run_ms(gg_graph_s* g, int32_t k, const uint32_t* given_sources, bool bc, int32_t* levels_out,
                  float* dep_out, float* np_out, gg_run_stats* st) {
  const uint32_t n = g->n;
  std::vector<uint32_t> dev_sources(given_sources, given_sources + k);
  for (auto& v : dev_sources) v = g->device_id(v);
  const uint32_t* sources = dev_sources.data();
  const uint64_t n64 = (uint64_t)n * 64;
  const uint64_t nk = (uint64_t)n * k;
  const uint64_t kmask = k == 64 ? ~0ull : ((1ull << k) - 1);
  DevAllocs mem(g->stream, g->device);
  uint64_t *seen, *visit, *next, *mask_a, *mask_b, *qmask = nullptr;
  float *sigma = nullptr, *dep = nullptr;
  uint32_t *d_src, *queue, *qdeg, *qoff;
  unsigned char* scan_tmp;
  unsigned long long* d_stats;
  GG_TRY(mem.get(&seen, n));
  GG_TRY(mem.get(&visit, n));
  GG_TRY(mem.get(&next, n));
  GG_TRY(mem.get(&d_src, 64));
  GG_TRY(mem.get(&d_stats, 4));
  GG_TRY(mem.get(&queue, n));
  GG_TRY(mem.get(&qdeg, n));
  GG_TRY(mem.get(&qoff, n));
  size_t scan_bytes = 0;
  GG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, qdeg, qoff, (int)n, g->stream));
  GG_TRY(mem.get(&scan_tmp, scan_bytes));
  if (bc) {
    GG_TRY(mem.get(&sigma, n64));
    GG_TRY(mem.get(&dep, n64));
    GG_TRY(mem.get(&qmask, n));
  }
  // multi-source BFS writes its levels straight into the n x k output
  DevBuf<int32_t> lout;
  int32_t* out_lv = nullptr;
  if (!bc && levels_out) {
    GG_TRY(lout.alloc(g, nk));
    out_lv = lout.p;
  }
  const uint32_t* old_of_new = g->relabeled ? g->d_old_of_new : nullptr;
  // the first frontier: the distinct sources, with their first-edge offsets
  std::vector<uint32_t> uq(sources, sources + k);
  std::sort(uq.begin(), uq.end());
  uq.erase(std::unique(uq.begin(), uq.end()), uq.end());
  std::vector<uint32_t> uoff(uq.size());
  uint64_t f_edges = 0;
  for (size_t i = 0; i < uq.size(); ++i) {
    uoff[i] = (uint32_t)f_edges;
    f_edges += g->h_out_off()[uq[i] + 1] - g->h_out_off()[uq[i]];
  }
  uint64_t f_cnt = uq.size();
  // BC: every level's vertices, their level masks and out-degrees, for the
  // backward pass (level 0: the distinct sources)
  std::vector<uint32_t*> r_list, r_deg;
  std::vector<uint64_t*> r_mask;
  std::vector<uint64_t> r_cnt, r_edges;
  std::vector<uint64_t> umask(uq.size(), 0);
  std::vector<uint32_t> udeg(uq.size());
  for (size_t i = 0; i < uq.size(); ++i) {
    udeg[i] = g->h_out_off()[uq[i] + 1] - g->h_out_off()[uq[i]];
    for (int32_t j = 0; j < k; ++j)
      if (sources[j] == uq[i]) umask[i] |= 1ull << j;
  }
  unsigned long long* h_stats = reinterpret_cast<unsigned long long*>(g->ws.h_red);
  g->kernels = 0;
  EventTimer tm(g->stream);
  GG_CUDA(cudaMemcpyAsync(d_src, sources, 4 * k, cudaMemcpyHostToDevice, g->stream));
  GG_CUDA(cudaMemcpyAsync(queue, uq.data(), 4 * uq.size(), cudaMemcpyHostToDevice, g->stream));
  GG_CUDA(cudaMemcpyAsync(qoff, uoff.data(), 4 * uoff.size(), cudaMemcpyHostToDevice, g->stream));
  GG_CUDA(cudaMemsetAsync(seen, 0, 8 * (uint64_t)n, g->stream));
  GG_CUDA(cudaMemsetAsync(visit, 0, 8 * (uint64_t)n, g->stream));
  GG_CUDA(cudaMemsetAsync(next, 0, 8 * (uint64_t)n, g->stream));
  if (out_lv) GG_CUDA(cudaMemsetAsync(out_lv, 0xff, 4 * nk, g->stream));
  if (bc) {
    GG_CUDA(cudaMemsetAsync(sigma, 0, 4 * n64, g->stream));
    uint32_t *l0, *d0;
    uint64_t* m0;
    GG_TRY(mem.get(&l0, uq.size()));
    GG_TRY(mem.get(&d0, uq.size()));
    GG_TRY(mem.get(&m0, uq.size()));
    GG_CUDA(cudaMemcpyAsync(l0, uq.data(), 4 * uq.size(), cudaMemcpyHostToDevice, g->stream));
    GG_CUDA(cudaMemcpyAsync(d0, udeg.data(), 4 * uq.size(), cudaMemcpyHostToDevice, g->stream));
    GG_CUDA(cudaMemcpyAsync(m0, umask.data(), 8 * uq.size(), cudaMemcpyHostToDevice, g->stream));
    r_list.push_back(l0);
    r_deg.push_back(d0);
    r_mask.push_back(m0);
    r_cnt.push_back(uq.size());
    r_edges.push_back(f_edges);
  }
  k_ms_seed<<<1, 64, 0, g->stream>>>(d_src, (uint32_t)k, seen, visit, out_lv, old_of_new, sigma);
  g->kernels++;
  uint64_t trav = 0;
  for (int32_t j = 0; j < k; ++j) trav += g->h_out_off()[sources[j] + 1] - g->h_out_off()[sources[j]];
  std::vector<uint64_t> level_trav{trav};
  int32_t L = 0;
  const int vgrid = generic_grid(g, n);
  const int64_t thr = app_threshold(g);
  for (int32_t r = 1;; ++r) {
    // edgeMap's direction rule on the frontier (vertices + out-edges against
    // m / 20): a sparse frontier pushes its out-edges, a dense one is pulled
    if ((int64_t)(f_cnt + f_edges) <= thr) {
      if (f_edges > 0) {
        k_ms_push<<<generic_grid(g, f_edges), kGenericThreads, 0, g->stream>>>(
            queue, qoff, (uint32_t)f_cnt, f_edges, g->out_off(), g->out_idx(), visit, seen, kmask, next, sigma);
        g->kernels++;
      }
    } else {
      GG_TRY(ms_pull(g, bc, true, true, seen, ~0ull, kmask, visit, sigma, next));
    }
    GG_CUDA(cudaMemsetAsync(d_stats, 0, 32, g->stream));
    k_ms_fwd_vertex<<<vgrid, kGenericThreads, 0, g->stream>>>(n, r, seen, visit, next, out_lv, (uint32_t)k,
                                                              old_of_new, g->out_off(), queue, qdeg, qmask, d_stats);
    g->kernels++;
    GG_CUDA(cudaMemcpyAsync(h_stats, d_stats, 24, cudaMemcpyDeviceToHost, g->stream));
    GG_CUDA(cudaStreamSynchronize(g->stream));
    if (h_stats[0] == 0) break;
    L = r;
    level_trav.push_back(h_stats[1]);
    trav += h_stats[1];
    f_cnt = h_stats[0];
    f_edges = h_stats[2];
    if (bc) {  // keep this level's vertex list for the backward pass
      uint32_t *lr, *dr;
      uint64_t* mr;
      GG_TRY(mem.get(&lr, f_cnt));
      GG_TRY(mem.get(&dr, f_cnt));
      GG_TRY(mem.get(&mr, f_cnt));
      GG_CUDA(cudaMemcpyAsync(lr, queue, 4 * f_cnt, cudaMemcpyDeviceToDevice, g->stream));
      GG_CUDA(cudaMemcpyAsync(dr, qdeg, 4 * f_cnt, cudaMemcpyDeviceToDevice, g->stream));
      GG_CUDA(cudaMemcpyAsync(mr, qmask, 8 * f_cnt, cudaMemcpyDeviceToDevice, g->stream));
      r_list.push_back(lr);
      r_deg.push_back(dr);
      r_mask.push_back(mr);
      r_cnt.push_back(f_cnt);
      r_edges.push_back(f_edges);
    }
    if ((int64_t)(f_cnt + f_edges) <= thr && f_edges > 0) {
      GG_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, qdeg, qoff, (int)f_cnt, g->stream));
    }
  }
  if (bc) {
    GG_TRY(mem.get(&mask_a, n));
    GG_TRY(mem.get(&mask_b, n));
    GG_CUDA(cudaMemsetAsync(mask_b, 0, 8 * (uint64_t)n, g->stream));
    GG_CUDA(cudaMemsetAsync(dep, 0, 4 * n64, g->stream));
    uint64_t *cur = mask_a, *prev = mask_b;
    for (int32_t r = L; r >= 0; --r) {
      // cur = the level-r masks (zero elsewhere), dep seeded with 1/paths there
      GG_CUDA(cudaMemsetAsync(cur, 0, 8 * (uint64_t)n, g->stream));
      k_ms_level_seed<<<generic_grid(g, r_cnt[r] * 32), kGenericThreads, 0, g->stream>>>(r_list[r], r_mask[r],
                                                                                         (uint32_t)r_cnt[r], cur,
                                                                                         sigma, dep);
      g->kernels++;
      if (r < L) {
        if ((int64_t)(r_cnt[r] + r_edges[r]) <= thr) {  // few edges leave level r: walk only them
          if (r_edges[r] > 0) {
            GG_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, r_deg[r], qoff, (int)r_cnt[r], g->stream));
            k_ms_back_edges<<<generic_grid(g, r_edges[r]), kGenericThreads, 0, g->stream>>>(
                r_list[r], qoff, (uint32_t)r_cnt[r], r_edges[r], g->out_off(), g->out_idx(), cur, prev, dep);
            g->kernels++;
          }
        } else {
          GG_TRY(ms_pull(g, true, false, false, cur, 0, kmask, prev, dep, nullptr));
        }
        trav += level_trav[r + 1];
      }
      std::swap(cur, prev);
    }
  }
  DevBuf<float> dout, sout;
  if (bc) {
    GG_TRY(dout.alloc(g, nk));
    if (np_out) GG_TRY(sout.alloc(g, nk));
    k_ms_bc_final<<<generic_grid(g, nk), kGenericThreads, 0, g->stream>>>(
        n, (uint32_t)k, g->relabeled ? g->d_new_of_old : nullptr, dep, sigma, dout.p, np_out ? sout.p : nullptr);
    g->kernels++;
  }
  GG_CUDA(cudaGetLastError());
  const double ms = tm.stop();
  if (bc) {
    GG_CUDA(cudaMemcpyAsync(dep_out, dout.p, 4 * nk, cudaMemcpyDeviceToHost, g->stream));
    if (np_out) GG_CUDA(cudaMemcpyAsync(np_out, sout.p, 4 * nk, cudaMemcpyDeviceToHost, g->stream));
  } else if (levels_out) {
    GG_CUDA(cudaMemcpyAsync(levels_out, lout.p, 4 * nk, cudaMemcpyDeviceToHost, g->stream));
  }
  GG_CUDA(cudaStreamSynchronize(g->stream));
  if (st) {
    st->ms = ms;
    st->rounds = L + 1;
    st->edges_traversed = trav;
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

static int check_sources(gg_graph_t g, int32_t k, const uint32_t* sources, const char* who) {
  if (!graph_live(g) || k < 1 || k > 64 || !sources) return fail(GG_ERR_INVALID_ARG, "%s: 1 <= k <= 64 sources", who);
  for (int32_t j = 0; j < k; ++j)
    if (sources[j] >= g->n) return fail(GG_ERR_INVALID_ARG, "%s: source %u out of range", who, sources[j]);
  return GG_OK;
}

extern "C" int gg_msbfs(gg_graph_t g, int32_t k, const uint32_t* sources, int32_t* levels, gg_run_stats* st) {
  GG_TRY(check_sources(g, k, sources, "gg_msbfs"));
  return run_ms(g, k, sources, false, levels, nullptr, nullptr, st);
}

extern "C" int gg_msbc(gg_graph_t g, int32_t k, const uint32_t* sources, float* dependencies, float* num_paths,
                       gg_run_stats* st) {
  GG_TRY(check_sources(g, k, sources, "gg_msbc"));
  if (!dependencies) return fail(GG_ERR_INVALID_ARG, "gg_msbc: null dependencies");
  return run_ms(g, k, sources, true, nullptr, dependencies, num_paths, st);
}
