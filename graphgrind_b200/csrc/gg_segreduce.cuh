// Row reductions over a segmented edge stream (CSC in-edges or CSR
// out-edges of the current orientation) with one lane per edge.
#pragma once
#include "gg_runtime.cuh"

namespace gg {

struct SegStream {
  const uint32_t* idx;
  const uint32_t* head;
  const uint32_t* blk;
  const uint32_t* rows;
  uint64_t nblocks, m;
};

__device__ __forceinline__ float seg_shfl_up(float v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
__device__ __forceinline__ float2 seg_shfl_up(float2 v, int d) {
  return make_float2(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d));
}
__device__ __forceinline__ float seg_shfl(float v, int l) { return __shfl_sync(0xffffffffu, v, l); }
__device__ __forceinline__ float2 seg_shfl(float2 v, int l) {
  return make_float2(__shfl_sync(0xffffffffu, v.x, l), __shfl_sync(0xffffffffu, v.y, l));
}

// For every row: op.flush(row, combine over the row's edges e of
// op.val(e, y, row), complete) with y the edge's other end.  One warp per
// 256-edge block, lane l takes edge 32 i + l; a segmented shuffle scan
// combines each row's lanes.  A row that lies inside the block is flushed
// once with complete = true; a row split across blocks is flushed once per
// block with complete = false (the op combines those atomically).
template <class Op>
__global__ void __launch_bounds__(256) k_seg_reduce(SegStream p, Op op) {
  using T = typename Op::T;
  __shared__ uint32_t s_row[8][kSegBlock + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lanemask_le = 0xffffffffu >> (31 - lane);
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t b = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp; b < p.nblocks; b += warps) {
    const uint64_t e0 = b * kSegBlock;
    // row of each slot: slot 0 continues from the previous block, one slot per head
    const uint32_t h0 = __ldg(p.blk + b), nr = __ldg(p.blk + b + 1) - h0 + 1;
    for (uint32_t i = lane; i < nr; i += 32) s_row[warp][i] = (i > 0 || h0 > 0) ? __ldg(p.rows + h0 - 1 + i) : 0u;
    __syncwarp();
    const uint64_t nb = e0 + kSegBlock;
    const bool ends_block = nb >= p.m || (__ldg(p.head + (nb >> 5)) & 1u);
    uint32_t running = 0;
    T carry = Op::identity();
    uint32_t hw = __ldg(p.head + b * 8);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const uint32_t hw_next = i < 7 ? __ldg(p.head + b * 8 + i + 1) : 0u;
      const uint64_t e = e0 + 32 * i + lane;
      const uint32_t rel = running + __popc(hw & lanemask_le);
      T v = Op::identity();
      if (e < p.m) v = op.val(e, Op::kNeedsIdx ? __ldg(p.idx + e) : 0u, s_row[warp][rel]);
      const uint32_t hb = hw & lanemask_le;
      const int seg0 = hb ? 31 - __clz(hb) : 0;
      if (lane == 0 && !(hw & 1u)) v = Op::combine(carry, v);
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const T t = seg_shfl_up(v, d);
        if (lane >= seg0 + d) v = Op::combine(t, v);
      }
      const bool ends = lane < 31 ? ((hw >> (lane + 1)) & 1u) : (i < 7 ? (hw_next & 1u) : ends_block);
      if ((ends || (lane == 31 && i == 7)) && (rel > 0 || h0 > 0)) op.flush(s_row[warp][rel], v, rel > 0 && ends);
      const T v31 = seg_shfl(v, 31);
      carry = (i < 7 && !(hw_next & 1u)) ? v31 : Op::identity();
      running += __popc(hw);
      hw = hw_next;
    }
    __syncwarp();
  }
}

template <class Op>
inline int seg_reduce(gg_graph_s* g, bool in_edges, Op op) {
  if (g->m == 0) return GG_OK;
  const int seg = g->symmetric ? 0 : ((in_edges != g->transposed) ? 0 : 1);
  const SegIndex& si = g->seg[seg];
  SegStream p{in_edges ? g->in_idx() : g->out_idx(), si.d_head, si.d_blk, si.d_rows,
              (g->m + kSegBlock - 1) / kSegBlock, g->m};
  const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>((p.nblocks + 7) / 8, (uint64_t)g->num_sms * 8));
  k_seg_reduce<Op><<<grid, 256, 0, g->stream>>>(p, op);
  g->kernels++;
  GG_CUDA(cudaGetLastError());
  return GG_OK;
}

}  // namespace gg
