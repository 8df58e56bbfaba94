// Loopy belief propagation, the Compute() loop of app/BP.C:152-212 with
// inputs the library defines (app/BP.C leaves the potentials and products
// uninitialised, indexes edge slots by offsets[s] + in-list position on its
// CSC path and by offsets[d] + 1 on its COO path, and resets products with a
// shadowed index, :136-149).  Here every edge e (its in-edge slot in the
// current orientation) holds a 2x2 potential, every vertex a 2-state
// potential, and per iteration, with products reset to 1:
//   belief_e[i]  = sum_k vert_pot[d][k] * edge_pot[e][i][k] * prod_cur[d][k]
//   prod_next[d][i] = product over d's in-edges e of belief_e[i]
// (BP_F::update, app/BP.C:80-94, which reads only the destination's data).
#include "gg_segreduce.cuh"

namespace gg {

__device__ __forceinline__ void atomic_mul(float* a, float b) {
  unsigned* p = reinterpret_cast<unsigned*>(a);
  unsigned old = *p, assumed;
  do {  // a compare-and-swap retry: ends once no other block changed the word in between
    assumed = old;
    old = atomicCAS(p, assumed, __float_as_uint(__uint_as_float(assumed) * b));
  } while (old != assumed);
}

struct BpOp {
  using T = float2;
  static constexpr bool kNeedsIdx = false;
  const float2* vp;   // [n] vertex potentials
  const float4* ep;   // [m] edge potentials, (i, k) at component 2 i + k
  const float2* cur;  // [n] products of the previous iteration
  float2* next;       // [n] products of this iteration (reset to 1)
  __device__ static T identity() { return make_float2(1.f, 1.f); }
  __device__ static T combine(T a, T b) { return make_float2(a.x * b.x, a.y * b.y); }
  __device__ T val(uint64_t e, uint32_t, uint32_t row) const {
    const float2 p = __ldg(vp + row), c = __ldg(cur + row);
    const float4 w = __ldg(ep + e);
    return make_float2(p.x * w.x * c.x + p.y * w.y * c.y, p.x * w.z * c.x + p.y * w.w * c.y);
  }
  __device__ void flush(uint32_t row, T v, bool complete) const {
    if (complete) {
      next[row] = v;
    } else {
      atomic_mul(&next[row].x, v.x);
      atomic_mul(&next[row].y, v.y);
    }
  }
};

__global__ void k_bp_fill(uint32_t n, float2* a) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
    a[v] = make_float2(1.f, 1.f);
}

static int run_bp(gg_graph_s* g, int32_t iters, const float* vert_pot, const float* edge_pot, float* out,
                  gg_run_stats* st) {
  const uint32_t n = g->n;
  const uint64_t m = g->m;
  DevBuf<float2> vp, cur, nxt;
  DevBuf<float4> ep;
  GG_TRY(vp.alloc(g, n));
  GG_TRY(cur.alloc(g, n));
  GG_TRY(nxt.alloc(g, n));
  GG_TRY(ep.alloc(g, std::max<uint64_t>(m, 1)));
  GG_CUDA(cudaMemcpyAsync(vp.p, vert_pot, 8ull * n, cudaMemcpyHostToDevice, g->stream));
  if (m) GG_CUDA(cudaMemcpyAsync(ep.p, edge_pot, 16 * m, cudaMemcpyHostToDevice, g->stream));
  g->kernels = 0;
  EventTimer tm(g->stream);
  const int grid = generic_grid(g, n);
  k_bp_fill<<<grid, kGenericThreads, 0, g->stream>>>(n, cur.p);
  g->kernels++;
  float2 *c = cur.p, *x = nxt.p;
  for (int32_t it = 0; it < iters; ++it) {
    k_bp_fill<<<grid, kGenericThreads, 0, g->stream>>>(n, x);  // BP_Vertex_Reset
    g->kernels++;
    GG_TRY(seg_reduce(g, true, BpOp{vp.p, ep.p, c, x}));
    std::swap(c, x);
  }
  GG_CUDA(cudaGetLastError());
  const double ms = tm.stop();
  GG_CUDA(cudaMemcpyAsync(out, c, 8ull * n, cudaMemcpyDeviceToHost, g->stream));
  GG_CUDA(cudaStreamSynchronize(g->stream));
  if (st) {
    st->ms = ms;
    st->rounds = iters;
    st->edges_traversed = m * (uint64_t)iters;
    st->kernels = g->kernels;
  }
  return GG_OK;
}

}  // namespace gg

using namespace gg;

extern "C" int gg_bp(gg_graph_t g, int32_t iters, const float* vert_potential, const float* edge_potential,
                     float* vert_out, gg_run_stats* st) {
  if (!graph_live(g) || iters < 0 || !vert_potential || (g->m && !edge_potential) || !vert_out)
    return fail(GG_ERR_INVALID_ARG, "gg_bp: bad arguments");
  if (g->relabeled)
    return fail(GG_ERR_UNSUPPORTED, "gg_bp: edge potentials follow the in-edge slots of the given ids; build the "
                                    "graph with vertex_order = GG_VORDER_GIVEN");
  return run_bp(g, iters, vert_potential, edge_potential, vert_out, st);
}
