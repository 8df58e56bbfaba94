// Weighted PageRank / SPMV and its hand-written adjoint.
//
//   a_e = w_e, or w_e / (sum of w over the source's out-edges) when normalising
//   x_{t+1}[v] = d * sum_{e = u->v} a_e x_t[u] + (1 - d) * tele[v]
//
// the weighted form of PR_F / PR_Vertex_F (app/PageRank.C:28-100) with a_e in
// place of 1/outdeg(u), and SPMV_F (app/SPMV.C:7-48) at one step with d = 1.
// Forward steps pull over the in-edges (CSC); the adjoint is the transposed
// traversal, a pull over the out-edges (CSR):
//   lambda_T = dL/dx_T
//   dL/dtele += (1 - d) lambda_{t+1}
//   dL/da_e  += d lambda_{t+1}[v] x_t[u]          (e = u->v, fused into the pull)
//   lambda_t[u] = d * sum_{e = u->v} a_e lambda_{t+1}[v]
// The forward keeps x_t every `every` steps; the backward recomputes the
// steps of each segment from its checkpoint before reversing through it.
#include <algorithm>
#include <mutex>
#include <unordered_set>
#include <vector>

#include "gg_segreduce.cuh"

struct gg_wpr_s {
  gg_graph_s* g = nullptr;
  int32_t iters = 0, every = 1, normalize = 0;
  float damping = 0.85f;
  uint32_t n = 0;
  uint64_t m = 0;
  bool have_forward = false;
  // device, all owned
  uint32_t *row_of = nullptr, *perm = nullptr;
  float *w = nullptr, *a_csr = nullptr, *a_csc = nullptr, *wsum = nullptr, *tele = nullptr;
  float *ckpt = nullptr, *seg = nullptr, *S = nullptr, *lam = nullptr, *lam2 = nullptr, *ga = nullptr;
  float *gt = nullptr, *xa = nullptr, *xb = nullptr, *gw = nullptr;
};

namespace gg {

static std::mutex g_wpr_mu;
static std::unordered_set<const gg_wpr_s*> g_wprs;

static bool wpr_live(const gg_wpr_s* w) {
  std::lock_guard<std::mutex> lk(g_wpr_mu);
  return w && g_wprs.count(w) && graph_live(w->g);
}

// Sums into S: rows inside a block are stored, rows split across blocks added.
struct SumInto {
  using T = float;
  static constexpr bool kNeedsIdx = true;
  float* S;
  __device__ static T identity() { return 0.f; }
  __device__ static T combine(T a, T b) { return a + b; }
  __device__ void flush(uint32_t row, T v, bool complete) const {
    if (complete)
      S[row] = v;
    else
      atomicAdd(S + row, v);
  }
};

struct OpFwd : SumInto {  // a_e x[u] over in-edges
  const float* a;
  const float* x;
  __device__ float val(uint64_t e, uint32_t y, uint32_t) const { return __ldg(a + e) * __ldg(x + y); }
};
struct OpBwd : SumInto {  // a_e lambda[v] over out-edges; dL/da_e += d lambda[v] x_t[u]
  const float* a;
  const float* lam;
  const float* x;
  float* ga;
  float d;
  __device__ float val(uint64_t e, uint32_t y, uint32_t row) const {
    const float l = __ldg(lam + y);
    ga[e] += d * l * __ldg(x + row);
    return __ldg(a + e) * l;
  }
};
struct OpW : SumInto {  // sum of out-edge weights
  const float* w;
  __device__ float val(uint64_t e, uint32_t, uint32_t) const { return __ldg(w + e); }
};
struct OpNormBack : SumInto {  // sum of dL/da_e * a_e over out-edges
  const float* ga;
  const float* a;
  __device__ float val(uint64_t e, uint32_t, uint32_t) const { return __ldg(ga + e) * __ldg(a + e); }
};

template <class Op>
static int seg_sum(gg_graph_s* g, bool in_edges, float* S, Op op) {
  GG_CUDA(cudaMemsetAsync(S, 0, 4ull * g->n, g->stream));
  op.S = S;
  return seg_reduce(g, in_edges, op);
}

__global__ void k_wpr_row_of(uint64_t m, uint32_t n, const uint32_t* off, uint32_t* row_of) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = n - 1;  // last row whose offset is <= e
    while (lo < hi) {
      const uint32_t mid = lo + (hi - lo + 1) / 2;
      if (off[mid] <= e)
        lo = mid;
      else
        hi = mid - 1;
    }
    row_of[e] = lo;
  }
}

// Rows whose out-edge list is not sorted by destination (flag[u] = 1).
__global__ void k_wpr_row_unsorted(uint64_t m, const uint32_t* row_of, const uint32_t* out_idx, uint32_t* flag) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x + 1; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t u = row_of[e];
    if (row_of[e - 1] == u && out_idx[e - 1] > out_idx[e]) flag[u] = 1u;
  }
}

// perm[e] = position of out-edge e = u->v among v's in-edges (sorted by
// source).  An edge u->v present c > 1 times has c consecutive in-edge slots;
// the copy of rank r among u's out-edges to v takes slot r of them (binary
// search for the first copy in a sorted row, a scan of the row before e in an
// unsorted one), so the map is a bijection.
__global__ void k_wpr_perm(uint64_t m, const uint32_t* row_of, const uint32_t* out_off, const uint32_t* out_idx,
                           const uint32_t* unsorted, const uint32_t* in_off, const uint32_t* in_idx, uint32_t* perm,
                           unsigned* err) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t u = row_of[e], v = out_idx[e];
    const uint32_t end = in_off[v + 1];
    uint32_t lo = in_off[v], hi = end;
    while (lo < hi) {
      const uint32_t mid = lo + (hi - lo) / 2;
      if (in_idx[mid] < u)
        lo = mid + 1;
      else
        hi = mid;
    }
    uint32_t r = 0;
    if (lo + 1 < end && in_idx[lo] == u && in_idx[lo + 1] == u) {
      const uint32_t rb = out_off[u];
      if (unsorted[u]) {
        for (uint32_t f = rb; f < (uint32_t)e; ++f) r += out_idx[f] == v;
      } else {
        uint32_t a = rb, b = (uint32_t)e;  // first copy of v in the sorted row
        while (a < b) {
          const uint32_t mid = a + (b - a) / 2;
          if (out_idx[mid] < v)
            a = mid + 1;
          else
            b = mid;
        }
        r = (uint32_t)e - a;
      }
    }
    if (lo + r < end && in_idx[lo + r] == u)
      perm[e] = lo + r;
    else
      atomicOr(err, 1u);
  }
}

__global__ void k_wpr_coeffs(uint64_t m, const float* w, const float* wsum, const uint32_t* row_of,
                             const uint32_t* perm, float* a_csr, float* a_csc) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
    const float a = wsum ? w[e] / wsum[row_of[e]] : w[e];
    a_csr[e] = a;
    a_csc[perm[e]] = a;
  }
}

__global__ void k_wpr_fwd_vertex(uint32_t n, const float* S, const float* tele, float d, float* x) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
    x[v] = d * S[v] + (1.f - d) * tele[v];
}

__global__ void k_wpr_bwd_vertex(uint32_t n, const float* S, const float* lam_next, float d, float* lam, float* gt) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
    gt[v] += (1.f - d) * lam_next[v];
    lam[v] = d * S[v];
  }
}

__global__ void k_wpr_norm_back(uint64_t m, const float* ga, const float* R, const float* wsum, const uint32_t* row_of,
                                float* gw) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t u = row_of[e];
    gw[e] = (ga[e] - R[u]) / wsum[u];
  }
}

__global__ void k_wpr_fill(uint32_t n, float v, float* x) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    x[i] = v;
}

static int wpr_step(gg_wpr_s* c, const float* x, float* y) {
  gg_graph_s* g = c->g;
  GG_TRY(seg_sum(g, true, c->S, OpFwd{{}, c->a_csc, x}));
  k_wpr_fwd_vertex<<<generic_grid(g, c->n), kGenericThreads, 0, g->stream>>>(c->n, c->S, c->tele, c->damping, y);
  g->kernels++;
  return GG_OK;
}

static void wpr_release(gg_wpr_s* c) {
  if (!c) return;
  for (void* p : {(void*)c->row_of, (void*)c->perm, (void*)c->w, (void*)c->a_csr, (void*)c->a_csc, (void*)c->wsum,
                  (void*)c->tele, (void*)c->ckpt, (void*)c->seg, (void*)c->S, (void*)c->lam, (void*)c->lam2,
                  (void*)c->ga, (void*)c->gt, (void*)c->xa, (void*)c->xb, (void*)c->gw})
    cudaFree(p);
  delete c;
}

static int wpr_build(gg_wpr_s* c) {
  gg_graph_s* g = c->g;
  const uint32_t n = c->n;
  const uint64_t m = c->m, me = std::max<uint64_t>(m, 1);
  const int32_t K = (c->iters + c->every - 1) / c->every;
  GG_CUDA(cudaMalloc(&c->row_of, 4 * me));
  GG_CUDA(cudaMalloc(&c->perm, 4 * me));
  GG_CUDA(cudaMalloc(&c->w, 4 * me));
  GG_CUDA(cudaMalloc(&c->a_csr, 4 * me));
  GG_CUDA(cudaMalloc(&c->a_csc, 4 * me));
  GG_CUDA(cudaMalloc(&c->ga, 4 * me));
  GG_CUDA(cudaMalloc(&c->wsum, 4ull * n));
  GG_CUDA(cudaMalloc(&c->tele, 4ull * n));
  GG_CUDA(cudaMalloc(&c->ckpt, 4ull * n * std::max(K, 1)));
  GG_CUDA(cudaMalloc(&c->seg, 4ull * n * c->every));
  GG_CUDA(cudaMalloc(&c->S, 4ull * n));
  GG_CUDA(cudaMalloc(&c->lam, 4ull * n));
  GG_CUDA(cudaMalloc(&c->lam2, 4ull * n));
  GG_CUDA(cudaMalloc(&c->gt, 4ull * n));
  GG_CUDA(cudaMalloc(&c->xa, 4ull * n));
  GG_CUDA(cudaMalloc(&c->xb, 4ull * n));
  if (c->normalize) GG_CUDA(cudaMalloc(&c->gw, 4 * me));
  if (m) {
    unsigned* d_err = reinterpret_cast<unsigned*>(g->ws.d_red);
    GG_CUDA(cudaMemsetAsync(d_err, 0, 4, g->stream));
    const int grid = generic_grid(g, m);
    k_wpr_row_of<<<grid, kGenericThreads, 0, g->stream>>>(m, n, g->out_off(), c->row_of);
    uint32_t* unsorted = reinterpret_cast<uint32_t*>(c->S);  // n flags; S is free until the first forward
    GG_CUDA(cudaMemsetAsync(unsorted, 0, 4ull * n, g->stream));
    k_wpr_row_unsorted<<<grid, kGenericThreads, 0, g->stream>>>(m, c->row_of, g->out_idx(), unsorted);
    k_wpr_perm<<<grid, kGenericThreads, 0, g->stream>>>(m, c->row_of, g->out_off(), g->out_idx(), unsorted,
                                                        g->in_off(), g->in_idx(), c->perm, d_err);
    unsigned h_err = 0;
    GG_CUDA(cudaMemcpyAsync(&h_err, d_err, 4, cudaMemcpyDeviceToHost, g->stream));
    GG_CUDA(cudaStreamSynchronize(g->stream));
    if (h_err) return fail(GG_ERR_FORMAT, "weighted PageRank: in-edge lists are not sorted by source");
  }
  return GG_OK;
}

static int wpr_forward(gg_wpr_s* c, const float* w, const float* tele, const float* x0, float* x_out,
                       gg_run_stats* st) {
  gg_graph_s* g = c->g;
  const uint32_t n = c->n;
  const uint64_t m = c->m;
  if (m) GG_CUDA(cudaMemcpyAsync(c->w, w, 4 * m, cudaMemcpyHostToDevice, g->stream));
  GG_CUDA(cudaMemcpyAsync(c->tele, tele, 4ull * n, cudaMemcpyHostToDevice, g->stream));
  if (x0) GG_CUDA(cudaMemcpyAsync(c->ckpt, x0, 4ull * n, cudaMemcpyHostToDevice, g->stream));
  g->kernels = 0;
  EventTimer tm(g->stream);
  if (!x0) {
    k_wpr_fill<<<generic_grid(g, n), kGenericThreads, 0, g->stream>>>(n, 1.0f / n, c->ckpt);
    g->kernels++;
  }
  if (m) {
    if (c->normalize) GG_TRY(seg_sum(g, false, c->wsum, OpW{{}, c->w}));
    k_wpr_coeffs<<<generic_grid(g, m), kGenericThreads, 0, g->stream>>>(m, c->w, c->normalize ? c->wsum : nullptr,
                                                                        c->row_of, c->perm, c->a_csr, c->a_csc);
    g->kernels++;
  }
  const float* x = c->ckpt;
  for (int32_t t = 0; t < c->iters; ++t) {
    // x_{t+1} goes to its checkpoint slot when it starts a segment, else to a spare buffer
    float* y = ((t + 1) % c->every == 0 && t + 1 < c->iters) ? c->ckpt + (uint64_t)n * ((t + 1) / c->every)
                                                               : (x == c->xa ? c->xb : c->xa);
    GG_TRY(wpr_step(c, x, y));
    x = y;
  }
  GG_CUDA(cudaGetLastError());
  const double ms = tm.stop();
  GG_CUDA(cudaMemcpyAsync(x_out, x, 4ull * n, cudaMemcpyDeviceToHost, g->stream));
  GG_CUDA(cudaStreamSynchronize(g->stream));
  c->have_forward = true;
  if (st) {
    st->ms = ms;
    st->rounds = c->iters;
    st->edges_traversed = m * (uint64_t)c->iters;
    st->kernels = g->kernels;
  }
  return GG_OK;
}

static int wpr_backward(gg_wpr_s* c, const float* grad_x, float* grad_w, float* grad_tele, float* grad_x0,
                        gg_run_stats* st) {
  gg_graph_s* g = c->g;
  const uint32_t n = c->n;
  const uint64_t m = c->m;
  GG_CUDA(cudaMemcpyAsync(c->lam, grad_x, 4ull * n, cudaMemcpyHostToDevice, g->stream));
  g->kernels = 0;
  EventTimer tm(g->stream);
  if (m) GG_CUDA(cudaMemsetAsync(c->ga, 0, 4 * m, g->stream));
  GG_CUDA(cudaMemsetAsync(c->gt, 0, 4ull * n, g->stream));
  const int32_t K = (c->iters + c->every - 1) / c->every;
  uint64_t steps = 0;
  for (int32_t s = K - 1; s >= 0; --s) {
    const int32_t t0 = s * c->every, t1 = std::min(c->iters, t0 + c->every);
    // x_{t0} .. x_{t1-1} of this segment: the checkpoint, then recomputed steps
    GG_CUDA(cudaMemcpyAsync(c->seg, c->ckpt + (uint64_t)n * s, 4ull * n, cudaMemcpyDeviceToDevice, g->stream));
    for (int32_t j = 1; j < t1 - t0; ++j) {
      GG_TRY(wpr_step(c, c->seg + (uint64_t)n * (j - 1), c->seg + (uint64_t)n * j));
      ++steps;
    }
    for (int32_t t = t1 - 1; t >= t0; --t) {
      const float* xt = c->seg + (uint64_t)n * (t - t0);
      GG_TRY(seg_sum(g, false, c->S, OpBwd{{}, c->a_csr, c->lam, xt, c->ga, c->damping}));
      k_wpr_bwd_vertex<<<generic_grid(g, n), kGenericThreads, 0, g->stream>>>(n, c->S, c->lam, c->damping, c->lam2,
                                                                              c->gt);
      g->kernels++;
      std::swap(c->lam, c->lam2);
    }
  }
  float* gw = c->ga;
  if (m && c->normalize) {
    // dL/dw_e = (dL/da_e - sum_{e' of u} dL/da_e' a_e') / W_u
    GG_TRY(seg_sum(g, false, c->S, OpNormBack{{}, c->ga, c->a_csr}));
    k_wpr_norm_back<<<generic_grid(g, m), kGenericThreads, 0, g->stream>>>(m, c->ga, c->S, c->wsum, c->row_of,
                                                                           c->gw);
    g->kernels++;
    gw = c->gw;
  }
  GG_CUDA(cudaGetLastError());
  const double ms = tm.stop();
  if (m && grad_w) GG_CUDA(cudaMemcpyAsync(grad_w, gw, 4 * m, cudaMemcpyDeviceToHost, g->stream));
  if (grad_tele) GG_CUDA(cudaMemcpyAsync(grad_tele, c->gt, 4ull * n, cudaMemcpyDeviceToHost, g->stream));
  if (grad_x0) GG_CUDA(cudaMemcpyAsync(grad_x0, c->lam, 4ull * n, cudaMemcpyDeviceToHost, g->stream));
  GG_CUDA(cudaStreamSynchronize(g->stream));
  if (st) {
    st->ms = ms;
    st->rounds = c->iters;
    st->edges_traversed = m * ((uint64_t)c->iters + steps);
    st->kernels = g->kernels;
  }
  return GG_OK;
}

}  // namespace gg

using namespace gg;

extern "C" {

int gg_pagerank_weighted_create(gg_graph_t g, int32_t iters, float damping, int32_t checkpoint_every,
                                int32_t normalize, gg_wpr_t* out) {
  if (!graph_live(g) || !out || iters < 0 || checkpoint_every < 1 || !(damping >= 0.f && damping <= 1.f))
    return fail(GG_ERR_INVALID_ARG, "gg_pagerank_weighted_create: iters >= 0, checkpoint_every >= 1, 0 <= damping <= 1");
  if (g->relabeled)
    return fail(GG_ERR_UNSUPPORTED, "gg_pagerank_weighted_create: weights follow the out-edge order of the given "
                                    "ids; build the graph with vertex_order = GG_VORDER_GIVEN");
  gg_wpr_s* c = new (std::nothrow) gg_wpr_s;
  if (!c) return fail(GG_ERR_OOM, "weighted PageRank: out of host memory");
  c->g = g;
  c->iters = iters;
  c->every = std::min(checkpoint_every, std::max(iters, 1));
  c->normalize = normalize ? 1 : 0;
  c->damping = damping;
  c->n = g->n;
  c->m = g->m;
  const int rc = wpr_build(c);
  if (rc) {
    const std::string keep = last_error();
    wpr_release(c);
    set_error("%s", keep.c_str());
    return rc;
  }
  {
    std::lock_guard<std::mutex> lk(g_wpr_mu);
    g_wprs.insert(c);
  }
  *out = c;
  return GG_OK;
}

int gg_pagerank_weighted_destroy(gg_wpr_t c) {
  {
    std::lock_guard<std::mutex> lk(g_wpr_mu);
    if (!c || !g_wprs.erase(c)) return fail(GG_ERR_INVALID_ARG, "gg_pagerank_weighted_destroy: unknown context");
  }
  if (graph_live(c->g)) cudaStreamSynchronize(c->g->stream);
  wpr_release(c);
  return GG_OK;
}

int gg_pagerank_weighted_fwd(gg_wpr_t c, const float* weights, const float* tele, const float* x0, float* x_out,
                             gg_run_stats* st) {
  if (!wpr_live(c) || (c->m && !weights) || !tele || !x_out)
    return fail(GG_ERR_INVALID_ARG, "gg_pagerank_weighted_fwd: bad arguments");
  return wpr_forward(c, weights, tele, x0, x_out, st);
}

int gg_pagerank_weighted_bwd(gg_wpr_t c, const float* grad_x, float* grad_weights, float* grad_tele, float* grad_x0,
                             gg_run_stats* st) {
  if (!wpr_live(c) || !grad_x) return fail(GG_ERR_INVALID_ARG, "gg_pagerank_weighted_bwd: bad arguments");
  if (!c->have_forward) return fail(GG_ERR_INVALID_ARG, "gg_pagerank_weighted_bwd: run the forward first");
  return wpr_backward(c, grad_x, grad_weights, grad_tele, grad_x0, st);
}

}  // extern "C"
