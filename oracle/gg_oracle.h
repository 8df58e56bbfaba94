/*
 * gg_oracle.h -- TEST INFRASTRUCTURE ONLY.  A sequential CPU restatement of
 * GraphGrind's traversal engine and applications, used as the checker for the
 * GPU library.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it; the product never does.
 *
 * FP64 throughout for PageRank / PageRankDelta / SPMV / BC (the reference's
 * PR/PRDelta/SPMV are double, app/PageRank.C:30, and BC's float is widened,
 * app/BC.C:26); integer apps use int64 like the reference's intT.
 */
#ifndef GG_ORACLE_H
#define GG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_graph {
  uint32_t n;
  uint64_t m;
  int32_t symmetric;
  int32_t part_vertex;      /* -v vertex: no COO, dense always pulls (ligra-numa.h:957) */
  const uint32_t* out_off;  /* n+1 */
  const uint32_t* out_idx;  /* m   */
  const uint32_t* in_off;   /* n+1 */
  const uint32_t* in_idx;   /* m   */
  const double* out_w;      /* m or NULL (weights as read by the app: int or float) */
  const double* in_w;       /* m or NULL */
  /* COO edge order for the dense >m/2 branch: m (src,dst) pairs in partition
   * order, or NULL to use CSC order (dst-major). */
  const uint32_t* coo_src;
  const uint32_t* coo_dst;
  const double* coo_w;
} or_graph;

typedef struct or_stats {
  int32_t rounds;           /* edgeMap calls */
  int64_t edges_traversed;  /* sum of frontier num_out_edges (ligra-numa.h:945) */
  int32_t kinds[4];         /* edgeMaps per branch: empty, sparse, csc, coo */
} or_stats;

int or_bfs(const or_graph* g, uint32_t start, int64_t* parents, int32_t* levels, or_stats* st);
int or_cc(const or_graph* g, int64_t* ids, or_stats* st);
int or_pagerank(const or_graph* g, int32_t max_iter, int32_t bit_all, double* ranks, or_stats* st);
/* or_pagerank's traversed edges and rounds, counted without the arithmetic
 * (valid while the L1 test does not stop the loop early). */
int or_pagerank_edges(const or_graph* g, int32_t max_iter, int32_t bit_all, int64_t* edges, int32_t* rounds);
int or_pagerank_delta(const or_graph* g, double* ranks, or_stats* st);
int or_spmv(const or_graph* g, const double* x, double* y, or_stats* st);
int or_bellman_ford(const or_graph* g, uint32_t start, int64_t* dist, or_stats* st);
int or_bc(const or_graph* g, uint32_t start, double* dependencies, double* num_paths, or_stats* st);
/* The value app/BC.C:156-226 computes when every backward edgeMap follows the
 * transposed edges (always so on symmetric graphs): levels by BFS, path
 * counts summed over in-edges from the previous level, dependencies summed
 * over out-edges to the next level, dependencies = (dep - 1/paths) * paths
 * with dep = 1/paths + sum of successors' dep, NaN where unreached. */
int or_bc_brandes(const or_graph* g, uint32_t start, double* dependencies, double* num_paths);
int or_bp(const or_graph* g, int32_t iters, const double* vert_pot, const double* edge_pot,
          double* vert_out, or_stats* st);
/* PageRank iterated to convergence-free fixed count on every vertex (the
 * k-column personalised form uses this per column): x_{t+1} = d*A x_t + (1-d)*tele. */
int or_ppr(const or_graph* g, int32_t iters, double damping, const double* tele, double* x);

/* app/PageRankConverage.C:235-315: PageRank with the dangling mass spread
 * evenly and the ranks renormalised every iteration, until the L1 change
 * drops to eps or max_iter iterations ran.  ranks[n]; *iters = iterations;
 * l1[max_iter] (may be NULL) = each iteration's L1 change. */
int or_pagerank_converge(const or_graph* g, int32_t max_iter, double eps, double* ranks, int32_t* iters,
                         double* l1);

/* Weighted PageRank and its adjoint (no reference counterpart; the weighted
 * form of PR_F / PR_Vertex_F, app/PageRank.C:28-100, with the edge weight in
 * place of 1/outdeg, and SPMV_F, app/SPMV.C:7-48, at iters = 1, damping = 1):
 *   a_e = w_e (or w_e / sum of w over the source's out-edges when normalize)
 *   x_{t+1}[v] = damping * sum_{e = u->v} a_e x_t[u] + (1 - damping) * tele[v]
 * weights in out-edge (CSR) order; x0 NULL means 1/n.  The backward takes
 * dL/dx_iters and returns dL/dw (CSR order), dL/dtele and dL/dx0 (NULL to
 * skip), by reverse iteration over the transposed edges with every x_t kept. */
int or_wpr_forward(const or_graph* g, const double* w, const double* tele, const double* x0, int32_t iters,
                   double damping, int32_t normalize, double* x_out);
int or_wpr_backward(const or_graph* g, const double* w, const double* tele, const double* x0, int32_t iters,
                    double damping, int32_t normalize, const double* grad_x, double* grad_w, double* grad_tele,
                    double* grad_x0);

/* Partition sizes by the reference rules (same contract as gg_partition_sizes). */
int or_partition_sizes(const uint32_t* in_deg, const uint32_t* out_deg, uint32_t n, uint64_t m,
                       int32_t P, int32_t balance, int32_t part_how, int32_t relabel,
                       int64_t* coo_sizes, int64_t* csc_sizes);
int64_t or_hilbert_key(int64_t side_edges, int64_t x, int64_t y);

/* Inputs without the GPU library (gg_oracle_gen.c). */
/* The library's seeded R-MAT generator restated (gg_gen_rmat): offsets[n+1]
 * filled, *indices malloc'd (release with or_free), *m set. */
int or_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c, uint64_t seed,
                int32_t symmetric, uint32_t* offsets, uint32_t** indices, uint64_t* m);
void or_free(void* p);
/* gg_host_graph_add_weights restated: int32 in [lo,hi] or float in (0,1]. */
int or_add_weights(uint32_t n, const uint32_t* offsets, const uint32_t* indices, int32_t symmetric,
                   int32_t as_float, uint64_t seed, int32_t lo, int32_t hi, void* weights);
/* In-edge CSC (in-lists ascending by source); weights follow when given. */
int or_csc(uint32_t n, uint64_t m, const uint32_t* out_off, const uint32_t* out_idx, const double* out_w,
           uint32_t* in_off, uint32_t* in_idx, double* in_w);
/* Galois .gr v1 (graphgrind/IO.h:365-450); directed graphs also get path_t. */
int or_write_gr(const char* path, uint32_t n, uint64_t m, const uint32_t* off, const uint32_t* idx,
                const int32_t* w, int32_t symmetric);

#ifdef __cplusplus
}
#endif
#endif
