/*
 * gg_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * Sequential restatement of GraphGrind's edgeMap / vertexMap / vertexFilter
 * and of the Compute() loops of its applications.  Every function names the
 * reference lines it follows (paths inside the GraphGrind tree).  Parity of
 * this restatement with the reference itself is pinned by golden vectors that
 * the reference's own code produced (tests/golden/, made by
 * tests/golden/make_golden.py through oracle/ref_harness.cpp).
 */
#include "gg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------- frontier */
/* partitioned_vertices (graphgrind/ligra-numa.h:91-272): dense bool[n] and/or
 * sparse list, d_m active count, num_out_edges, bit = "all active". */
typedef struct {
  int bit;
  int has_dense;
  uint8_t* d;
  uint32_t* s;
  int64_t dm;
  int64_t out_edges;
  int empty;
} fr_t;

static fr_t fr_empty(void) {
  fr_t f;
  memset(&f, 0, sizeof f);
  f.empty = 1;
  return f;
}
static fr_t fr_single(uint32_t v, int64_t outdeg) { /* ::create :103-116 */
  fr_t f = fr_empty();
  f.empty = 0;
  f.s = (uint32_t*)malloc(sizeof(uint32_t));
  f.s[0] = v;
  f.dm = 1;
  f.out_edges = outdeg;
  return f;
}
static fr_t fr_all(uint32_t n, int64_t out_edges) { /* ::bits :169-180 */
  fr_t f = fr_empty();
  f.empty = 0;
  f.bit = 1;
  f.has_dense = 1;
  f.d = (uint8_t*)malloc(n ? n : 1);
  memset(f.d, 1, n);
  f.dm = n;
  f.out_edges = out_edges;
  return f;
}
static void fr_free(fr_t* f) {
  free(f->d);
  free(f->s);
  memset(f, 0, sizeof *f);
}
/* toDense :228-244 (only when no dense array exists) */
static void fr_to_dense(fr_t* f, uint32_t n) {
  if (!f->d) {
    f->d = (uint8_t*)calloc(n ? n : 1, 1);
    for (int64_t i = 0; i < f->dm; i++) f->d[f->s[i]] = 1;
  }
  f->has_dense = 1;
}
/* toSparse :246-260 (packIndex over d, ascending) */
static void fr_to_sparse(fr_t* f, uint32_t n) {
  if (!f->s) {
    int64_t c = 0;
    f->s = (uint32_t*)malloc(sizeof(uint32_t) * (f->dm ? f->dm : 1));
    for (uint32_t i = 0; i < n; i++)
      if (f->d[i]) f->s[c++] = i;
    f->dm = c;
  }
  f->has_dense = 0;
}
static int fr_is_empty(const fr_t* f) { return f->dm == 0; }

/* --------------------------------------------------------------- functor */
typedef struct {
  void* ctx;
  int (*cond)(void* ctx, uint32_t d);
  int (*update)(void* ctx, uint32_t s, uint32_t d, double w, int64_t pos);        /* non-atomic */
  int (*update_atomic)(void* ctx, uint32_t s, uint32_t d, double w, int64_t pos); /* push */
  int use_cache;
  void (*create_cache)(void* ctx, double* cache, uint32_t d);
  int (*update_cache)(void* ctx, double* cache, uint32_t s, uint32_t d, double w, int64_t pos);
  void (*commit_cache)(void* ctx, double* cache, uint32_t d);
} fn_t;

typedef struct {
  const or_graph* g;
  int transposed; /* BC backward phase (partitioned_graph::transpose, graph-numa.h:721-728) */
  or_stats* st;
  int error;      /* set when edgeMap would abort (ligra-numa.h:937-942) */
} eng_t;

static uint32_t outdeg(const eng_t* e, uint32_t v) {
  const or_graph* g = e->g;
  return e->transposed ? g->in_off[v + 1] - g->in_off[v] : g->out_off[v + 1] - g->out_off[v];
}

/* edgeMap, graphgrind/ligra-numa.h:919-1019 */
static fr_t edge_map(eng_t* e, fr_t* F, const fn_t* f, int64_t threshold) {
  const or_graph* g = e->g;
  const uint32_t n = g->n;
  const int64_t m = (int64_t)g->m;
  if (threshold == -1) threshold = m / 20;          /* :932 */
  const int64_t dense_threshold = m / 2;            /* :934 */
  const int64_t fm = F->dm;
  const int64_t tot = F->out_edges;
  if (F->empty) { /* partitioned_vertices::empty() has numVertices 0: "Sizes Don't match" */
    e->error = 1;
    return fr_empty();
  }
  if (e->st) {
    e->st->rounds++;
    e->st->edges_traversed += tot;                  /* :945 */
  }
  if (tot == 0) {                                   /* :947 */
    if (e->st) e->st->kinds[0]++;
    return fr_empty();
  }
  fr_t out = fr_empty();
  out.empty = 0;
  if (fm + tot > threshold) {                       /* :953 dense */
    fr_to_dense(F, n);
    uint8_t* next = (uint8_t*)calloc(n ? n : 1, 1);
    const uint8_t* fd = F->d;
    const int bit = F->bit;
    if (fm + tot > dense_threshold && !g->part_vertex) {
      /* edgeMapDense over the partitioned COO (:803-866), PART96: the
       * non-atomic update per edge, cond(dst) first.  COO is never transposed. */
      if (e->st) e->st->kinds[3]++;
      if (g->coo_src) {
        for (uint64_t k = 0; k < g->m; k++) {
          uint32_t s = g->coo_src[k], d = g->coo_dst[k];
          double w = g->coo_w ? g->coo_w[k] : 1.0;
          if (f->cond(f->ctx, d) && (bit || fd[s]) && f->update(f->ctx, s, d, w, 1)) next[d] = 1;
        }
      } else {
        for (uint32_t d = 0; d < n; d++)
          for (uint32_t j = g->in_off[d]; j < g->in_off[d + 1]; j++) {
            uint32_t s = g->in_idx[j];
            double w = g->in_w ? g->in_w[j] : 1.0;
            if (f->cond(f->ctx, d) && (bit || fd[s]) && f->update(f->ctx, s, d, w, 1)) next[d] = 1;
          }
      }
    } else {
      /* edgeMapDenseCSC (:549-729), destination partitioning: over the
       * compressed CSC list (vertices with original in-degree > 0), break
       * once cond(id) is false, functor cache when use_cache. */
      if (e->st) e->st->kinds[2]++;
      const uint32_t* off = e->transposed ? g->out_off : g->in_off;
      const uint32_t* idx = e->transposed ? g->out_idx : g->in_idx;
      const double* ww = e->transposed ? g->out_w : g->in_w;
      for (uint32_t id = 0; id < n; id++) {
        if (g->in_off[id + 1] == g->in_off[id]) continue; /* not in CSCV */
        if (!f->cond(f->ctx, id)) continue;
        uint32_t b = off[id], en = off[id + 1];
        if (f->use_cache) {
          double cache[4];
          f->create_cache(f->ctx, cache, id);
          for (uint32_t j = b; j < en; j++) {
            uint32_t s = idx[j];
            double w = ww ? ww[j] : 1.0;
            if ((bit || fd[s]) && f->update_cache(f->ctx, cache, s, id, w, (int64_t)(j - b))) next[id] = 1;
            if (!f->cond(f->ctx, id)) break;
          }
          f->commit_cache(f->ctx, cache, id);
        } else {
          for (uint32_t j = b; j < en; j++) {
            uint32_t s = idx[j];
            double w = ww ? ww[j] : 1.0;
            if ((bit || fd[s]) && f->update(f->ctx, s, id, w, (int64_t)(j - b))) next[id] = 1;
            if (!f->cond(f->ctx, id)) break;
          }
        }
      }
    }
    /* statistics :985-988 */
    int64_t c = 0, oe = 0;
    for (uint32_t i = 0; i < n; i++)
      if (next[i]) {
        c++;
        oe += outdeg(e, i);
      }
    out.has_dense = 1;
    out.d = next;
    out.dm = c;
    out.out_edges = oe;
  } else {
    /* edgeMapSparseWithG (:868-916) */
    if (e->st) e->st->kinds[1]++;
    fr_to_sparse(F, n);
    const uint32_t* off = e->transposed ? g->in_off : g->out_off;
    const uint32_t* idx = e->transposed ? g->in_idx : g->out_idx;
    const double* ww = e->transposed ? g->in_w : g->out_w;
    int64_t total = 0;
    for (int64_t k = 0; k < F->dm; k++) total += off[F->s[k] + 1] - off[F->s[k]];
    uint32_t* q = (uint32_t*)malloc(sizeof(uint32_t) * (total ? total : 1));
    int64_t c = 0;
    for (int64_t k = 0; k < F->dm; k++) {
      uint32_t v = F->s[k];
      for (uint32_t j = off[v]; j < off[v + 1]; j++) {
        uint32_t d = idx[j];
        double w = ww ? ww[j] : 1.0;
        if (f->cond(f->ctx, d) && f->update_atomic(f->ctx, v, d, w, (int64_t)(j - off[v]))) q[c++] = d;
      }
    }
    out.s = q;
    out.dm = c;
    int64_t oe = 0;
    for (int64_t k = 0; k < c; k++) oe += outdeg(e, q[k]); /* :1016 */
    out.out_edges = oe;
  }
  return out;
}

/* vertexMap :1023-1049 */
typedef int (*vfn_t)(void* ctx, uint32_t i);
static void vertex_map(uint32_t n, const fr_t* V, vfn_t fn, void* ctx) {
  if (V->has_dense) {
    for (uint32_t j = 0; j < n; j++)
      if (V->bit || V->d[j]) fn(ctx, j);
  } else {
    for (int64_t i = 0; i < V->dm; i++) fn(ctx, V->s[i]);
  }
}
/* vertexFilter :1053-1082 */
static fr_t vertex_filter(eng_t* e, fr_t* V, vfn_t fn, void* ctx) {
  const uint32_t n = e->g->n;
  fr_to_dense(V, n);
  uint8_t* d_out = (uint8_t*)calloc(n ? n : 1, 1);
  for (uint32_t j = 0; j < n; j++)
    if (V->bit || V->d[j]) d_out[j] = fn(ctx, j) ? 1 : 0;
  fr_t out = fr_empty();
  out.empty = 0;
  out.has_dense = 1;
  out.d = d_out;
  for (uint32_t j = 0; j < n; j++)
    if (d_out[j]) {
      out.dm++;
      out.out_edges += outdeg(e, j);
    }
  return out;
}

/* ================================================================== BFS */
/* app/BFS.C:26-75 */
typedef struct { int64_t* parents; } bfs_ctx;
static int bfs_cond(void* c, uint32_t d) { return ((bfs_ctx*)c)->parents[d] == -1; }
static int bfs_update(void* c, uint32_t s, uint32_t d, double w, int64_t pos) {
  (void)w; (void)pos;
  bfs_ctx* x = (bfs_ctx*)c;
  if (x->parents[d] == -1) {
    x->parents[d] = s;
    return 1;
  }
  return 0;
}

int or_bfs(const or_graph* g, uint32_t start, int64_t* parents, int32_t* levels, or_stats* st) {
  /* app/BFS.C:77-101 */
  if (!g || start >= g->n) return -1;
  eng_t e = {g, 0, st, 0};
  for (uint32_t i = 0; i < g->n; i++) {
    parents[i] = -1;
    if (levels) levels[i] = -1;
  }
  parents[start] = start;
  if (levels) levels[start] = 0;
  bfs_ctx c = {parents};
  fn_t f = {&c, bfs_cond, bfs_update, bfs_update, 0, 0, 0, 0};
  fr_t F = fr_single(start, g->out_off[start + 1] - g->out_off[start]);
  int32_t round = 0;
  while (!fr_is_empty(&F)) {
    fr_t out = edge_map(&e, &F, &f, (int64_t)g->m / 20);
    round++;
    if (levels) {
      if (out.has_dense) {
        for (uint32_t i = 0; i < g->n; i++)
          if (out.d[i]) levels[i] = round;
      } else {
        for (int64_t k = 0; k < out.dm; k++) levels[out.s[k]] = round;
      }
    }
    fr_free(&F);
    F = out;
  }
  fr_free(&F);
  return 0;
}

/* ================================================================ Components */
/* app/Components.C:26-99 */
typedef struct { int64_t* ids; int64_t* prev; } cc_ctx;
static int cc_cond(void* c, uint32_t d) { (void)c; (void)d; return 1; }
static int cc_update(void* c, uint32_t s, uint32_t d, double w, int64_t pos) {
  (void)w; (void)pos;
  cc_ctx* x = (cc_ctx*)c;
  int64_t orig = x->ids[d];
  if (x->ids[s] < orig) {
    x->ids[d] = orig < x->ids[s] ? orig : x->ids[s];
    if (orig == x->prev[d]) return 1;
  }
  return 0;
}
static int cc_update_atomic(void* c, uint32_t s, uint32_t d, double w, int64_t pos) {
  (void)w; (void)pos;
  cc_ctx* x = (cc_ctx*)c;
  int64_t orig = x->ids[d];
  int wrote = 0;
  if (x->ids[s] < x->ids[d]) { /* writeMin, graphgrind/utils.h:445-452 */
    x->ids[d] = x->ids[s];
    wrote = 1;
  }
  return wrote && orig == x->prev[d];
}
static void cc_create(void* c, double* cache, uint32_t d) {
  cc_ctx* x = (cc_ctx*)c;
  cache[0] = (double)x->ids[d];
  cache[1] = (double)x->prev[d];
}
static int cc_update_cache(void* c, double* cache, uint32_t s, uint32_t d, double w, int64_t pos) {
  (void)d; (void)w; (void)pos;
  cc_ctx* x = (cc_ctx*)c;
  double orig = cache[0];
  if ((double)x->prev[s] < orig) {
    cache[0] = orig < (double)x->prev[s] ? orig : (double)x->prev[s];
    if (orig == cache[1]) return 1;
  }
  return 0;
}
static void cc_commit(void* c, double* cache, uint32_t d) { ((cc_ctx*)c)->ids[d] = (int64_t)cache[0]; }
static int cc_vertex(void* c, uint32_t i) {
  cc_ctx* x = (cc_ctx*)c;
  x->prev[i] = x->ids[i];
  return 1;
}

int or_cc(const or_graph* g, int64_t* ids, or_stats* st) {
  /* app/Components.C:101-126 */
  if (!g) return -1;
  eng_t e = {g, 0, st, 0};
  int64_t* prev = (int64_t*)malloc(sizeof(int64_t) * (g->n ? g->n : 1));
  for (uint32_t i = 0; i < g->n; i++) ids[i] = i;
  cc_ctx c = {ids, prev};
  fn_t f = {&c, cc_cond, cc_update, cc_update_atomic, 1, cc_create, cc_update_cache, cc_commit};
  fr_t F = fr_all(g->n, (int64_t)g->m);
  while (!fr_is_empty(&F)) {
    vertex_map(g->n, &F, cc_vertex, &c);
    fr_t out = edge_map(&e, &F, &f, (int64_t)g->m / 20);
    fr_free(&F);
    F = out;
  }
  fr_free(&F);
  free(prev);
  return 0;
}

/* ================================================================== PageRank */
/* app/PageRank.C:28-100 */
typedef struct { double* p_curr; double* p_next; const eng_t* e; double damping, added; } pr_ctx;
static int true_cond(void* c, uint32_t d) { (void)c; (void)d; return 1; }
static int pr_update(void* c, uint32_t s, uint32_t d, double w, int64_t pos) {
  (void)w; (void)pos;
  pr_ctx* x = (pr_ctx*)c;
  x->p_next[d] += x->p_curr[s] / outdeg(x->e, s);
  return 1;
}
static void pr_create(void* c, double* cache, uint32_t d) { cache[0] = ((pr_ctx*)c)->p_next[d]; }
static int pr_update_cache(void* c, double* cache, uint32_t s, uint32_t d, double w, int64_t pos) {
  (void)d; (void)w; (void)pos;
  pr_ctx* x = (pr_ctx*)c;
  cache[0] += x->p_curr[s] / outdeg(x->e, s);
  return 1;
}
static void pr_commit(void* c, double* cache, uint32_t d) { ((pr_ctx*)c)->p_next[d] = cache[0]; }
static int pr_vertex(void* c, uint32_t i) {
  pr_ctx* x = (pr_ctx*)c;
  x->p_next[i] = x->damping * x->p_next[i] + x->added;
  return 1;
}
static int pr_reset(void* c, uint32_t i) {
  ((pr_ctx*)c)->p_curr[i] = 0.0;
  return 1;
}

int or_pagerank(const or_graph* g, int32_t max_iter, int32_t bit_all, double* ranks, or_stats* st) {
  /* app/PageRank.C:102-150; bit_all reproduces app/PageRankBit.C:145 */
  if (!g) return -1;
  const uint32_t n = g->n;
  eng_t e = {g, 0, st, 0};
  const double damping = 0.85, eps = 0.0000001;
  double one_over_n = 1 / (double)n;
  double* a = (double*)malloc(sizeof(double) * n);
  double* b = (double*)malloc(sizeof(double) * n);
  for (uint32_t j = 0; j < n; j++) {
    a[j] = one_over_n;
    b[j] = 0;
  }
  pr_ctx c = {a, b, &e, damping, (1 - damping) * (1 / (double)n)};
  fn_t f = {&c, true_cond, pr_update, pr_update, 1, pr_create, pr_update_cache, pr_commit};
  fr_t F = fr_all(n, (int64_t)g->m);
  int count = 0;
  double* last = b;
  while (count < max_iter) {
    count++;
    fr_t out = edge_map(&e, &F, &f, (int64_t)g->m / 20);
    if (e.error) {
      fr_free(&F);
      free(a);
      free(b);
      return -2;
    }
    vertex_map(n, &F, pr_vertex, &c);
    last = c.p_next;
    double l1 = 0;
    for (uint32_t j = 0; j < n; j++) {
      c.p_curr[j] = fabs(c.p_curr[j] - c.p_next[j]);
      l1 += c.p_curr[j];
    }
    if (l1 < eps) {
      fr_free(&out);
      break;
    }
    vertex_map(n, &F, pr_reset, &c);
    double* t = c.p_curr;
    c.p_curr = c.p_next;
    c.p_next = t;
    fr_free(&F);
    F = out;
    if (bit_all) F.bit = 1; /* output.bit = true */
  }
  fr_free(&F);
  memcpy(ranks, last, sizeof(double) * n);
  free(a);
  free(b);
  return 0;
}

/* The traversed-edge count of or_pagerank without its arithmetic: the
 * frontier sequence of app/PageRank.C:128-146 (all vertices first, then each
 * edgeMap's output: every destination of an edge leaving the frontier, since
 * PR_F::update always returns 1 and cond is cond_true; with bit_all every
 * vertex sends, app/PageRankBit.C:145), summing each frontier's out-degrees (graphgrind/ligra-numa.h:944-945).  It assumes the
 * L1 test (:139-140) does not end the loop before max_iter, which holds when
 * a vertex without in-edges exists: its rank is left out of every later
 * frontier, so |p_curr - p_next| keeps its 0.15/n there. */
int or_pagerank_edges(const or_graph* g, int32_t max_iter, int32_t bit_all, int64_t* edges, int32_t* rounds) {
  if (!g || !edges || !rounds) return -1;
  const uint32_t n = g->n;
  uint8_t* cur = (uint8_t*)malloc(n ? n : 1);
  uint8_t* nxt = (uint8_t*)malloc(n ? n : 1);
  if (!cur || !nxt) {
    free(cur);
    free(nxt);
    return -2;
  }
  memset(cur, 1, n);
  int all = 1;
  int64_t total = 0;
  int32_t r = 0;
  for (; r < max_iter; r++) {
    memset(nxt, 0, n);
    for (uint32_t u = 0; u < n; u++) {
      /* the frontier's out-degrees count; with bit set (PageRankBit's
       * output.bit = true) every source sends */
      if (cur[u]) total += (int64_t)(g->out_off[u + 1] - g->out_off[u]);
      if (!all && !cur[u]) continue;
      for (uint32_t j = g->out_off[u]; j < g->out_off[u + 1]; j++) nxt[g->out_idx[j]] = 1;
    }
    uint8_t* t = cur;
    cur = nxt;
    nxt = t;
    all = bit_all;
  }
  free(cur);
  free(nxt);
  *edges = total;
  *rounds = r;
  return 0;
}

/* ============================================================ PageRankDelta */
/* app/PageRankDelta.C:29-117 */
typedef struct { double* p; double* delta; double* ngh; const eng_t* e; double damping, added, one_over_n, eps2; } prd_ctx;
static int prd_update(void* c, uint32_t s, uint32_t d, double w, int64_t pos) {
  (void)w; (void)pos;
  prd_ctx* x = (prd_ctx*)c;
  x->ngh[d] += x->delta[s] / outdeg(x->e, s);
  return 1;
}
static void prd_create(void* c, double* cache, uint32_t d) { cache[0] = ((prd_ctx*)c)->ngh[d]; }
static int prd_update_cache(void* c, double* cache, uint32_t s, uint32_t d, double w, int64_t pos) {
  (void)d; (void)w; (void)pos;
  prd_ctx* x = (prd_ctx*)c;
  cache[0] += x->delta[s] / outdeg(x->e, s);
  return 1;
}
static void prd_commit(void* c, double* cache, uint32_t d) { ((prd_ctx*)c)->ngh[d] = cache[0]; }
static int prd_first(void* c, uint32_t i) {
  prd_ctx* x = (prd_ctx*)c;
  x->delta[i] = x->damping * (x->p[i] + x->ngh[i]) + x->added - x->p[i];
  x->p[i] += x->delta[i];
  x->delta[i] -= x->one_over_n;
  return fabs(x->delta[i]) > x->eps2 * x->p[i];
}
static int prd_vertex(void* c, uint32_t i) {
  prd_ctx* x = (prd_ctx*)c;
  x->delta[i] = x->ngh[i] * x->damping;
  x->p[i] += x->delta[i];
  return fabs(x->delta[i]) > x->eps2 * x->p[i];
}

int or_pagerank_delta(const or_graph* g, double* ranks, or_stats* st) {
  /* app/PageRankDelta.C:120-174 */
  if (!g) return -1;
  const uint32_t n = g->n;
  eng_t e = {g, 0, st, 0};
  const double damping = 0.85, eps = 0.0000001, eps2 = 0.01;
  double one_over_n = 1 / (double)n;
  double* delta = (double*)malloc(sizeof(double) * n);
  double* ngh = (double*)malloc(sizeof(double) * n);
  for (uint32_t j = 0; j < n; j++) {
    ranks[j] = 0.0;
    delta[j] = one_over_n;
    ngh[j] = 0.0;
  }
  prd_ctx c = {ranks, delta, ngh, &e, damping, (1 - damping) * one_over_n, one_over_n, eps2};
  fn_t f = {&c, true_cond, prd_update, prd_update, 1, prd_create, prd_update_cache, prd_commit};
  fr_t F = fr_all(n, (int64_t)g->m);
  fr_t All = fr_all(n, (int64_t)g->m);
  int round = 0;
  for (;;) {
    round++;
    fr_t out = edge_map(&e, &F, &f, (int64_t)g->m / 20);
    fr_free(&out);
    fr_t active = vertex_filter(&e, &All, round == 1 ? prd_first : prd_vertex, &c);
    double l1 = 0;
    for (uint32_t j = 0; j < n; j++) {
      ngh[j] = fabs(delta[j]);
      l1 += ngh[j];
    }
    if (l1 < eps) {
      fr_free(&active);
      break;
    }
    for (uint32_t j = 0; j < n; j++) ngh[j] = 0.0;
    fr_free(&F);
    F = active;
  }
  fr_free(&F);
  fr_free(&All);
  free(delta);
  free(ngh);
  return 0;
}

/* ===================================================================== SPMV */
/* app/SPMV.C:7-92 */
typedef struct { const double* x; double* y; } spmv_ctx;
static int spmv_update(void* c, uint32_t s, uint32_t d, double w, int64_t pos) {
  (void)pos;
  spmv_ctx* z = (spmv_ctx*)c;
  z->y[d] += z->x[s] * w;
  return 1;
}
static void spmv_create(void* c, double* cache, uint32_t d) { cache[0] = ((spmv_ctx*)c)->y[d]; }
static int spmv_update_cache(void* c, double* cache, uint32_t s, uint32_t d, double w, int64_t pos) {
  (void)d; (void)pos;
  cache[0] += ((spmv_ctx*)c)->x[s] * w;
  return 1;
}
static void spmv_commit(void* c, double* cache, uint32_t d) { ((spmv_ctx*)c)->y[d] = cache[0]; }

int or_spmv(const or_graph* g, const double* x, double* y, or_stats* st) {
  if (!g) return -1;
  const uint32_t n = g->n;
  eng_t e = {g, 0, st, 0};
  double* xv = (double*)malloc(sizeof(double) * n);
  for (uint32_t j = 0; j < n; j++) {
    xv[j] = x ? x[j] : 1 / (double)n;
    y[j] = 0;
  }
  spmv_ctx c = {xv, y};
  fn_t f = {&c, true_cond, spmv_update, spmv_update, 1, spmv_create, spmv_update_cache, spmv_commit};
  fr_t F = fr_all(n, (int64_t)g->m);
  fr_t out = edge_map(&e, &F, &f, (int64_t)g->m / 20);
  fr_free(&out);
  fr_free(&F);
  free(xv);
  return 0;
}

/* ============================================================== BellmanFord */
/* app/BellmanFord.C:28-103 */
typedef struct { int64_t* sp; int64_t* visited; } bf_ctx;
static int bf_update(void* c, uint32_t s, uint32_t d, double w, int64_t pos) {
  (void)pos;
  bf_ctx* x = (bf_ctx*)c;
  int64_t nd = x->sp[s] + (int64_t)w;
  if (x->sp[d] > nd) {
    x->sp[d] = nd;
    if (x->visited[d] == 0) {
      x->visited[d] = 1;
      return 1;
    }
  }
  return 0;
}
static int bf_update_atomic(void* c, uint32_t s, uint32_t d, double w, int64_t pos) {
  (void)pos;
  bf_ctx* x = (bf_ctx*)c;
  int64_t nd = x->sp[s] + (int64_t)w;
  if (nd < x->sp[d]) { /* writeMin */
    x->sp[d] = nd;
    if (x->visited[d] == 0) { /* CAS(&Visited[d],0,1) */
      x->visited[d] = 1;
      return 1;
    }
  }
  return 0;
}
static void bf_create(void* c, double* cache, uint32_t d) {
  bf_ctx* x = (bf_ctx*)c;
  cache[0] = (double)x->sp[d];
  cache[1] = (double)x->visited[d];
}
static int bf_update_cache(void* c, double* cache, uint32_t s, uint32_t d, double w, int64_t pos) {
  (void)d; (void)pos;
  bf_ctx* x = (bf_ctx*)c;
  double nd = (double)(x->sp[s] + (int64_t)w);
  if (cache[0] > nd) {
    cache[0] = nd;
    if (cache[1] == 0) {
      cache[1] = 1;
      return 1;
    }
  }
  return 0;
}
static void bf_commit(void* c, double* cache, uint32_t d) {
  bf_ctx* x = (bf_ctx*)c;
  x->visited[d] = (int64_t)cache[1];
  x->sp[d] = (int64_t)cache[0];
}
static int bf_vertex(void* c, uint32_t i) {
  ((bf_ctx*)c)->visited[i] = 0;
  return 1;
}

int or_bellman_ford(const or_graph* g, uint32_t start, int64_t* sp, or_stats* st) {
  /* app/BellmanFord.C:106-145 */
  if (!g || start >= g->n) return -1;
  const uint32_t n = g->n;
  eng_t e = {g, 0, st, 0};
  const int64_t inf = 2147483647 / 2;
  int64_t* visited = (int64_t*)calloc(n, sizeof(int64_t));
  for (uint32_t j = 0; j < n; j++) sp[j] = inf;
  sp[start] = 0;
  bf_ctx c = {sp, visited};
  fn_t f = {&c, true_cond, bf_update, bf_update_atomic, 1, bf_create, bf_update_cache, bf_commit};
  fr_t F = fr_single(start, g->out_off[start + 1] - g->out_off[start]);
  int64_t round = 0;
  while (!fr_is_empty(&F)) {
    if (round == n) {
      for (uint32_t j = 0; j < n; j++) sp[j] = -inf;
      break;
    }
    fr_t out = edge_map(&e, &F, &f, (int64_t)g->m / 20);
    vertex_map(n, &out, bf_vertex, &c);
    fr_free(&F);
    F = out;
    round++;
  }
  fr_free(&F);
  free(visited);
  return 0;
}

/* ======================================================================= BC */
/* app/BC.C:28-154 with fType widened to double */
typedef struct { double* v; uint8_t* visited; } bc_ctx;
static int bc_cond(void* c, uint32_t d) { return ((bc_ctx*)c)->visited[d] == 0; }
static int bc_update(void* c, uint32_t s, uint32_t d, double w, int64_t pos) {
  (void)w; (void)pos;
  bc_ctx* x = (bc_ctx*)c;
  double old = x->v[d];
  x->v[d] += x->v[s];
  return old == 0.0;
}
static void bc_create(void* c, double* cache, uint32_t d) { cache[0] = ((bc_ctx*)c)->v[d]; }
static int bc_update_cache(void* c, double* cache, uint32_t s, uint32_t d, double w, int64_t pos) {
  (void)d; (void)w; (void)pos;
  double old = cache[0];
  cache[0] += ((bc_ctx*)c)->v[s];
  return old == 0.0;
}
static void bc_commit(void* c, double* cache, uint32_t d) { ((bc_ctx*)c)->v[d] = cache[0]; }
static int bc_mark(void* c, uint32_t i) {
  ((bc_ctx*)c)->visited[i] = 1;
  return 1;
}
typedef struct { uint8_t* visited; double* dep; const double* inv; } bcb_ctx;
static int bc_back_vertex(void* c, uint32_t i) {
  bcb_ctx* x = (bcb_ctx*)c;
  x->visited[i] = 1;
  x->dep[i] += x->inv[i];
  return 1;
}

int or_bc(const or_graph* g, uint32_t start, double* dep, double* num_paths, or_stats* st) {
  /* app/BC.C:156-226 */
  if (!g || start >= g->n) return -1;
  const uint32_t n = g->n;
  eng_t e = {g, 0, st, 0};
  double* np = (double*)calloc(n, sizeof(double));
  uint8_t* visited = (uint8_t*)calloc(n, 1);
  np[start] = 1.0;
  visited[start] = 1;
  int cap = 64, nl = 0;
  fr_t* levels = (fr_t*)malloc(sizeof(fr_t) * cap);
  levels[nl++] = fr_single(start, g->out_off[start + 1] - g->out_off[start]);
  bc_ctx c = {np, visited};
  fn_t f = {&c, bc_cond, bc_update, bc_update, 1, bc_create, bc_update_cache, bc_commit};
  int round = 0;
  fr_t* F = &levels[0];
  while (!fr_is_empty(F)) {
    round++;
    fr_t out = edge_map(&e, F, &f, (int64_t)g->m / 20);
    vertex_map(n, &out, bc_mark, &c);
    if (nl == cap) {
      cap *= 2;
      levels = (fr_t*)realloc(levels, sizeof(fr_t) * cap);
    }
    levels[nl++] = out;
    F = &levels[nl - 1];
  }
  if (num_paths) memcpy(num_paths, np, sizeof(double) * n);
  for (uint32_t j = 0; j < n; j++) dep[j] = 0.0;
  for (uint32_t j = 0; j < n; j++) np[j] = 1 / np[j]; /* inverseNumPaths aliases NumPaths */
  for (uint32_t j = 0; j < n; j++) visited[j] = 0;
  bcb_ctx bb = {visited, dep, np};
  bc_ctx cb = {dep, visited};
  fn_t fb = {&cb, bc_cond, bc_update, bc_update, 1, bc_create, bc_update_cache, bc_commit};
  fr_t* Fr = &levels[round - 1];
  vertex_map(n, Fr, bc_back_vertex, &bb);
  e.transposed = g->symmetric ? 0 : 1; /* GA.transpose() is a no-op when symmetric */
  for (int r = round - 2; r >= 0; r--) {
    fr_t out = edge_map(&e, Fr, &fb, (int64_t)g->m / 20);
    fr_free(&out);
    Fr = &levels[r];
    vertex_map(n, Fr, bc_back_vertex, &bb);
  }
  for (uint32_t j = 0; j < n; j++) dep[j] = (dep[j] - np[j]) / np[j];
  for (int k = 0; k < nl; k++) fr_free(&levels[k]);
  free(levels);
  free(np);
  free(visited);
  return 0;
}

int or_bc_brandes(const or_graph* g, uint32_t start, double* dep, double* num_paths) {
  if (!g || start >= g->n) return -1;
  const uint32_t n = g->n;
  int32_t* lev = (int32_t*)malloc(sizeof(int32_t) * n);
  uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * n);
  double* np = (double*)calloc(n, sizeof(double));
  for (uint32_t v = 0; v < n; v++) lev[v] = -1;
  lev[start] = 0;
  np[start] = 1.0;
  order[0] = start;
  uint64_t head = 0, tail = 1;
  while (head < tail) { /* queue BFS: vertices leave in level order */
    const uint32_t v = order[head++];
    for (uint32_t e = g->out_off[v]; e < g->out_off[v + 1]; e++) {
      const uint32_t u = g->out_idx[e];
      if (lev[u] < 0) {
        lev[u] = lev[v] + 1;
        order[tail++] = u;
      }
    }
  }
  for (uint64_t i = 1; i < tail; i++) { /* path counts from in-edges of the previous level */
    const uint32_t u = order[i];
    double s = 0;
    for (uint32_t e = g->in_off[u]; e < g->in_off[u + 1]; e++)
      if (lev[g->in_idx[e]] == lev[u] - 1) s += np[g->in_idx[e]];
    np[u] = s;
  }
  if (num_paths) memcpy(num_paths, np, sizeof(double) * n);
  for (uint32_t v = 0; v < n; v++) dep[v] = 0.0;
  for (uint64_t i = tail; i-- > 0;) { /* successors first */
    const uint32_t v = order[i];
    double s = 0;
    for (uint32_t e = g->out_off[v]; e < g->out_off[v + 1]; e++)
      if (lev[g->out_idx[e]] == lev[v] + 1) s += dep[g->out_idx[e]];
    dep[v] = s + 1.0 / np[v];
  }
  for (uint32_t v = 0; v < n; v++) {
    const double inv = 1.0 / np[v]; /* inf where unreached, giving NaN below */
    dep[v] = (dep[v] - inv) / inv;
  }
  free(lev);
  free(order);
  free(np);
  return 0;
}

/* ======================================================================= BP */
/* Two-state belief propagation in the form the GPU library defines
 * (app/BP.C:54-149 leaves vertex/edge potentials uninitialised and resets
 * with a shadowed index, :145; here every vertex's product is reset to 1 and
 * the potentials are inputs).  Per iteration, for every edge s->d at in-list
 * position j of d (edge index e = in_off[d]+j):
 *   belief[e][i] = sum_k vert_pot[d][k] * edge_pot[e][i][k] * prod_cur[d][k]
 *   prod_next[d][i] *= belief[e][i]                                        */
int or_bp(const or_graph* g, int32_t iters, const double* vert_pot, const double* edge_pot,
          double* vert_out, or_stats* st) {
  (void)st;
  if (!g) return -1;
  const uint32_t n = g->n;
  double* cur = (double*)malloc(sizeof(double) * 2 * n);
  double* nxt = (double*)malloc(sizeof(double) * 2 * n);
  for (uint32_t i = 0; i < 2 * n; i++) cur[i] = 1.0;
  for (int it = 0; it < iters; it++) {
    for (uint32_t i = 0; i < 2 * n; i++) nxt[i] = 1.0;
    for (uint32_t d = 0; d < n; d++) {
      for (uint32_t e = g->in_off[d]; e < g->in_off[d + 1]; e++) {
        for (int i = 0; i < 2; i++) {
          double b = 0;
          for (int k = 0; k < 2; k++) b += vert_pot[2 * d + k] * edge_pot[4 * (uint64_t)e + 2 * i + k] * cur[2 * d + k];
          nxt[2 * d + i] *= b;
        }
      }
    }
    double* t = cur;
    cur = nxt;
    nxt = t;
  }
  memcpy(vert_out, cur, sizeof(double) * 2 * n);
  free(cur);
  free(nxt);
  return 0;
}

/* ======================================================== personalised PR */
int or_ppr(const or_graph* g, int32_t iters, double damping, const double* tele, double* x) {
  if (!g) return -1;
  const uint32_t n = g->n;
  double* y = (double*)malloc(sizeof(double) * n);
  for (uint32_t i = 0; i < n; i++) x[i] = tele[i];
  for (int it = 0; it < iters; it++) {
    for (uint32_t d = 0; d < n; d++) {
      double acc = 0;
      for (uint32_t j = g->in_off[d]; j < g->in_off[d + 1]; j++) {
        uint32_t s = g->in_idx[j];
        acc += x[s] / (double)(g->out_off[s + 1] - g->out_off[s]);
      }
      y[d] = damping * acc + (1 - damping) * tele[d];
    }
    memcpy(x, y, sizeof(double) * n);
  }
  free(y);
  return 0;
}

/* ================================================ PageRankConverage */
int or_pagerank_converge(const or_graph* g, int32_t max_iter, double eps, double* ranks, int32_t* iters,
                         double* l1) {
  if (!g || max_iter < 0) return -1;
  const uint32_t n = g->n;
  double* pc = (double*)malloc(sizeof(double) * n);
  double* pn = (double*)malloc(sizeof(double) * n);
  double* add = (double*)malloc(sizeof(double) * n);
  for (uint32_t j = 0; j < n; j++) {
    pc[j] = 1 / (double)n;
    pn[j] = 0;
  }
  int32_t count = 0;
  double L1 = 2;
  while (count < max_iter && L1 > eps) {
    for (uint32_t j = 0; j < n; j++) { /* edge_factor * p_curr; sinks are never gathered */
      const uint32_t d = g->out_off[j + 1] - g->out_off[j];
      add[j] = d ? 0.85 / d * pc[j] : 0.0;
    }
    for (uint32_t d = 0; d < n; d++)
      for (uint32_t e = g->in_off[d]; e < g->in_off[d + 1]; e++) pn[d] += add[g->in_idx[e]];
    double s = 0;
    for (uint32_t j = 0; j < n; j++) s += pn[j];
    const double c = (1 - s) / n; /* PR_Vertex_Csum with sum(..., scale=1) */
    L1 = 0;
    double s2 = 0;
    for (uint32_t j = 0; j < n; j++) {
      pn[j] += c;
      L1 += fabs(pc[j] - pn[j]);
    }
    for (uint32_t j = 0; j < n; j++) s2 += pn[j];
    if (l1) l1[count] = L1;
    for (uint32_t j = 0; j < n; j++) {
      pn[j] /= s2; /* PR_Vertex_norm */
      pc[j] = 0;   /* PR_Vertex_Reset */
    }
    count++;
    double* t = pc;
    pc = pn;
    pn = t;
  }
  memcpy(ranks, pc, sizeof(double) * n);
  if (iters) *iters = count;
  free(pc);
  free(pn);
  free(add);
  return 0;
}

/* ======================================================= weighted PageRank */
static double* wpr_coeffs(const or_graph* g, const double* w, int32_t normalize) {
  double* a = (double*)malloc(sizeof(double) * (g->m ? g->m : 1));
  for (uint32_t u = 0; u < g->n; u++) {
    double s = 0;
    for (uint32_t e = g->out_off[u]; e < g->out_off[u + 1]; e++) s += w[e];
    for (uint32_t e = g->out_off[u]; e < g->out_off[u + 1]; e++) a[e] = normalize ? w[e] / s : w[e];
  }
  return a;
}

/* x_{t+1} from x_t over out-edges (the same sums as a pull over in-edges). */
static void wpr_step(const or_graph* g, const double* a, const double* tele, double damping, const double* x,
                     double* y) {
  for (uint32_t v = 0; v < g->n; v++) y[v] = 0;
  for (uint32_t u = 0; u < g->n; u++)
    for (uint32_t e = g->out_off[u]; e < g->out_off[u + 1]; e++) y[g->out_idx[e]] += a[e] * x[u];
  for (uint32_t v = 0; v < g->n; v++) y[v] = damping * y[v] + (1 - damping) * tele[v];
}

static double* wpr_states(const or_graph* g, const double* a, const double* tele, const double* x0, int32_t iters,
                          double damping) {
  const uint32_t n = g->n;
  double* xs = (double*)malloc(sizeof(double) * n * (iters + 1));
  for (uint32_t v = 0; v < n; v++) xs[v] = x0 ? x0[v] : 1.0 / n;
  for (int32_t t = 0; t < iters; t++) wpr_step(g, a, tele, damping, xs + (size_t)t * n, xs + (size_t)(t + 1) * n);
  return xs;
}

int or_wpr_forward(const or_graph* g, const double* w, const double* tele, const double* x0, int32_t iters,
                   double damping, int32_t normalize, double* x_out) {
  if (!g || iters < 0) return -1;
  double* a = wpr_coeffs(g, w, normalize);
  double* xs = wpr_states(g, a, tele, x0, iters, damping);
  memcpy(x_out, xs + (size_t)iters * g->n, sizeof(double) * g->n);
  free(xs);
  free(a);
  return 0;
}

int or_wpr_backward(const or_graph* g, const double* w, const double* tele, const double* x0, int32_t iters,
                    double damping, int32_t normalize, const double* grad_x, double* grad_w, double* grad_tele,
                    double* grad_x0) {
  if (!g || iters < 0) return -1;
  const uint32_t n = g->n;
  double* a = wpr_coeffs(g, w, normalize);
  double* xs = wpr_states(g, a, tele, x0, iters, damping);
  double* lam = (double*)malloc(sizeof(double) * n);
  double* nl = (double*)malloc(sizeof(double) * n);
  double* ga = (double*)calloc(g->m ? g->m : 1, sizeof(double));
  memcpy(lam, grad_x, sizeof(double) * n);
  for (uint32_t v = 0; v < n; v++) grad_tele[v] = 0;
  for (int32_t t = iters - 1; t >= 0; t--) {
    const double* x = xs + (size_t)t * n;
    for (uint32_t v = 0; v < n; v++) grad_tele[v] += (1 - damping) * lam[v];
    for (uint32_t u = 0; u < n; u++) {
      double s = 0;
      for (uint32_t e = g->out_off[u]; e < g->out_off[u + 1]; e++) {
        const uint32_t v = g->out_idx[e];
        ga[e] += damping * lam[v] * x[u];
        s += a[e] * lam[v];
      }
      nl[u] = damping * s;
    }
    memcpy(lam, nl, sizeof(double) * n);
  }
  if (grad_x0) memcpy(grad_x0, lam, sizeof(double) * n);
  for (uint32_t u = 0; u < n; u++) { /* chain rule through the normalisation */
    double W = 0, r = 0;
    for (uint32_t e = g->out_off[u]; e < g->out_off[u + 1]; e++) {
      W += w[e];
      r += ga[e] * a[e];
    }
    for (uint32_t e = g->out_off[u]; e < g->out_off[u + 1]; e++) grad_w[e] = normalize ? (ga[e] - r) / W : ga[e];
  }
  free(a);
  free(xs);
  free(lam);
  free(nl);
  free(ga);
  return 0;
}

/* ============================================================== partitioner */
/* graphgrind/graph-numa.h:1287-1357 (partitionByDegree), :1208-1256
 * (cscpartitionByDegree); degrees[cnt] read as 0. */
static int or_greedy(const uint32_t* deg, uint64_t cnt, uint64_t m, int32_t P, int64_t* sizes) {
  int64_t* edges = (int64_t*)calloc((size_t)P, sizeof(int64_t));
  int64_t avg = (int64_t)m / P, counter = 0;
  int rc = 0;
  for (int p = 0; p < P; p++) sizes[p] = 0;
  for (uint64_t i = 0; i < cnt; i++) {
    edges[counter] += deg[i];
    sizes[counter]++;
    int64_t nx = i + 1 < cnt ? (int64_t)deg[i + 1] : 0;
    if (edges[counter] < avg && (double)(nx + edges[counter]) > 1.1 * (double)avg) counter++;
    if (counter >= P) {
      rc = -4;
      break;
    }
    if (edges[counter] >= avg && counter < P - 1) counter++;
  }
  if (!rc && counter + 1 != P) rc = -4;
  free(edges);
  return rc;
}
static int or_relabel(const uint32_t* indeg, uint64_t cnt, int32_t P, int64_t* sizes, int check) {
  int64_t counter = 0;
  for (int p = 0; p < P; p++) sizes[p] = 0;
  for (uint64_t j = 0; j < cnt; j++) {
    sizes[counter]++;
    if (j + 1 < cnt && indeg[j + 1] > indeg[j] && counter < P - 1) counter++;
  }
  return (check && counter + 1 != P) ? -4 : 0;
}
static void or_even(uint64_t cnt, int32_t P, int64_t* sizes) {
  int64_t chunk = 0;
  for (int i = 0; i < P - 1; i++) {
    sizes[i] = (int64_t)cnt / P;
    chunk += sizes[i];
  }
  sizes[P - 1] = (int64_t)cnt - chunk;
}

int or_partition_sizes(const uint32_t* in_deg, const uint32_t* out_deg, uint32_t n, uint64_t m, int32_t P,
                       int32_t balance, int32_t part_how, int32_t relabel, int64_t* coo, int64_t* csc) {
  int rc = 0;
  if (P < 1 || n < 1) return -1;
  if (balance == 1) {
    if (relabel) or_relabel(in_deg, n, P, coo, 0);
    else or_even(n, P, coo);
  } else {
    rc = relabel ? or_relabel(in_deg, n, P, coo, 1) : or_greedy(part_how ? out_deg : in_deg, n, m, P, coo);
  }
  if (rc) return rc;
  uint32_t* ci = (uint32_t*)malloc(sizeof(uint32_t) * n);
  uint32_t* co = (uint32_t*)malloc(sizeof(uint32_t) * n);
  uint64_t cn = 0;
  for (uint32_t i = 0; i < n; i++)
    if (in_deg[i]) {
      ci[cn] = in_deg[i];
      co[cn] = out_deg[i];
      cn++;
    }
  if (balance == 1) {
    if (relabel) or_relabel(ci, cn, P, csc, 0);
    else or_even(cn, P, csc);
  } else {
    rc = relabel ? or_relabel(ci, cn, P, csc, 1) : or_greedy(part_how ? co : ci, cn, m, P, csc);
  }
  free(ci);
  free(co);
  return rc;
}

/* HilbertEdgeSort::xy2d/rot, graphgrind/graph-numa.h:353-415 */
int64_t or_hilbert_key(int64_t side_edges, int64_t x, int64_t y) {
  uint64_t s64 = (uint64_t)side_edges;
  unsigned sh;
  int64_t n, s, d = 0;
  --s64;
  for (sh = 1; sh < 64; sh <<= 1) s64 |= s64 >> sh;
  ++s64;
  n = (int64_t)s64;
  for (s = n / 2; s > 0; s /= 2) {
    int64_t rx = (x & s) > 0, ry = (y & s) > 0;
    d += s * s * ((3 * rx) ^ ry);
    if (ry == 0) {
      if (rx == 1) {
        x = s - 1 - x;
        y = s - 1 - y;
      }
      {
        int64_t t = x;
        x = y;
        y = t;
      }
    }
  }
  return d;
}
