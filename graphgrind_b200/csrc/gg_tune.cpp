// Autotuner: picks the engine's knobs for one application on one graph by
// timing it.  Runtime knobs (dense-pull layout policy, COO pull kernel,
// push/pull threshold m/div, and for Components on a symmetric graph the
// union-find pass) are searched on a built graph; build knobs
// (partition count, CTA tile size, COO window order) by building the graph
// once per candidate; the personalised-PageRank column count by timing one
// k-column pass per candidate k.  Every knob leaves edgeMap's results as they
// are (integer results bit-exact, FP32 sums up to their order), so tuning is
// safe to apply.  Written over the public C ABI only.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gg.h"
#include "gg_common.h"

namespace {

struct HostBufs {
  std::vector<int32_t> i0, i1;
  std::vector<float> f0, f1;
  explicit HostBufs(uint32_t n) : i0(n), i1(n), f0(n), f1(n) {}
};

// One run of `app`; *ms = its device time.
int run_app(gg_graph_t g, int32_t app, uint32_t start, HostBufs& b, double* ms) {
  gg_run_stats st{};
  int rc = GG_OK;
  switch (app) {
    case GG_APP_BFS:
      rc = gg_bfs(g, start, b.i0.data(), b.i1.data(), &st);
      break;
    case GG_APP_COMPONENTS:
      rc = gg_components(g, b.i0.data(), &st);
      break;
    case GG_APP_PAGERANK:
      rc = gg_pagerank(g, 10, 0, b.f0.data(), &st);
      break;
    case GG_APP_PAGERANK_DELTA:
      rc = gg_pagerank_delta(g, b.f0.data(), &st);
      break;
    case GG_APP_SPMV:
      rc = gg_spmv(g, nullptr, b.f0.data(), &st);
      break;
    case GG_APP_BELLMAN_FORD:
      rc = gg_bellman_ford(g, start, b.i0.data(), &st);
      break;
    case GG_APP_BC:
      rc = gg_bc(g, start, b.f0.data(), b.f1.data(), &st);
      break;
    default:
      return gg::fail(GG_ERR_INVALID_ARG, "autotune: unknown application %d", app);
  }
  *ms = st.ms;
  return rc;
}

int time_app(gg_graph_t g, int32_t app, uint32_t start, HostBufs& b, int reps, double* best) {
  double ms = 0;
  GG_TRY_HOST(run_app(g, app, start, b, &ms));  // warm-up
  *best = 1e300;
  for (int r = 0; r < reps; ++r) {
    GG_TRY_HOST(run_app(g, app, start, b, &ms));
    *best = std::min(*best, ms);
  }
  return GG_OK;
}

int set_knobs(gg_graph_t g, const gg_tune_trial& t) {
  GG_TRY_HOST(gg_graph_set_tuning(g, GG_TUNE_DENSE_POLICY, t.dense_policy));
  GG_TRY_HOST(gg_graph_set_tuning(g, GG_TUNE_COO_KERNEL, t.coo_kernel));
  GG_TRY_HOST(gg_graph_set_tuning(g, GG_TUNE_SPARSE_DIV, t.sparse_div));
  GG_TRY_HOST(gg_graph_set_tuning(g, GG_TUNE_CC_ALGO, t.cc_algo));
  return GG_OK;
}

}  // namespace

extern "C" {

int gg_autotune(gg_graph_t g, int32_t app, uint32_t start, gg_tune_trial* trials, int32_t max_trials,
                int32_t* n_trials) {
  gg_graph_info info{};
  GG_TRY_HOST(gg_graph_get_info(g, &info));
  if (start >= info.n) return gg::fail(GG_ERR_INVALID_ARG, "gg_autotune: start %u out of range", start);
  int64_t keep[4];
  GG_TRY_HOST(gg_graph_get_tuning(g, GG_TUNE_DENSE_POLICY, &keep[0]));
  GG_TRY_HOST(gg_graph_get_tuning(g, GG_TUNE_COO_KERNEL, &keep[1]));
  GG_TRY_HOST(gg_graph_get_tuning(g, GG_TUNE_SPARSE_DIV, &keep[2]));
  GG_TRY_HOST(gg_graph_get_tuning(g, GG_TUNE_CC_ALGO, &keep[3]));
  HostBufs bufs(info.n);
  std::vector<gg_tune_trial> tried;
  const bool has_coo = info.num_coo_tiles > 0;
  std::vector<int> kernels = {7, 6, 1, 5, 0};
  if (keep[1] == 4) kernels.push_back(4);  // lane-contiguous pull: graphs built with source-ordered windows
  const int policies[3] = {0, 1, 2};
  const int divs[3] = {20, 10, 40};
  auto restore = [&]() {
    gg_graph_set_tuning(g, GG_TUNE_DENSE_POLICY, keep[0]);
    gg_graph_set_tuning(g, GG_TUNE_COO_KERNEL, keep[1]);
    gg_graph_set_tuning(g, GG_TUNE_SPARSE_DIV, keep[2]);
    gg_graph_set_tuning(g, GG_TUNE_CC_ALGO, keep[3]);
  };
  for (int pol : policies) {
    if (pol == 2 && !has_coo) continue;
    for (int k : kernels) {
      if ((pol == 1 || !has_coo) && k != kernels[0]) continue;  // the COO kernel matters only where the COO runs
      for (int dv : divs) {
        gg_tune_trial t{};
        t.dense_policy = pol;
        t.coo_kernel = k;
        t.sparse_div = dv;
        int rc = set_knobs(g, t);
        if (!rc) rc = time_app(g, app, start, bufs, 3, &t.ms);
        if (rc) {
          const std::string keep_msg = gg_last_error_string();
          restore();
          return gg::fail(rc, "%s", keep_msg.c_str());
        }
        tried.push_back(t);
      }
    }
  }
  if (app == GG_APP_COMPONENTS && info.symmetric) {  // union-find: no edgeMap knob applies
    gg_tune_trial t{};
    t.dense_policy = 0;
    t.coo_kernel = kernels[0];
    t.sparse_div = 20;
    t.cc_algo = 1;
    int rc = set_knobs(g, t);
    if (!rc) rc = time_app(g, app, start, bufs, 3, &t.ms);
    if (rc) {
      const std::string keep_msg = gg_last_error_string();
      restore();
      return gg::fail(rc, "%s", keep_msg.c_str());
    }
    tried.push_back(t);
  }
  std::stable_sort(tried.begin(), tried.end(), [](const gg_tune_trial& a, const gg_tune_trial& b) { return a.ms < b.ms; });
  if (tried.empty()) {  // unreachable: policy 0 is always tried
    restore();
    return gg::fail(GG_ERR_UNSUPPORTED, "gg_autotune: no trial ran");
  }
  GG_TRY_HOST(set_knobs(g, tried[0]));
  if (trials)
    for (int32_t i = 0; i < max_trials && i < (int32_t)tried.size(); ++i) trials[i] = tried[i];
  if (n_trials) *n_trials = (int32_t)tried.size();
  return GG_OK;
}

int gg_autotune_build(const gg_host_graph* hg, int32_t app, uint32_t start, const gg_build_opts* candidates,
                      int32_t n_candidates, gg_build_opts* best_opts, gg_tune_trial* best) {
  if (!hg || !candidates || n_candidates <= 0 || !best_opts)
    return gg::fail(GG_ERR_INVALID_ARG, "gg_autotune_build: bad arguments");
  double best_ms = 1e300;
  int found = 0;
  std::string last;
  for (int32_t c = 0; c < n_candidates; ++c) {
    gg_graph_t g = nullptr;
    const int rc = gg_graph_build(hg, &candidates[c], &g);
    if (rc == GG_ERR_PARTITION) {  // the reference partitioner rejects this (graph, P): skip it
      last = gg_last_error_string();
      continue;
    }
    if (rc) return rc;
    gg_tune_trial t{};
    int32_t nt = 0;
    const int tr = gg_autotune(g, app, start, &t, 1, &nt);
    gg_graph_destroy(g);
    if (tr) return tr;
    t.partitions = candidates[c].num_partitions;
    t.tile_vertices = candidates[c].tile_vertices;
    t.tile_edges = candidates[c].tile_edges;
    t.coo_window = candidates[c].coo_window;
    if (t.ms < best_ms) {
      best_ms = t.ms;
      *best_opts = candidates[c];
      if (best) *best = t;
      found = 1;
    }
  }
  if (!found) return gg::fail(GG_ERR_PARTITION, "gg_autotune_build: no candidate could be built (%s)", last.c_str());
  return GG_OK;
}

int gg_autotune_ppr_k(gg_graph_t g, int32_t iters, int32_t* best_k, double* column_edges_per_s) {
  gg_graph_info info{};
  GG_TRY_HOST(gg_graph_get_info(g, &info));
  if (!best_k || iters < 1) return gg::fail(GG_ERR_INVALID_ARG, "gg_autotune_ppr_k: bad arguments");
  const int ks[3] = {1, 32, 64};
  double best_rate = -1;
  for (int k : ks) {
    std::vector<uint32_t> seeds(k);
    for (int j = 0; j < k; ++j) seeds[j] = (uint32_t)(((uint64_t)j * 2654435761u) % info.n);
    double ms = 1e300;
    for (int r = 0; r < 3; ++r) {
      gg_run_stats st{};
      GG_TRY_HOST(gg_ppr_k(g, k, iters, 0.85f, nullptr, seeds.data(), nullptr, &st));
      if (r) ms = std::min(ms, st.ms);
    }
    const double rate = (double)k * (double)info.m * iters / (ms * 1e-3);
    if (rate > best_rate) {
      best_rate = rate;
      *best_k = k;
    }
  }
  if (column_edges_per_s) *column_edges_per_s = best_rate;
  return GG_OK;
}

}  // extern "C"
