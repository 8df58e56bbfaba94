// gg_run: the command-line driver, a flag-compatible replacement for
// parallel_main (graphgrind/ligra-numa.h:1094-1200) with the application
// named on the command line instead of linked in:
//
//   gg_run <App> [-s] [-b] [-r start] [-rounds R] [-p nodes] [-c P]
//          [-P dest|source] [-v edge|vertex] [-o] <inFile>
//
// App: BFS, BC, Components, PageRank, PageRankBit, PageRankDelta,
// PageRankConverage, SPMV, BellmanFord, BP.  Prints "Running : <seconds>" per round and
// "Average : <seconds>" like the reference timer (graphgrind/gettime.h:88-131);
// the time is the device time of the application's Compute() loop.  -p (NUMA
// nodes) is accepted and ignored.  BellmanFord and SPMV read weighted graphs,
// as the reference builds them with WEIGHTED.  BP uses seeded potentials
// (the reference leaves them uninitialised).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gg.h"

namespace {

int usage() {
  std::fprintf(stderr,
               "usage: gg_run <BFS|BC|Components|PageRank|PageRankBit|PageRankDelta|PageRankConverage|SPMV|BellmanFord|BP> "
               "[-s] [-b] [-r start] [-rounds R] [-p nodes] [-c P] [-P dest|source] [-v edge|vertex] [-o] <inFile>\n");
  return 1;
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) return usage();
  const std::string app = argv[1];
  bool symmetric = false, binary = false, relabel = false;
  long start = 100, rounds = 3, parts = 384;
  const char* part_how = nullptr;
  const char* vertex_edge = nullptr;
  const char* file = nullptr;
  for (int i = 2; i < argc; ++i) {
    const std::string a = argv[i];
    auto val = [&]() -> const char* { return i + 1 < argc ? argv[++i] : nullptr; };
    if (a == "-s") symmetric = true;
    else if (a == "-b") binary = true;
    else if (a == "-o") relabel = true;
    else if (a == "-r") { const char* v = val(); if (!v) return usage(); start = std::atol(v); }
    else if (a == "-rounds") { const char* v = val(); if (!v) return usage(); rounds = std::atol(v); }
    else if (a == "-p") { if (!val()) return usage(); }
    else if (a == "-c") { const char* v = val(); if (!v) return usage(); parts = std::atol(v); }
    else if (a == "-P") { part_how = val(); if (!part_how) return usage(); }
    else if (a == "-v") { vertex_edge = val(); if (!vertex_edge) return usage(); }
    else if (a[0] == '-') return usage();
    else file = argv[i];
  }
  if (!file) return usage();
  gg_build_opts o;
  std::memset(&o, 0, sizeof(o));
  o.num_partitions = (int32_t)parts;
  o.relabel = relabel;
  o.order = GG_ORDER_HILBERT;
  if (!part_how || !std::strcmp(part_how, "dest")) {
    o.part_how = GG_PART_DEST;
  } else if (!std::strcmp(part_how, "source")) {
    o.part_how = GG_PART_SOURCE;
  } else {
    std::fprintf(stderr, "Illegal value for -P: \"%s\". Allowed values: dest source. Default: dest\n", part_how);
    return 1;
  }
  if (!vertex_edge || !std::strcmp(vertex_edge, "edge")) {
    o.balance = GG_BALANCE_EDGE;
  } else if (!std::strcmp(vertex_edge, "vertex")) {
    o.balance = GG_BALANCE_VERTEX;
  } else {
    std::fprintf(stderr, "Illegal value for -v: \"%s\". Allowed values: edge vertex. Default: edge\n", vertex_edge);
    return 1;
  }
  const bool weighted = app == "BellmanFord" || app == "SPMV";
  gg_host_graph hg;
  std::memset(&hg, 0, sizeof(hg));
  std::fprintf(stderr, "Loading Graph \n");
  if (gg_host_graph_read(file, binary, symmetric, weighted, &hg) != GG_OK) {
    std::fprintf(stderr, "%s\n", gg_last_error_string());
    return 1;
  }
  gg_graph_t g = nullptr;
  if (gg_graph_build(&hg, &o, &g) != GG_OK) {
    std::fprintf(stderr, "%s\n", gg_last_error_string());
    gg_host_graph_free(&hg);
    return 1;
  }
  const uint32_t n = hg.n;
  const uint64_t m = hg.m;
  if (start < 0 || (uint64_t)start >= n) {
    std::fprintf(stderr, "start vertex %ld is not in [0, %u)\n", start, n);
    gg_graph_destroy(g);
    gg_host_graph_free(&hg);
    return 1;
  }
  std::vector<int32_t> i0(n), i1(n);
  std::vector<float> f0(2ull * n), f1(n), vp, ep;
  if (app == "BP") {
    uint64_t s = 7;
    vp.resize(2ull * n);
    ep.resize(4ull * m);
    for (auto& x : vp) x = 0.9f + 0.2f * (float)(splitmix(s) >> 40) / (float)(1u << 24);
    for (auto& x : ep) x = 0.45f + 0.1f * (float)(splitmix(s) >> 40) / (float)(1u << 24);
  }
  double total = 0;
  int rc = GG_OK;
  for (long r = 0; r < rounds && rc == GG_OK; ++r) {
    gg_run_stats st{};
    if (app == "BFS") rc = gg_bfs(g, (uint32_t)start, i0.data(), i1.data(), &st);
    else if (app == "BC") rc = gg_bc(g, (uint32_t)start, f0.data(), f1.data(), &st);
    else if (app == "Components") rc = gg_components(g, i0.data(), &st);
    else if (app == "PageRank") rc = gg_pagerank(g, 10, 0, f0.data(), &st);
    else if (app == "PageRankBit") rc = gg_pagerank(g, 10, 1, f0.data(), &st);
    else if (app == "PageRankDelta") rc = gg_pagerank_delta(g, f0.data(), &st);
    else if (app == "PageRankConverage") rc = gg_pagerank_converge(g, 100, 0.0000001, f0.data(), &st);
    else if (app == "SPMV") rc = gg_spmv(g, nullptr, f0.data(), &st);
    else if (app == "BellmanFord") rc = gg_bellman_ford(g, (uint32_t)start, i0.data(), &st);
    else if (app == "BP") rc = gg_bp(g, 10, vp.data(), ep.data(), f0.data(), &st);
    else {
      gg_graph_destroy(g);
      gg_host_graph_free(&hg);
      return usage();
    }
    if (rc == GG_OK) {
      std::printf("Running : %.6g\n", st.ms / 1e3);
      total += st.ms / 1e3;
    }
  }
  if (rc != GG_OK) {
    std::fprintf(stderr, "%s\n", gg_last_error_string());
  } else {
    std::printf("Average : %.6g\n", rounds > 0 ? total / rounds : 0.0);
  }
  gg_graph_destroy(g);
  gg_host_graph_free(&hg);
  return rc == GG_OK ? 0 : 1;
}
