/*
 * ligra_b200_main.h -- the command-line driver of a GraphGrind application
 * compiled against ligra_b200.h: include it after the application source.
 *
 * parallel_main (graphgrind/ligra-numa.h:1095-1208) restated over the C
 * ABI: the same flags (-s symmetric, -b Galois binary, -r start (100),
 * -rounds (3), -p NUMA nodes (accepted, one GPU), -c partitions (384),
 * -P dest|source, -v edge|vertex, -o relabel), the graph read by
 * gg_host_graph_read and built by gg_graph_build with the given vertex ids,
 * then `rounds` calls of Compute(PG, start), each reported as
 * "Running : t" (seconds, the device finished), and "Average : t".  As in
 * the reference, graph load and partition build are outside the timed
 * region, and a directed graph is transposed back between rounds when
 * Compute left it transposed.
 */
#ifndef LIGRA_B200_MAIN_H
#define LIGRA_B200_MAIN_H

#undef inline

#ifndef LIGRA_B200_H
#error "include ligra_b200.h (as ligra-numa.h) and the application source first"
#endif

namespace lb {
inline const char* arg_value(int argc, char** argv, const char* flag) {
  for (int i = 1; i + 1 < argc; i++)
    if (!strcmp(argv[i], flag)) return argv[i + 1];
  return nullptr;
}
inline bool arg_flag(int argc, char** argv, const char* flag) {
  for (int i = 1; i < argc; i++)
    if (!strcmp(argv[i], flag)) return true;
  return false;
}

template <class vertex>
inline int run_rounds(gg_graph_t g, bool vertex_balanced, long start, long rounds) {
  partitioned_graph<vertex> PG(g, vertex_balanced);
  if (PG.transposed()) PG.transpose();
  double total = 0;
  for (long r = 0; r < rounds; r++) {
    sync();
    const auto t0 = std::chrono::steady_clock::now();
    Compute(PG, start);
    sync();
    const double t = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    total += t;
    std::cout << "Running : " << std::setprecision(6) << t << std::endl;
    if (PG.transposed()) PG.transpose();
  }
  std::cout << "Average : " << std::setprecision(6) << (rounds ? total / rounds : 0.0) << std::endl;
  PG.del();
  return 0;
}
}  // namespace lb

int main(int argc, char* argv[]) {
  if (argc < 2) {
    std::cerr << "usage: " << argv[0] << " [-s] [-b] [-r start] [-rounds R] [-c P] [-P dest|source] "
                                         "[-v edge|vertex] [-o] <graph>" << std::endl;
    return 1;
  }
  const char* path = argv[argc - 1];
  const bool symmetric = lb::arg_flag(argc, argv, "-s");
  const bool binary = lb::arg_flag(argc, argv, "-b");
  const char* r = lb::arg_value(argc, argv, "-r");
  const char* rr = lb::arg_value(argc, argv, "-rounds");
  const char* c = lb::arg_value(argc, argv, "-c");
  const char* ph = lb::arg_value(argc, argv, "-P");
  const char* ve = lb::arg_value(argc, argv, "-v");
  const long start = r ? atol(r) : 100;
  const long rounds = rr ? atol(rr) : 3;
  gg_build_opts o;
  memset(&o, 0, sizeof o);
  o.num_partitions = c ? atoi(c) : 384;
  o.order = GG_ORDER_HILBERT;
  o.relabel = lb::arg_flag(argc, argv, "-o") ? 1 : 0;
  if (ph && strcmp(ph, "dest") && strcmp(ph, "source")) {
    std::cerr << "Illegal value for -P: \"" << ph << "\". Allowed values: dest source. Default: dest\n";
    return 1;
  }
  o.part_how = ph && !strcmp(ph, "source") ? GG_PART_SOURCE : GG_PART_DEST;
  if (ve && strcmp(ve, "edge") && strcmp(ve, "vertex")) {
    std::cerr << "Illegal value for -v: \"" << ve << "\". Allowed values: edge vertex. Default: edge\n";
    return 1;
  }
  const bool vertex_balanced = ve && !strcmp(ve, "vertex");
  o.balance = vertex_balanced ? GG_BALANCE_VERTEX : GG_BALANCE_EDGE;
#ifdef WEIGHTED
  const int weighted = 1;
#else
  const int weighted = 0;
#endif
  gg_host_graph hg;
  if (gg_host_graph_read(path, binary, symmetric, weighted, &hg) != GG_OK) {
    std::cerr << gg_last_error_string() << std::endl;
    return 1;
  }
  gg_graph_t g;
  if (gg_graph_build(&hg, &o, &g) != GG_OK) {
    std::cerr << gg_last_error_string() << std::endl;
    gg_host_graph_free(&hg);
    return 1;
  }
  gg_host_graph_free(&hg);
  const int rc = symmetric ? lb::run_rounds<symmetricVertex>(g, vertex_balanced, start, rounds)
                           : lb::run_rounds<asymmetricVertex>(g, vertex_balanced, start, rounds);
  gg_graph_destroy(g);
  return rc;
}

#endif  // LIGRA_B200_MAIN_H
