// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Builds one GraphGrind application straight from the reference source tree
// (the app's .C file and the graphgrind/ headers, included where they lie;
// nothing is copied) and adds two entry points beside the reference's own
// driver:
//   ref_<App> run  <reference flags> <graph>   -> the reference's parallel_main
//                                                 (graphgrind/ligra-numa.h:1095),
//                                                 prints "Running : t" lines
//   ref_<App> dump <out.bin> <flags> <graph>   -> re-runs the app's Compute()
//                                                 control flow with the
//                                                 reference's own functors,
//                                                 edgeMap/vertexMap/vertexFilter,
//                                                 and writes the result arrays
//   ref_<App> parts <out.bin> <flags> <graph>  -> partition sizes and the
//                                                 partitioned COO edge order
//
// The reference reads degrees[n] one past the end of a new[] array
// (graphgrind/graph-numa.h:1248, :1335).  Instead of editing the source, this
// file replaces operator new[] so that every array carries 64 zeroed bytes
// past its end; the read then yields 0, the same as the guard
// (i+1<n ? degrees[i+1] : 0).
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

void* operator new[](std::size_t sz) {
  void* p = std::malloc(sz + 64);
  if (!p) throw std::bad_alloc();
  std::memset(static_cast<char*>(p) + sz, 0, 64);
  return p;
}
void* operator new[](std::size_t sz, const std::nothrow_t&) noexcept {
  void* p = std::malloc(sz + 64);
  if (p) std::memset(static_cast<char*>(p) + sz, 0, 64);
  return p;
}
void operator delete[](void* p) noexcept { std::free(p); }
void operator delete[](void* p, std::size_t) noexcept { std::free(p); }

#define main gg_reference_main
#include GG_APP_FILE
#undef main

// ----------------------------------------------------------------- dumping
static FILE* g_out = nullptr;
static void put(const char* name, char type, const void* p, uint64_t count, size_t esize) {
  char hdr[24];
  std::memset(hdr, 0, sizeof hdr);
  std::strncpy(hdr, name, 15);
  hdr[16] = type;
  std::fwrite(hdr, 1, 24, g_out);
  std::fwrite(&count, 8, 1, g_out);
  if (count) std::fwrite(p, esize, count, g_out);
}
static void put_i64(const char* name, const intT* p, uint64_t n) {
  std::vector<int64_t> v(p, p + n);
  put(name, 'q', v.data(), n, 8);
}
static void put_f64(const char* name, const double* p, uint64_t n) { put(name, 'd', p, n, 8); }

// frontier trace entry: (dense?, d_m, num_out_edges)
struct Trace {
  std::vector<int64_t> v;
  void add(partitioned_vertices& f) {
    v.push_back(f.has_dense ? 1 : 0);
    v.push_back(f.d_m);
    v.push_back(f.num_out_edges);
  }
  void put_as(const char* name) { put(name, 'q', v.data(), v.size(), 8); }
};

static void mark_levels(partitioned_vertices& out, intT n, std::vector<int32_t>& lev, int32_t round) {
  if (out.isEmpty()) return;
  if (out.has_dense) {
    for (intT i = 0; i < n; i++)
      if (out.d[i] && lev[i] < 0) lev[i] = round;
  } else {
    for (intT k = 0; k < out.d_m; k++)
      if (lev[out.s[k]] < 0) lev[out.s[k]] = round;
  }
}

// ----------------------------------------------------------- replays
// Each replay repeats the named Compute() loop step for step, with the
// reference's functor structs and engine calls, and dumps the arrays that
// Compute() frees before returning.
#if defined(GG_APP_BFS)
template <class G>
static void replay(G& GA, long start) {  // app/BFS.C:77-101
  const intT n = GA.n, m = GA.m;
  const partitioner& part = GA.get_partitioner();
  mmap_ptr<intT> Parents;
  Parents.part_allocate(part);
  map_vertexL(part, [&](intT j) { Parents[j] = -1; });
  Parents[start] = start;
  std::vector<int32_t> lev(n, -1);
  lev[start] = 0;
  Trace tr;
  partitioned_vertices F = partitioned_vertices::create(n, start, GA.get_partition().V[start].getOutDegree());
  int32_t round = 0;
  while (!F.isEmpty()) {
    partitioned_vertices out = edgeMap(GA, F, BFS_F(Parents), m / 20);
    round++;
    tr.add(out);
    mark_levels(out, n, lev, round);
    F.del();
    F = out;
  }
  F.del();
  put_i64("parents", Parents.get(), n);
  put("levels", 'i', lev.data(), n, 4);
  tr.put_as("trace");
  Parents.del();
}
#elif defined(GG_APP_CC)
template <class G>
static void replay(G& GA, long) {  // app/Components.C:101-126
  const intT n = GA.n, m = GA.m;
  const partitioner& part = GA.get_partitioner();
  mmap_ptr<intT> IDs, prevIDs;
  IDs.part_allocate(part);
  prevIDs.part_allocate(part);
  map_vertexL(part, [&](intT j) { IDs[j] = j; });
  Trace tr;
  partitioned_vertices F = partitioned_vertices::bits(part, n, m);
  while (!F.isEmpty()) {
    vertexMap(part, F, CC_Vertex_F(IDs, prevIDs));
    partitioned_vertices out = edgeMap(GA, F, CC_F(IDs, prevIDs), m / 20);
    tr.add(out);
    F.del();
    F = out;
  }
  F.del();
  put_i64("ids", IDs.get(), n);
  tr.put_as("trace");
  IDs.del();
  prevIDs.del();
}
#elif defined(GG_APP_PR) || defined(GG_APP_PRBIT)
template <class G>
static void replay(G& GA, long) {  // app/PageRank.C:102-150, app/PageRankBit.C:103-151
  typedef typename G::vertex_type vertex;
  const partitioner& part = GA.get_partitioner();
  graph<vertex>& WG = GA.get_partition();
  const intT n = GA.n, m = GA.m;
  const double damping = 0.85, epsilon = 0.0000001;
  double one_over_n = 1 / (double)n;
  mmap_ptr<double> p_curr, p_next;
  p_curr.part_allocate(part);
  p_next.part_allocate(part);
  map_vertexL(part, [&](intT j) { p_curr[j] = one_over_n; });
  map_vertexL(part, [&](intT j) { p_next[j] = 0; });
  std::vector<double> ranks(n);
  Trace tr;
  int count = 0;
  partitioned_vertices F = partitioned_vertices::bits(part, n, m);
  while (count < MaxIter) {
    count++;
    partitioned_vertices out = edgeMap(GA, F, PR_F<vertex>(p_curr, p_next, WG.V), m / 20);
    vertexMap(part, F, PR_Vertex_F(p_curr, p_next, damping, n));
    for (intT j = 0; j < n; j++) ranks[j] = p_next[j];
    tr.add(out);
    map_vertexL(part, [&](intT j) { p_curr[j] = fabs(p_curr[j] - p_next[j]); });
    double L1 = sequence::plusReduce(p_curr.get(), n);
    if (L1 < epsilon) break;
    vertexMap(part, F, PR_Vertex_Reset(p_curr));
    swap(p_curr, p_next);
    F.del();
#if defined(GG_APP_PRBIT)
    out.bit = true;
#endif
    F = out;
  }
  F.del();
  put_f64("ranks", ranks.data(), n);
  tr.put_as("trace");
  p_curr.del();
  p_next.del();
}
#elif defined(GG_APP_PRC)
template <class G>
static void replay(G& GA, long) {  // app/PageRankConverage.C:235-315
  typedef typename G::vertex_type vertex;
  const partitioner& part = GA.get_partitioner();
  graph<vertex>& WG = GA.get_partition();
  const intT n = GA.n, m = GA.m;
  const double epsilon = 0.0000001;
  double one_over_n = 1 / (double)n;
  mmap_ptr<double> p_curr, p_next, edge_factor, add_factor;
  p_curr.part_allocate(part);
  p_next.part_allocate(part);
  edge_factor.part_allocate(part);
  add_factor.part_allocate(part);
  map_vertexL(part, [&](intT j) { p_curr[j] = one_over_n; });
  map_vertexL(part, [&](intT j) { p_next[j] = 0; });
  map_vertexL(part, [&](intT j) { edge_factor[j] = (double)0.85 / (WG.V[j].getOutDegree()); });
  int count = 0;
  double L1_norm = 2;
  std::vector<double> l1s;
  partitioned_vertices F = partitioned_vertices::bits(part, n, m);
  while (count < MaxIter && L1_norm > epsilon) {
    map_vertexL(part, [&](intT j) { add_factor[j] = (double)edge_factor[j] * p_curr[j]; });
    partitioned_vertices out = edgeMap(GA, F, PR_F<vertex>(p_curr, p_next, WG.V, add_factor), m / 20);
    vertexMap(part, F, PR_Vertex_Csum(p_next, sum(part, p_next, n, 1), n));
    L1_norm = normdiff(part, p_curr, p_next, n);
    l1s.push_back(L1_norm);
    vertexMap(part, F, PR_Vertex_norm(p_next, sum(part, p_next, n, 0), n));
    vertexMap(part, F, PR_Vertex_Reset(p_curr));
    count++;
    swap(p_curr, p_next);
    out.del();
  }
  F.del();
  put_f64("ranks", p_curr.get(), n);
  put_f64("l1", l1s.data(), l1s.size());
  p_curr.del();
  p_next.del();
  edge_factor.del();
  add_factor.del();
}
#elif defined(GG_APP_PRD)
template <class G>
static void replay(G& GA, long) {  // app/PageRankDelta.C:120-174
  typedef typename G::vertex_type vertex;
  const partitioner& part = GA.get_partitioner();
  const double damping = 0.85, epsilon = 0.0000001, epsilon2 = 0.01;
  const intT n = GA.n, m = GA.m;
  double one_over_n = 1 / (double)n;
  mmap_ptr<double> p, nghSum, Delta;
  p.part_allocate(part);
  nghSum.part_allocate(part);
  Delta.part_allocate(part);
  map_vertexL(part, [&](intT j) { p[j] = 0.0; });
  map_vertexL(part, [&](intT j) { Delta[j] = one_over_n; });
  map_vertexL(part, [&](intT j) { nghSum[j] = 0.0; });
  partitioned_vertices F = partitioned_vertices::bits(part, n, m);
  partitioned_vertices All = partitioned_vertices::bits(part, n, m);
  Trace tr;
  intT round = 0;
  while (1) {
    round++;
    partitioned_vertices out = edgeMap(GA, F, PR_F<vertex>(GA.get_partition().V, Delta, nghSum), m / 20);
    out.del();
    partitioned_vertices active =
        (round == 1) ? vertexFilter(GA, All, PR_Vertex_F_FirstRound(p, Delta, nghSum, damping, one_over_n, epsilon2))
                     : vertexFilter(GA, All, PR_Vertex_F(p, Delta, nghSum, damping, epsilon2));
    tr.add(active);
    map_vertexL(part, [&](intT j) { nghSum[j] = fabs(Delta[j]); });
    double L1 = sequence::plusReduce(nghSum.get(), n);
    if (L1 < epsilon) break;
    vertexMap(part, All, PR_Vertex_Reset(nghSum));
    F.del();
    F = active;
  }
  F.del();
  put_f64("ranks", p.get(), n);
  tr.put_as("trace");
  p.del();
  Delta.del();
  nghSum.del();
}
#elif defined(GG_APP_SPMV)
template <class G>
static void replay(G& GA, long) {  // app/SPMV.C:64-92
  typedef typename G::vertex_type vertex;
  const partitioner& part = GA.get_partitioner();
  const intT n = GA.n, m = GA.m;
  double one_over_n = 1 / (double)n;
  mmap_ptr<double> p_curr, p_next;
  p_curr.part_allocate(part);
  p_next.part_allocate(part);
  map_vertexL(part, [&](intT j) { p_curr[j] = one_over_n; });
  map_vertexL(part, [&](intT j) { p_next[j] = 0; });
  partitioned_vertices F = partitioned_vertices::bits(part, n, m);
  partitioned_vertices out = edgeMap(GA, F, SPMV_F<vertex>(p_curr, p_next), m / 20);
  vertexMap(part, F, SPMV_Vertex_Reset(p_curr));
  swap(p_curr, p_next);
  put_f64("y", p_curr.get(), n);
  F.del();
  p_curr.del();
  p_next.del();
}
#elif defined(GG_APP_BF)
template <class G>
static void replay(G& GA, long start) {  // app/BellmanFord.C:106-145
  const intT n = GA.n, m = GA.m;
  const partitioner& part = GA.get_partitioner();
  mmap_ptr<intT> SP, Visited;
  SP.part_allocate(part);
  map_vertexL(part, [&](intT j) { SP[j] = INT_MAX / 2; });
  SP[start] = 0;
  Visited.part_allocate(part);
  map_vertexL(part, [&](intT j) { Visited[j] = 0; });
  partitioned_vertices F = partitioned_vertices::create(n, start, GA.get_partition().V[start].getOutDegree());
  intT round = 0;
  while (!F.isEmpty()) {
    if (round == n) {
      map_vertexL(part, [&](intT j) { SP[j] = -(INT_MAX / 2); });
      break;
    }
    partitioned_vertices out = edgeMap(GA, F, BF_F(SP, Visited), m / 20);
    vertexMap(part, out, BF_Vertex_F(Visited));
    F.del();
    F = out;
    round++;
  }
  F.del();
  put_i64("dist", SP.get(), n);
  SP.del();
  Visited.del();
}
#elif defined(GG_APP_BC)
template <class G>
static void replay(G& GA, long start) {  // app/BC.C:156-226
  const partitioner& part = GA.get_partitioner();
  const intT n = GA.n, m = GA.m;
  mmap_ptr<fType> NumPaths;
  NumPaths.part_allocate(part);
  mmap_ptr<bool> Visited;
  Visited.part_allocate(part);
  map_vertexL(part, [&](intT j) { NumPaths[j] = 0.0; });
  map_vertexL(part, [&](intT j) { Visited[j] = false; });
  NumPaths[start] = 1.0;
  Visited[start] = true;
  partitioned_vertices F = partitioned_vertices::create(n, start, GA.get_partition().V[start].getOutDegree());
  vector<partitioned_vertices> Levels;
  Levels.push_back(F);
  intT round = 0;
  while (!F.isEmpty()) {
    round++;
    partitioned_vertices out = edgeMap(GA, F, BC_F(NumPaths, Visited), m / 20);
    vertexMap(part, out, BC_Vertex_F(Visited));
    Levels.push_back(out);
    F = out;
  }
  std::vector<double> np(NumPaths.get(), NumPaths.get() + n);
  mmap_ptr<fType> Dependencies;
  Dependencies.part_allocate(part);
  map_vertexL(part, [&](intT j) { Dependencies[j] = 0.0; });
  mmap_ptr<fType> inverseNumPaths;
  inverseNumPaths = NumPaths;
  map_vertexL(part, [&](intT j) { inverseNumPaths[j] = 1 / inverseNumPaths[j]; });
  Levels[round].del();
  map_vertexL(part, [&](intT j) { Visited[j] = false; });
  F = Levels[round - 1];
  vertexMap(part, F, BC_Back_Vertex_F(Visited, Dependencies, inverseNumPaths));
  GA.transpose();
  for (intT r = round - 2; r >= 0; r--) {
    partitioned_vertices out = edgeMap(GA, F, BC_Back_F(Dependencies, Visited), m / 20);
    out.del();
    F.del();
    F = Levels[r];
    vertexMap(part, F, BC_Back_Vertex_F(Visited, Dependencies, inverseNumPaths));
  }
  F.del();
  map_vertexL(part, [&](intT j) { Dependencies[j] = (Dependencies[j] - inverseNumPaths[j]) / inverseNumPaths[j]; });
  std::vector<double> dep(Dependencies.get(), Dependencies.get() + n);
  put_f64("dependencies", dep.data(), n);
  put_f64("num_paths", np.data(), n);
  GA.transpose();
  inverseNumPaths.del();
  Visited.del();
  Dependencies.del();
}
#else
template <class G>
static void replay(G&, long) {}
#endif

template <class G>
static void dump_parts(G& PG) {
  const partitioner& cp = PG.get_coo_partitioner();
  const partitioner& sp = PG.get_partition().get_csc_partitioner();
  const int P = cp.get_num_partitions();
  std::vector<int64_t> a(P), b(P);
  for (int p = 0; p < P; p++) {
    a[p] = cp.get_size(p);
    b[p] = sp.get_size(p);
  }
  put("coo_sizes", 'q', a.data(), P, 8);
  put("csc_sizes", 'q', b.data(), P, 8);
  if (!PG.part_ver) {
    std::vector<int64_t> src, dst, bounds;
    bounds.push_back(0);
    for (int p = 0; p < P; p++) {
      const auto& el = PG.get_edge_list_partition(p);
      for (auto it = el.cbegin(); it != el.cend(); ++it) {
        src.push_back(it->getSource());
        dst.push_back(it->getDestination());
      }
      bounds.push_back((int64_t)src.size());
    }
    put("coo_src", 'q', src.data(), src.size(), 8);
    put("coo_dst", 'q', dst.data(), dst.size(), 8);
    put("coo_bounds", 'q', bounds.data(), bounds.size(), 8);
  }
}

template <class V>
static int dump_mode(commandLine& P, const char* out, bool parts_only) {
  char* iFile = P.getArgument(0);
  bool symmetric = P.getOptionValue("-s");
  bool binary = P.getOptionValue("-b");
  long start = P.getOptionLongValue("-r", 100);
  int numOfCoo = P.getOptionLongValue("-c", 384);
  char* part_how = P.getOptionValue("-P");
  char* vertex_edge = P.getOptionValue("-v");
  bool relabel = P.getOptionValue("-o");
  bool part_src = part_how && !strcmp(part_how, "source");
  bool part_vertex = vertex_edge && !strcmp(vertex_edge, "vertex");
  g_out = std::fopen(out, "wb");
  if (!g_out) return 2;
  wholeGraph<V> G = readGraph<V>(iFile, symmetric, binary);
  partitioned_graph<V> PG(G, numOfCoo, part_src, part_vertex, relabel);
  if (PG.transposed()) PG.transpose();
  if (parts_only) dump_parts(PG);
  else replay(PG, start);
  std::fclose(g_out);
  PG.del();
  G.del();
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s run <flags> <graph> | dump <out> <flags> <graph> | parts <out> <flags> <graph>\n",
                 argv[0]);
    return 2;
  }
  if (!std::strcmp(argv[1], "run")) {
    argv[1] = argv[0];
    return gg_reference_main(argc - 1, argv + 1);
  }
  if ((!std::strcmp(argv[1], "dump") || !std::strcmp(argv[1], "parts")) && argc >= 4) {
    const bool parts_only = !std::strcmp(argv[1], "parts");
    const char* out = argv[2];
    argv[2] = argv[0];
    commandLine P(argc - 2, argv + 2, " [-s] <inFile>");
    if (P.getOptionValue("-s")) return dump_mode<symmetricVertex>(P, out, parts_only);
    return dump_mode<asymmetricVertex>(P, out, parts_only);
  }
  std::fprintf(stderr, "unknown mode %s\n", argv[1]);
  return 2;
}
