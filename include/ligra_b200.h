/*
 * ligra_b200.h -- source-compatible front end of the B200 engine for
 * GraphGrind application sources.
 *
 * A GraphGrind application is a C++ file that includes "ligra-numa.h",
 * defines its edge and vertex functors and a `template <class G> void
 * Compute(G&, long)` loop over edgeMap / vertexMap / vertexFilter.  This
 * header stands in for "ligra-numa.h" (graphgrind/ligra-numa.h and the
 * headers it includes): the same names, argument meanings and value
 * semantics, with every edgeMap and vertexMap running on the GPU and the
 * application's own functor structs executing inside the kernels.  An
 * application source compiles with nvcc unchanged; the only layer is the
 * macro at the end of this header that makes the functors' `inline` member
 * functions `__host__ __device__`.  ligra_b200_main.h supplies the
 * command-line driver (parallel_main, graphgrind/ligra-numa.h:1095-1208).
 *
 *   nvcc -x cu -std=c++17 -DLONG --expt-relaxed-constexpr -I include \
 *        -gencode arch=compute_100a,code=sm_100a  app_main.cu -lgg
 *   where app_main.cu is:  #include "BFS.C"  #include "ligra_b200_main.h"
 *   and "ligra-numa.h", found beside BFS.C first, is this file.
 *
 * What maps to what:
 *   partitioned_graph<V>  (graph-numa.h:642-728)  a gg_graph_t built by the
 *       library (device CSR + CSC, the -c partitions); V[] holds each
 *       vertex's degrees in managed memory
 *   partitioned_vertices  (ligra-numa.h:91-272)   dense bool[n] and/or
 *       sparse intT list in managed memory, d_m, num_out_edges, bit
 *   edgeMap               (ligra-numa.h:919-1019)  the same direction rule:
 *       m_f + outdeg(F) > threshold (m/20 by default) pulls over the CSC
 *       (edgeMapDenseCSC, :549-729: per destination, cond, the functor's cache
 *       protocol or update, early exit once cond turns false), otherwise
 *       pushes over the CSR (edgeMapSparseWithG, :868-916: cond &&
 *       updateAtomic per out-edge).  The reference's third branch, the
 *       partitioned COO above m/2, also pulls over the CSC here: for a
 *       destination-owned update both give the same edgeMap result, and
 *       the library's applications (gg.h) are the path with the tuned COO
 *       kernels.  A vertex reached by several pushes enters the sparse
 *       output once.
 *   vertexMap / vertexFilter (ligra-numa.h:1023-1082)  one kernel over the
 *       members, the functor called once per member
 *   map_vertexL / map_partitionL (partitioner.h:337-387)  run on the host,
 *       as the applications' lambdas capture host references; every host
 *       loop first waits for the device
 *   mmap_ptr<T> (mm.h:246-324)  a managed-memory array with the same manual
 *       del(); sequence::plusReduce, CAS, writeMin, writeAdd, cond_true
 *       (utils.h) work on the host and, for the atomics, on the device.
 *
 * Errors: like the reference, a fatal condition prints to stderr and
 * aborts (CUDA errors included).  Dump mode: with LIGRA_B200_DUMP=<file>,
 * every application array of n elements released by mmap_ptr::del() is
 * appended to <file> (16-byte name "del<k>", type char, u64 count, data) in
 * the order of release, so that tests can read the results a Compute()
 * computes and frees.
 */
#ifndef LIGRA_B200_H
#define LIGRA_B200_H

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <iomanip>
#include <iostream>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "gg.h"

using namespace std;

#ifdef LONG
typedef long intT;
typedef unsigned long uintT;
#else
typedef int intT;
typedef unsigned int uintT;
#endif
typedef int intE;
typedef unsigned int uintE;

#define newA(__E, __n) (__E*)malloc((__n) * sizeof(__E))
#define parallel_for for
#define parallel_for_1 for
#define parallel_for_256 for

enum options { DENSE, DENSE_FORWARD };

namespace lb {

inline void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::cerr << "ligra_b200: " << what << ": " << cudaGetErrorString(e) << std::endl;
    abort();
  }
}
#define LB_CUDA(x) ::lb::cuda_check((x), #x)

inline void sync() { LB_CUDA(cudaDeviceSynchronize()); }

template <class T>
inline T* alloc(size_t count) {
  void* p = nullptr;
  LB_CUDA(cudaMallocManaged(&p, (count ? count : 1) * sizeof(T)));
  return static_cast<T*>(p);
}

inline void release(void* p) {
  if (p) {
    sync();
    LB_CUDA(cudaFree(p));
  }
}

constexpr int kThreads = 256;
inline unsigned grid_for(uint64_t items) {
  uint64_t b = (items + kThreads - 1) / kThreads;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(b, 148ull * 32));
}

// ----------------------------------------------------------- dump mode
inline FILE* dump_file() {
  static FILE* f = nullptr;
  static bool opened = false;
  if (!opened) {
    opened = true;
    const char* p = getenv("LIGRA_B200_DUMP");
    if (p && *p) f = fopen(p, "ab");
  }
  return f;
}
inline int& dump_seq() {
  static int k = 0;
  return k;
}
template <class T>
inline void dump(const T* p, uint64_t count) {
  FILE* f = dump_file();
  if (!f || !p) return;
  char type = 'B';
  if (std::is_floating_point<T>::value)
    type = sizeof(T) == 8 ? 'd' : 'f';
  else if (sizeof(T) == 8)
    type = 'q';
  else if (sizeof(T) == 4)
    type = 'i';
  char hdr[24];
  memset(hdr, 0, sizeof hdr);
  snprintf(hdr, 16, "del%d", dump_seq()++);
  hdr[16] = type;
  fwrite(hdr, 1, 24, f);
  fwrite(&count, 8, 1, f);
  fwrite(p, sizeof(T), count, f);
  fflush(f);
}

}  // namespace lb

// ============================================================ partitioner
// partitioner (graphgrind/partitioner.h:38-200): P destination ranges of the
// vertex set; one memory domain here, so every partition is "per node".
class partitioner {
 public:
  int num_partitions = 1;
  intT elements = 0;
  std::vector<intT> starts;
  partitioner() {}
  partitioner(int P, intT n) : num_partitions(P), elements(n), starts(P + 1, 0) { starts[P] = n; }
  int get_num_partitions() const { return num_partitions; }
  int get_num_per_node_partitions() const { return num_partitions; }
  intT get_num_elements() const { return elements; }
  intT start_of(int p) const { return starts[p]; }
  intT get_size(int p) const { return starts[p + 1] - starts[p]; }
};

// map_vertexL / map_partitionL (graphgrind/partitioner.h:337-387): host
// loops (the applications' lambdas capture host references).
template <class F>
inline void map_vertexL(const partitioner& part, F f) {
  lb::sync();
  const intT n = part.get_num_elements();
  for (intT j = 0; j < n; j++) f(j);
}
template <class F>
inline void map_partitionL(const partitioner& part, F f) {
  lb::sync();
  for (int p = 0; p < part.get_num_partitions(); p++) f(p);
}

// ================================================================ mmap_ptr
// mmap_ptr<T> (graphgrind/mm.h:246-324): a raw owner with manual del() and
// shallow copies; the storage is managed memory, so the host loops and the
// kernels both index it.
template <typename T>
class mmap_ptr {
  T* mem = nullptr;
  size_t count = 0;
  bool app = false;  // allocated by the application (dumped on del in dump mode)

 public:
  mmap_ptr() {}
  mmap_ptr(const partitioner& part) { part_allocate(part); }
  mmap_ptr(size_t elements) { Interleave_allocate(elements); }
  mmap_ptr(size_t elements, size_t) { Interleave_allocate(elements); }
  void part_allocate(const partitioner& part) { take(part.get_num_elements(), true); }
  void Interleave_allocate(size_t elements) { take(elements, true); }
  void local_allocate(size_t elements, int) { take(elements, true); }
  void internal_allocate(size_t elements) { take(elements, false); }
  void del() {
    if (mem) {
      lb::sync();
      if (app) lb::dump(mem, count);
      lb::release(mem);
    }
    mem = nullptr;
    count = 0;
  }
  operator T*() const { return mem; }
  operator bool() const { return mem != nullptr; }
  size_t get_bytes() const { return count * sizeof(T); }
  T* get() const { return mem; }

 private:
  void take(size_t elements, bool by_app) {
    mem = lb::alloc<T>(elements);
    count = elements;
    app = by_app;
  }
};

// ============================================================ the graph
// symmetricVertex / asymmetricVertex (graphgrind/graph-numa.h:39-217): the
// degrees the functors ask for; neighbour lists live in the library's CSR/CSC.
struct symmetricVertex {
  uint32_t out_deg = 0, in_deg = 0;
  __host__ __device__ intT getOutDegree() const { return out_deg; }
  __host__ __device__ intT getInDegree() const { return in_deg; }
  __host__ __device__ void setOutDegree(intT d) { out_deg = (uint32_t)d; }
  __host__ __device__ void setInDegree(intT d) { in_deg = (uint32_t)d; }
};
struct asymmetricVertex : symmetricVertex {};

namespace lb {
static __global__ void k_degrees(const uint32_t* out_off, const uint32_t* in_off, symmetricVertex* V, intT n) {
  for (intT v = blockIdx.x * (intT)blockDim.x + threadIdx.x; v < n; v += (intT)gridDim.x * blockDim.x) {
    V[v].out_deg = out_off[v + 1] - out_off[v];
    V[v].in_deg = in_off[v + 1] - in_off[v];
  }
}
}  // namespace lb

// graph<vertex> (the CSC view, graphgrind/graph-numa.h:500-620)
template <class vertex>
class graph {
 public:
  vertex* V = nullptr;
  intT n = 0, m = 0;
  const uint32_t *out_off = nullptr, *out_idx = nullptr, *in_off = nullptr, *in_idx = nullptr;
  const intE *out_w = nullptr, *in_w = nullptr;
  partitioner csc_part;
  const partitioner& get_csc_partitioner() const { return csc_part; }
};

// partitioned_graph (graphgrind/graph-numa.h:642-728)
template <class vertex>
class partitioned_graph {
 public:
  typedef vertex vertex_type;
  intT n = 0, m = 0;
  bool part_ver = false;
  bool source = false;
  gg_graph_t h = nullptr;
  partitioner part;
  graph<vertex> G;

  partitioned_graph() {}
  // Wraps a graph built by gg_graph_build (given vertex ids).
  explicit partitioned_graph(gg_graph_t g, bool vertex_balanced = false) : h(g), part_ver(vertex_balanced) {
    gg_graph_info info;
    if (gg_graph_get_info(g, &info) != GG_OK) {
      std::cerr << "partitioned_graph: " << gg_last_error_string() << std::endl;
      abort();
    }
    n = info.n;
    m = (intT)info.m;
    part = partitioner(info.num_partitions, n);
    std::vector<int64_t> st(info.num_partitions + 1);
    gg_graph_partition_starts(g, st.data());
    for (int p = 0; p <= info.num_partitions; p++) part.starts[p] = (intT)st[p];
    G.n = n;
    G.m = m;
    G.csc_part = part;
    G.V = lb::alloc<vertex>(n);
    refresh();
  }
  // Re-reads the orientation's device lists and degrees (after transpose).
  void refresh() {
    gg_graph_device_arrays(h, &G.out_off, &G.out_idx, &G.in_off, &G.in_idx);
    const void *ow = nullptr, *iw = nullptr;
    gg_graph_device_weights(h, &ow, &iw);
    G.out_w = static_cast<const intE*>(ow);
    G.in_w = static_cast<const intE*>(iw);
    lb::k_degrees<<<lb::grid_for(n), lb::kThreads>>>(G.out_off, G.in_off, G.V, n);
    LB_CUDA(cudaGetLastError());
    lb::sync();
  }
  const partitioner& get_partitioner() const { return part; }
  const partitioner& get_coo_partitioner() const { return part; }
  graph<vertex>& get_partition() { return G; }
  bool transposed() const {
    int64_t t = 0;
    gg_graph_info info;
    if (gg_graph_get_info(h, &info) == GG_OK) t = info.transposed;
    return t != 0;
  }
  void transpose() {
    gg_graph_transpose(h);
    refresh();
  }
  void del() {
    lb::release(G.V);
    G.V = nullptr;
  }
};

// ================================================= utils.h arithmetic
__host__ __device__ inline bool cond_true(intT) { return 1; }

// CAS / writeMin / writeAdd (graphgrind/utils.h:423-477) on the host (GCC
// builtins, as the reference) and on the device (atomicCAS).
template <class ET>
__host__ __device__ inline bool CAS(ET* ptr, ET oldv, ET newv) {
  static_assert(sizeof(ET) == 8 || sizeof(ET) == 4, "CAS bad length");
#ifdef __CUDA_ARCH__
  if (sizeof(ET) == 8) {
    unsigned long long o, nw;
    memcpy(&o, &oldv, 8);
    memcpy(&nw, &newv, 8);
    return atomicCAS(reinterpret_cast<unsigned long long*>(ptr), o, nw) == o;
  } else {
    unsigned int o, nw;
    memcpy(&o, &oldv, 4);
    memcpy(&nw, &newv, 4);
    return atomicCAS(reinterpret_cast<unsigned int*>(ptr), o, nw) == o;
  }
#else
  if (sizeof(ET) == 8) {
    long o, nw;
    memcpy(&o, &oldv, 8);
    memcpy(&nw, &newv, 8);
    return __sync_bool_compare_and_swap(reinterpret_cast<long*>(ptr), o, nw);
  } else {
    int o, nw;
    memcpy(&o, &oldv, 4);
    memcpy(&nw, &newv, 4);
    return __sync_bool_compare_and_swap(reinterpret_cast<int*>(ptr), o, nw);
  }
#endif
}

template <class ET>
__host__ __device__ inline bool writeMin(ET* a, ET b) {
  ET c;
  bool r = 0;
  do c = *(volatile ET*)a;
  while (c > b && !(r = CAS(a, c, b)));
  return r;
}

template <class ET>
__host__ __device__ inline void writeAdd(ET* a, ET b) {
  ET o, nw;
  do {
    o = *(volatile ET*)a;
    nw = o + b;
  } while (!CAS(a, o, nw));
}

template <class ET>
__host__ __device__ inline void writeOr(ET* a, ET b) {
  ET o, nw;
  do {
    o = *(volatile ET*)a;
    nw = o | b;
  } while (o != nw && !CAS(a, o, nw));
}

namespace lb {
template <class T>
__global__ void k_sum(const T* a, intT n, double* out) {
  double s = 0;
  for (intT i = blockIdx.x * (intT)blockDim.x + threadIdx.x; i < n; i += (intT)gridDim.x * blockDim.x) s += a[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}
}  // namespace lb

namespace sequence {
// plusReduce (graphgrind/utils.h:192): a device reduction for arrays the
// device can read (managed or device memory), a host loop otherwise.
template <class OT>
inline OT plusReduce(OT* A, intT n) {
  lb::sync();
  cudaPointerAttributes at;
  const bool dev = cudaPointerGetAttributes(&at, A) == cudaSuccess &&
                   (at.type == cudaMemoryTypeManaged || at.type == cudaMemoryTypeDevice);
  cudaGetLastError();
  if (dev && std::is_arithmetic<OT>::value) {
    double* acc = lb::alloc<double>(1);
    *acc = 0;
    lb::k_sum<<<lb::grid_for(n), lb::kThreads>>>(A, n, acc);
    LB_CUDA(cudaGetLastError());
    lb::sync();
    const OT r = (OT)*acc;
    lb::release(acc);
    return r;
  }
  OT r = 0;
  for (intT i = 0; i < n; i++) r += A[i];
  return r;
}
}  // namespace sequence

// ======================================================== vertexSubset
// partitioned_vertices (graphgrind/ligra-numa.h:91-272)
class partitioned_vertices {
 public:
  intT numVertices = 0;
  intT d_m = 0;
  mmap_ptr<bool> d;
  bool has_dense = false;
  intT* s = nullptr;
  intT num_out_edges = 0;
  bool bit = false;

  static partitioned_vertices create(intT n, intT v, intT initialOutdegree) {
    partitioned_vertices pv;
    pv.numVertices = n;
    pv.d_m = 1;
    pv.s = lb::alloc<intT>(1);
    pv.s[0] = v;
    pv.num_out_edges = initialOutdegree;
    return pv;
  }
  static partitioned_vertices empty() { return partitioned_vertices(); }
  static partitioned_vertices dense(intT n, const partitioner&) {
    partitioned_vertices pv;
    pv.numVertices = n;
    pv.d.internal_allocate(n);
    LB_CUDA(cudaMemset(pv.d.get(), 0, n ? n : 1));
    pv.has_dense = true;
    return pv;
  }
  static partitioned_vertices sparse(intT n) {
    partitioned_vertices pv;
    pv.numVertices = n;
    return pv;
  }
  static partitioned_vertices bits(const partitioner&, intT n, intT initialOutdegree) {
    partitioned_vertices pv;
    pv.num_out_edges = initialOutdegree;
    pv.numVertices = n;
    pv.d.internal_allocate(n);
    pv.bit = true;
    pv.d_m = n;
    pv.has_dense = true;
    return pv;
  }
  static partitioned_vertices boolean(intT n, mmap_ptr<bool> b, intT activeM, intT out_edges) {
    partitioned_vertices pv;
    pv.numVertices = n;
    pv.num_out_edges = out_edges;
    pv.d_m = activeM;
    pv.d = b;
    pv.has_dense = true;
    return pv;
  }
  static partitioned_vertices indice(intT n, mmap_ptr<intT> idx, intT activeM, intT out_edges) {
    partitioned_vertices pv;
    pv.numVertices = n;
    pv.num_out_edges = out_edges;
    pv.d_m = activeM;
    pv.s = idx.get();
    return pv;
  }
  void del() {
    lb::release(s);
    s = nullptr;
    d.del();
  }
  intT* get_partition(unsigned) { return s; }
  bool isEmpty() { return d_m == 0; }
  void toDense(const partitioner& part);
  void toSparse();
  intT numRows() { return numVertices; }
  intT numNonzeros() { return d_m; }
};

namespace lb {
static __global__ void k_scatter(const intT* s, intT k, bool* d) {
  for (intT i = blockIdx.x * (intT)blockDim.x + threadIdx.x; i < k; i += (intT)gridDim.x * blockDim.x) d[s[i]] = 1;
}
static __global__ void k_pack(const bool* d, intT n, intT* s, unsigned long long* cnt) {
  for (intT i = blockIdx.x * (intT)blockDim.x + threadIdx.x; i < n; i += (intT)gridDim.x * blockDim.x)
    if (d[i]) s[atomicAdd(cnt, 1ull)] = i;
}
// (members, out-degree sum) of a dense set (GoutDegree, ligra-numa.h:274-311)
static __global__ void k_dense_stats(const bool* d, intT n, const uint32_t* out_off, unsigned long long* st) {
  unsigned long long c = 0, e = 0;
  for (intT i = blockIdx.x * (intT)blockDim.x + threadIdx.x; i < n; i += (intT)gridDim.x * blockDim.x)
    if (d[i]) {
      c++;
      e += out_off[i + 1] - out_off[i];
    }
  for (int o = 16; o > 0; o >>= 1) {
    c += __shfl_xor_sync(0xffffffffu, c, o);
    e += __shfl_xor_sync(0xffffffffu, e, o);
  }
  if ((threadIdx.x & 31) == 0 && (c || e)) {
    atomicAdd(st, c);
    atomicAdd(st + 1, e);
  }
}
static __global__ void k_list_outdeg(const intT* s, intT k, const uint32_t* out_off, unsigned long long* st) {
  unsigned long long e = 0;
  for (intT i = blockIdx.x * (intT)blockDim.x + threadIdx.x; i < k; i += (intT)gridDim.x * blockDim.x)
    e += out_off[s[i] + 1] - out_off[s[i]];
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  if ((threadIdx.x & 31) == 0 && e) atomicAdd(st + 1, e);
}
inline unsigned long long* counters() {
  static unsigned long long* c = nullptr;
  if (!c) c = alloc<unsigned long long>(2);
  return c;
}
}  // namespace lb

inline void partitioned_vertices::toDense(const partitioner&) {
  if (!d) {
    d.internal_allocate(numVertices);
    LB_CUDA(cudaMemset(d.get(), 0, numVertices ? numVertices : 1));
    if (d_m) lb::k_scatter<<<lb::grid_for(d_m), lb::kThreads>>>(s, d_m, d.get());
    LB_CUDA(cudaGetLastError());
  }
  has_dense = true;
}

inline void partitioned_vertices::toSparse() {
  if (s == nullptr) {
    if (bit) {
      std::cerr << "toSparse of an all-vertices frontier" << std::endl;  // the reference packs garbage here
      abort();
    }
    s = lb::alloc<intT>(d_m ? d_m : 1);
    unsigned long long* c = lb::counters();
    lb::sync();
    c[0] = 0;
    lb::k_pack<<<lb::grid_for(numVertices), lb::kThreads>>>(d.get(), numVertices, s, c);
    LB_CUDA(cudaGetLastError());
    lb::sync();
    if ((intT)c[0] != d_m) {  // ligra-numa.h:251-255
      cout << "bad stored value of m" << endl;
      abort();
    }
  }
  has_dense = false;
}

// ============================================================ edgeMap
static long edgesTraversed = 0;

namespace lb {
// edgeOpIn / edgeOpBwd (graphgrind/ligra-numa.h:364-543) for one in-edge
template <class F>
__device__ __forceinline__ bool bwd(F& f, intT s, intT d, intE w) {
#ifdef WEIGHTED
  return f.update(s, d, w);
#else
  (void)w;
  return f.update(s, d);
#endif
}
template <class F>
__device__ __forceinline__ bool bwd_cache(F& f, typename F::cache_t& c, intT s, intE w) {
#ifdef WEIGHTED
  return f.update(c, s, w);
#else
  (void)w;
  return f.update(c, s);
#endif
}
template <class F>
__device__ __forceinline__ bool fwd_atomic(F& f, intT s, intT d, intE w) {
#ifdef WEIGHTED
  return f.updateAtomic(s, d, w);
#else
  (void)w;
  return f.updateAtomic(s, d);
#endif
}

// edgeMapDenseCSC (graphgrind/ligra-numa.h:549-729), destination-owned: one
// thread per destination walks its in-edges in order.
template <class F>
__global__ void k_dense_pull(F f, const uint32_t* __restrict__ in_off, const uint32_t* __restrict__ in_idx,
                             const intE* __restrict__ in_w, const bool* __restrict__ frontier, bool bit, bool* next,
                             intT n) {
  for (intT id = blockIdx.x * (intT)blockDim.x + threadIdx.x; id < n; id += (intT)gridDim.x * blockDim.x) {
    if (!f.cond(id)) continue;
    const uint32_t b = in_off[id], e = in_off[id + 1];
    if (F::use_cache) {
      typename F::cache_t cache;
      f.create_cache(cache, id);
      for (uint32_t j = b; j < e; j++) {
        const intT s = in_idx[j];
        if ((bit || frontier[s]) && bwd_cache(f, cache, s, in_w ? in_w[j] : 1)) next[id] = 1;
        if (!f.cond(id)) break;
      }
      f.commit_cache(cache, id);
    } else {
      for (uint32_t j = b; j < e; j++) {
        const intT s = in_idx[j];
        if ((bit || frontier[s]) && bwd(f, s, id, in_w ? in_w[j] : 1)) next[id] = 1;
        if (!f.cond(id)) break;
      }
    }
  }
}

// edgeMapSparseWithG (graphgrind/ligra-numa.h:868-916): one warp per
// frontier vertex, lanes over its out-edges; a destination whose update
// succeeds enters the output once (bitmap).
template <class F>
__global__ void k_sparse_push(F f, const uint32_t* __restrict__ out_off, const uint32_t* __restrict__ out_idx,
                              const intE* __restrict__ out_w, const intT* __restrict__ fr, intT k, uint32_t* seen,
                              intT* out, unsigned long long* cnt) {
  const int lane = threadIdx.x & 31;
  const intT warps = ((intT)gridDim.x * blockDim.x) >> 5;
  for (intT w = (blockIdx.x * (intT)blockDim.x + threadIdx.x) >> 5; w < k; w += warps) {
    const intT src = fr[w];
    const uint32_t b = out_off[src], e = out_off[src + 1];
    for (uint32_t j = b + lane; j < e; j += 32) {
      const intT dst = out_idx[j];
      if (f.cond(dst) && fwd_atomic(f, src, dst, out_w ? out_w[j] : 1)) {
        const uint32_t bitm = 1u << (dst & 31);
        if (!(atomicOr(seen + (dst >> 5), bitm) & bitm)) out[atomicAdd(cnt, 1ull)] = dst;
      }
    }
  }
}

template <class F>
__global__ void k_vertex_all(F f, intT n) {
  for (intT i = blockIdx.x * (intT)blockDim.x + threadIdx.x; i < n; i += (intT)gridDim.x * blockDim.x) f(i);
}
template <class F>
__global__ void k_vertex_dense(F f, const bool* d, intT n) {
  for (intT i = blockIdx.x * (intT)blockDim.x + threadIdx.x; i < n; i += (intT)gridDim.x * blockDim.x)
    if (d[i]) f(i);
}
template <class F>
__global__ void k_vertex_list(F f, const intT* s, intT k) {
  for (intT i = blockIdx.x * (intT)blockDim.x + threadIdx.x; i < k; i += (intT)gridDim.x * blockDim.x) f(s[i]);
}
template <class F>
__global__ void k_vertex_filter(F f, const bool* d, bool bit, bool* out, intT n) {
  for (intT i = blockIdx.x * (intT)blockDim.x + threadIdx.x; i < n; i += (intT)gridDim.x * blockDim.x)
    out[i] = (bit || d[i]) ? (bool)f(i) : false;
}
}  // namespace lb

template <class F, class vertex>
partitioned_vertices edgeMap(partitioned_graph<vertex> GA, partitioned_vertices Localfrontier, F f,
                             intT threshold = -1, char option = DENSE, bool remDups = false) {
  (void)option;
  (void)remDups;
  const intT numVertices = GA.n;
  if (threshold == -1) threshold = GA.m / 20;
  const intT m = Localfrontier.numNonzeros();
  if (numVertices != Localfrontier.numRows()) {  // ligra-numa.h:937-942
    cerr << "numVertices" << numVertices << " and rows" << Localfrontier.numRows() << endl;
    cerr << "edgeMap: Sizes Don't match" << endl;
    abort();
  }
  const intT TotalOutDegrees = Localfrontier.num_out_edges;
  edgesTraversed += TotalOutDegrees;
  if (TotalOutDegrees == 0) return partitioned_vertices::empty();
  graph<vertex>& WG = GA.get_partition();
  unsigned long long* c = lb::counters();
  partitioned_vertices v1;
  // representations made here live only in this call's copy of the frontier
  const bool made_dense = !Localfrontier.d, made_sparse = Localfrontier.s == nullptr;
  if (m + TotalOutDegrees > threshold) {
    Localfrontier.toDense(GA.get_coo_partitioner());
    v1 = partitioned_vertices::dense(numVertices, GA.get_coo_partitioner());
    lb::k_dense_pull<<<lb::grid_for(numVertices), lb::kThreads>>>(f, WG.in_off, WG.in_idx, WG.in_w,
                                                                  Localfrontier.d.get(), Localfrontier.bit,
                                                                  v1.d.get(), numVertices);
    LB_CUDA(cudaGetLastError());
    lb::sync();
    c[0] = c[1] = 0;
    lb::k_dense_stats<<<lb::grid_for(numVertices), lb::kThreads>>>(v1.d.get(), numVertices, WG.out_off, c);
    LB_CUDA(cudaGetLastError());
    lb::sync();
    v1.d_m = (intT)c[0];
    v1.num_out_edges = (intT)c[1];
    if (made_dense) Localfrontier.d.del();
  } else {
    Localfrontier.toSparse();
    v1 = partitioned_vertices::sparse(numVertices);
    uint32_t* seen = nullptr;
    const size_t words = ((size_t)numVertices + 31) / 32;
    LB_CUDA(cudaMalloc(&seen, 4 * (words ? words : 1)));
    LB_CUDA(cudaMemset(seen, 0, 4 * (words ? words : 1)));
    v1.s = lb::alloc<intT>(std::min<intT>(numVertices, TotalOutDegrees));
    lb::sync();
    c[0] = c[1] = 0;
    lb::k_sparse_push<<<lb::grid_for((uint64_t)m * 32), lb::kThreads>>>(f, WG.out_off, WG.out_idx, WG.out_w,
                                                                       Localfrontier.s, m, seen, v1.s, c);
    LB_CUDA(cudaGetLastError());
    lb::sync();
    v1.d_m = (intT)c[0];
    if (v1.d_m) lb::k_list_outdeg<<<lb::grid_for(v1.d_m), lb::kThreads>>>(v1.s, v1.d_m, WG.out_off, c);
    LB_CUDA(cudaGetLastError());
    lb::sync();
    v1.num_out_edges = v1.d_m ? (intT)c[1] : 0;
    LB_CUDA(cudaFree(seen));
    if (made_sparse) {
      lb::release(Localfrontier.s);
      Localfrontier.s = nullptr;
    }
  }
  return v1;
}

// vertexMap (graphgrind/ligra-numa.h:1023-1049)
template <class F>
void vertexMap(const partitioner& part, partitioned_vertices V, F add) {
  const intT n = part.get_num_elements();
  if (V.has_dense) {
    if (V.bit)
      lb::k_vertex_all<<<lb::grid_for(n), lb::kThreads>>>(add, n);
    else
      lb::k_vertex_dense<<<lb::grid_for(n), lb::kThreads>>>(add, V.d.get(), n);
  } else if (V.d_m) {
    lb::k_vertex_list<<<lb::grid_for(V.d_m), lb::kThreads>>>(add, V.s, V.d_m);
  }
  LB_CUDA(cudaGetLastError());
}

// vertexFilter (graphgrind/ligra-numa.h:1053-1082)
template <typename vertex, class F>
partitioned_vertices vertexFilter(partitioned_graph<vertex> GA, partitioned_vertices V, F filter) {
  const partitioner& part = GA.get_partitioner();
  const intT n = V.numRows();
  const bool made_dense = !V.d;
  V.toDense(part);
  mmap_ptr<bool> d_out;
  d_out.internal_allocate(n);
  lb::k_vertex_filter<<<lb::grid_for(n), lb::kThreads>>>(filter, V.d.get(), V.bit, d_out.get(), n);
  LB_CUDA(cudaGetLastError());
  lb::sync();
  unsigned long long* c = lb::counters();
  c[0] = c[1] = 0;
  lb::k_dense_stats<<<lb::grid_for(n), lb::kThreads>>>(d_out.get(), n, GA.get_partition().out_off, c);
  LB_CUDA(cudaGetLastError());
  lb::sync();
  if (made_dense) V.d.del();
  return partitioned_vertices::boolean(n, d_out, (intT)c[0], (intT)c[1]);
}

// The functors of an application are defined after this header; their
// `inline` member functions become callable from the kernels above.
#define inline __host__ __device__ inline

#endif  // LIGRA_B200_H
