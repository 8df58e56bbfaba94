// VEBO reordering on the GPU (graphtools/VEBO.C:56-395; the host restatement
// is gg_vebo in gg_host.cpp, which gives the same result).
//
// The tool's three phases map to the device as follows.
//   1. In-degrees (an atomic histogram of the destinations, or the degrees of
//      a symmetric graph) and the order of the vertices by (in-degree
//      descending, id): one 64-bit radix sort of (~degree << 32 | id).
//   2. The deal of each run of equal degree to the partitions
//      (graphtools/VEBO.C:180-262) depends on the edge totals of all earlier
//      deals, so it stays sequential; it only needs the runs (degree, count),
//      which a run-length encoding of the sorted degrees gives.  The host runs
//      it (vebo_deal, shared with gg_vebo) on those few numbers.
//   3. Placement (:276-300): the vertices of run i dealt to partition p take
//      consecutive ids after everything dealt to p from earlier runs.  With
//      per-(run, partition) tables (first position inside the run, first new
//      id) every vertex finds its new id by two binary searches, and the
//      graph is relabelled (:330-343) by a scan of the new degrees and a
//      warp per new vertex copying its renamed neighbour list (and weights).
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "gg_common.h"

namespace gg {
namespace {

struct DBuf {
  void* p = nullptr;
  cudaError_t alloc(size_t bytes) { return cudaMalloc(&p, bytes ? bytes : 16); }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
  ~DBuf() {
    if (p) cudaFree(p);
  }
};

__global__ void k_vebo_indeg(const uint32_t* idx, uint64_t m, uint32_t* deg) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x)
    atomicAdd(deg + idx[e], 1u);
}

__global__ void k_vebo_outdeg(const uint32_t* off, uint32_t n, uint32_t* deg) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
    deg[v] = off[v + 1] - off[v];
}

// ascending keys = descending degree, then ascending id (LargePairSort)
__global__ void k_vebo_keys(const uint32_t* deg, uint32_t n, uint64_t* keys) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
    keys[v] = ((uint64_t)(~deg[v]) << 32) | v;
}

__global__ void k_vebo_split(const uint64_t* keys, uint32_t n, uint32_t* sdeg, uint32_t* sv) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    sdeg[i] = ~(uint32_t)(keys[i] >> 32);
    sv[i] = (uint32_t)keys[i];
  }
}

// last index j in [0, len) with a[j] <= x (a ascending, a[0] <= x)
__device__ __forceinline__ uint32_t last_le(const uint32_t* a, uint32_t len, uint32_t x) {
  uint32_t lo = 0, hi = len;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a[mid] <= x)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// sorted position r -> run g, offset k in the run -> partition p (the last
// one whose first position in the run is <= k) -> new id
__global__ void k_vebo_place(const uint32_t* sv, uint32_t n, const uint32_t* run_start, uint32_t runs,
                             const uint32_t* cum, const uint32_t* base, uint32_t P, uint32_t* new_of_old,
                             uint32_t* old_of_new) {
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t g = last_le(run_start, runs, (uint32_t)r);
    const uint32_t k = (uint32_t)r - run_start[g];
    const uint32_t p = last_le(cum + (size_t)g * P, P, k);
    const uint32_t id = base[(size_t)g * P + p] + (k - cum[(size_t)g * P + p]);
    new_of_old[sv[r]] = id;
    old_of_new[id] = sv[r];
  }
}

__global__ void k_vebo_newdeg(const uint32_t* off, const uint32_t* old_of_new, uint32_t n, uint32_t* nd) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += (uint64_t)gridDim.x * blockDim.x)
    nd[i] = i < n ? off[old_of_new[i] + 1] - off[old_of_new[i]] : 0;
}

// one warp per new vertex: its old row, renamed, in order (weights carried)
__global__ void k_vebo_relabel(const uint32_t* off, const uint32_t* idx, const uint32_t* w, const uint32_t* old_of_new,
                               const uint32_t* new_of_old, const uint32_t* noff, uint32_t n, uint32_t* nidx,
                               uint32_t* nw) {
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    const uint32_t o = old_of_new[i];
    const uint32_t b = off[o], d = off[o + 1] - b, dst = noff[i];
    for (uint32_t j = lane; j < d; j += 32) {
      nidx[dst + j] = new_of_old[idx[b + j]];
      if (w) nw[dst + j] = w[b + j];
    }
  }
}

}  // namespace
}  // namespace gg

using namespace gg;

#define GG_VB(call)                                                                \
  do {                                                                             \
    cudaError_t e__ = (call);                                                      \
    if (e__ != cudaSuccess) {                                                      \
      gg_host_graph_free(out);                                                     \
      return fail(GG_ERR_CUDA, "gg_vebo_gpu: %s: %s", #call, cudaGetErrorString(e__)); \
    }                                                                              \
  } while (0)

extern "C" int gg_vebo_gpu(const gg_host_graph* g, int32_t partitions, uint32_t* new_of_old, int64_t* part_sizes,
                           gg_host_graph* out) {
  if (!g || !out || !g->offsets || (g->m && !g->indices) || partitions < 1 || g->n == 0)
    return fail(GG_ERR_INVALID_ARG, "gg_vebo_gpu: bad arguments");
  memset(out, 0, sizeof *out);
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0)
    return fail(GG_ERR_NO_DEVICE, "gg_vebo_gpu: no CUDA device");
  const uint32_t n = g->n;
  const uint64_t m = g->m;
  const int64_t P = partitions;
  const int grid = 148 * 8, threads = 256;
  DBuf off, idx, w, deg, keys, keys2, sdeg, sv, uniq, counts, nruns, tmp;
  GG_VB(off.alloc(4ull * (n + 1)));
  GG_VB(idx.alloc(4 * m));
  GG_VB(cudaMemcpy(off.p, g->offsets, 4ull * (n + 1), cudaMemcpyHostToDevice));
  if (m) GG_VB(cudaMemcpy(idx.p, g->indices, 4 * m, cudaMemcpyHostToDevice));
  if (g->weights) {
    GG_VB(w.alloc(4 * m));
    if (m) GG_VB(cudaMemcpy(w.p, g->weights, 4 * m, cudaMemcpyHostToDevice));
  }
  // 1. in-degrees and the sorted order
  GG_VB(deg.alloc(4ull * n));
  GG_VB(cudaMemset(deg.p, 0, 4ull * n));
  if (g->symmetric)
    k_vebo_outdeg<<<grid, threads>>>(off.as<uint32_t>(), n, deg.as<uint32_t>());
  else if (m)
    k_vebo_indeg<<<grid, threads>>>(idx.as<uint32_t>(), m, deg.as<uint32_t>());
  GG_VB(keys.alloc(8ull * n));
  GG_VB(keys2.alloc(8ull * n));
  k_vebo_keys<<<grid, threads>>>(deg.as<uint32_t>(), n, keys.as<uint64_t>());
  GG_VB(cudaGetLastError());
  size_t tb = 0, tb2 = 0;
  GG_VB(cub::DeviceRadixSort::SortKeys(nullptr, tb, keys.as<uint64_t>(), keys2.as<uint64_t>(), (int64_t)n));
  GG_VB(sdeg.alloc(4ull * n));
  GG_VB(sv.alloc(4ull * n));
  GG_VB(uniq.alloc(4ull * n));
  GG_VB(counts.alloc(4ull * n));
  GG_VB(nruns.alloc(8));
  GG_VB(cub::DeviceRunLengthEncode::Encode(nullptr, tb2, sdeg.as<uint32_t>(), uniq.as<uint32_t>(),
                                           counts.as<uint32_t>(), nruns.as<int64_t>(), (int64_t)n));
  GG_VB(tmp.alloc(std::max(tb, tb2)));
  GG_VB(cub::DeviceRadixSort::SortKeys(tmp.p, tb, keys.as<uint64_t>(), keys2.as<uint64_t>(), (int64_t)n));
  k_vebo_split<<<grid, threads>>>(keys2.as<uint64_t>(), n, sdeg.as<uint32_t>(), sv.as<uint32_t>());
  GG_VB(cudaGetLastError());
  GG_VB(cub::DeviceRunLengthEncode::Encode(tmp.p, tb2, sdeg.as<uint32_t>(), uniq.as<uint32_t>(),
                                           counts.as<uint32_t>(), nruns.as<int64_t>(), (int64_t)n));
  int64_t c = 0;
  GG_VB(cudaMemcpy(&c, nruns.p, 8, cudaMemcpyDeviceToHost));
  std::vector<uint32_t> hu(c), hc(c);
  GG_VB(cudaMemcpy(hu.data(), uniq.p, 4 * c, cudaMemcpyDeviceToHost));
  GG_VB(cudaMemcpy(hc.data(), counts.p, 4 * c, cudaMemcpyDeviceToHost));
  // 2. the deal, on the runs
  std::vector<std::pair<int64_t, int64_t>> runs(c);
  for (int64_t i = 0; i < c; i++) runs[i] = {(int64_t)hu[i], (int64_t)hc[i]};
  std::vector<int64_t> perDeg, vsize;
  const int rc = vebo_deal(runs, n, P, perDeg, vsize);
  if (rc) return rc;
  // 3. placement tables: first sorted position of each run; per (run,
  // partition) the first offset inside the run and the first new id
  std::vector<uint32_t> run_start(c), cum((size_t)c * P), base((size_t)c * P);
  std::vector<int64_t> next_id(P, 0);
  for (int64_t p = 1; p < P; p++) next_id[p] = next_id[p - 1] + vsize[p - 1];
  int64_t pos = 0;
  for (int64_t i = 0; i < c; i++) {
    run_start[i] = (uint32_t)pos;
    int64_t k = 0;
    for (int64_t p = 0; p < P; p++) {
      cum[(size_t)i * P + p] = (uint32_t)k;
      base[(size_t)i * P + p] = (uint32_t)next_id[p];
      const int64_t cnt = perDeg[(size_t)p * c + i];
      k += cnt;
      next_id[p] += cnt;
    }
    pos += k;
  }
  DBuf d_rs, d_cum, d_base, nofo, oofn, nd, noff, nidx, nw;
  GG_VB(d_rs.alloc(4 * c));
  GG_VB(d_cum.alloc(4 * cum.size()));
  GG_VB(d_base.alloc(4 * base.size()));
  GG_VB(cudaMemcpy(d_rs.p, run_start.data(), 4 * c, cudaMemcpyHostToDevice));
  GG_VB(cudaMemcpy(d_cum.p, cum.data(), 4 * cum.size(), cudaMemcpyHostToDevice));
  GG_VB(cudaMemcpy(d_base.p, base.data(), 4 * base.size(), cudaMemcpyHostToDevice));
  GG_VB(nofo.alloc(4ull * n));
  GG_VB(oofn.alloc(4ull * n));
  k_vebo_place<<<grid, threads>>>(sv.as<uint32_t>(), n, d_rs.as<uint32_t>(), (uint32_t)c, d_cum.as<uint32_t>(),
                                  d_base.as<uint32_t>(), (uint32_t)P, nofo.as<uint32_t>(), oofn.as<uint32_t>());
  GG_VB(cudaGetLastError());
  // relabelled CSR
  GG_VB(nd.alloc(4ull * (n + 1)));
  GG_VB(noff.alloc(4ull * (n + 1)));
  k_vebo_newdeg<<<grid, threads>>>(off.as<uint32_t>(), oofn.as<uint32_t>(), n, nd.as<uint32_t>());
  GG_VB(cudaGetLastError());
  size_t tb3 = 0;
  GG_VB(cub::DeviceScan::ExclusiveSum(nullptr, tb3, nd.as<uint32_t>(), noff.as<uint32_t>(), (int64_t)n + 1));
  DBuf tmp3;
  GG_VB(tmp3.alloc(tb3));
  GG_VB(cub::DeviceScan::ExclusiveSum(tmp3.p, tb3, nd.as<uint32_t>(), noff.as<uint32_t>(), (int64_t)n + 1));
  GG_VB(nidx.alloc(4 * m));
  if (g->weights) GG_VB(nw.alloc(4 * m));
  k_vebo_relabel<<<grid, threads>>>(off.as<uint32_t>(), idx.as<uint32_t>(), g->weights ? w.as<uint32_t>() : nullptr,
                                    oofn.as<uint32_t>(), nofo.as<uint32_t>(), noff.as<uint32_t>(), n,
                                    nidx.as<uint32_t>(), g->weights ? nw.as<uint32_t>() : nullptr);
  GG_VB(cudaGetLastError());
  out->n = n;
  out->m = m;
  out->symmetric = g->symmetric;
  out->weight_type = g->weight_type;
  out->offsets = static_cast<uint32_t*>(malloc(4ull * (n + 1)));
  out->indices = static_cast<uint32_t*>(malloc(4 * (m ? m : 1)));
  if (g->weights) out->weights = malloc(4 * (m ? m : 1));
  if (!out->offsets || !out->indices || (g->weights && !out->weights)) {
    gg_host_graph_free(out);
    return fail(GG_ERR_OOM, "gg_vebo_gpu: out of host memory");
  }
  GG_VB(cudaMemcpy(out->offsets, noff.p, 4ull * (n + 1), cudaMemcpyDeviceToHost));
  if (m) GG_VB(cudaMemcpy(out->indices, nidx.p, 4 * m, cudaMemcpyDeviceToHost));
  if (g->weights && m) GG_VB(cudaMemcpy(out->weights, nw.p, 4 * m, cudaMemcpyDeviceToHost));
  if (new_of_old) GG_VB(cudaMemcpy(new_of_old, nofo.p, 4ull * n, cudaMemcpyDeviceToHost));
  if (part_sizes) std::copy(vsize.begin(), vsize.end(), part_sizes);
  return GG_OK;
}
