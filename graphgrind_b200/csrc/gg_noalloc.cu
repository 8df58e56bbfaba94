// One sparse-push BFS level that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc: an application that owns
// every byte of device memory and hands the library fixed buffers (a memory
// budget enforced by the embedding program), or a latency-critical loop where
// cudaMalloc/cudaFree would add allocator latency and, for cudaFree, an
// implicit device-wide synchronisation.  gg_bfs_push_step_noalloc serves
// them: it runs the same kernels as the push branch of gg_edge_map for the
// BFS functor, but every temporary it needs lives in one file-scope device
// array whose size is fixed at build time.
//
// Limits: frontiers of at most GG_NOALLOC_MAX_FRONTIER vertices and graphs of
// at most GG_NOALLOC_MAX_VERTICES vertices (sizes above are rejected with
// GG_ERR_SIZE).  Every GPU that loads the library holds the array
// (GG_NOALLOC_SCRATCH_BYTES) until the process exits.  All calls share it,
// so calls whose work overlaps on the GPU (different streams, or different
// host threads) race with each other; issue them one after another.  The
// first call on a device looks up the array's device address on that device
// (host code only sees a host-side stand-in for the array's name); make that
// first call before any stream capture.
#include <mutex>

#include "gg_runtime.cuh"

namespace {

constexpr size_t kAlign = 256;
constexpr size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }
constexpr size_t kStatsBytes = align_up(sizeof(unsigned long long) * 8);
constexpr size_t kDedupBytes = align_up(sizeof(uint32_t) * (GG_NOALLOC_MAX_VERTICES / 32 + 4));
constexpr size_t kScanBytes = align_up(sizeof(uint32_t) * (GG_NOALLOC_MAX_FRONTIER + 4));
constexpr size_t kBsumBytes =
    align_up(sizeof(uint32_t) * ((GG_NOALLOC_MAX_FRONTIER + gg::kScanTile - 1) / gg::kScanTile + 32));
constexpr size_t kScratchBytes = kStatsBytes + kDedupBytes + kScanBytes + kBsumBytes;
static_assert(kScratchBytes <= GG_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the stated size");

}  // namespace

// The scratch of gg_bfs_push_step_noalloc (stats | dedup bitmap | scan | block sums).
static __device__ __align__(256) unsigned char g_noalloc_scratch[GG_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned char* g_scratch_addr[kMaxDevices] = {};
int g_num_sms[kMaxDevices] = {};

// Device address of the scratch array on the current device (set up once).
int scratch_on_current_device(unsigned char** out, int* num_sms) {
  int dev = 0;
  GG_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return gg::fail(GG_ERR_UNSUPPORTED, "device ordinal %d not supported", dev);
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return gg::fail(GG_ERR_CUDA, "cudaGetSymbolAddress(scratch) on device %d: %s", dev, cudaGetErrorString(e));
    // the dedup bitmap is zero between calls (each call clears the words its
    // output set); make it so once, whatever the array held at load
    GG_CUDA(cudaMemset(p, 0, GG_NOALLOC_SCRATCH_BYTES));
    GG_CUDA(cudaDeviceSynchronize());
    int sms = 0;
    GG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    g_scratch_addr[dev] = static_cast<unsigned char*>(p);
    g_num_sms[dev] = sms > 0 ? sms : 1;
  }
  *out = g_scratch_addr[dev];
  *num_sms = g_num_sms[dev];
  return GG_OK;
}

}  // namespace

extern "C" int gg_bfs_push_step_noalloc(const uint32_t* out_offsets, const uint32_t* out_indices, uint32_t n,
                                        const uint32_t* frontier, uint32_t frontier_len, int32_t* parents,
                                        int32_t* levels, int32_t round, uint32_t* next_frontier,
                                        uint64_t* next_counts, void* stream) {
  if (!out_offsets || !out_indices || !parents || !next_frontier || !next_counts || (frontier_len && !frontier))
    return gg::fail(GG_ERR_INVALID_ARG, "gg_bfs_push_step_noalloc: null pointer argument");
  if (n == 0 || n > GG_NOALLOC_MAX_VERTICES)
    return gg::fail(GG_ERR_SIZE, "gg_bfs_push_step_noalloc: n=%u outside 1..%u (GG_NOALLOC_MAX_VERTICES)", n,
                    (unsigned)GG_NOALLOC_MAX_VERTICES);
  if (frontier_len > GG_NOALLOC_MAX_FRONTIER || frontier_len > n)
    return gg::fail(GG_ERR_SIZE, "gg_bfs_push_step_noalloc: frontier of %u vertices exceeds %u (GG_NOALLOC_MAX_FRONTIER)",
                    frontier_len, (unsigned)GG_NOALLOC_MAX_FRONTIER);
  unsigned char* base = nullptr;
  int num_sms = 1;
  GG_TRY(scratch_on_current_device(&base, &num_sms));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned long long* stats = reinterpret_cast<unsigned long long*>(base);
  uint32_t* dedup = reinterpret_cast<uint32_t*>(base + kStatsBytes);
  uint32_t* scan = reinterpret_cast<uint32_t*>(base + kStatsBytes + kDedupBytes);
  uint32_t* bsum = reinterpret_cast<uint32_t*>(base + kStatsBytes + kDedupBytes + kScanBytes);
  // The array keeps the previous call's contents: the counters start at zero
  // here; the dedup bitmap is zero on entry (cleared at set-up, then by every
  // call for the vertices it output), so no call pays for an n-bit clear.
  GG_CUDA(cudaMemsetAsync(stats, 0, kStatsBytes, st));
  if (frontier_len > 0) {
    const uint32_t nb = (frontier_len + gg::kScanTile - 1) / gg::kScanTile;
    gg::k_scan_sums<<<nb, gg::kScanThreads, 0, st>>>(frontier, frontier_len, out_offsets, bsum);
    gg::k_scan_blocks<<<1, 1024, 0, st>>>(bsum, nb, stats + 5);
    gg::k_scan_write<<<nb, gg::kScanThreads, 0, st>>>(frontier, frontier_len, out_offsets, bsum, scan);
    gg::PushParams p{};
    p.q = frontier;
    p.k = frontier_len;
    p.offs = scan;
    p.total = stats + 5;
    p.off = out_offsets;
    p.idx = out_indices;
    p.wts = nullptr;
    p.deg_off = out_offsets;
    p.dedup = dedup;
    p.out_q = next_frontier;
    p.stats = stats;
    gg::BfsF f;
    f.parents = parents;
    f.levels = levels;
    f.round = round;
    gg::k_push<gg::BfsF, false><<<num_sms * 8, gg::kPushThreads, 0, st>>>(p, f);
    GG_CUDA(cudaGetLastError());
    // the output's dedup words back to zero for the next call
    gg::k_clear_dedup<<<num_sms * 4, 256, 0, st>>>(next_frontier, stats + 2, dedup);
    GG_CUDA(cudaGetLastError());
  }
  // next_counts[0] = output frontier size, next_counts[1] = its out-degree sum
  GG_CUDA(cudaMemcpyAsync(next_counts, stats + 2, sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
  GG_CUDA(cudaMemcpyAsync(next_counts + 1, stats + 1, sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
  return GG_OK;
}
