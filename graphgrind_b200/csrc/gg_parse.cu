// GPU parsing of the reference's PBBS text graph format (graphgrind/IO.h:136-199,
// readGraphFromFile: "AdjacencyGraph" or "WeightedAdjacencyGraph", n, m, n
// offsets, m neighbours, [m weights], separated by whitespace).  The host reads
// the file and the header; the body goes to the device in chunks cut at
// whitespace, where one pass marks the first byte of every number, a select
// compacts those positions, and one thread per number converts and range-checks
// it into its slot of the offsets / neighbours / weights arrays.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cstring>
#include <vector>

#include "gg_common.h"

namespace gg {

constexpr int kParseThreads = 256;
constexpr size_t kMaxToken = 32;  // a longer run of non-blank bytes is no number

__host__ __device__ inline bool blank(char c) { return c == ' ' || c == '\n' || c == '\r' || c == '\t'; }

struct TokenStart {
  const char* c;
  __device__ bool operator()(uint32_t i) const { return !blank(c[i]) && (i == 0 || blank(c[i - 1])); }
};

enum : unsigned { kBadNumber = 1u, kBadOffset = 2u, kBadEdge = 4u };

// Number t of the chunk is number base + t of the body: offsets [0, n),
// neighbours [n, n + m), weights [n + m, n + 2m).
__global__ void k_parse_numbers(const char* c, uint32_t len, const uint32_t* starts, uint32_t count, uint64_t base,
                                uint64_t n, uint64_t m, uint64_t total, uint32_t* off, uint32_t* idx, int32_t* w,
                                unsigned* err) {
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < count; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t gi = base + t;
    if (gi >= total) return;  // numbers past the body are ignored, as by the host reader
    uint32_t p = starts[t];
    bool neg = false;
    if (c[p] == '-') {
      neg = true;
      ++p;
    }
    long long v = 0;
    int digits = 0;
    bool ok = true;
    while (p < len && !blank(c[p])) {
      const char ch = c[p++];
      if (ch < '0' || ch > '9' || digits == 18) {
        ok = false;
        break;
      }
      v = v * 10 + (ch - '0');
      ++digits;
    }
    if (!ok || digits == 0) {
      atomicOr(err, kBadNumber);
      continue;
    }
    if (neg) v = -v;
    if (gi < n) {
      if (v < 0 || (uint64_t)v > m) atomicOr(err, kBadOffset);
      else off[gi] = (uint32_t)v;
    } else if (gi < n + m) {
      if (v < 0 || (uint64_t)v >= n) atomicOr(err, kBadEdge);
      else idx[gi - n] = (uint32_t)v;
    } else {
      w[gi - n - m] = (int32_t)v;  // the host reader's cast of any integer
    }
  }
}

struct ParseBufs {
  char* h_file = nullptr;  // pinned
  char* d_chunk = nullptr;
  uint32_t *d_starts = nullptr, *d_count = nullptr, *d_off = nullptr, *d_idx = nullptr;
  int32_t* d_w = nullptr;
  unsigned* d_err = nullptr;
  void* d_tmp = nullptr;
  cudaStream_t st = nullptr;
  ~ParseBufs() {
    if (st) cudaStreamSynchronize(st);
    if (h_file) cudaFreeHost(h_file);
    for (void* p : {(void*)d_chunk, (void*)d_starts, (void*)d_count, (void*)d_off, (void*)d_idx, (void*)d_w,
                    (void*)d_err, d_tmp})
      cudaFree(p);
    if (st) cudaStreamDestroy(st);
  }
};

#define GG_PARSE_CUDA(call)                                                               \
  do {                                                                                    \
    cudaError_t e__ = (call);                                                             \
    if (e__ != cudaSuccess) return fail(GG_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e__)); \
  } while (0)

static int parse_adj(const char* path, int32_t symmetric, int32_t weighted, int64_t chunk_bytes, gg_host_graph* out) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(GG_ERR_NO_DEVICE, "no CUDA device is visible");
  }
  const size_t chunk = chunk_bytes > 0 ? (size_t)chunk_bytes : (size_t)256 << 20;
  if (chunk >= (1ull << 31)) return fail(GG_ERR_INVALID_ARG, "read_gpu: chunk_bytes must be below 2^31");
  int fd = open(path, O_RDONLY);
  if (fd < 0) return fail(GG_ERR_IO, "cannot open %s: %s", path, strerror(errno));
  struct stat sb;
  if (fstat(fd, &sb)) {
    close(fd);
    return fail(GG_ERR_IO, "cannot stat %s", path);
  }
  const size_t len = (size_t)sb.st_size;
  ParseBufs b;
  if (cudaMallocHost((void**)&b.h_file, len + 1) != cudaSuccess) {
    close(fd);
    cudaGetLastError();
    return fail(GG_ERR_OOM, "read_gpu: no pinned host memory for %zu bytes", len);
  }
  size_t got = 0;
  while (got < len) {
    const ssize_t r = read(fd, b.h_file + got, len - got);
    if (r <= 0) break;
    got += (size_t)r;
  }
  close(fd);
  if (got != len) return fail(GG_ERR_IO, "short read on %s", path);
  b.h_file[len] = 0;
  // header on the host
  const char* p = b.h_file;
  const char* end = p + len;
  while (p < end && blank(*p)) ++p;
  const char* hdr = weighted ? "WeightedAdjacencyGraph" : "AdjacencyGraph";
  const size_t hl = strlen(hdr);
  if ((size_t)(end - p) < hl || strncmp(p, hdr, hl) != 0 || (p + hl < end && !blank(p[hl])))
    return fail(GG_ERR_FORMAT, "Bad input file: %s (expected header %s)", path, hdr);
  p += hl;
  long long hv[2];
  for (long long& x : hv) {
    while (p < end && blank(*p)) ++p;
    char* q;
    errno = 0;
    x = strtoll(p, &q, 10);
    if (q == p || errno || (q < end && !blank(*q))) return fail(GG_ERR_FORMAT, "Bad input file (n,m): %s", path);
    p = q;
  }
  const long long n = hv[0], m = hv[1];
  if (n < 1 || m < 0 || n > 0xffffffffLL || m >= (1LL << 32) - 64)
    return fail(GG_ERR_FORMAT, "Bad input file (n,m): %s", path);
  const uint64_t total = (uint64_t)n + (uint64_t)m * (weighted ? 2 : 1);
  GG_PARSE_CUDA(cudaStreamCreateWithFlags(&b.st, cudaStreamNonBlocking));
  GG_PARSE_CUDA(cudaMalloc(&b.d_chunk, chunk + kMaxToken + 1));
  GG_PARSE_CUDA(cudaMalloc(&b.d_starts, sizeof(uint32_t) * (chunk + kMaxToken + 1) / 2 + 16));
  GG_PARSE_CUDA(cudaMalloc(&b.d_count, sizeof(uint32_t)));
  GG_PARSE_CUDA(cudaMalloc(&b.d_off, sizeof(uint32_t) * ((size_t)n + 1)));
  GG_PARSE_CUDA(cudaMalloc(&b.d_idx, sizeof(uint32_t) * (size_t)(m ? m : 1)));
  if (weighted) GG_PARSE_CUDA(cudaMalloc(&b.d_w, sizeof(int32_t) * (size_t)(m ? m : 1)));
  GG_PARSE_CUDA(cudaMalloc(&b.d_err, sizeof(unsigned)));
  GG_PARSE_CUDA(cudaMemsetAsync(b.d_err, 0, sizeof(unsigned), b.st));
  size_t tmp_bytes = 0;
  thrust::counting_iterator<uint32_t> pos(0);
  GG_PARSE_CUDA(cub::DeviceSelect::If(nullptr, tmp_bytes, pos, b.d_starts, b.d_count, (int)(chunk + kMaxToken),
                                      TokenStart{b.d_chunk}, b.st));
  GG_PARSE_CUDA(cudaMalloc(&b.d_tmp, tmp_bytes));
  int sms = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // chunks of the body, each ending where a number ends
  size_t at = (size_t)(p - b.h_file);
  uint64_t seen = 0;
  while (at < len && seen < total) {
    size_t stop = std::min(len, at + chunk);
    const size_t cut = stop;
    while (stop < len && !blank(b.h_file[stop])) ++stop;
    if (stop - cut > kMaxToken) return fail(GG_ERR_FORMAT, "Bad input file (a number of over %zu bytes): %s", kMaxToken, path);
    const uint32_t L = (uint32_t)(stop - at);
    GG_PARSE_CUDA(cudaMemcpyAsync(b.d_chunk, b.h_file + at, L, cudaMemcpyHostToDevice, b.st));
    GG_PARSE_CUDA(cub::DeviceSelect::If(b.d_tmp, tmp_bytes, pos, b.d_starts, b.d_count, (int)L, TokenStart{b.d_chunk},
                                        b.st));
    uint32_t cnt = 0;
    GG_PARSE_CUDA(cudaMemcpyAsync(&cnt, b.d_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, b.st));
    GG_PARSE_CUDA(cudaStreamSynchronize(b.st));
    if (cnt) {
      const int grid = (int)std::min<uint64_t>((cnt + kParseThreads - 1) / kParseThreads, (uint64_t)sms * 8);
      k_parse_numbers<<<grid, kParseThreads, 0, b.st>>>(b.d_chunk, L, b.d_starts, cnt, seen, (uint64_t)n, (uint64_t)m,
                                                       total, b.d_off, b.d_idx, b.d_w, b.d_err);
      GG_PARSE_CUDA(cudaGetLastError());
    }
    seen += cnt;
    at = stop;
  }
  unsigned err = 0;
  GG_PARSE_CUDA(cudaMemcpyAsync(&err, b.d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, b.st));
  GG_PARSE_CUDA(cudaStreamSynchronize(b.st));
  if (err & kBadNumber) return fail(GG_ERR_FORMAT, "Bad input file (not a number): %s", path);
  if (err & kBadOffset) return fail(GG_ERR_FORMAT, "Bad input file (offsets): %s", path);
  if (err & kBadEdge) return fail(GG_ERR_FORMAT, "Bad input file (edges): %s", path);
  if (seen < total)
    return fail(GG_ERR_FORMAT, "Bad input file (%s): %s", seen < (uint64_t)n ? "offsets"
                               : seen < (uint64_t)(n + m) ? "edges" : "weights", path);
  memset(out, 0, sizeof *out);
  out->n = (uint32_t)n;
  out->m = (uint64_t)m;
  out->symmetric = symmetric;
  out->weight_type = weighted ? GG_W_INT32 : GG_W_NONE;
  out->offsets = (uint32_t*)malloc(4 * ((size_t)n + 1));
  out->indices = (uint32_t*)malloc(4 * (size_t)(m ? m : 1));
  if (weighted) out->weights = malloc(4 * (size_t)(m ? m : 1));
  if (!out->offsets || !out->indices || (weighted && !out->weights)) {
    gg_host_graph_free(out);
    return fail(GG_ERR_OOM, "read_gpu: out of host memory");
  }
  int rc = GG_OK;
  if (cudaMemcpyAsync(out->offsets, b.d_off, 4 * (size_t)n, cudaMemcpyDeviceToHost, b.st) != cudaSuccess ||
      (m && cudaMemcpyAsync(out->indices, b.d_idx, 4 * (size_t)m, cudaMemcpyDeviceToHost, b.st) != cudaSuccess) ||
      (weighted && m &&
       cudaMemcpyAsync(out->weights, b.d_w, 4 * (size_t)m, cudaMemcpyDeviceToHost, b.st) != cudaSuccess) ||
      cudaStreamSynchronize(b.st) != cudaSuccess)
    rc = fail(GG_ERR_CUDA, "read_gpu: copy of the parsed arrays failed");
  out->offsets[n] = (uint32_t)m;
  for (long long i = 0; !rc && i < n; i++)
    if (out->offsets[i] > out->offsets[i + 1]) rc = fail(GG_ERR_FORMAT, "Bad input file (offsets not monotone): %s", path);
  if (rc) gg_host_graph_free(out);
  return rc;
}

}  // namespace gg

extern "C" int gg_host_graph_read_gpu(const char* path, int32_t binary, int32_t symmetric, int32_t weighted,
                                      int64_t chunk_bytes, gg_host_graph* out) {
  if (!path || !out || chunk_bytes < 0) return gg::fail(GG_ERR_INVALID_ARG, "gg_host_graph_read_gpu: bad arguments");
  if (binary) return gg_host_graph_read(path, 1, symmetric, weighted, out);  // nothing to parse in a .gr file
  return gg::parse_adj(path, symmetric, weighted, chunk_bytes, out);
}
