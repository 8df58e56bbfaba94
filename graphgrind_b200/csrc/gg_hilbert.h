// Hilbert-curve key of an edge, shared by host and device builds.
// HilbertEdgeSort (graphgrind/graph-numa.h:353-415): xy2d on a square grid
// whose side is roundUpPow2(n_) (:302-313, :358); the reference constructs
// the sorter with the partition's EDGE count (:487), so the grid side is the
// next power of two of the number of edges in the partition, not of n.
// Signed 64-bit arithmetic as the reference's intT.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define GG_HD __host__ __device__ __forceinline__
#else
#define GG_HD inline
#endif

namespace gg {

GG_HD int64_t hilbert_side(int64_t edges) {
  uint64_t s = (uint64_t)edges;
  --s;
  for (unsigned sh = 1; sh < 64; sh <<= 1) s |= s >> sh;
  ++s;
  return (int64_t)s;
}

GG_HD int64_t hilbert_xy2d(int64_t side, int64_t x, int64_t y) {
  int64_t d = 0;
  for (int64_t s = side / 2; s > 0; s /= 2) {
    const int64_t rx = (x & s) > 0;
    const int64_t ry = (y & s) > 0;
    d += s * s * ((3 * rx) ^ ry);
    if (ry == 0) {
      if (rx == 1) {
        x = s - 1 - x;
        y = s - 1 - y;
      }
      const int64_t t = x;
      x = y;
      y = t;
    }
  }
  return d;
}

}  // namespace gg
