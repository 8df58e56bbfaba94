// Shared host-side helpers of libgg: status codes, thread-local error text.
#pragma once
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>
#include <utility>
#include <vector>

#include "../../include/gg.h"

namespace gg {

void set_error(const char* fmt, ...);
const char* last_error();

// Return `code` after recording a formatted message.
int fail(int code, const char* fmt, ...);

#define GG_TRY_HOST(expr)         \
  do {                            \
    int r__ = (expr);             \
    if (r__ != GG_OK) return r__; \
  } while (0)

// Rows of g renumbered: new vertex i holds the out-edges of old vertex
// old_of_new[i], in their order, with neighbour ids mapped through new_of_old
// and the weights carried along.  out is allocated like gg_host_graph_read's.
int relabel_host_graph(const gg_host_graph* g, const uint32_t* old_of_new, const uint32_t* new_of_old,
                       gg_host_graph* out);
// GG_VORDER_HOT_FIRST: inside every [starts[p], starts[p+1]) the vertices by
// descending out-degree, ties by id.  starts has P+1 ascending entries, 0 .. n.
void hot_first_order(const gg_host_graph* g, const int64_t* starts, int32_t P, uint32_t* old_of_new,
                     uint32_t* new_of_old);

// The deal of VEBO over runs of equal in-degree (degree, vertices) of the
// vertices sorted by (in-degree descending, id): perDeg[p * runs + i] and
// vsize[p]; GG_ERR_PARTITION where the reference's zero-degree fill breaks.
int vebo_deal(const std::vector<std::pair<int64_t, int64_t>>& runs, int64_t n, int64_t P, std::vector<int64_t>& perDeg,
              std::vector<int64_t>& vsize);

inline uint64_t mix64(uint64_t z) {
  // SplitMix64 output function (Steele, Lea & Flood, OOPSLA 2014).
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

}  // namespace gg
