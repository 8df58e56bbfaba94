// Device forms of the applications' functor structs (app/*.C).  Each edge
// functor states the reference member functions it replaces; the pull path
// runs gather/combine/commit (the functor-cache protocol, create_cache /
// update(cache, s) / commit_cache), the push path runs update_atomic.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "gg_device.cuh"

namespace gg {

struct MinI32 {
  using value_t = int32_t;
  static constexpr bool kIdentityCommitNoop = false;
  bool frontier_in_values = false;  // gathered values already mark frontier membership
  bool outside_inert = false;       // a source outside the frontier cannot change any result
  __device__ static value_t identity() { return 0x7fffffff; }
  __device__ static value_t combine(value_t a, value_t b) { return a < b ? a : b; }
  __device__ static void atomic_combine(value_t* s, value_t v) { atomicMin(s, v); }
};
struct MinU32 {
  using value_t = uint32_t;
  static constexpr bool kIdentityCommitNoop = false;
  bool frontier_in_values = false;  // gathered values already mark frontier membership
  bool outside_inert = false;       // a source outside the frontier cannot change any result
  __device__ static value_t identity() { return 0xffffffffu; }
  __device__ static value_t combine(value_t a, value_t b) { return a < b ? a : b; }
  __device__ static void atomic_combine(value_t* s, value_t v) { atomicMin(s, v); }
};
struct SumF32 {
  using value_t = float;
  static constexpr bool kIdentityCommitNoop = false;  // set by functors whose commit is "+= acc" alone
  bool frontier_in_values = false;  // gathered values already mark frontier membership
  bool outside_inert = false;       // a source outside the frontier cannot change any result
  __device__ static value_t identity() { return 0.0f; }
  __device__ static value_t combine(value_t a, value_t b) { return a + b; }
  __device__ static void atomic_combine(value_t* s, value_t v) { atomicAdd(s, v); }
};

// BFS_F, app/BFS.C:26-75.  cond = unvisited; update = first writer becomes
// the parent (the pull keeps the smallest frontier in-neighbour; parents are
// order-dependent in the reference too); updateAtomic = CAS(-1 -> s).
// Also records the level (edgeMap round) of every newly reached vertex.
struct BfsF : MinU32 {
  static constexpr bool kPositive = false;
  static constexpr bool kEarlyExit = true;
  static constexpr bool kCondTrue = false;
  static constexpr bool kUsesWeight = false;
  int32_t* parents;
  int32_t* levels;
  int32_t round;
  __device__ bool cond(uint32_t d) const { return __ldcg(parents + d) == -1; }
  __device__ value_t gather(uint32_t s, uint32_t) const { return s; }
  __device__ bool commit(uint32_t d, value_t acc) const {
    parents[d] = (int32_t)acc;
    if (levels) levels[d] = round;
    return true;
  }
  __device__ bool update_atomic(uint32_t s, uint32_t d, uint32_t) const {
    if (atomicCAS(parents + d, -1, (int32_t)s) == -1) {
      if (levels) levels[d] = round;
      return true;
    }
    return false;
  }
};

// CC_F, app/Components.C:26-85.  Pull = the cached form (:57-79):
// min over prevIDs[s]; output iff the label drops and IDs[d]==prevIDs[d].
// Push = updateAtomic (:152-157): writeMin(IDs[d], IDs[s]) && orig==prevIDs[d].
struct CcF : MinI32 {
  static constexpr bool kPositive = false;
  static constexpr bool kEarlyExit = false;
  static constexpr bool kCondTrue = true;
  static constexpr bool kUsesWeight = false;
  int32_t* ids;
  int32_t* prev;
  __device__ bool cond(uint32_t) const { return true; }
  __device__ value_t gather(uint32_t s, uint32_t) const { return __ldg(prev + s); }
  __device__ bool commit(uint32_t d, value_t acc) const {
    const int32_t orig = ids[d];
    if (acc < orig) {
      ids[d] = acc;
      return orig == prev[d];
    }
    return false;
  }
  __device__ bool update_atomic(uint32_t s, uint32_t d, uint32_t) const {
    const int32_t v = __ldcg(ids + s);
    const int32_t old = atomicMin(ids + d, v);
    return v < old && old == prev[d];
  }
};

// PR_F, app/PageRank.C:28-70: p_next[d] += p_curr[s]/outdeg(s).  The
// division is done once per source (contrib[s] = p_curr[s]/outdeg(s)) by the
// iteration's vertex pass; the per-edge value is the same FP32 quotient.
// Also PageRankDelta's PR_F (app/PageRankDelta.C:29-71) with contrib = Delta/outdeg.
// POS: every contribution is > 0 (PageRank: frontier sources have p > 0), so
// a destination was updated iff its accumulator differs from 0 and the pull
// needs no separate "touched" flag.  PageRankDelta's Delta can be 0 or < 0.
template <bool POS>
struct PrT : SumF32 {
  static constexpr bool kIdentityCommitNoop = true;  // commit is acc_out[d] += acc
  static constexpr bool kEarlyExit = false;
  static constexpr bool kCondTrue = true;
  static constexpr bool kPositive = POS;
  static constexpr bool kUsesWeight = false;
  const float* contrib;
  float* acc_out;
  __device__ bool cond(uint32_t) const { return true; }
  __device__ value_t gather(uint32_t s, uint32_t) const { return __ldg(contrib + s); }
  // gather with an L2 eviction policy (kept ahead of the streamed edges)
  __device__ value_t gather_pol(uint32_t s, uint32_t, uint64_t pol) const {
    return gg::ld_keep_f32(contrib + s, pol);
  }
  __device__ bool commit(uint32_t d, value_t acc) const {
    acc_out[d] += acc;
    return true;
  }
  __device__ bool update_atomic(uint32_t s, uint32_t d, uint32_t) const {
    atomicAdd(acc_out + d, __ldg(contrib + s));
    return true;
  }
};
using PrF = PrT<false>;
using PrPosF = PrT<true>;

// PageRank's pull with the vertex step of app/PageRank.C (PR_Vertex_F and
// PR_Vertex_Reset, :84-100, and the L1 term of :136-139) applied where the
// per-warp COO pull commits a tile's destinations (each destination belongs
// to one tile, so its sum is final there): rank = the accumulated sum, for
// input-frontier members damping * rank + (1 - damping)/n; L1 += |previous -
// rank|; the previous-rank buffer becomes the next accumulator (0 for members,
// the difference for the others); the next contribution rank/outdeg, -1 for
// sources outside the output when the output marks the frontier.  The
// contributions are double-buffered: the pull reads contrib and writes
// contrib_next.  Other kernels apply PrT's commit and leave the vertex step
// to a separate pass.
struct PrFinishF : PrT<true> {
  static constexpr bool kFinish = true;
  static constexpr bool kIdentityCommitNoop = false;  // the vertex step visits every destination
  float* p_prev;            // ranks of the previous iteration, reset in place
  const uint32_t* fbits;    // input frontier (null: every vertex)
  float* contrib_next;
  double* l1;
  float damping, added;
  int masked;               // the output marks the next frontier in contrib_next
  // vertex v of the tile: s = its accumulated sum (touched: s came from an
  // edge), d = its out-degree; returns its L1 term
  __device__ float finish(uint32_t v, bool touched, float s, uint32_t d) const {
    return finish_apply(v, finish_load(v), touched, s, d);
  }
  // The vertex step split into its loads and the rest, so that a caller can
  // issue the loads of several vertices before it needs any of them.
  struct FinishIn {
    float acc, prev;
    bool in;
  };
  __device__ FinishIn finish_load(uint32_t v) const {
    FinishIn x;
    x.acc = acc_out[v];
    x.prev = p_prev[v];
    x.in = !fbits || ((fbits[v >> 5] >> (v & 31)) & 1u);
    return x;
  }
  __device__ float finish_apply(uint32_t v, const FinishIn& x, bool touched, float s, uint32_t d) const {
    float pn = x.acc;
    if (touched) pn += s;
    if (x.in) pn = damping * pn + added;
    const float diff = fabsf(x.prev - pn);
    acc_out[v] = pn;
    p_prev[v] = x.in ? 0.0f : diff;
    contrib_next[v] = d ? ((!masked || touched) ? pn / (float)d : -1.0f) : 0.0f;
    return diff;
  }
};

// SPMV_F, app/SPMV.C:7-48: p_next[d] += p_curr[s] * edgeLen.  Weights are
// the reference's int edge lengths, or FP32 when the graph carries FP32 weights.
struct SpmvF : SumF32 {
  static constexpr bool kIdentityCommitNoop = true;  // commit is y[d] += acc
  static constexpr bool kPositive = false;
  static constexpr bool kEarlyExit = false;
  static constexpr bool kCondTrue = true;
  static constexpr bool kUsesWeight = true;
  const float* x;
  float* y;
  int float_w;
  const uint32_t* y_map = nullptr;  // y is indexed by y_map[d] (the given ids of a renumbered graph), else by d
  __device__ float wv(uint32_t w) const { return float_w ? __uint_as_float(w) : (float)(int32_t)w; }
  __device__ uint32_t yi(uint32_t d) const { return y_map ? __ldg(y_map + d) : d; }
  __device__ bool cond(uint32_t) const { return true; }
  __device__ value_t gather(uint32_t s, uint32_t w) const { return __ldg(x + s) * wv(w); }
  __device__ value_t gather_pol(uint32_t s, uint32_t w, uint64_t pol) const {
    return gg::ld_keep_f32(x + s, pol) * wv(w);
  }
  __device__ bool commit(uint32_t d, value_t acc) const {
    y[yi(d)] += acc;
    return true;
  }
  __device__ bool update_atomic(uint32_t s, uint32_t d, uint32_t w) const {
    atomicAdd(y + yi(d), __ldg(x + s) * wv(w));
    return true;
  }
};

// BF_F, app/BellmanFord.C:28-91.  Pull = cached form: min of SP[s]+w over the
// frontier in-neighbours; output iff it lowers SP[d] and Visited[d] was 0.
// Push = writeMin(SP[d], SP[s]+w) && CAS(Visited[d], 0, 1).
struct BfF : MinI32 {
  static constexpr bool kPositive = false;
  static constexpr bool kEarlyExit = false;
  static constexpr bool kCondTrue = true;
  static constexpr bool kUsesWeight = true;
  int32_t* sp;
  int32_t* visited;
  __device__ bool cond(uint32_t) const { return true; }
  __device__ value_t gather(uint32_t s, uint32_t w) const { return __ldcg(sp + s) + (int32_t)w; }
  __device__ bool commit(uint32_t d, value_t acc) const {
    if (acc < sp[d]) {
      sp[d] = acc;
      if (visited[d] == 0) {
        visited[d] = 1;
        return true;
      }
    }
    return false;
  }
  __device__ bool update_atomic(uint32_t s, uint32_t d, uint32_t w) const {
    const int32_t nd = __ldcg(sp + s) + (int32_t)w;
    const int32_t old = atomicMin(sp + d, nd);
    if (nd < old) return atomicCAS(visited + d, 0, 1) == 0;
    return false;
  }
};

// BC_F / BC_Back_F, app/BC.C:28-126: value[d] += value[s] for unvisited d;
// output iff value[d] was 0 before (first path reaching d).
struct BcF : SumF32 {
  static constexpr bool kPositive = false;
  static constexpr bool kEarlyExit = false;
  static constexpr bool kCondTrue = false;
  static constexpr bool kUsesWeight = false;
  float* values;
  const uint8_t* visited;
  __device__ bool cond(uint32_t d) const { return visited[d] == 0; }
  __device__ value_t gather(uint32_t s, uint32_t) const { return __ldcg(values + s); }
  __device__ bool commit(uint32_t d, value_t acc) const {
    const float old = values[d];
    values[d] = old + acc;
    return old == 0.0f;
  }
  __device__ bool update_atomic(uint32_t s, uint32_t d, uint32_t) const {
    return atomicAdd(values + d, __ldcg(values + s)) == 0.0f;
  }
};

// ------------------------------------------------------- vertex functors
// CC_Vertex_F, app/Components.C:88-99
struct VCcCopy {
  int32_t* ids;
  int32_t* prev;
  __device__ bool operator()(uint32_t i) const {
    prev[i] = ids[i];
    return true;
  }
};
// PR_Vertex_F, app/PageRank.C:73-87
struct VPrUpdate {
  float* p_next;
  float damping, added;
  __device__ bool operator()(uint32_t i) const {
    p_next[i] = damping * p_next[i] + added;
    return true;
  }
};
template <class T>
struct VFill {
  T* a;
  T value;
  __device__ bool operator()(uint32_t i) const {
    a[i] = value;
    return true;
  }
};
// PR_Vertex_F_FirstRound, app/PageRankDelta.C:73-89
struct VPrdFirst {
  float* p;
  float* delta;
  const float* ngh;
  float damping, added, one_over_n, eps2;
  __device__ bool operator()(uint32_t i) const {
    float d = damping * (p[i] + ngh[i]) + added - p[i];
    const float pi = p[i] + d;
    p[i] = pi;
    d -= one_over_n;
    delta[i] = d;
    return fabsf(d) > eps2 * pi;
  }
};
// PR_Vertex_F, app/PageRankDelta.C:91-105
struct VPrd {
  float* p;
  float* delta;
  const float* ngh;
  float damping, eps2;
  __device__ bool operator()(uint32_t i) const {
    const float d = ngh[i] * damping;
    delta[i] = d;
    const float pi = p[i] + d;
    p[i] = pi;
    return fabsf(d) > eps2 * pi;
  }
};
// BC_Vertex_F, app/BC.C:129-138
struct VBcMark {
  uint8_t* visited;
  __device__ bool operator()(uint32_t i) const {
    visited[i] = 1;
    return true;
  }
};
// BC_Back_Vertex_F, app/BC.C:142-154
struct VBcBack {
  uint8_t* visited;
  float* dep;
  const float* inv;
  __device__ bool operator()(uint32_t i) const {
    visited[i] = 1;
    dep[i] += inv[i];
    return true;
  }
};

}  // namespace gg
