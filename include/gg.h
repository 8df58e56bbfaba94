/*
 * gg.h -- C ABI of the B200 traversal engine (edgeMap / vertexMap / vertexFilter
 * over a destination-range partitioned, Hilbert-ordered graph).
 *
 * The reference (GraphGrind) has no FFI: its interface is header-only C++
 * templates instantiated by each application's Compute().  Every entry point
 * below names the reference interface it replaces (file:line inside the
 * GraphGrind source tree).  Conventions:
 *   - every function returns an int status: GG_OK (0) or a negative GG_ERR_*;
 *     the library never aborts; gg_last_error_string() explains the last error
 *     of the calling thread (the reference abort()s / assert()s instead,
 *     graphgrind/ligra-numa.h:937-942, graphgrind/graph-numa.h:1253,1353);
 *   - vertex ids and CSR/CSC offsets are uint32 (m < 2^32);
 *   - device memory is owned by the library and released by *_destroy;
 *   - a graph handle is not thread-safe; distinct handles may be used from
 *     distinct threads.
 * Functions under "host-only" touch no GPU and work on machines without one.
 */
#ifndef GG_H
#define GG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define GG_OK 0
#define GG_ERR_INVALID_ARG -1
#define GG_ERR_CUDA -2
#define GG_ERR_OOM -3
#define GG_ERR_PARTITION -4   /* reference partitioner would assert/overflow */
#define GG_ERR_IO -5
#define GG_ERR_FORMAT -6
#define GG_ERR_NO_DEVICE -7
#define GG_ERR_UNSUPPORTED -8
#define GG_ERR_TIMEOUT -9     /* a bounded device-side wait gave up */
#define GG_ERR_SIZE -10       /* n or m beyond the uint32 limits */

/* Human-readable text of the calling thread's last error. */
const char* gg_last_error_string(void);
/* Library version string. */
const char* gg_version(void);

/* ------------------------------------------------------ enums and flags */
enum gg_weight_type { GG_W_NONE = 0, GG_W_INT32 = 1, GG_W_FLOAT32 = 2 };
enum gg_balance { GG_BALANCE_EDGE = 0, GG_BALANCE_VERTEX = 1 };     /* -v edge|vertex */
enum gg_part_how { GG_PART_DEST = 0, GG_PART_SOURCE = 1 };          /* -P dest|source */
enum gg_order { GG_ORDER_HILBERT = 1, GG_ORDER_CSR = 0 };           /* EDGES_HILBERT */

/* Options of gg_graph_build, mirroring parallel_main's flags
 * (graphgrind/ligra-numa.h:1097-1130) plus GPU tiling knobs (0 = default). */
typedef struct gg_build_opts {
  int32_t num_partitions;   /* -c   (default 384)                           */
  int32_t balance;          /* -v   gg_balance                              */
  int32_t part_how;         /* -P   gg_part_how                             */
  int32_t relabel;          /* -o   partition boundaries at degree rises    */
  int32_t order;            /* EDGES_HILBERT: gg_order                      */
  int32_t tile_vertices;    /* GPU: max destinations per CTA tile (<=4096;
                               0 or larger values give 4096)             */
  int32_t tile_edges;       /* GPU: target edges per CTA tile               */
  int32_t build_coo;        /* 1 = build the partitioned COO (default when balance==edge) */
  int32_t coo_window;       /* GPU: order inside a COO tile after the Hilbert sort:
                               0 = destination order inside 256-edge windows;
                               W > 0 = source order inside windows of W edges
                               (rounded up to a multiple of 256), which lets a
                               warp's 32 gathers share cache lines          */
  int32_t coo_dst_window;   /* GPU: edges per destination-ordered window when
                               coo_window == 0 (multiple of 256; 0 = 256)    */
  int32_t vertex_order;     /* GPU: gg_vertex_order (0 = the given ids)      */
  int32_t coo_tile_vertices;/* GPU: max destinations per COO tile (<= 16384;
                               0 = tile_vertices); the CSC tiles keep
                               tile_vertices                                 */
} gg_build_opts;

/* Device-side vertex numbering of a graph (gg_build_opts.vertex_order).
 * GG_VORDER_HOT_FIRST renumbers the vertices inside every partition of the
 * COO partitioner (computed on the given ids) by descending out-degree, ties
 * by id: each partition keeps its vertex set and size, and the sources a
 * dense pull gathers most share cache lines.  The
 * applications (gg_bfs ... gg_msbc) take and return the given ids and arrays
 * in the given order, with results equal to the unrenumbered graph's (FP32
 * sums up to their summation order; BFS parents are another valid tree).
 * The low-level API (frontiers, edgeMap / vertexMap arrays, device arrays,
 * gg_bfs_push_step_noalloc on the device arrays) speaks the device ids:
 * gg_graph_vertex_order gives the map.  gg_bp and gg_pagerank_weighted_*,
 * whose inputs are per-edge arrays, return GG_ERR_UNSUPPORTED on such graphs. */
enum gg_vertex_order { GG_VORDER_GIVEN = 0, GG_VORDER_HOT_FIRST = 1 };

typedef struct gg_graph_info {
  uint32_t n;
  uint64_t m;
  int32_t symmetric;
  int32_t weight_type;
  int32_t num_partitions;
  int32_t has_coo;
  int32_t transposed;
  int32_t num_csc_tiles;
  int32_t num_coo_tiles;
  uint64_t device_bytes;    /* HBM held by the graph */
  int32_t num_coo_gaps;     /* destination ranges with no in-edges, outside every COO tile */
} gg_graph_info;

/* ==================================================== host-only: graphs */
/* A host CSR graph (out-edges).  offsets has n+1 entries. */
typedef struct gg_host_graph {
  uint32_t n;
  uint64_t m;
  int32_t symmetric;
  int32_t weight_type;      /* gg_weight_type */
  uint32_t* offsets;        /* n+1 */
  uint32_t* indices;        /* m   */
  void* weights;            /* m x 4 bytes or NULL */
} gg_host_graph;

/* Seeded generators (replace the absent rMatGraph inputs of the reference
 * README; no generator exists in the reference).  Self-loops and duplicate
 * edges are removed; symmetric=1 adds the reverse of every edge first.
 * RMAT: 2^scale vertices, edge_factor*2^scale sampled edges, (a,b,c,d). */
int gg_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c,
                uint64_t seed, int32_t symmetric, gg_host_graph* out);
/* 2D side x side 4-neighbour grid (symmetric) plus long_range_frac * grid-edges
 * uniformly random extra undirected edges. */
int gg_gen_grid(int32_t side, double long_range_frac, uint64_t seed, gg_host_graph* out);
/* Erdos-Renyi G(n, m): m uniformly random (src,dst) samples. */
int gg_gen_er(uint32_t n, uint64_t m, uint64_t seed, int32_t symmetric, gg_host_graph* out);
/* Attach weights: GG_W_INT32 uniform in [lo,hi]; GG_W_FLOAT32 uniform in (0,1].
 * The weight is a hash of (seed, src, dst), so an edge and its reverse view
 * in the CSC carry the same weight. */
int gg_host_graph_add_weights(gg_host_graph* g, int32_t weight_type, uint64_t seed,
                              int32_t lo, int32_t hi);
/* Read/write the reference's input formats (graphgrind/IO.h:136-199 PBBS
 * text, graphgrind/IO.h:365-450 Galois .gr v1).  A directed .gr/.adj also gets
 * its "<path>_t" transpose file on write, which the reference loads when present. */
int gg_host_graph_write_adj(const gg_host_graph* g, const char* path);
int gg_host_graph_write_gr(const gg_host_graph* g, const char* path);
int gg_host_graph_read(const char* path, int32_t binary, int32_t symmetric,
                       int32_t weighted, gg_host_graph* out);
/* The same reader with the PBBS text body parsed on the GPU (readGraphFromFile,
 * graphgrind/IO.h:136-199): the file is read once into pinned memory, its
 * header on the host, and the body crosses to the device in chunks of
 * chunk_bytes (0 = 256 MiB; cut where a number ends), where the numbers are
 * found, converted and range-checked in parallel.  Same result and the same
 * GG_ERR_FORMAT cases as gg_host_graph_read (a number of more than 18 digits
 * is also one); binary != 0 reads a .gr file as gg_host_graph_read does.
 * Needs a CUDA device; the device memory it takes is released on return. */
int gg_host_graph_read_gpu(const char* path, int32_t binary, int32_t symmetric,
                           int32_t weighted, int64_t chunk_bytes, gg_host_graph* out);
/* VEBO reordering (graphtools/VEBO.C:56-395, the tool that prepares graphs
 * for -o): vertices sorted by in-degree are dealt to `partitions` partitions
 * that balance edges first and vertices second, and renumbered partition by
 * partition.  out: the relabelled graph (out-edges of the old vertex at each
 * new id, neighbour order kept, weights carried along); new_of_old[n] and
 * part_sizes[partitions] may be NULL.  GG_ERR_PARTITION where the reference's
 * zero-degree fill would place a different number of vertices than n. */
int gg_vebo(const gg_host_graph* g, int32_t partitions, uint32_t* new_of_old, int64_t* part_sizes,
            gg_host_graph* out);
/* gg_vebo computed on the GPU (the same arguments, result, bit for bit, and
 * errors): the in-degree histogram, the (in-degree, id) sort, the runs of
 * equal degree and the placement and relabelling run on the device; the deal
 * of the runs to partitions, which depends on every earlier deal, runs on the
 * host over the runs alone.  The host graph crosses to the device and back;
 * needs a CUDA device, whose memory it takes is released on return. */
int gg_vebo_gpu(const gg_host_graph* g, int32_t partitions, uint32_t* new_of_old, int64_t* part_sizes,
                gg_host_graph* out);
/* CSC (in-edges) of a host graph: in_offsets n+1, in_indices m, in_weights m. */
int gg_host_graph_transpose(const gg_host_graph* g, gg_host_graph* out);
void gg_host_graph_free(gg_host_graph* g);

/* Partition sizes exactly as the reference computes them
 * (partitionByDegree graphgrind/graph-numa.h:1287-1357, partitionByVertex
 * :1177-1206) for the COO partitions, and (cscpartitionByDegree :1208-1256,
 * cscpartitionByVertex :1258-1285) for the compressed CSC ranges.  The one
 * deviation: degrees[n] (read one past the end at :1335 / :1248) is taken as 0.
 * Returns GG_ERR_PARTITION where the reference asserts (counter+1 != P) or
 * would index past its P-entry arrays.  sizes has P entries. */
int gg_partition_sizes(const uint32_t* in_degrees, const uint32_t* out_degrees, uint32_t n,
                       uint64_t m, int32_t P, int32_t balance, int32_t part_how,
                       int32_t relabel, int64_t* coo_sizes, int64_t* csc_sizes);
/* GG_VORDER_HOT_FIRST for graph g built with opts (num_partitions, balance,
 * part_how, relabel): the COO partition starts (P+1 entries, may be NULL) of
 * the given ids, and new_of_old[n], the device id gg_graph_build gives each
 * vertex: inside every partition, the vertices by descending out-degree, ties
 * by id.  Host-only; gg_graph_build with vertex_order = GG_VORDER_HOT_FIRST
 * uses the same order. */
int gg_hot_first_order(const gg_host_graph* g, const gg_build_opts* opts, uint32_t* new_of_old,
                       int64_t* starts);
/* Hilbert key of edge (x=src, y=dst) on the reference's grid, whose side is
 * roundUpPow2(edges in the partition) (graphgrind/graph-numa.h:353-386, 487). */
int64_t gg_hilbert_key(int64_t side_edges, int64_t x, int64_t y);

/* ============================================================ device graph */
typedef struct gg_graph_s* gg_graph_t;
typedef struct gg_frontier_s* gg_frontier_t;

/* partitioned_graph constructor (graphgrind/graph-numa.h:642-685): uploads the
 * CSR, builds CSC, the -c destination-range partitions and, for -v edge, the
 * Hilbert/CSR-sorted partitioned COO, cut into CTA tiles sized to shared memory. */
int gg_graph_build(const gg_host_graph* g, const gg_build_opts* opts, gg_graph_t* out);
int gg_graph_destroy(gg_graph_t g);
/* Waits for the graph's work and for the result copies that
 * GG_TUNE_ASYNC_RESULTS left in flight. */
int gg_graph_synchronize(gg_graph_t g);
int gg_graph_get_info(gg_graph_t g, gg_graph_info* info);
/* Partition starts (P+1 entries) of the COO partitioner (partitioner::start_of,
 * graphgrind/partitioner.h:153-165). */
int gg_graph_partition_starts(gg_graph_t g, int64_t* starts);
/* The partitioned COO as the device holds it (COOPartitionByDest /
 * COOPartitionBySour + hilbert_sort, graphgrind/graph-numa.h:482-490,
 * 1116-1171), for inspection: *num_tiles CTA tiles in the order the
 * persistent kernels take them, tiles[4 t .. 4 t + 3] = {first destination,
 * destinations, first slot, slots} (for -P source: one entry per source
 * partition, {first source, sources, first slot, edges}); src/dst[coo_len]
 * the edge of every slot, 0xffffffff in the padding that rounds a tile up
 * to 8 slots.  Inside a tile the edges follow the partition's Hilbert (or
 * CSRDestSort) order at 256-slot granularity and go by destination inside
 * each 256-slot window.  tiles, src and dst may be NULL (sizes only).
 * GG_ERR_UNSUPPORTED for a graph without a COO (-v vertex). */
int gg_graph_coo_layout(gg_graph_t g, uint64_t* num_tiles, uint32_t* tiles, uint64_t* coo_len, uint32_t* src,
                        uint32_t* dst);
/* partitioned_graph::transpose (graphgrind/graph-numa.h:721-728): swaps the
 * out/in roles of CSR and CSC for symmetric=0 graphs; the COO partitions are
 * NOT transposed, as in the reference. */
int gg_graph_transpose(gg_graph_t g);
/* new_of_old[n]: the device id of every given vertex id (the identity unless
 * the graph was built with a vertex_order). */
int gg_graph_vertex_order(gg_graph_t g, uint32_t* new_of_old);
/* Device CSR (out-edges) and CSC (in-edges) of the current orientation, in
 * the device ids (the vertex array and neighbour lists that
 * symmetricVertex/asymmetricVertex wrap, graphgrind/graph-numa.h:39-217);
 * any output may be NULL.  Owned by the graph. */
int gg_graph_device_arrays(gg_graph_t g, const uint32_t** out_offsets,
                           const uint32_t** out_indices, const uint32_t** in_offsets,
                           const uint32_t** in_indices);
/* The edge weights beside those lists (int32 or float32 by the graph's
 * weight_type; getOutWeight/getInWeight, graphgrind/graph-numa.h:63-86),
 * NULL for an unweighted graph. */
int gg_graph_device_weights(gg_graph_t g, const void** out_weights, const void** in_weights);

/* ===================================================== vertexSubset API */
/* partitioned_vertices (graphgrind/ligra-numa.h:91-272). */
int gg_frontier_single(gg_graph_t g, uint32_t v, gg_frontier_t* out);   /* ::create :103 */
int gg_frontier_all(gg_graph_t g, gg_frontier_t* out);                  /* ::bits   :169 */
int gg_frontier_empty(gg_graph_t g, gg_frontier_t* out);                /* ::empty  :119 */
/* From a host byte mask (1 = active); the frontier is dense with exact stats. */
int gg_frontier_from_mask(gg_graph_t g, const uint8_t* mask, gg_frontier_t* out);
/* From a host vertex list (must be duplicate-free); the frontier is sparse. */
int gg_frontier_from_list(gg_graph_t g, const uint32_t* verts, uint64_t count,
                          gg_frontier_t* out);
int gg_frontier_destroy(gg_frontier_t f);                               /* ::del    :210 */
/* numNonzeros (:268) and num_out_edges (:99). */
int gg_frontier_stats(gg_frontier_t f, uint64_t* active, uint64_t* out_edges);
/* Dense byte mask (n bytes) of the members, copied to the host. */
int gg_frontier_to_mask(gg_frontier_t f, uint8_t* mask);
/* Force representation: toDense (:228) / toSparse (:246). */
int gg_frontier_to_dense(gg_frontier_t f);
int gg_frontier_to_sparse(gg_frontier_t f);
/* 1 if the frontier currently holds a dense bitmap, 2 if sparse, 3 both, 4 'bit' (all). */
int gg_frontier_repr(gg_frontier_t f);

/* ================================================== built-in functors */
/* The functor structs of the app/ sources re-hosted as device functors.  Arguments
 * point at device vertex arrays allocated with gg_vertex_array_alloc. */
enum gg_functor_id {
  GG_F_BFS = 1,            /* app/BFS.C:26-75            args: gg_bfs_args      */
  GG_F_CC = 2,             /* app/Components.C:26-85     args: gg_cc_args       */
  GG_F_PR = 3,             /* app/PageRank.C:28-70       args: gg_pr_args       */
  GG_F_PRDELTA = 4,        /* app/PageRankDelta.C:29-71  args: gg_prdelta_args  */
  GG_F_SPMV = 5,           /* app/SPMV.C:7-48            args: gg_spmv_args     */
  GG_F_BF = 6,             /* app/BellmanFord.C:28-91    args: gg_bf_args       */
  GG_F_BC = 7,             /* app/BC.C:28-77 (BC_F)      args: gg_bc_args       */
  GG_F_BC_BACK = 8,        /* app/BC.C:79-126 (BC_Back_F) args: gg_bc_args      */
  GG_F_BP = 9              /* app/BP.C:54-133            args: gg_bp_args       */
};
typedef struct { int32_t* parents; int32_t* levels; int32_t round; } gg_bfs_args;
typedef struct { int32_t* ids; int32_t* prev_ids; } gg_cc_args;
typedef struct { const float* p_curr; float* p_next; } gg_pr_args;
typedef struct { const float* delta; float* ngh_sum; } gg_prdelta_args;
typedef struct { const float* p_curr; float* p_next; } gg_spmv_args;
typedef struct { int32_t* sp_len; int32_t* visited; } gg_bf_args;
typedef struct { float* values; uint8_t* visited; } gg_bc_args;
typedef struct { const float* edge_pot; const float* vert_pot; const float* edge_cur;
                 float* edge_next; const float* vert_cur; float* vert_next; } gg_bp_args;

/* edgeMap flags */
#define GG_EM_FORCE_SPARSE 0x1u   /* take the push branch regardless of size   */
#define GG_EM_FORCE_CSC 0x2u      /* dense branch: pull over CSC                */
#define GG_EM_FORCE_COO 0x4u      /* dense branch: partitioned COO              */
#define GG_EM_NO_OUTPUT 0x8u      /* caller discards the output (output.del()):
                                     a dense COO pull of a sum functor (GG_F_SPMV)
                                     then skips building it and *out is empty  */

/* Per-call statistics of the last edgeMap on a graph handle. */
typedef struct gg_edge_map_stats {
  int32_t kind;             /* 0 empty, 1 sparse push, 2 dense CSC pull, 3 dense COO */
  uint64_t frontier_active;
  uint64_t frontier_out_edges;
  uint64_t output_active;
  uint64_t output_out_edges;
} gg_edge_map_stats;

/* edgeMap (graphgrind/ligra-numa.h:919-1019): threshold < 0 means m/20;
 * direction switch m_f + outdeg(F) > threshold -> dense, > m/2 (and
 * balance==edge) -> COO else CSC pull; otherwise sparse push over CSR. */
int gg_edge_map(gg_graph_t g, gg_frontier_t in, int32_t functor_id, const void* functor_args,
                int64_t threshold, uint32_t flags, gg_frontier_t* out);
int gg_last_edge_map_stats(gg_graph_t g, gg_edge_map_stats* stats);

/* Kernel timing (replaces the reference's per-phase tmlog accumulators,
 * graphgrind/ligra-numa.h:61-79): when enabled, every edgeMap kernel is
 * bracketed by CUDA events on the graph's stream.  kind: 0 sparse push,
 * 1 dense CSC pull, 2 dense COO pull, 3 early-exit pull. */
typedef struct gg_profile {
  uint64_t launches[4];
  double ms[4];
  uint64_t edges[4];        /* edges streamed by those launches */
} gg_profile;
int gg_graph_set_profiling(gg_graph_t g, int32_t enable);
/* Copies the accumulated profile and resets it. */
int gg_graph_get_profile(gg_graph_t g, gg_profile* out);
/* Dense-branch kernel policy: 0 = the reference's rule (COO above m/2 when
 * the COO exists, else CSC), 1 = always CSC pull, 2 = always COO pull. */
int gg_graph_set_dense_policy(gg_graph_t g, int32_t policy);
/* Engine tuning knobs (all keep edgeMap's results; they pick kernels):
 *   GG_TUNE_DENSE_POLICY  as gg_graph_set_dense_policy
 *   GG_TUNE_COO_KERNEL    0 CTA-wide bulk-copy ring, 1 per-warp direct loads,
 *                         2/3 per-warp bulk-copy ring with 2/3 stages,
 *                         4 per-warp direct loads with lane-contiguous edges
 *                         and one shared-memory accumulation per edge (the
 *                         default for graphs built with coo_window > 0),
 *                         5 per-warp direct loads with the next block's edge
 *                         stream prefetched into registers, 6 per-warp direct
 *                         loads with destination runs merged across lanes;
 *                         7 kernel 6 with cache hints (the default for graphs
 *                         built with coo_window == 0): the edge stream read
 *                         past L1 and marked evict-first in L2, the source
 *                         gathers of PageRank and SpMV marked evict-last in
 *                         L1 and L2; PageRank's vertex step at the commits
 *                         loads four 32-vertex groups ahead
 *   GG_TUNE_SPARSE_DIV    the application loops (gg_bfs ... gg_bc) call edgeMap
 *                         with threshold m / value (20 in the reference apps)
 *   GG_TUNE_DEVICE_LOOP   2 (default): gg_bfs runs the whole BFS in one
 *                         cooperative launch, dense levels bottom-up over the
 *                         in-edges (first frontier in-neighbour, as
 *                         edgeMapDenseCSC with BFS_F) and sparse levels
 *                         top-down, the direction rule and the queue/bitmap
 *                         conversions done on the device (transposed graphs
 *                         and dense policy 2 take mode 1); 1: runs of
 *                         consecutive sparse levels in one cooperative launch
 *                         each, dense levels from the host; 0: one host round
 *                         trip per level
 *   GG_TUNE_ROUND_GRAPH   1 (default): gg_bellman_ford, gg_components and
 *                         gg_pagerank_delta run each stretch of rounds that
 *                         edgeMap sends to the dense COO pull as one CUDA
 *                         graph (the round's edgeMap and vertex step, then a
 *                         check kernel that applies the loop's tests, L1 <
 *                         eps for PageRankDelta, and the direction rule on
 *                         the device); the graph and the application's
 *                         n-entry arrays (two, four for PageRankDelta) stay
 *                         with the graph handle.  0: one host round trip per
 *                         round.  Falls back to 0 by itself when the
 *                         driver refuses the capture; profiling also takes
 *                         the host loop
 *   GG_TUNE_LOOP_CTAS     CTAs per SM of those cooperative launches, 0..16
 *                         (0, the default: 4 for mode 1, 8 for mode 2; capped
 *                         by the kernel's occupancy)
 *   GG_TUNE_CC_ALGO       0 (default): gg_components runs app/Components.C's
 *                         label propagation through edgeMap; 1: on symmetric
 *                         graphs, a union-find pass over the edges (each root
 *                         hooked under the smaller one), which ends with the
 *                         same labels (the smallest id of each component) and
 *                         reports 1 round; directed graphs keep label
 *                         propagation, whose labels are not components
 *   GG_TUNE_PR_GRAPH      1 (default): gg_pagerank runs its iterations as one
 *                         CUDA graph (a while node; L1, the iteration count and
 *                         the direction rule are checked on the device) while
 *                         each edgeMap takes the dense COO pull, and hands the
 *                         loop back to the host otherwise; the graph and its
 *                         rank buffers (16 bytes per vertex) stay with the
 *                         graph handle.  Falls back to 0 by itself when the
 *                         driver refuses the capture; profiling (see
 *                         gg_graph_set_profiling) also takes the host loop.
 *                         0: one host round trip per iteration
 *   GG_TUNE_ASYNC_RESULTS 0 (default): the applications return once their
 *                         results are in the host arrays; 1: a result bound
 *                         for pinned host memory (cudaMallocHost or
 *                         cudaHostRegister) is copied on a second stream
 *                         while the call returns, so that the copy overlaps
 *                         the next call's work; gg_graph_synchronize waits
 *                         for every such copy (read the arrays after it).
 *                         Pageable arrays are filled before the call
 *                         returns in both modes.  The mode holds three
 *                         n-entry staging arrays per graph (BFS's parents
 *                         have one of their own); small control results
 *                         (loop states, statistics) never take a copy engine,
 *                         so the calls do not wait behind these copies
 *   GG_TUNE_LOOP_WAIT_BUDGET  probes of the grid-barrier wait of the device
 *                         BFS level loop (GG_TUNE_DEVICE_LOOP) before it gives
 *                         up: 0..2^22 (default 2^22, seconds at most).  When a
 *                         wait runs out, every CTA returns, and gg_bfs returns
 *                         GG_ERR_TIMEOUT with the graph left usable; tests set
 *                         it to 0 to drive that path on a healthy graph
 *   GG_TUNE_EARLY_KERNEL  the dense pull with early exit (BFS's bottom-up
 *                         step, edgeMapDenseCSC's break, ligra-numa.h:621-626, 708-713):
 *                         0 one lane per destination, one edge per step; 1 8
 *                         lanes walk a destination's in-list 8 edges per step,
 *                         4 destinations per warp (faster on long rows, slower
 *                         on R-MAT-24: 0.67 against 0.46 ms for BFS's three
 *                         bottom-up levels); 2 one lane per destination
 *                         reading its in-list 4 edges per 16-byte load, the 4
 *                         frontier tests issued together (also in the
 *                         bottom-up levels of GG_TUNE_DEVICE_LOOP 2: BFS on
 *                         R-MAT-24 0.453 against 0.473 ms with 0); 3
 *                         (default) as 2, and the bottom-up levels of
 *                         GG_TUNE_DEVICE_LOOP 2 walk a copy of the in-lists
 *                         with each list's sources by descending out-degree
 *                         (a vertex meets a frontier in-neighbour sooner:
 *                         0.438 against 0.452 ms); the first such BFS builds
 *                         the copy (one segmented sort), which stays with the
 *                         graph: 4 bytes per edge (a graph past 2^31 edges,
 *                         or one the copy does not fit beside, walks the
 *                         CSC's own in-lists)
 *   GG_TUNE_PUSH_DENSE_DIV  a dense edgeMap of BFS (an early-exit functor)
 *                         whose frontier has at most n / value vertices runs
 *                         top-down instead (the frontier's out-edges pushed,
 *                         the output built as a bitmap): after a level of a
 *                         few hubs, the bottom-up step would walk every
 *                         unvisited in-list.  Same levels; 0 (default) =
 *                         never: on RMAT-24 the bottom-up step measured faster
 *                         (0.224 ms against 0.29 ms for the hub level) */
#define GG_TUNE_DENSE_POLICY 1
#define GG_TUNE_COO_KERNEL 2
#define GG_TUNE_SPARSE_DIV 3
#define GG_TUNE_DEVICE_LOOP 4
#define GG_TUNE_CC_ALGO 5
#define GG_TUNE_PR_GRAPH 6
#define GG_TUNE_ASYNC_RESULTS 7
#define GG_TUNE_LOOP_WAIT_BUDGET 8
#define GG_TUNE_EARLY_KERNEL 9
#define GG_TUNE_PUSH_DENSE_DIV 10
#define GG_TUNE_LOOP_CTAS 11
#define GG_TUNE_ROUND_GRAPH 12
int gg_graph_set_tuning(gg_graph_t g, int32_t key, int64_t value);
int gg_graph_get_tuning(gg_graph_t g, int32_t key, int64_t* value);

/* Vertex functors for vertexMap / vertexFilter (graphgrind/ligra-numa.h:1023-1082). */
enum gg_vertex_functor_id {
  GG_V_CC_COPY = 101,      /* app/Components.C:88-99    prevIDs[i]=IDs[i]      args gg_cc_args   */
  GG_V_PR_UPDATE = 102,    /* app/PageRank.C:73-87      p=d*p+(1-d)/n          args gg_pr_vertex_args */
  GG_V_FILL_F32 = 103,     /* PR/SPMV reset: a[i]=value                        args gg_fill_args */
  GG_V_FILL_I32 = 104,     /* BF_Vertex_F: a[i]=value                          args gg_fill_args */
  GG_V_PRDELTA_FIRST = 105,/* app/PageRankDelta.C:73-89 (filter)             args gg_prdelta_vertex_args */
  GG_V_PRDELTA = 106,      /* app/PageRankDelta.C:91-105 (filter)            args gg_prdelta_vertex_args */
  GG_V_BC_MARK = 107,      /* app/BC.C:129-138 Visited[i]=1                  args gg_bc_args */
  GG_V_BC_BACK = 108,      /* app/BC.C:142-154                               args gg_bc_back_vertex_args */
  GG_V_FILL_U8 = 109       /* a[i]=value (bytes)                              args gg_fill_args */
};
typedef struct { float* p_next; float damping; uint32_t n; } gg_pr_vertex_args;
typedef struct { void* array; double value; } gg_fill_args;
typedef struct { float* p; float* delta; const float* ngh_sum; float damping; float one_over_n;
                 float epsilon2; } gg_prdelta_vertex_args;
typedef struct { uint8_t* visited; float* dependencies; const float* inv_num_paths; } gg_bc_back_vertex_args;

int gg_vertex_map(gg_graph_t g, gg_frontier_t f, int32_t vfunctor_id, const void* args);
int gg_vertex_filter(gg_graph_t g, gg_frontier_t f, int32_t vfunctor_id, const void* args,
                     gg_frontier_t* out);

/* Device vertex arrays (mmap_ptr<T>::part_allocate, graphgrind/mm.h:246-324). */
int gg_vertex_array_alloc(gg_graph_t g, size_t elem_bytes, void** dev_ptr);
int gg_vertex_array_free(gg_graph_t g, void* dev_ptr);
int gg_memcpy_h2d(void* dev_dst, const void* host_src, size_t bytes);
int gg_memcpy_d2h(void* host_dst, const void* dev_src, size_t bytes);
/* Page-locked host buffers for the host<->device copies of the app calls. */
int gg_host_alloc_pinned(size_t bytes, void** host_ptr);
int gg_host_free_pinned(void* host_ptr);

/* =========================================== push step without allocation */
/* No counterpart in the reference.  One BFS level on the sparse-push path
 * (the same kernels as gg_edge_map's push branch with GG_F_BFS) for callers
 * that must not let the library allocate device memory: programs that own
 * all device memory and give the library fixed buffers, and latency-critical
 * loops where cudaMalloc/cudaFree would add allocator latency or an implicit
 * device synchronisation.  Its temporaries live in one static device array of
 * GG_NOALLOC_SCRATCH_BYTES that every GPU using the library holds until exit.
 *   out_offsets/out_indices: device CSR of the graph (n+1 / m entries)
 *   frontier[frontier_len]:  device queue of the current level (no duplicates)
 *   parents/levels[n]:       device BFS state (-1 = unvisited); levels may be NULL
 *   next_frontier[n]:        device output queue (caller-allocated, n entries)
 *   next_counts[2]:          device output: {output size, its out-degree sum}
 *   stream:                  a cudaStream_t (NULL = legacy default stream)
 * Sizes above GG_NOALLOC_MAX_VERTICES / GG_NOALLOC_MAX_FRONTIER return
 * GG_ERR_SIZE.  The call is asynchronous on `stream`.  All calls share the
 * array: calls that overlap on the GPU race, so issue them in sequence.  The
 * first call on each device looks up the array's device address and zeroes
 * the array (a synchronous memset); make it before any stream capture.
 * Later calls clear only the bitmap words of the vertices they output. */
#define GG_NOALLOC_MAX_VERTICES (1u << 24)
#define GG_NOALLOC_MAX_FRONTIER (1u << 19)
#define GG_NOALLOC_SCRATCH_BYTES ((4u << 20) + (64u << 10))
int gg_bfs_push_step_noalloc(const uint32_t* out_offsets, const uint32_t* out_indices, uint32_t n,
                             const uint32_t* frontier, uint32_t frontier_len, int32_t* parents,
                             int32_t* levels, int32_t round, uint32_t* next_frontier,
                             uint64_t* next_counts, void* stream);

/* ====================================================== applications */
/* Each runs the Compute() loop of the named app on the device and copies its
 * result to host arrays of n entries.  Timing (device, ms) of the loop alone
 * is returned in *ms when ms != NULL, like the reference's "Running : t". */
typedef struct gg_run_stats {
  double ms;                /* device time of the Compute loop               */
  int32_t rounds;           /* edgeMap calls (levels / iterations)           */
  uint64_t edges_traversed; /* sum of frontier out-degrees (ligra-numa.h:945) */
  int32_t kernels;          /* kernels launched by the loop                  */
} gg_run_stats;

/* app/BFS.C:77-101: parents[n] (-1 unreached), levels[n] (-1 unreached); either
 * output may be NULL (app/BFS.C's result is the parents). */
int gg_bfs(gg_graph_t g, uint32_t start, int32_t* parents, int32_t* levels, gg_run_stats* st);
/* app/Components.C:101-126: ids[n]. */
int gg_components(gg_graph_t g, int32_t* ids, gg_run_stats* st);
/* app/PageRank.C:102-150 (bit_all=0) and app/PageRankBit.C (bit_all=1):
 * ranks[n] in FP32, max_iter iterations (10 in the reference). */
int gg_pagerank(gg_graph_t g, int32_t max_iter, int32_t bit_all, float* ranks, gg_run_stats* st);
/* app/PageRankConverage.C:235-315: PageRank whose dangling mass is spread
 * evenly and whose ranks are renormalised every iteration, until the L1
 * change is at most eps or max_iter iterations ran (100 and 1e-7 in the
 * reference).  ranks[n]; st->rounds = iterations. */
int gg_pagerank_converge(gg_graph_t g, int32_t max_iter, double eps, float* ranks, gg_run_stats* st);
/* app/PageRankDelta.C:120-174: ranks[n]. */
int gg_pagerank_delta(gg_graph_t g, float* ranks, gg_run_stats* st);
/* app/SPMV.C:64-92 with x = 1/n (x_in == NULL) or x_in[n]: y[n] = A^T-weighted sum. */
int gg_spmv(gg_graph_t g, const float* x_in, float* y, gg_run_stats* st);
/* gg_spmv with its input uploaded ahead: gg_spmv_stage_input starts the
 * upload of x[n] (pinned host memory) on the graph's copy stream after the
 * work already queued (so it overlaps the preceding call, e.g. a PageRank),
 * and gg_spmv_staged runs SPMV on it (its device work waits for the
 * upload).  Needs GG_TUNE_ASYNC_RESULTS 1; x must stay unchanged until
 * gg_spmv_staged returns; one input is staged at a time (a second stage call
 * replaces it), and a call in between that stages a result in the same
 * array (BFS levels, SpMV, BC dependencies) gives it up: gg_spmv_staged then
 * returns GG_ERR_INVALID_ARG. */
int gg_spmv_stage_input(gg_graph_t g, const float* x_in);
int gg_spmv_staged(gg_graph_t g, float* y, gg_run_stats* st);
/* app/BellmanFord.C:106-145: dist[n] (1073741823 = unreached). */
int gg_bellman_ford(gg_graph_t g, uint32_t start, int32_t* dist, gg_run_stats* st);
/* app/BC.C:156-226 single source: dependencies[n], num_paths[n] (forward counts). */
int gg_bc(gg_graph_t g, uint32_t start, float* dependencies, float* num_paths, gg_run_stats* st);
/* app/BP.C:152-212 with defined inputs (the reference leaves them
 * uninitialised): vert_potential[2n], edge_potential[4m] with edge e's 2x2
 * potential (i, k) at 4e + 2i + k, e = the edge's in-edge slot of the current
 * orientation (CSC position); per iteration, products reset to 1,
 *   belief_e[i] = sum_k vert_potential[d][k] edge_potential[e][i][k] prod[d][k]
 *   prod_next[d][i] = product of belief_e[i] over d's in-edges.
 * vert_out[2n] = the products after iters iterations. */
int gg_bp(gg_graph_t g, int32_t iters, const float* vert_potential, const float* edge_potential,
          float* vert_out, gg_run_stats* st);

/* ============================================================ batching */
/* k-column personalised PageRank, the batched form of PR_F/PR_Vertex_F
 * (app/PageRank.C:28-87) with every vertex active (app/PageRankBit.C:145)
 * and a teleport matrix in place of the uniform 1/n:
 *   X_0 = T,  X_{t+1} = damping * A X_t + (1 - damping) * T,  A[v,u] = 1/outdeg(u)
 * k = 32 or 64 runs all columns in one SpMM-shaped pull per iteration (each
 * edge moves a whole k-column row); k = 1 runs the scalar engine pull.
 * tele: host n x k row-major ([v][j]), or NULL with seeds[k] (one-hot columns).
 * out: host n x k row-major result X_iters. */
int gg_ppr_k(gg_graph_t g, int32_t k, int32_t iters, float damping, const float* tele,
             const uint32_t* seeds, float* out, gg_run_stats* st);

/* Multi-source BFS: k <= 64 sources in one level-synchronous traversal, with
 * a 64-bit mask per vertex (bit j: reached from sources[j]) moved along every
 * edge once per level.  levels: host n x k row-major ([v][j]); levels[v][j] is
 * gg_bfs's level of v from sources[j] (app/BFS.C:77-101), -1 if unreached.
 * Duplicate sources are allowed.  st->edges_traversed sums the per-source
 * counts of gg_bfs. */
int gg_msbfs(gg_graph_t g, int32_t k, const uint32_t* sources, int32_t* levels, gg_run_stats* st);

/* Multi-source betweenness contributions (app/BC.C:156-226 for each of k <= 64
 * sources): dependencies and num_paths are host n x k row-major (num_paths may
 * be NULL).  num_paths = forward path counts (0 where unreached);
 * dependencies = (dep - 1/paths) * paths with dep = 1/paths + the successors'
 * dep, NaN where unreached.  The backward pass follows the out-edges of the
 * current orientation on every level, which is app/BC.C's result on symmetric
 * graphs; on directed graphs app/BC.C also pulls some levels through the
 * untransposed COO (graphgrind/ligra-numa.h:957-966 after GA.transpose()),
 * which gg_bc reproduces and this call does not. */
int gg_msbc(gg_graph_t g, int32_t k, const uint32_t* sources, float* dependencies, float* num_paths,
            gg_run_stats* st);

/* ======================================================== many graphs */
/* No single counterpart in the reference (one graph per process there).  A
 * batch of independent graphs of uneven size held in one device arena, for
 * running one traversal over all of them in a single persistent launch. */
typedef struct gg_graph_batch_s* gg_graph_batch_t;
/* Uploads `count` host graphs (out-edge CSR each; weights ignored). */
int gg_batch_create(int32_t count, const gg_host_graph* graphs, gg_graph_batch_t* out);
int gg_batch_destroy(gg_graph_batch_t b);
/* Sum of vertices and edges over the batch; firsts[count] (may be NULL)
 * receives each graph's first slot in the level output. */
int gg_batch_info(gg_graph_batch_t b, uint64_t* total_vertices, uint64_t* total_edges, uint64_t* firsts);
/* BFS from sources[i] in graph i for every graph (app/BFS.C:77-101 levels),
 * in one persistent launch whose CTAs take graphs, largest first, from a
 * device work queue and traverse each inside the CTA.  levels: host array of
 * total_vertices int32 (may be NULL), graph i's at firsts[i], -1 unreached.
 * The sequence source upload -> traversal -> level download is a CUDA graph
 * captured at gg_batch_create and replayed by every call; st->ms is its
 * device time, st->edges_traversed the sum over graphs of gg_bfs's count. */
int gg_batch_bfs(gg_graph_batch_t b, const uint32_t* sources, int32_t* levels, gg_run_stats* st);

/* ==================================================== differentiation */
/* No counterpart in the reference.  Weighted PageRank
 *   a_e = w_e, or w_e / (sum of w over u's out-edges) when normalize != 0
 *   x_{t+1}[v] = damping * sum_{e = u->v} a_e x_t[u] + (1 - damping) * tele[v]
 * for t < iters from x_0 (x0, or 1/n when x0 == NULL): PR_F / PR_Vertex_F
 * (app/PageRank.C:28-100) with a_e in place of 1/outdeg(u) (a_e = 1/outdeg(u),
 * tele = 1/n gives PageRankBit), and SPMV_F (app/SPMV.C:7-48) at iters = 1,
 * damping = 1.  Its adjoint is the transposed traversal (a pull over the
 * out-edges where the forward pulls the in-edges).  A context holds the
 * forward's checkpoints (x_t every checkpoint_every steps) for the backward,
 * which recomputes each segment from its checkpoint and reverses through it.
 * weights / grad_weights: host, m entries in the graph's out-edge order
 * (gg_host_graph offsets/indices of the current orientation); tele, x0, x_out,
 * grad_x, grad_tele, grad_x0: host, n entries (grad_* may be NULL).
 * Repeated edges u->v carry one weight each.  create returns GG_ERR_FORMAT
 * when an in-edge list of the current orientation is not sorted by source: the
 * library builds a directed graph's in-edges sorted, the given rows are used as
 * they are (a symmetric graph's in-edges, a transposed graph's in-edges). */
typedef struct gg_wpr_s* gg_wpr_t;
int gg_pagerank_weighted_create(gg_graph_t g, int32_t iters, float damping, int32_t checkpoint_every,
                                int32_t normalize, gg_wpr_t* out);
int gg_pagerank_weighted_destroy(gg_wpr_t ctx);
/* x_out = x_iters; keeps the checkpoints in ctx. */
int gg_pagerank_weighted_fwd(gg_wpr_t ctx, const float* weights, const float* tele, const float* x0, float* x_out,
                             gg_run_stats* st);
/* Given grad_x = dL/dx_iters of the last forward: dL/dweights, dL/dtele, dL/dx0. */
int gg_pagerank_weighted_bwd(gg_wpr_t ctx, const float* grad_x, float* grad_weights, float* grad_tele,
                             float* grad_x0, gg_run_stats* st);

/* ========================================================= autotuner */
/* No counterpart in the reference (its knobs are command-line flags).  The
 * tuner times an application and keeps the fastest knobs; no knob changes
 * results beyond the summation order of FP32 sums. */
enum gg_tune_app {
  GG_APP_BFS = 1,            /* gg_bfs from `start`                 */
  GG_APP_COMPONENTS = 2,     /* gg_components                       */
  GG_APP_PAGERANK = 3,       /* gg_pagerank, 10 iterations          */
  GG_APP_PAGERANK_DELTA = 4, /* gg_pagerank_delta                   */
  GG_APP_SPMV = 5,           /* gg_spmv with x = 1/n                */
  GG_APP_BELLMAN_FORD = 6,   /* gg_bellman_ford from `start`        */
  GG_APP_BC = 7              /* gg_bc from `start`                  */
};
typedef struct gg_tune_trial {
  int32_t dense_policy;   /* GG_TUNE_DENSE_POLICY                       */
  int32_t coo_kernel;     /* GG_TUNE_COO_KERNEL                         */
  int32_t sparse_div;     /* GG_TUNE_SPARSE_DIV                         */
  int32_t partitions;     /* build knobs of gg_autotune_build (else 0)  */
  int32_t tile_vertices;
  int32_t tile_edges;
  int32_t coo_window;
  int32_t cc_algo;        /* GG_TUNE_CC_ALGO                            */
  double ms;              /* best of 3 device times of the application  */
} gg_tune_trial;
/* Runtime search on a built graph: every combination of dense policy, COO
 * kernel (where a COO exists) and threshold divisor {20, 10, 40}, plus the
 * union-find pass for GG_APP_COMPONENTS on a symmetric graph; the fastest
 * is left set on g.  trials[max_trials] (may be NULL) receives the trials,
 * fastest first; *n_trials the number run. */
int gg_autotune(gg_graph_t g, int32_t app, uint32_t start, gg_tune_trial* trials, int32_t max_trials,
                int32_t* n_trials);
/* Build-time search: builds hg under each candidate option set (candidates
 * the reference partitioner rejects are skipped), runs gg_autotune on each
 * and returns the fastest options in *best_opts and its trial in *best. */
int gg_autotune_build(const gg_host_graph* hg, int32_t app, uint32_t start, const gg_build_opts* candidates,
                      int32_t n_candidates, gg_build_opts* best_opts, gg_tune_trial* best);
/* Column count for gg_ppr_k on g: the k in {1, 32, 64} with the most
 * column-edges per second over `iters` iterations. */
int gg_autotune_ppr_k(gg_graph_t g, int32_t iters, int32_t* best_k, double* column_edges_per_s);

#ifdef __cplusplus
}
#endif
#endif /* GG_H */
