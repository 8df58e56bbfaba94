"""Python binding of the B200 traversal engine (libgg.so, C ABI in include/gg.h).

The binding is a thin ctypes layer: graphs, frontiers and vertex arrays live
on the GPU inside the library; results come back as numpy arrays.  There is
no CPU fallback: importing works without a GPU (host-only functions such as
the generators and the partitioner run anywhere), but every device call fails
with a GGError when no CUDA device is present, and importing fails when the
compiled library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# GG_LIBRARY names another build of the same C ABI (for side-by-side builds)
LIB_PATH = os.environ.get("GG_LIBRARY") or os.path.join(_HERE, "libgg.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"graphgrind_b200: compiled library {LIB_PATH} is missing; build it with "
        "`make -C graphgrind_b200` (or __graft_entry__.build())")

lib = C.CDLL(LIB_PATH)

# ------------------------------------------------------------------ status
GG_OK = 0
ERRORS = {
    -1: "INVALID_ARG", -2: "CUDA", -3: "OOM", -4: "PARTITION", -5: "IO", -6: "FORMAT",
    -7: "NO_DEVICE", -8: "UNSUPPORTED", -9: "TIMEOUT", -10: "SIZE",
}
ERR_INVALID_ARG, ERR_CUDA, ERR_OOM, ERR_PARTITION, ERR_IO, ERR_FORMAT = -1, -2, -3, -4, -5, -6
ERR_NO_DEVICE, ERR_UNSUPPORTED, ERR_TIMEOUT, ERR_SIZE = -7, -8, -9, -10
W_NONE, W_INT32, W_FLOAT32 = 0, 1, 2
BALANCE_EDGE, BALANCE_VERTEX = 0, 1
PART_DEST, PART_SOURCE = 0, 1
ORDER_CSR, ORDER_HILBERT = 0, 1
VORDER_GIVEN, VORDER_HOT_FIRST = 0, 1
EM_FORCE_SPARSE, EM_FORCE_CSC, EM_FORCE_COO, EM_NO_OUTPUT = 0x1, 0x2, 0x4, 0x8
F_BFS, F_CC, F_PR, F_PRDELTA, F_SPMV, F_BF, F_BC, F_BC_BACK, F_BP = range(1, 10)


class GGError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        msg = lib.gg_last_error_string().decode(errors="replace")
        super().__init__(f"{where}: GG_ERR_{ERRORS.get(code, code)} ({code}): {msg}")


def check(rc: int, where: str) -> None:
    if rc != GG_OK:
        raise GGError(rc, where)


# ----------------------------------------------------------------- structs
class HostGraphC(C.Structure):
    _fields_ = [("n", C.c_uint32), ("m", C.c_uint64), ("symmetric", C.c_int32),
                ("weight_type", C.c_int32), ("offsets", C.POINTER(C.c_uint32)),
                ("indices", C.POINTER(C.c_uint32)), ("weights", C.c_void_p)]


class BuildOpts(C.Structure):
    _fields_ = [("num_partitions", C.c_int32), ("balance", C.c_int32), ("part_how", C.c_int32),
                ("relabel", C.c_int32), ("order", C.c_int32), ("tile_vertices", C.c_int32),
                ("tile_edges", C.c_int32), ("build_coo", C.c_int32), ("coo_window", C.c_int32),
                ("coo_dst_window", C.c_int32), ("vertex_order", C.c_int32), ("coo_tile_vertices", C.c_int32)]


class TuneTrial(C.Structure):
    _fields_ = [("dense_policy", C.c_int32), ("coo_kernel", C.c_int32), ("sparse_div", C.c_int32),
                ("partitions", C.c_int32), ("tile_vertices", C.c_int32), ("tile_edges", C.c_int32),
                ("coo_window", C.c_int32), ("cc_algo", C.c_int32), ("ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class GraphInfo(C.Structure):
    _fields_ = [("n", C.c_uint32), ("m", C.c_uint64), ("symmetric", C.c_int32),
                ("weight_type", C.c_int32), ("num_partitions", C.c_int32), ("has_coo", C.c_int32),
                ("transposed", C.c_int32), ("num_csc_tiles", C.c_int32),
                ("num_coo_tiles", C.c_int32), ("device_bytes", C.c_uint64), ("num_coo_gaps", C.c_int32)]


class RunStats(C.Structure):
    _fields_ = [("ms", C.c_double), ("rounds", C.c_int32), ("edges_traversed", C.c_uint64),
                ("kernels", C.c_int32)]


class EdgeMapStats(C.Structure):
    _fields_ = [("kind", C.c_int32), ("frontier_active", C.c_uint64),
                ("frontier_out_edges", C.c_uint64), ("output_active", C.c_uint64),
                ("output_out_edges", C.c_uint64)]


class Profile(C.Structure):
    _fields_ = [("launches", C.c_uint64 * 4), ("ms", C.c_double * 4), ("edges", C.c_uint64 * 4)]


PROFILE_KINDS = ("push", "csc_pull", "coo_pull", "early_pull")


class BfsArgs(C.Structure):
    _fields_ = [("parents", C.c_void_p), ("levels", C.c_void_p), ("round", C.c_int32)]


class CcArgs(C.Structure):
    _fields_ = [("ids", C.c_void_p), ("prev_ids", C.c_void_p)]


class PairArgs(C.Structure):  # gg_pr_args / gg_prdelta_args / gg_spmv_args / gg_bf_args / gg_bc_args
    _fields_ = [("a", C.c_void_p), ("b", C.c_void_p)]


_P = C.c_void_p
_u32p = C.POINTER(C.c_uint32)
_i64p = C.POINTER(C.c_int64)


def _sig(name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


_sig("gg_last_error_string", C.c_char_p)
_sig("gg_version", C.c_char_p)
_sig("gg_gen_rmat", C.c_int, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_uint64,
     C.c_int32, C.POINTER(HostGraphC))
_sig("gg_gen_grid", C.c_int, C.c_int32, C.c_double, C.c_uint64, C.POINTER(HostGraphC))
_sig("gg_gen_er", C.c_int, C.c_uint32, C.c_uint64, C.c_uint64, C.c_int32, C.POINTER(HostGraphC))
_sig("gg_host_graph_add_weights", C.c_int, C.POINTER(HostGraphC), C.c_int32, C.c_uint64, C.c_int32, C.c_int32)
_sig("gg_host_graph_write_adj", C.c_int, C.POINTER(HostGraphC), C.c_char_p)
_sig("gg_host_graph_write_gr", C.c_int, C.POINTER(HostGraphC), C.c_char_p)
_sig("gg_host_graph_read", C.c_int, C.c_char_p, C.c_int32, C.c_int32, C.c_int32, C.POINTER(HostGraphC))
_sig("gg_host_graph_transpose", C.c_int, C.POINTER(HostGraphC), C.POINTER(HostGraphC))
_sig("gg_host_graph_free", None, C.POINTER(HostGraphC))
_sig("gg_vebo", C.c_int, C.POINTER(HostGraphC), C.c_int32, _P, _P, C.POINTER(HostGraphC))
_sig("gg_vebo_gpu", C.c_int, C.POINTER(HostGraphC), C.c_int32, _P, _P, C.POINTER(HostGraphC))
_sig("gg_partition_sizes", C.c_int, _u32p, _u32p, C.c_uint32, C.c_uint64, C.c_int32, C.c_int32, C.c_int32,
     C.c_int32, _i64p, _i64p)
_sig("gg_hilbert_key", C.c_int64, C.c_int64, C.c_int64, C.c_int64)
_sig("gg_hot_first_order", C.c_int, C.POINTER(HostGraphC), C.POINTER(BuildOpts), _P, _P)
_sig("gg_host_graph_read_gpu", C.c_int, C.c_char_p, C.c_int32, C.c_int32, C.c_int32, C.c_int64,
     C.POINTER(HostGraphC))
_sig("gg_graph_build", C.c_int, C.POINTER(HostGraphC), C.POINTER(BuildOpts), C.POINTER(_P))
_sig("gg_graph_destroy", C.c_int, _P)
_sig("gg_graph_synchronize", C.c_int, _P)
_sig("gg_graph_get_info", C.c_int, _P, C.POINTER(GraphInfo))
_sig("gg_graph_partition_starts", C.c_int, _P, _i64p)
_sig("gg_graph_transpose", C.c_int, _P)
_sig("gg_graph_device_arrays", C.c_int, _P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P), C.POINTER(_P))
_sig("gg_graph_vertex_order", C.c_int, _P, _P)
_sig("gg_graph_device_weights", C.c_int, _P, C.POINTER(_P), C.POINTER(_P))
_sig("gg_graph_coo_layout", C.c_int, _P, C.POINTER(C.c_uint64), _P, C.POINTER(C.c_uint64), _P, _P)
_sig("gg_spmv_stage_input", C.c_int, _P, _P)
_sig("gg_spmv_staged", C.c_int, _P, _P, C.POINTER(RunStats))
_sig("gg_frontier_single", C.c_int, _P, C.c_uint32, C.POINTER(_P))
_sig("gg_frontier_all", C.c_int, _P, C.POINTER(_P))
_sig("gg_frontier_empty", C.c_int, _P, C.POINTER(_P))
_sig("gg_frontier_from_mask", C.c_int, _P, C.POINTER(C.c_uint8), C.POINTER(_P))
_sig("gg_frontier_from_list", C.c_int, _P, _u32p, C.c_uint64, C.POINTER(_P))
_sig("gg_frontier_destroy", C.c_int, _P)
_sig("gg_frontier_stats", C.c_int, _P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64))
_sig("gg_frontier_to_mask", C.c_int, _P, C.POINTER(C.c_uint8))
_sig("gg_frontier_to_dense", C.c_int, _P)
_sig("gg_frontier_to_sparse", C.c_int, _P)
_sig("gg_frontier_repr", C.c_int, _P)
_sig("gg_edge_map", C.c_int, _P, _P, C.c_int32, _P, C.c_int64, C.c_uint32, C.POINTER(_P))
_sig("gg_last_edge_map_stats", C.c_int, _P, C.POINTER(EdgeMapStats))
_sig("gg_graph_set_profiling", C.c_int, _P, C.c_int32)
_sig("gg_graph_get_profile", C.c_int, _P, C.POINTER(Profile))
_sig("gg_graph_set_dense_policy", C.c_int, _P, C.c_int32)
_sig("gg_graph_set_tuning", C.c_int, _P, C.c_int32, C.c_int64)
_sig("gg_graph_get_tuning", C.c_int, _P, C.c_int32, C.POINTER(C.c_int64))
TUNE_DENSE_POLICY, TUNE_COO_KERNEL, TUNE_SPARSE_DIV, TUNE_DEVICE_LOOP, TUNE_CC_ALGO, TUNE_PR_GRAPH = 1, 2, 3, 4, 5, 6
TUNE_ASYNC_RESULTS = 7
TUNE_LOOP_WAIT_BUDGET = 8
TUNE_EARLY_KERNEL = 9
TUNE_PUSH_DENSE_DIV = 10
TUNE_LOOP_CTAS = 11
TUNE_ROUND_GRAPH = 12
APP_BFS, APP_COMPONENTS, APP_PAGERANK, APP_PAGERANK_DELTA, APP_SPMV, APP_BELLMAN_FORD, APP_BC = range(1, 8)
_sig("gg_vertex_map", C.c_int, _P, _P, C.c_int32, _P)
_sig("gg_vertex_filter", C.c_int, _P, _P, C.c_int32, _P, C.POINTER(_P))
_sig("gg_vertex_array_alloc", C.c_int, _P, C.c_size_t, C.POINTER(_P))
_sig("gg_vertex_array_free", C.c_int, _P, _P)
_sig("gg_memcpy_h2d", C.c_int, _P, _P, C.c_size_t)
_sig("gg_memcpy_d2h", C.c_int, _P, _P, C.c_size_t)
_sig("gg_host_alloc_pinned", C.c_int, C.c_size_t, C.POINTER(_P))
_sig("gg_host_free_pinned", C.c_int, _P)
_sig("gg_bfs", C.c_int, _P, C.c_uint32, _P, _P, C.POINTER(RunStats))
_sig("gg_components", C.c_int, _P, _P, C.POINTER(RunStats))
_sig("gg_pagerank", C.c_int, _P, C.c_int32, C.c_int32, _P, C.POINTER(RunStats))
_sig("gg_pagerank_delta", C.c_int, _P, _P, C.POINTER(RunStats))
_sig("gg_spmv", C.c_int, _P, _P, _P, C.POINTER(RunStats))
_sig("gg_bellman_ford", C.c_int, _P, C.c_uint32, _P, C.POINTER(RunStats))
_sig("gg_bc", C.c_int, _P, C.c_uint32, _P, _P, C.POINTER(RunStats))
_sig("gg_bp", C.c_int, _P, C.c_int32, _P, _P, _P, C.POINTER(RunStats))
_sig("gg_bfs_push_step_noalloc", C.c_int, _P, _P, C.c_uint32, _P, C.c_uint32, _P, _P, C.c_int32, _P, _P, _P)
_sig("gg_pagerank_converge", C.c_int, _P, C.c_int32, C.c_double, _P, C.POINTER(RunStats))
_sig("gg_ppr_k", C.c_int, _P, C.c_int32, C.c_int32, C.c_float, _P, _P, _P, C.POINTER(RunStats))
_sig("gg_msbfs", C.c_int, _P, C.c_int32, _P, _P, C.POINTER(RunStats))
_sig("gg_msbc", C.c_int, _P, C.c_int32, _P, _P, _P, C.POINTER(RunStats))
_sig("gg_batch_create", C.c_int, C.c_int32, _P, C.POINTER(_P))
_sig("gg_batch_destroy", C.c_int, _P)
_sig("gg_batch_info", C.c_int, _P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), _P)
_sig("gg_batch_bfs", C.c_int, _P, _P, _P, C.POINTER(RunStats))
_sig("gg_autotune", C.c_int, _P, C.c_int32, C.c_uint32, _P, C.c_int32, C.POINTER(C.c_int32))
_sig("gg_autotune_build", C.c_int, _P, C.c_int32, C.c_uint32, _P, C.c_int32, _P, _P)
_sig("gg_autotune_ppr_k", C.c_int, _P, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double))
_sig("gg_pagerank_weighted_create", C.c_int, _P, C.c_int32, C.c_float, C.c_int32, C.c_int32, C.POINTER(_P))
_sig("gg_pagerank_weighted_destroy", C.c_int, _P)
_sig("gg_pagerank_weighted_fwd", C.c_int, _P, _P, _P, _P, _P, C.POINTER(RunStats))
_sig("gg_pagerank_weighted_bwd", C.c_int, _P, _P, _P, _P, _P, C.POINTER(RunStats))

# Every symbol declared in include/gg.h (checked by the tests).
EXPORTED = [
    "gg_last_error_string", "gg_version", "gg_gen_rmat", "gg_gen_grid", "gg_gen_er",
    "gg_host_graph_add_weights", "gg_host_graph_write_adj", "gg_host_graph_write_gr",
    "gg_host_graph_read", "gg_host_graph_transpose", "gg_host_graph_free", "gg_partition_sizes",
    "gg_hilbert_key", "gg_graph_build", "gg_graph_destroy", "gg_graph_synchronize", "gg_graph_get_info",
    "gg_graph_partition_starts", "gg_graph_transpose", "gg_graph_device_arrays",
    "gg_frontier_single", "gg_frontier_all", "gg_frontier_empty", "gg_frontier_from_mask",
    "gg_frontier_from_list", "gg_frontier_destroy", "gg_frontier_stats", "gg_frontier_to_mask",
    "gg_frontier_to_dense", "gg_frontier_to_sparse", "gg_frontier_repr", "gg_edge_map",
    "gg_last_edge_map_stats", "gg_graph_set_profiling", "gg_graph_get_profile",
    "gg_graph_set_dense_policy", "gg_graph_set_tuning", "gg_graph_get_tuning", "gg_vertex_map", "gg_vertex_filter", "gg_vertex_array_alloc",
    "gg_vertex_array_free", "gg_memcpy_h2d", "gg_memcpy_d2h", "gg_host_alloc_pinned", "gg_host_free_pinned", "gg_bfs", "gg_components",
    "gg_pagerank", "gg_pagerank_delta", "gg_spmv", "gg_bellman_ford", "gg_bc", "gg_bp",
    "gg_bfs_push_step_noalloc", "gg_ppr_k", "gg_pagerank_converge", "gg_vebo", "gg_msbfs", "gg_msbc",
    "gg_batch_create", "gg_batch_destroy", "gg_batch_info", "gg_batch_bfs",
    "gg_pagerank_weighted_create", "gg_pagerank_weighted_destroy", "gg_pagerank_weighted_fwd",
    "gg_pagerank_weighted_bwd", "gg_autotune", "gg_autotune_build", "gg_autotune_ppr_k",
    "gg_hot_first_order", "gg_graph_vertex_order", "gg_host_graph_read_gpu", "gg_graph_device_weights",
    "gg_graph_coo_layout", "gg_vebo_gpu", "gg_spmv_stage_input", "gg_spmv_staged",
]


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def _view(addr: int, count: int, ctype, dtype, owner) -> np.ndarray:
    """numpy view of library-owned memory that keeps `owner` alive."""
    if count == 0 or not addr:
        return np.zeros(0, dtype)
    buf = (ctype * count).from_address(addr)
    buf._gg_owner = owner
    return np.frombuffer(buf, dtype=dtype)


# -------------------------------------------------------------- host graph
class HostGraph:
    """A host CSR graph owned by the library (gg_host_graph)."""

    def __init__(self, c: HostGraphC):
        self.c = c

    def __del__(self):
        try:
            lib.gg_host_graph_free(C.byref(self.c))
        except Exception:
            pass

    @property
    def n(self) -> int:
        return int(self.c.n)

    @property
    def m(self) -> int:
        return int(self.c.m)

    @property
    def symmetric(self) -> bool:
        return bool(self.c.symmetric)

    @property
    def weight_type(self) -> int:
        return int(self.c.weight_type) if self.c.weights else W_NONE

    @property
    def offsets(self) -> np.ndarray:
        return _view(C.cast(self.c.offsets, C.c_void_p).value, self.n + 1, C.c_uint32, np.uint32, self)

    @property
    def indices(self) -> np.ndarray:
        return _view(C.cast(self.c.indices, C.c_void_p).value, self.m, C.c_uint32, np.uint32, self)

    @property
    def weights(self):
        if not self.c.weights or self.m == 0:
            return None
        a = _view(self.c.weights, self.m, C.c_uint32, np.uint32, self)
        return a.view(np.float32) if self.weight_type == W_FLOAT32 else a.view(np.int32)

    def degrees(self) -> np.ndarray:
        return np.diff(self.offsets.astype(np.int64)).astype(np.uint32)

    @staticmethod
    def rmat(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=1, symmetric=True) -> "HostGraph":
        g = HostGraphC()
        check(lib.gg_gen_rmat(scale, edge_factor, a, b, c, seed, int(symmetric), C.byref(g)), "gg_gen_rmat")
        return HostGraph(g)

    @staticmethod
    def grid(side, long_range_frac=0.001, seed=3) -> "HostGraph":
        g = HostGraphC()
        check(lib.gg_gen_grid(side, long_range_frac, seed, C.byref(g)), "gg_gen_grid")
        return HostGraph(g)

    @staticmethod
    def er(n, m, seed=4, symmetric=False) -> "HostGraph":
        g = HostGraphC()
        check(lib.gg_gen_er(n, m, seed, int(symmetric), C.byref(g)), "gg_gen_er")
        return HostGraph(g)

    @staticmethod
    def read(path, binary=False, symmetric=False, weighted=False) -> "HostGraph":
        g = HostGraphC()
        check(lib.gg_host_graph_read(str(path).encode(), int(binary), int(symmetric), int(weighted), C.byref(g)),
              "gg_host_graph_read")
        return HostGraph(g)

    @staticmethod
    def read_gpu(path, binary=False, symmetric=False, weighted=False, chunk_bytes=0) -> "HostGraph":
        """gg_host_graph_read_gpu: the PBBS text body parsed on the GPU."""
        g = HostGraphC()
        check(lib.gg_host_graph_read_gpu(str(path).encode(), int(binary), int(symmetric), int(weighted),
                                         int(chunk_bytes), C.byref(g)), "gg_host_graph_read_gpu")
        return HostGraph(g)

    @staticmethod
    def from_csr(offsets, indices, weights=None, symmetric=False) -> "HostGraph":
        """Copy a CSR given as numpy arrays into a library-owned host graph."""
        import tempfile
        offsets = np.ascontiguousarray(offsets, dtype=np.uint32)
        indices = np.ascontiguousarray(indices, dtype=np.uint32)
        n = len(offsets) - 1
        with tempfile.TemporaryDirectory() as d:  # round trip through the .gr writer/reader
            p = os.path.join(d, "g.gr")
            hdr = np.array([1, 4 if weights is not None else 0, n, len(indices)], np.uint64)
            with open(p, "wb") as f:
                f.write(hdr.tobytes())
                f.write(offsets[1:].astype(np.uint64).tobytes())
                f.write(indices.tobytes())
                if len(indices) & 1:
                    f.write(b"\0\0\0\0")
                if weights is not None:
                    f.write(np.ascontiguousarray(weights, dtype=np.int32).tobytes())
            return HostGraph.read(p, binary=True, symmetric=symmetric, weighted=weights is not None)

    def add_weights(self, weight_type=W_INT32, seed=7, lo=1, hi=100) -> "HostGraph":
        check(lib.gg_host_graph_add_weights(C.byref(self.c), weight_type, seed, lo, hi), "gg_host_graph_add_weights")
        return self

    def write_adj(self, path):
        check(lib.gg_host_graph_write_adj(C.byref(self.c), str(path).encode()), "gg_host_graph_write_adj")

    def write_gr(self, path):
        check(lib.gg_host_graph_write_gr(C.byref(self.c), str(path).encode()), "gg_host_graph_write_gr")

    def transpose(self) -> "HostGraph":
        t = HostGraphC()
        check(lib.gg_host_graph_transpose(C.byref(self.c), C.byref(t)), "gg_host_graph_transpose")
        return HostGraph(t)

    def hot_first_order(self, partitions=384, balance=BALANCE_EDGE, part_how=PART_DEST, relabel=False):
        """gg_hot_first_order: (new_of_old[n], COO partition starts[P+1]) of VORDER_HOT_FIRST."""
        o = BuildOpts(partitions, balance, part_how, int(relabel), ORDER_HILBERT, 0, 0, 0, 0, 0, VORDER_HOT_FIRST)
        new_of_old = np.empty(self.n, np.uint32)
        starts = np.empty(partitions + 1, np.int64)
        check(lib.gg_hot_first_order(C.byref(self.c), C.byref(o), _ptr(new_of_old), _ptr(starts)),
              "gg_hot_first_order")
        return new_of_old, starts

    def vebo(self, partitions=384):
        """VEBO reordering: (relabelled HostGraph, new_of_old[n], vertices per partition[P])."""
        t = HostGraphC()
        new_of_old = np.empty(self.n, np.uint32)
        sizes = np.empty(partitions, np.int64)
        check(lib.gg_vebo(C.byref(self.c), partitions, _ptr(new_of_old), _ptr(sizes), C.byref(t)), "gg_vebo")
        return HostGraph(t), new_of_old, sizes

    def vebo_gpu(self, partitions=384):
        """gg_vebo_gpu: vebo() computed on the GPU, the same result."""
        t = HostGraphC()
        new_of_old = np.empty(self.n, np.uint32)
        sizes = np.empty(partitions, np.int64)
        check(lib.gg_vebo_gpu(C.byref(self.c), partitions, _ptr(new_of_old), _ptr(sizes), C.byref(t)), "gg_vebo_gpu")
        return HostGraph(t), new_of_old, sizes


def partition_sizes(in_deg, out_deg, m, P, balance=BALANCE_EDGE, part_how=PART_DEST, relabel=False):
    """Reference partition sizes (coo, csc); raises GGError(PARTITION) where the reference asserts."""
    in_deg = np.ascontiguousarray(in_deg, np.uint32)
    out_deg = np.ascontiguousarray(out_deg, np.uint32)
    coo = np.zeros(P, np.int64)
    csc = np.zeros(P, np.int64)
    check(lib.gg_partition_sizes(in_deg.ctypes.data_as(_u32p), out_deg.ctypes.data_as(_u32p), len(in_deg), m, P,
                                 balance, part_how, int(relabel), coo.ctypes.data_as(_i64p),
                                 csc.ctypes.data_as(_i64p)), "gg_partition_sizes")
    return coo, csc


def hilbert_key(side_edges: int, x: int, y: int) -> int:
    return int(lib.gg_hilbert_key(side_edges, x, y))


class PinnedArray:
    """A page-locked host buffer viewed as a numpy array (for timed H2D/D2H)."""

    def __init__(self, count: int, dtype):
        self.dtype = np.dtype(dtype)
        p = C.c_void_p()
        check(lib.gg_host_alloc_pinned(max(1, count) * self.dtype.itemsize, C.byref(p)), "gg_host_alloc_pinned")
        self.ptr = p
        buf = (C.c_uint8 * (max(1, count) * self.dtype.itemsize)).from_address(p.value)
        buf._gg_owner = self
        self.array = np.frombuffer(buf, dtype=self.dtype)[:count]

    def __del__(self):
        if getattr(self, "ptr", None):
            lib.gg_host_free_pinned(self.ptr)
            self.ptr = None


# ------------------------------------------------------------ device graph
@dataclass
class Run:
    ms: float
    rounds: int
    edges_traversed: int
    kernels: int


def _run(st: RunStats) -> Run:
    return Run(st.ms, st.rounds, st.edges_traversed, st.kernels)


class Frontier:
    """partitioned_vertices on the device."""

    def __init__(self, graph: "Graph", handle: C.c_void_p):
        self.graph = graph
        self.h = handle
        graph._deps.add(self)

    def __del__(self):
        self.close()

    def close(self):
        if getattr(self, "h", None):
            if getattr(self.graph, "h", None):
                lib.gg_frontier_destroy(self.h)
            self.h = None

    def stats(self):
        a, b = C.c_uint64(), C.c_uint64()
        check(lib.gg_frontier_stats(self.h, C.byref(a), C.byref(b)), "gg_frontier_stats")
        return int(a.value), int(b.value)

    def mask(self) -> np.ndarray:
        out = np.zeros(self.graph.n, np.uint8)
        check(lib.gg_frontier_to_mask(self.h, out.ctypes.data_as(C.POINTER(C.c_uint8))), "gg_frontier_to_mask")
        return out

    def to_dense(self):
        check(lib.gg_frontier_to_dense(self.h), "gg_frontier_to_dense")

    def to_sparse(self):
        check(lib.gg_frontier_to_sparse(self.h), "gg_frontier_to_sparse")

    def repr(self) -> int:
        return int(lib.gg_frontier_repr(self.h))


class DeviceArray:
    """A device vertex array (n entries) owned by a Graph."""

    def __init__(self, graph: "Graph", dtype, init=None):
        self.graph = graph
        self.dtype = np.dtype(dtype)
        p = C.c_void_p()
        check(lib.gg_vertex_array_alloc(graph.h, self.dtype.itemsize, C.byref(p)), "gg_vertex_array_alloc")
        self.ptr = p
        graph._deps.add(self)
        if init is not None:
            self.upload(np.full(graph.n, init, self.dtype) if np.isscalar(init) else init)

    def upload(self, a):
        a = np.ascontiguousarray(a, self.dtype)
        check(lib.gg_memcpy_h2d(self.ptr, _ptr(a), a.nbytes), "gg_memcpy_h2d")

    def download(self) -> np.ndarray:
        out = np.empty(self.graph.n, self.dtype)
        check(lib.gg_memcpy_d2h(_ptr(out), self.ptr, out.nbytes), "gg_memcpy_d2h")
        return out

    def close(self):
        if getattr(self, "ptr", None):
            if getattr(self.graph, "h", None):
                lib.gg_vertex_array_free(self.graph.h, self.ptr)
            self.ptr = None

    def __del__(self):
        self.close()


class Graph:
    """partitioned_graph on the device (gg_graph_build)."""

    def __init__(self, host: HostGraph, partitions=384, balance=BALANCE_EDGE, part_how=PART_DEST, relabel=False,
                 order=ORDER_HILBERT, tile_vertices=0, tile_edges=0, build_coo=0, coo_window=0, coo_dst_window=0,
                 vertex_order=VORDER_GIVEN, coo_tile_vertices=0):
        self.host = host
        self._deps = weakref.WeakSet()
        o = BuildOpts(partitions, balance, part_how, int(relabel), order, tile_vertices, tile_edges, build_coo,
                      coo_window, coo_dst_window, vertex_order, coo_tile_vertices)
        h = C.c_void_p()
        check(lib.gg_graph_build(C.byref(host.c), C.byref(o), C.byref(h)), "gg_graph_build")
        self.h = h
        self.n = host.n
        self.m = host.m

    def close(self):
        if getattr(self, "h", None):
            for d in list(getattr(self, "_deps", ())):  # frontiers / arrays first
                d.close()
            lib.gg_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def info(self) -> GraphInfo:
        i = GraphInfo()
        check(lib.gg_graph_get_info(self.h, C.byref(i)), "gg_graph_get_info")
        return i

    def partition_starts(self) -> np.ndarray:
        P = self.info().num_partitions
        s = np.zeros(P + 1, np.int64)
        check(lib.gg_graph_partition_starts(self.h, s.ctypes.data_as(_i64p)), "gg_graph_partition_starts")
        return s

    def coo_layout(self):
        """The device COO (gg_graph_coo_layout): (tiles[T, 4] {first vertex,
        vertices, first slot, slots} in work order, src[slots], dst[slots];
        padding slots hold 0xffffffff)."""
        nt, ln = C.c_uint64(), C.c_uint64()
        check(lib.gg_graph_coo_layout(self.h, C.byref(nt), None, C.byref(ln), None, None), "gg_graph_coo_layout")
        tiles = np.empty((max(nt.value, 1), 4), np.uint32)
        src = np.empty(max(ln.value, 1), np.uint32)
        dst = np.empty(max(ln.value, 1), np.uint32)
        check(lib.gg_graph_coo_layout(self.h, C.byref(nt), _ptr(tiles), C.byref(ln), _ptr(src), _ptr(dst)),
              "gg_graph_coo_layout")
        return tiles[:nt.value], src[:ln.value], dst[:ln.value]

    def vertex_order(self) -> np.ndarray:
        """new_of_old[n]: the device id of every given vertex (gg_graph_vertex_order)."""
        a = np.empty(self.n, np.uint32)
        check(lib.gg_graph_vertex_order(self.h, _ptr(a)), "gg_graph_vertex_order")
        return a

    def transpose(self):
        check(lib.gg_graph_transpose(self.h), "gg_graph_transpose")

    def synchronize(self):
        """Waits for the result copies TUNE_ASYNC_RESULTS leaves in flight."""
        check(lib.gg_graph_synchronize(self.h), "gg_graph_synchronize")

    def set_profiling(self, enable=True):
        check(lib.gg_graph_set_profiling(self.h, int(enable)), "gg_graph_set_profiling")

    def profile(self) -> dict:
        """Per kernel kind: launches, device ms (CUDA events), edges streamed; resets."""
        p = Profile()
        check(lib.gg_graph_get_profile(self.h, C.byref(p)), "gg_graph_get_profile")
        return {k: {"launches": int(p.launches[i]), "ms": float(p.ms[i]), "edges": int(p.edges[i])}
                for i, k in enumerate(PROFILE_KINDS)}

    def set_dense_policy(self, policy: int):
        """0: reference rule (COO above m/2), 1: always CSC pull, 2: always COO pull."""
        check(lib.gg_graph_set_dense_policy(self.h, policy), "gg_graph_set_dense_policy")

    def set_tuning(self, key: int, value: int):
        check(lib.gg_graph_set_tuning(self.h, key, value), "gg_graph_set_tuning")

    def get_tuning(self, key: int) -> int:
        v = C.c_int64()
        check(lib.gg_graph_get_tuning(self.h, key, C.byref(v)), "gg_graph_get_tuning")
        return int(v.value)

    # vertexSubset constructors
    def frontier_single(self, v) -> Frontier:
        h = C.c_void_p()
        check(lib.gg_frontier_single(self.h, v, C.byref(h)), "gg_frontier_single")
        return Frontier(self, h)

    def frontier_all(self) -> Frontier:
        h = C.c_void_p()
        check(lib.gg_frontier_all(self.h, C.byref(h)), "gg_frontier_all")
        return Frontier(self, h)

    def frontier_from_mask(self, mask) -> Frontier:
        mask = np.ascontiguousarray(mask, np.uint8)
        h = C.c_void_p()
        check(lib.gg_frontier_from_mask(self.h, mask.ctypes.data_as(C.POINTER(C.c_uint8)), C.byref(h)),
              "gg_frontier_from_mask")
        return Frontier(self, h)

    def frontier_from_list(self, verts) -> Frontier:
        verts = np.ascontiguousarray(verts, np.uint32)
        h = C.c_void_p()
        check(lib.gg_frontier_from_list(self.h, verts.ctypes.data_as(_u32p), len(verts), C.byref(h)),
              "gg_frontier_from_list")
        return Frontier(self, h)

    def edge_map(self, frontier: Frontier, functor_id: int, args: C.Structure, threshold=-1, flags=0) -> Frontier:
        h = C.c_void_p()
        check(lib.gg_edge_map(self.h, frontier.h, functor_id, C.cast(C.byref(args), C.c_void_p), threshold, flags,
                              C.byref(h)), "gg_edge_map")
        return Frontier(self, h)

    def last_edge_map_stats(self) -> EdgeMapStats:
        s = EdgeMapStats()
        check(lib.gg_last_edge_map_stats(self.h, C.byref(s)), "gg_last_edge_map_stats")
        return s

    # applications
    def bfs(self, start=100, out=None):
        """app/BFS.C: (parents, levels, Run); out=(parents, None) skips the levels."""
        par, lev = out if out is not None else (np.empty(self.n, np.int32), np.empty(self.n, np.int32))
        st = RunStats()
        check(lib.gg_bfs(self.h, start, _ptr(par), None if lev is None else _ptr(lev), C.byref(st)), "gg_bfs")
        return par, lev, _run(st)

    def components(self):
        ids = np.empty(self.n, np.int32)
        st = RunStats()
        check(lib.gg_components(self.h, _ptr(ids), C.byref(st)), "gg_components")
        return ids, _run(st)

    def pagerank(self, max_iter=10, bit_all=False, out=None):
        r = out if out is not None else np.empty(self.n, np.float32)
        st = RunStats()
        check(lib.gg_pagerank(self.h, max_iter, int(bit_all), _ptr(r), C.byref(st)), "gg_pagerank")
        return r, _run(st)

    def pagerank_delta(self):
        r = np.empty(self.n, np.float32)
        st = RunStats()
        check(lib.gg_pagerank_delta(self.h, _ptr(r), C.byref(st)), "gg_pagerank_delta")
        return r, _run(st)

    def spmv(self, x=None, out=None):
        y = out if out is not None else np.empty(self.n, np.float32)
        st = RunStats()
        xp = None
        if x is not None:
            x = np.ascontiguousarray(x, np.float32)
            xp = _ptr(x)
        check(lib.gg_spmv(self.h, xp, _ptr(y), C.byref(st)), "gg_spmv")
        return y, _run(st)

    def spmv_stage_input(self, x):
        """gg_spmv_stage_input: start the upload of x (keep it alive and unchanged
        until spmv_staged returns; pinned memory overlaps best)."""
        self._staged = x if isinstance(x, np.ndarray) and x.dtype == np.float32 else np.ascontiguousarray(x, np.float32)
        check(lib.gg_spmv_stage_input(self.h, _ptr(self._staged)), "gg_spmv_stage_input")

    def spmv_staged(self, out=None):
        """gg_spmv_staged: SpMV on the staged input; (y, Run)."""
        y = out if out is not None else np.empty(self.n, np.float32)
        st = RunStats()
        check(lib.gg_spmv_staged(self.h, _ptr(y), C.byref(st)), "gg_spmv_staged")
        self._staged = None
        return y, _run(st)

    def bellman_ford(self, start=100):
        d = np.empty(self.n, np.int32)
        st = RunStats()
        check(lib.gg_bellman_ford(self.h, start, _ptr(d), C.byref(st)), "gg_bellman_ford")
        return d, _run(st)

    def pagerank_converge(self, max_iter=100, eps=1e-7, out=None):
        """app/PageRankConverage.C: (ranks, Run)."""
        r = out if out is not None else np.empty(self.n, np.float32)
        st = RunStats()
        check(lib.gg_pagerank_converge(self.h, max_iter, eps, _ptr(r), C.byref(st)), "gg_pagerank_converge")
        return r, _run(st)

    def ppr_k(self, k=64, iters=20, damping=0.85, tele=None, seeds=None, out=None):
        """k-column personalised PageRank; returns (X[n, k] float32, Run)."""
        y = out if out is not None else np.empty((self.n, k), np.float32)
        tp = sp = None
        if tele is not None:
            tele = np.ascontiguousarray(tele, np.float32).reshape(self.n, k)
            tp = _ptr(tele)
        else:
            seeds = np.ascontiguousarray(seeds, np.uint32)
            assert len(seeds) == k
            sp = _ptr(seeds)
        st = RunStats()
        check(lib.gg_ppr_k(self.h, k, iters, damping, tp, sp, _ptr(y), C.byref(st)), "gg_ppr_k")
        return y, _run(st)

    def bp(self, iters, vert_pot, edge_pot):
        """Belief propagation products after `iters` iterations: (prod[n, 2], Run)."""
        vp = np.ascontiguousarray(vert_pot, np.float32).reshape(self.n, 2)
        ep = np.ascontiguousarray(edge_pot, np.float32).reshape(self.m, 2, 2)
        out = np.empty((self.n, 2), np.float32)
        st = RunStats()
        check(lib.gg_bp(self.h, iters, _ptr(vp), _ptr(ep), _ptr(out), C.byref(st)), "gg_bp")
        return out, _run(st)

    def autotune(self, app=APP_PAGERANK, start=0):
        """Time `app` under every runtime knob combination; the fastest stays
        set on the graph.  Returns the trials (dicts), fastest first."""
        trials = (TuneTrial * 64)()
        nt = C.c_int32()
        check(lib.gg_autotune(self.h, app, start, trials, 64, C.byref(nt)), "gg_autotune")
        return [trials[i].as_dict() for i in range(min(nt.value, 64))]

    def autotune_ppr_k(self, iters=5):
        """(k, column-edges/s) of the fastest gg_ppr_k column count on this graph."""
        k, rate = C.c_int32(), C.c_double()
        check(lib.gg_autotune_ppr_k(self.h, iters, C.byref(k), C.byref(rate)), "gg_autotune_ppr_k")
        return k.value, rate.value

    def msbfs(self, sources, out=None):
        """Levels from up to 64 sources in one traversal: (levels[n, k] int32, Run)."""
        src = np.ascontiguousarray(sources, np.uint32)
        lev = out if out is not None else np.empty((self.n, len(src)), np.int32)
        st = RunStats()
        check(lib.gg_msbfs(self.h, len(src), _ptr(src), _ptr(lev), C.byref(st)), "gg_msbfs")
        return lev, _run(st)

    def msbc(self, sources, dep_out=None, paths_out=None):
        """BC contributions of up to 64 sources: (dependencies[n, k], num_paths[n, k], Run)."""
        src = np.ascontiguousarray(sources, np.uint32)
        k = len(src)
        dep = dep_out if dep_out is not None else np.empty((self.n, k), np.float32)
        npth = paths_out if paths_out is not None else np.empty((self.n, k), np.float32)
        st = RunStats()
        check(lib.gg_msbc(self.h, k, _ptr(src), _ptr(dep), _ptr(npth), C.byref(st)), "gg_msbc")
        return dep, npth, _run(st)

    def bc(self, start=100):
        dep = np.empty(self.n, np.float32)
        npaths = np.empty(self.n, np.float32)
        st = RunStats()
        check(lib.gg_bc(self.h, start, _ptr(dep), _ptr(npaths), C.byref(st)), "gg_bc")
        return dep, npaths, _run(st)


def version() -> str:
    return lib.gg_version().decode()


class GraphBatch:
    """Many independent graphs in one device arena (gg_batch_*)."""

    def __init__(self, host_graphs):
        arr = (HostGraphC * len(host_graphs))(*[hg.c for hg in host_graphs])
        self._hosts = list(host_graphs)
        h = _P()
        check(lib.gg_batch_create(len(host_graphs), arr, C.byref(h)), "gg_batch_create")
        self.h = h
        self.count = len(host_graphs)
        tn, tm = C.c_uint64(), C.c_uint64()
        self.firsts = np.empty(self.count, np.uint64)
        check(lib.gg_batch_info(self.h, C.byref(tn), C.byref(tm), _ptr(self.firsts)), "gg_batch_info")
        self.total_vertices, self.total_edges = tn.value, tm.value

    def bfs(self, sources, out=None):
        """Levels of every graph from its source: (flat levels[total_vertices], Run)."""
        src = np.ascontiguousarray(sources, np.uint32)
        assert len(src) == self.count
        lev = out if out is not None else np.empty(self.total_vertices, np.int32)
        st = RunStats()
        check(lib.gg_batch_bfs(self.h, _ptr(src), _ptr(lev), C.byref(st)), "gg_batch_bfs")
        return lev, _run(st)

    def split(self, flat):
        """Per-graph views of a flat per-vertex array."""
        ends = list(self.firsts[1:]) + [self.total_vertices]
        return [flat[int(a):int(b)] for a, b in zip(self.firsts, ends)]

    def close(self):
        if self.h:
            check(lib.gg_batch_destroy(self.h), "gg_batch_destroy")
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class WeightedPageRank:
    """Weighted PageRank with its adjoint (gg_pagerank_weighted_*): forward
    keeps checkpoints every `checkpoint_every` steps, backward returns
    (dL/dweights, dL/dtele, dL/dx0) for dL/dx of the last forward."""

    def __init__(self, graph, iters=30, damping=0.85, checkpoint_every=5, normalize=False):
        h = _P()
        check(lib.gg_pagerank_weighted_create(graph.h, iters, damping, checkpoint_every, int(normalize), C.byref(h)),
              "gg_pagerank_weighted_create")
        self.h, self.graph, self.n, self.m = h, graph, graph.n, graph.m
        graph._deps.add(self)

    def forward(self, weights, tele, x0=None):
        w = np.ascontiguousarray(weights, np.float32)
        t = np.ascontiguousarray(tele, np.float32)
        x0a = None if x0 is None else np.ascontiguousarray(x0, np.float32)
        x = np.empty(self.n, np.float32)
        st = RunStats()
        check(lib.gg_pagerank_weighted_fwd(self.h, _ptr(w), _ptr(t), None if x0a is None else _ptr(x0a), _ptr(x),
                                           C.byref(st)), "gg_pagerank_weighted_fwd")
        return x, _run(st)

    def backward(self, grad_x):
        g = np.ascontiguousarray(grad_x, np.float32)
        gw = np.empty(self.m, np.float32)
        gt = np.empty(self.n, np.float32)
        g0 = np.empty(self.n, np.float32)
        st = RunStats()
        check(lib.gg_pagerank_weighted_bwd(self.h, _ptr(g), _ptr(gw), _ptr(gt), _ptr(g0), C.byref(st)),
              "gg_pagerank_weighted_bwd")
        return gw, gt, g0, _run(st)

    def close(self):
        if self.h:
            check(lib.gg_pagerank_weighted_destroy(self.h), "gg_pagerank_weighted_destroy")
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune_build(host, app=APP_PAGERANK, start=0, candidates=()):
    """Build `host` under each candidate (dicts of Graph keyword options),
    autotune each, and return (best options dict, best trial dict)."""
    names = ("partitions", "balance", "part_how", "relabel", "order", "tile_vertices", "tile_edges", "build_coo",
             "coo_window", "coo_dst_window", "vertex_order", "coo_tile_vertices")
    defaults = dict(partitions=384, balance=BALANCE_EDGE, part_how=PART_DEST, relabel=0, order=ORDER_HILBERT,
                    tile_vertices=0, tile_edges=0, build_coo=0, coo_window=0, coo_dst_window=0,
                    vertex_order=VORDER_GIVEN, coo_tile_vertices=0)
    cands = (BuildOpts * len(candidates))()
    for i, c in enumerate(candidates):
        d = dict(defaults, **c)
        cands[i] = BuildOpts(*[int(d[k]) for k in names])
    best = BuildOpts()
    trial = TuneTrial()
    check(lib.gg_autotune_build(C.byref(host.c), app, start, cands, len(candidates), C.byref(best), C.byref(trial)),
          "gg_autotune_build")
    return {k: getattr(best, f) for k, f in zip(names, [f for f, _ in BuildOpts._fields_])}, trial.as_dict()
