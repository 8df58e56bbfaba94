"""TEST INFRASTRUCTURE ONLY: Python access to the oracle.

Two checkers live here:
  * liboracle.so -- a sequential C restatement of GraphGrind's engine and apps
    (gg_oracle.c), FP64 for the floating-point apps;
  * _ref/ref_<App> -- the reference's own applications compiled from the
    GraphGrind source tree by oracle/Makefile (`make -C oracle ref`), driven
    through their 'dump' mode.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package; the product (graphgrind_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")


def reference_tree() -> str:
    """The GraphGrind source tree: $GG_REFERENCE, or a checkout named
    `reference` beside this repository."""
    return os.environ.get("GG_REFERENCE") or os.path.normpath(os.path.join(HERE, "..", "..", "reference"))


def build(ref: bool = False) -> None:
    """Compile liboracle.so (and the reference harness when ref=True and the
    reference tree is present)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    if ref and os.path.isdir(os.path.join(reference_tree(), "graphgrind")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", "REF=" + reference_tree()], check=True)


if not os.path.exists(LIB):
    build()
_lib = C.CDLL(LIB)


class OrGraph(C.Structure):
    _fields_ = [("n", C.c_uint32), ("m", C.c_uint64), ("symmetric", C.c_int32), ("part_vertex", C.c_int32),
                ("out_off", C.c_void_p), ("out_idx", C.c_void_p), ("in_off", C.c_void_p), ("in_idx", C.c_void_p),
                ("out_w", C.c_void_p), ("in_w", C.c_void_p), ("coo_src", C.c_void_p), ("coo_dst", C.c_void_p),
                ("coo_w", C.c_void_p)]


class OrStats(C.Structure):
    _fields_ = [("rounds", C.c_int32), ("edges_traversed", C.c_int64), ("kinds", C.c_int32 * 4)]


_P = C.c_void_p
for name, args in {
    "or_bfs": [C.POINTER(OrGraph), C.c_uint32, _P, _P, C.POINTER(OrStats)],
    "or_cc": [C.POINTER(OrGraph), _P, C.POINTER(OrStats)],
    "or_pagerank": [C.POINTER(OrGraph), C.c_int32, C.c_int32, _P, C.POINTER(OrStats)],
    "or_pagerank_delta": [C.POINTER(OrGraph), _P, C.POINTER(OrStats)],
    "or_pagerank_edges": [C.POINTER(OrGraph), C.c_int32, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int32)],
    "or_spmv": [C.POINTER(OrGraph), _P, _P, C.POINTER(OrStats)],
    "or_bellman_ford": [C.POINTER(OrGraph), C.c_uint32, _P, C.POINTER(OrStats)],
    "or_bc": [C.POINTER(OrGraph), C.c_uint32, _P, _P, C.POINTER(OrStats)],
    "or_bc_brandes": [C.POINTER(OrGraph), C.c_uint32, _P, _P],
    "or_bp": [C.POINTER(OrGraph), C.c_int32, _P, _P, _P, C.POINTER(OrStats)],
    "or_ppr": [C.POINTER(OrGraph), C.c_int32, C.c_double, _P, _P],
    "or_pagerank_converge": [C.POINTER(OrGraph), C.c_int32, C.c_double, _P, C.POINTER(C.c_int32), _P],
    "or_wpr_forward": [C.POINTER(OrGraph), _P, _P, _P, C.c_int32, C.c_double, C.c_int32, _P],
    "or_wpr_backward": [C.POINTER(OrGraph), _P, _P, _P, C.c_int32, C.c_double, C.c_int32, _P, _P, _P, _P],
    "or_partition_sizes": [_P, _P, C.c_uint32, C.c_uint64, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _P, _P],
    "or_hilbert_key": [C.c_int64, C.c_int64, C.c_int64],
    "or_gen_rmat": [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_int32, _P,
                    C.POINTER(C.c_void_p), C.POINTER(C.c_uint64)],
    "or_add_weights": [C.c_uint32, _P, _P, C.c_int32, C.c_int32, C.c_uint64, C.c_int32, C.c_int32, _P],
    "or_csc": [C.c_uint32, C.c_uint64, _P, _P, _P, _P, _P, _P],
    "or_write_gr": [C.c_char_p, C.c_uint32, C.c_uint64, _P, _P, _P, C.c_int32],
}.items():
    f = getattr(_lib, name)
    f.argtypes = args
    f.restype = C.c_int64 if name == "or_hilbert_key" else C.c_int
_lib.or_free.argtypes = [C.c_void_p]
_lib.or_free.restype = None


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def csc_of(offsets, indices, weights=None):
    """In-edge CSC of a CSR, in-lists ordered by source id (host; or_csc)."""
    off = np.ascontiguousarray(offsets, np.uint32)
    idx = np.ascontiguousarray(indices, np.uint32)
    n, m = len(off) - 1, len(idx)
    w = None if weights is None else np.ascontiguousarray(weights, np.float64)
    in_off = np.empty(n + 1, np.uint32)
    in_idx = np.empty(max(m, 1), np.uint32)
    in_w = None if w is None else np.empty(max(m, 1), np.float64)
    assert _lib.or_csc(n, m, _p(off), _p(idx), _p(w), _p(in_off), _p(in_idx), _p(in_w)) == 0
    return in_off, in_idx[:m], None if in_w is None else in_w[:m]


class Graph:
    """Oracle view of a CSR graph (numpy arrays kept alive here)."""

    def __init__(self, offsets, indices, weights=None, symmetric=False, part_vertex=False, coo=None):
        self.out_off = np.ascontiguousarray(offsets, np.uint32)
        self.out_idx = np.ascontiguousarray(indices, np.uint32)
        self.n = len(self.out_off) - 1
        self.m = len(self.out_idx)
        self.out_w = None if weights is None else np.ascontiguousarray(weights, np.float64)
        in_off, in_idx, in_w = csc_of(self.out_off, self.out_idx, self.out_w)
        self.in_off, self.in_idx = in_off, in_idx
        self.in_w = None if in_w is None else np.ascontiguousarray(in_w, np.float64)
        self.coo = None
        if coo is not None:
            self.coo = (np.ascontiguousarray(coo[0], np.uint32), np.ascontiguousarray(coo[1], np.uint32),
                        None if coo[2] is None else np.ascontiguousarray(coo[2], np.float64))
        self.c = OrGraph(self.n, self.m, int(symmetric), int(part_vertex), _p(self.out_off), _p(self.out_idx),
                         _p(self.in_off), _p(self.in_idx), _p(self.out_w), _p(self.in_w),
                         _p(self.coo[0]) if self.coo else None, _p(self.coo[1]) if self.coo else None,
                         _p(self.coo[2]) if self.coo else None)

    @staticmethod
    def from_host(hg, part_vertex=False, float_weights=False):
        w = hg.weights
        if w is not None:
            w = w.astype(np.float64)
        return Graph(hg.offsets.copy(), hg.indices.copy(), w, hg.symmetric, part_vertex)

    def _st(self):
        return OrStats()

    def bfs(self, start):
        par = np.empty(self.n, np.int64)
        lev = np.empty(self.n, np.int32)
        st = self._st()
        assert _lib.or_bfs(C.byref(self.c), start, _p(par), _p(lev), C.byref(st)) == 0
        return par, lev, st

    def cc(self):
        ids = np.empty(self.n, np.int64)
        st = self._st()
        assert _lib.or_cc(C.byref(self.c), _p(ids), C.byref(st)) == 0
        return ids, st

    def pagerank(self, max_iter=10, bit_all=False):
        r = np.empty(self.n, np.float64)
        st = self._st()
        assert _lib.or_pagerank(C.byref(self.c), max_iter, int(bit_all), _p(r), C.byref(st)) == 0
        return r, st

    def pagerank_edges(self, max_iter=10, bit_all=False):
        """(traversed edges, rounds) of pagerank(max_iter, bit_all), counted
        without the arithmetic (valid while the L1 test does not stop early)."""
        e, r = C.c_int64(), C.c_int32()
        assert _lib.or_pagerank_edges(C.byref(self.c), max_iter, int(bit_all), C.byref(e), C.byref(r)) == 0
        return int(e.value), int(r.value)

    def pagerank_delta(self):
        r = np.empty(self.n, np.float64)
        st = self._st()
        assert _lib.or_pagerank_delta(C.byref(self.c), _p(r), C.byref(st)) == 0
        return r, st

    def spmv(self, x=None):
        y = np.empty(self.n, np.float64)
        xx = None if x is None else np.ascontiguousarray(x, np.float64)
        st = self._st()
        assert _lib.or_spmv(C.byref(self.c), _p(xx), _p(y), C.byref(st)) == 0
        return y, st

    def bellman_ford(self, start):
        d = np.empty(self.n, np.int64)
        st = self._st()
        assert _lib.or_bellman_ford(C.byref(self.c), start, _p(d), C.byref(st)) == 0
        return d, st

    def bc(self, start):
        dep = np.empty(self.n, np.float64)
        np_ = np.empty(self.n, np.float64)
        st = self._st()
        assert _lib.or_bc(C.byref(self.c), start, _p(dep), _p(np_), C.byref(st)) == 0
        return dep, np_, st

    def bc_brandes(self, start):
        dep = np.empty(self.n, np.float64)
        np_ = np.empty(self.n, np.float64)
        assert _lib.or_bc_brandes(C.byref(self.c), start, _p(dep), _p(np_)) == 0
        return dep, np_

    def bp(self, iters, vert_pot, edge_pot):
        out = np.empty(2 * self.n, np.float64)
        vp = np.ascontiguousarray(vert_pot, np.float64)
        ep = np.ascontiguousarray(edge_pot, np.float64)
        assert _lib.or_bp(C.byref(self.c), iters, _p(vp), _p(ep), _p(out), None) == 0
        return out

    def pagerank_converge(self, max_iter=100, eps=1e-7):
        """(ranks, iterations, per-iteration L1 changes) of app/PageRankConverage.C (FP64)."""
        ranks = np.empty(self.n, np.float64)
        l1 = np.zeros(max(max_iter, 1), np.float64)
        it = C.c_int32()
        assert _lib.or_pagerank_converge(C.byref(self.c), max_iter, eps, _p(ranks), C.byref(it), _p(l1)) == 0
        return ranks, it.value, l1[:it.value]

    def wpr_forward(self, w, tele, iters, damping, normalize=False, x0=None):
        """Weighted PageRank x_iters (FP64); w in out-edge order."""
        w = np.ascontiguousarray(w, np.float64)
        t = np.ascontiguousarray(tele, np.float64)
        x0a = None if x0 is None else np.ascontiguousarray(x0, np.float64)  # kept alive across the call
        out = np.empty(self.n, np.float64)
        assert _lib.or_wpr_forward(C.byref(self.c), _p(w), _p(t), _p(x0a), iters, damping, int(normalize), _p(out)) == 0
        return out

    def wpr_backward(self, w, tele, iters, damping, grad_x, normalize=False, x0=None):
        """(dL/dw, dL/dtele, dL/dx0) of weighted PageRank for dL/dx_iters = grad_x (FP64)."""
        w = np.ascontiguousarray(w, np.float64)
        t = np.ascontiguousarray(tele, np.float64)
        gx = np.ascontiguousarray(grad_x, np.float64)
        x0a = None if x0 is None else np.ascontiguousarray(x0, np.float64)
        gw = np.empty(len(w), np.float64)
        gt = np.empty(self.n, np.float64)
        g0 = np.empty(self.n, np.float64)
        assert _lib.or_wpr_backward(C.byref(self.c), _p(w), _p(t), None if x0a is None else _p(x0a), iters, damping,
                                    int(normalize), _p(gx), _p(gw), _p(gt), _p(g0)) == 0
        return gw, gt, g0

    def ppr(self, iters, damping, tele):
        x = np.empty(self.n, np.float64)
        t = np.ascontiguousarray(tele, np.float64)
        assert _lib.or_ppr(C.byref(self.c), iters, damping, _p(t), _p(x)) == 0
        return x


def partition_sizes(in_deg, out_deg, m, P, balance=0, part_how=0, relabel=False):
    in_deg = np.ascontiguousarray(in_deg, np.uint32)
    out_deg = np.ascontiguousarray(out_deg, np.uint32)
    coo = np.zeros(P, np.int64)
    csc = np.zeros(P, np.int64)
    rc = _lib.or_partition_sizes(_p(in_deg), _p(out_deg), len(in_deg), m, P, balance, part_how, int(relabel),
                                 _p(coo), _p(csc))
    return rc, coo, csc


def hilbert_key(side_edges, x, y):
    return int(_lib.or_hilbert_key(side_edges, x, y))


# ------------------------------------------------ inputs without the library
class RmatGraph:
    """A seeded R-MAT CSR made by the oracle's restatement of the library's
    generator (or_gen_rmat), for processes that must not load the library."""

    def __init__(self, scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=1, symmetric=False):
        n = 1 << scale
        self.n, self.symmetric = n, bool(symmetric)
        self.offsets = np.empty(n + 1, np.uint32)
        ptr, m = C.c_void_p(), C.c_uint64()
        rc = _lib.or_gen_rmat(scale, edge_factor, a, b, c, seed, int(symmetric), _p(self.offsets), C.byref(ptr),
                              C.byref(m))
        if rc:
            raise RuntimeError(f"or_gen_rmat failed ({rc})")
        self.m = int(m.value)
        try:
            self.indices = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_uint32)), (max(self.m, 1),))[:self.m].copy()
        finally:
            _lib.or_free(ptr)
        self.weights = None

    def add_weights(self, as_float: bool, seed: int, lo: int = 1, hi: int = 100):
        w = np.empty(max(self.m, 1), np.float32 if as_float else np.int32)
        assert _lib.or_add_weights(self.n, _p(self.offsets), _p(self.indices), int(self.symmetric), int(as_float),
                                   seed, lo, hi, _p(w)) == 0
        self.weights = w[:self.m]
        return self

    def write_gr(self, path: str):
        """Galois .gr (plus path_t for a directed graph); float weights are
        written rounded to integers, as the library's writer does."""
        w = None
        if self.weights is not None:
            w = self.weights if self.weights.dtype == np.int32 else np.rint(self.weights).astype(np.int32)
            w = np.ascontiguousarray(w)
        assert _lib.or_write_gr(path.encode(), self.n, self.m, _p(self.offsets), _p(self.indices), _p(w),
                                int(self.symmetric)) == 0, f"cannot write {path}"

    def out_degrees(self):
        return np.diff(self.offsets.astype(np.int64))


# ------------------------------------------------------- reference harness
def ref_binary(app: str) -> str:
    return os.path.join(REF_DIR, "ref_" + app)


def ref_available(app: str = "BFS") -> bool:
    return os.path.exists(ref_binary(app))


def read_dump(path):
    """Parse the ref_harness dump format: 16-byte name, type char, count, data."""
    out = {}
    with open(path, "rb") as f:
        b = f.read()
    o = 0
    types = {"q": "<i8", "i": "<i4", "d": "<f8", "f": "<f4", "B": "u1"}
    while o < len(b):
        name = b[o:o + 16].split(b"\0")[0].decode()
        t = chr(b[o + 16])
        o += 24
        (cnt,) = struct.unpack("<Q", b[o:o + 8])
        o += 8
        dt = np.dtype(types[t])
        out[name] = np.frombuffer(b[o:o + cnt * dt.itemsize], dtype=dt).copy()
        o += cnt * dt.itemsize
    return out


def run_ref(app: str, mode: str, graph_path: str, out_path: str, flags=(), timeout=600, threads=None):
    """Run the reference harness; returns (returncode, parsed dump or None, stderr)."""
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    cmd = [ref_binary(app), mode, out_path, *map(str, flags), graph_path]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, env=env)
    if p.returncode != 0:
        return p.returncode, None, p.stderr
    return 0, read_dump(out_path), p.stderr


def time_ref(app: str, graph_path: str, flags=(), rounds=3, threads=None, timeout=900):
    """The reference's own driver: returns the list of 'Running : t' seconds."""
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    cmd = [ref_binary(app), "run", *map(str, flags), "-rounds", str(rounds), graph_path]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, env=env)
    if p.returncode != 0:
        raise RuntimeError(f"reference {app} failed ({p.returncode}): {p.stderr[-500:]}")
    return [float(l.split(":")[1]) for l in p.stdout.splitlines() if l.startswith("Running")]
