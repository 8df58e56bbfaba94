"""Generate tests/golden/adjoint_fd_rmat22.npz: FP64 central finite
differences of the weighted-PageRank loss on the differentiation workload.

Workload (the benchmark's adjoint line): R-MAT scale 22, edge factor 16,
seed 6, directed; edge weights U(0,1] normalised per source inside the
function, teleport 1/n, damping 0.85, 30 iterations, loss = c . x_30 with
c ~ N(0,1) (bench.adjoint_inputs).  For 256 edges drawn with
numpy.random.default_rng(9) (indices in the out-edge order) and 16 teleport
entries, the derivative (L(w + h e) - L(w - h e)) / 2h, h = 1e-4, is taken
with the oracle's FP64 forward (oracle.Graph.wpr_forward).  That is 544 FP64
forward runs of 30 iterations over 65M edges, too slow for a test run, so
the values are made once, in parallel worker processes, and committed.
h = 1e-4 (weights are U(0,1], the loss sums 4M ranks of about 2.4e-7): with
h = 1e-6 the rounding of the loss reached several percent of a single
edge's derivative (about 1e-8), while the O(h^2) truncation stays many
orders below it at 1e-4.  The test regenerates the graph and inputs, checks their
fingerprints against the ones stored here and compares the GPU adjoint with
these derivatives.

    python tests/golden/make_fullsize.py [--workers 8]
"""
from __future__ import annotations

import argparse
import hashlib
import multiprocessing as mp
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
OUT = os.path.join(ROOT, "tests", "golden", "adjoint_fd_rmat22.npz")
SCALE, SEED, ITERS, DAMPING, H = 22, 6, 30, 0.85, 1e-4

_state = {}


def fingerprint(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def _init():
    import bench
    import oracle

    r = oracle.RmatGraph(SCALE, 16, seed=SEED, symmetric=False)
    _state["og"] = oracle.Graph(r.offsets, r.indices)
    w, tele, c = bench.adjoint_inputs(r.n, r.m)
    _state["w"], _state["t"], _state["c"] = (w.astype(np.float64), tele.astype(np.float64), c.astype(np.float64))


def _loss(w, t):
    og = _state["og"]
    return float(_state["c"] @ og.wpr_forward(w, t, ITERS, DAMPING, True))


def _fd_edge(e):
    w = _state["w"]
    wp, wm = w.copy(), w.copy()
    wp[e] += H
    wm[e] -= H
    return (_loss(wp, _state["t"]) - _loss(wm, _state["t"])) / (2 * H)


def _fd_tele(v):
    t = _state["t"]
    tp, tm = t.copy(), t.copy()
    tp[v] += H
    tm[v] -= H
    return (_loss(_state["w"], tp) - _loss(_state["w"], tm)) / (2 * H)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workers", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--sample", type=int, default=0, help="only this many edges, printed (no file written)")
    a = ap.parse_args()
    import bench
    import oracle

    r = oracle.RmatGraph(SCALE, 16, seed=SEED, symmetric=False)
    w, tele, c = bench.adjoint_inputs(r.n, r.m)
    rng = np.random.default_rng(9)
    edges = np.sort(rng.choice(r.m, 256, replace=False)).astype(np.int64)
    verts = np.sort(rng.choice(r.n, 16, replace=False)).astype(np.int64)
    if a.sample:
        edges, verts = edges[:a.sample], verts[:0]
    with mp.get_context("spawn").Pool(a.workers, initializer=_init) as pool:
        fd_w = np.array(pool.map(_fd_edge, edges.tolist(), chunksize=1))
        fd_t = np.array(pool.map(_fd_tele, verts.tolist(), chunksize=1))
    if a.sample:
        print(edges.tolist(), fd_w.tolist())
        return
    np.savez_compressed(OUT, edges=edges, fd_w=fd_w, verts=verts, fd_tele=fd_t, h=np.float64(H),
                        graph_sha=np.array(fingerprint(r.offsets, r.indices)),
                        inputs_sha=np.array(fingerprint(w, tele, c)))
    print(f"wrote {OUT}: |fd_w| = {np.linalg.norm(fd_w):.3e}, |fd_tele| = {np.linalg.norm(fd_t):.3e}")


if __name__ == "__main__":
    main()
