"""Oracle jobs of the full-size parity tests (tests/test_gpu_fullsize.py).

Each job runs in a worker process started with `spawn` (so no CUDA state is
ever inherited) and computes one oracle result on a graph the test process
saved as .npy files, or -- for the many small R-MAT graphs -- generated with
the oracle's own restatement of the library's generator.  Only the tests use
this module; it is the checker, never the thing measured.
"""
from __future__ import annotations

import os

import numpy as np

_cache: dict = {}


def save_graph(d: str, name: str, hg, weights=None) -> None:
    """Write a host graph's CSR (and optional per-edge weights) for the workers."""
    np.save(os.path.join(d, f"{name}_off.npy"), hg.offsets)
    np.save(os.path.join(d, f"{name}_idx.npy"), hg.indices)
    if weights is not None:
        np.save(os.path.join(d, f"{name}_w.npy"), np.asarray(weights))
    with open(os.path.join(d, f"{name}_sym"), "w") as f:
        f.write("1" if hg.symmetric else "0")


def _graph(d: str, name: str, weighted: bool):
    import oracle

    key = (d, name, weighted)
    if key not in _cache:
        _cache.clear()  # one graph per worker at a time
        off = np.load(os.path.join(d, f"{name}_off.npy"))
        idx = np.load(os.path.join(d, f"{name}_idx.npy"))
        w = np.load(os.path.join(d, f"{name}_w.npy")).astype(np.float64) if weighted else None
        sym = open(os.path.join(d, f"{name}_sym")).read() == "1"
        _cache[key] = oracle.Graph(off, idx, w, symmetric=sym)
    return _cache[key]


def run(job: dict):
    """One oracle computation; returns a dict of numpy arrays and counts."""
    app = job["app"]
    if app == "many_bfs":  # app/BFS.C levels of each small graph from vertex 0
        import oracle

        out = []
        for scale, ef, seed in job["graphs"]:
            r = oracle.RmatGraph(int(scale), int(ef), seed=int(seed), symmetric=False)
            og = oracle.Graph(r.offsets, r.indices)
            _, lev, st = og.bfs(0)
            out.append((lev, st.edges_traversed))
        return {"levels": [o[0] for o in out], "edges": [o[1] for o in out]}
    og = _graph(job["dir"], job["graph"], job.get("weighted", False))
    if app == "bfs":
        _, lev, st = og.bfs(job["start"])
        return {"levels": lev, "edges": st.edges_traversed, "rounds": st.rounds}
    if app == "bfs_many_sources":
        res = [og.bfs(int(s)) for s in job["sources"]]
        return {"levels": [r[1] for r in res], "edges": [r[2].edges_traversed for r in res]}
    if app == "cc":
        ids, st = og.cc()
        return {"ids": ids, "rounds": st.rounds}
    if app == "pagerank":
        r, st = og.pagerank(job["iters"])
        return {"ranks": r, "rounds": st.rounds, "edges": st.edges_traversed}
    if app == "pagerank_delta":
        r, st = og.pagerank_delta()
        return {"ranks": r, "rounds": st.rounds}
    if app == "spmv":
        y, st = og.spmv(np.load(os.path.join(job["dir"], job["x"])))
        return {"y": y}
    if app == "bellman_ford":
        dist, st = og.bellman_ford(job["start"])
        return {"dist": dist, "rounds": st.rounds}
    if app == "ppr":
        cols = []
        for s in job["seeds"]:
            t = np.zeros(og.n)
            t[int(s)] = 1.0
            cols.append(og.ppr(job["iters"], job["damping"], t))
        return {"cols": cols}
    if app == "bc_brandes":
        res = [og.bc_brandes(int(s)) for s in job["sources"]]
        return {"dep": [r[0] for r in res], "paths": [r[1] for r in res]}
    if app == "wpr":
        d = job["dir"]
        w = np.load(os.path.join(d, "wpr_w.npy"))
        tele = np.load(os.path.join(d, "wpr_tele.npy"))
        c = np.load(os.path.join(d, "wpr_c.npy"))
        x = og.wpr_forward(w, tele, job["iters"], job["damping"], job["normalize"])
        gw, gt, _ = og.wpr_backward(w, tele, job["iters"], job["damping"], c, job["normalize"])
        return {"x": x, "grad_w": gw, "grad_tele": gt}
    raise ValueError(f"unknown oracle job {app}")
