"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs GraphGrind's own applications, compiled from the reference source tree
by `make -C oracle ref` (oracle/ref_harness.cpp), on small graphs and stores
inputs (CSR) and outputs as .npz files.  Run it in a container that has the
reference tree; the fixtures are committed and the tests only read them.

    python tests/golden/make_golden.py [--reference <GraphGrind tree>]
    (default: $GG_REFERENCE, or a checkout named `reference` beside this repository)
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import graphgrind_b200 as gg  # noqa: E402  (host-only generators and writers)
import oracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
UNWEIGHTED = {"BFS": ["levels", "trace"], "CC": ["ids"], "PR": ["ranks", "trace"], "PRBIT": ["ranks", "trace"],
              "PRD": ["ranks", "trace"], "PRC": ["ranks", "l1"], "BC": ["dependencies", "num_paths"]}
WEIGHTED = {"SPMV": ["y"], "BF": ["dist"]}


def csr_arrays(hg):
    d = {"offsets": hg.offsets.copy(), "indices": hg.indices.copy(), "symmetric": np.int32(hg.symmetric)}
    if hg.weights is not None:
        d["weights"] = hg.weights.astype(np.int32)
    return d


def hand_graph(edges, n, symmetric):
    e = np.array(edges, np.int64).reshape(-1, 2)
    if symmetric:
        e = np.concatenate([e, e[:, ::-1]])
    e = np.unique(e, axis=0)
    off = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(e[:, 0], minlength=n), out=off[1:])
    return gg.HostGraph.from_csr(off.astype(np.uint32), e[:, 1].astype(np.uint32), symmetric=symmetric)


def run_case(name, hg, apps, flags, start, tmp, path=None):
    if path is None:
        path = os.path.join(tmp, name + ".adj")
        hg.write_adj(path)
    out = {**csr_arrays(hg), "start": np.int64(start), "flags": np.array(" ".join(flags))}
    for app, keys in apps.items():
        rc, dump, err = oracle.run_ref(app, "dump", path, os.path.join(tmp, "o.bin"), [*flags, "-r", str(start)])
        if rc != 0:  # the reference aborted: record the failure and its message
            out[f"{app}_error"] = np.array(err.strip().splitlines()[-1] if err.strip() else f"rc={rc}")
            print(f"  {name}/{app}: reference aborted ({out[f'{app}_error']})")
            continue
        for k in keys:
            out[f"{app}_{k}"] = dump[k]
    rc, dump, err = oracle.run_ref("BFS", "parts", path, os.path.join(tmp, "p.bin"), flags)
    if rc == 0:
        for k, v in dump.items():
            out["parts_" + k] = v
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **out)
    print(f"{name}: n={hg.n} m={hg.m} -> {name}.npz")


def partition_cases(tmp):
    """Partition sizes (and failures) of the reference for several -c/-v/-o."""
    out = {}
    g = gg.HostGraph.rmat(12, 16, seed=21, symmetric=True)
    path = os.path.join(tmp, "parts.adj")
    g.write_adj(path)
    out.update({"offsets": g.offsets.copy(), "indices": g.indices.copy()})
    for P in (1, 2, 8, 64, 200, 384):
        for mode, fl in (("edge", []), ("vertex", ["-v", "vertex"]), ("relabel", ["-o"])):
            rc, dump, err = oracle.run_ref("BFS", "parts", path, os.path.join(tmp, "p.bin"), ["-s", "-c", str(P), *fl])
            key = f"P{P}_{mode}"
            out[key + "_rc"] = np.int32(0 if rc == 0 else 1)
            if rc == 0:
                out[key + "_coo"] = dump["coo_sizes"]
                out[key + "_csc"] = dump["csc_sizes"]
    np.savez_compressed(os.path.join(OUT, "partitions.npz"), **out)
    print("partitions.npz")


def partition_src_cases(tmp):
    """-P source on a directed graph: the reference's partition sizes for several
    P, and its source-partitioned COO order (edges of each partition in its
    sorted order) for one P."""
    out = {}
    g = gg.HostGraph.rmat(12, 16, seed=22, symmetric=False)
    path = os.path.join(tmp, "parts_src.adj")
    g.write_adj(path)
    out.update({"offsets": g.offsets.copy(), "indices": g.indices.copy()})
    for P in (1, 2, 8, 64):
        for how in ("source", "dest"):
            rc, dump, err = oracle.run_ref("BFS", "parts", path, os.path.join(tmp, "p.bin"), ["-c", str(P), "-P", how])
            key = f"P{P}_{how}"
            out[key + "_rc"] = np.int32(0 if rc == 0 else 1)
            if rc == 0:
                out[key + "_coo"] = dump["coo_sizes"]
                out[key + "_csc"] = dump["csc_sizes"]
                if P == 8 and how == "source":
                    for k in ("coo_src", "coo_dst", "coo_bounds"):
                        out["P8_source_" + k] = dump[k]
    np.savez_compressed(os.path.join(OUT, "partitions_src.npz"), **out)
    print("partitions_src.npz")


def read_adj_text(path):
    """CSR of a PBBS AdjacencyGraph text file, neighbour order as written."""
    tok = open(path).read().split()
    assert tok[0] == "AdjacencyGraph"
    n, m = int(tok[1]), int(tok[2])
    off = np.array(tok[3:3 + n] + [m], np.int64)
    idx = np.array(tok[3 + n:3 + n + m], np.int64)
    return off, idx


def vebo_cases(tmp):
    """The reference's VEBO tool (graphtools/VEBO.C) on directed graphs; a
    symmetric graph goes in as a directed file holding both directions, whose
    in-degrees are its degrees."""
    out = {}
    cases = [("rmat10_P8", gg.HostGraph.rmat(10, 8, seed=11, symmetric=False), 8),
             ("rmat10_P3", gg.HostGraph.rmat(10, 8, seed=11, symmetric=False), 3),
             ("rmat12_P64", gg.HostGraph.rmat(12, 16, seed=14, symmetric=False), 64),
             ("rmat11sym_P16", gg.HostGraph.rmat(11, 8, seed=15, symmetric=True), 16)]
    for name, hg, P in cases:
        gin = os.path.join(tmp, name + ".gr")
        d = gg.HostGraph.from_csr(hg.offsets.copy(), hg.indices.copy(), symmetric=False)
        d.write_gr(gin)
        adj = os.path.join(tmp, name + ".vebo.adj")
        r = subprocess.run([oracle.ref_binary("VEBO"), "-p", str(P), gin, adj], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-500:]
        off, idx = read_adj_text(adj)
        out.update({f"{name}_in_offsets": hg.offsets.copy(), f"{name}_in_indices": hg.indices.copy(),
                    f"{name}_P": np.int32(P), f"{name}_sym": np.int32(hg.symmetric),
                    f"{name}_offsets": off, f"{name}_indices": idx})
        print(f"vebo {name}: n={hg.n} m={hg.m} P={P}")
    np.savez_compressed(os.path.join(OUT, "vebo.npz"), **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=oracle.reference_tree())
    a = ap.parse_args()
    os.environ["GG_REFERENCE"] = a.reference
    oracle.build(ref=True)
    tmp = tempfile.mkdtemp()
    six = gg.HostGraph.read(os.path.join(a.reference, "sixnode"))
    run_case("sixnode", six, UNWEIGHTED, ["-c", "2"], 0, tmp, path=os.path.join(a.reference, "sixnode"))
    for sym in (True, False):
        tag = "sym" if sym else "dir"
        g = gg.HostGraph.rmat(10, 8, seed=11, symmetric=sym)
        run_case(f"rmat10_{tag}", g, UNWEIGHTED, (["-s"] if sym else []) + ["-c", "8"], 5, tmp)
        w = gg.HostGraph.rmat(10, 8, seed=12, symmetric=sym).add_weights(gg.W_INT32, seed=3, lo=1, hi=100)
        run_case(f"rmat10w_{tag}", w, WEIGHTED, (["-s"] if sym else []) + ["-c", "8"], 5, tmp)
    g = gg.HostGraph.rmat(10, 8, seed=13, symmetric=True)
    run_case("rmat10_vertex", g, UNWEIGHTED, ["-s", "-c", "8", "-v", "vertex"], 7, tmp)
    # hand graphs: directed path, star, two components with isolated vertices
    run_case("path8", hand_graph([(i, i + 1) for i in range(7)], 8, False), UNWEIGHTED, ["-c", "2"], 0, tmp)
    run_case("star9", hand_graph([(0, i) for i in range(1, 9)], 9, True), UNWEIGHTED, ["-s", "-c", "2"], 3, tmp)
    two = [(0, 1), (1, 2), (2, 0), (4, 5), (5, 6), (6, 7), (7, 4), (4, 6)]
    run_case("twocomp10", hand_graph(two, 10, True), UNWEIGHTED, ["-s", "-c", "2"], 4, tmp)
    partition_cases(tmp)
    partition_src_cases(tmp)
    vebo_cases(tmp)


if __name__ == "__main__":
    main()
