"""The oracle's input builders (oracle/gg_oracle_gen.c) against the library's.

The process that times the reference (bench.py --impl reference) generates
its graph with the oracle's restatement of the library's R-MAT generator, so
that it loads no library of the product; these tests pin that restatement to
gg_gen_rmat / gg_host_graph_add_weights / gg_host_graph_write_gr edge for
edge and byte for byte, and the oracle's CSC builder to a plain sort.
"""
import os

import numpy as np
import pytest

import graphgrind_b200 as gg
import oracle


@pytest.mark.parametrize("scale,ef,seed,sym", [(8, 16, 1, True), (10, 8, 2, False), (12, 16, 5, False),
                                               (11, 32, 1000, False), (9, 4, 3, True)])
def test_rmat_matches_library(scale, ef, seed, sym):
    a = gg.HostGraph.rmat(scale, ef, 0.57, 0.19, 0.19, seed=seed, symmetric=sym)
    b = oracle.RmatGraph(scale, ef, 0.57, 0.19, 0.19, seed=seed, symmetric=sym)
    assert (a.n, a.m) == (b.n, b.m)
    assert np.array_equal(a.offsets, b.offsets)
    assert np.array_equal(a.indices, b.indices)


@pytest.mark.parametrize("sym", [True, False])
def test_weights_match_library(sym):
    a = gg.HostGraph.rmat(10, 16, seed=4, symmetric=sym)
    b = oracle.RmatGraph(10, 16, seed=4, symmetric=sym)
    a.add_weights(gg.W_INT32, seed=102, lo=1, hi=100)
    b.add_weights(False, seed=102, lo=1, hi=100)
    assert np.array_equal(a.weights, b.weights)
    a.add_weights(gg.W_FLOAT32, seed=102)
    b.add_weights(True, seed=102)
    assert np.array_equal(a.weights, b.weights)


@pytest.mark.parametrize("sym,weighted", [(False, False), (False, True), (True, True)])
def test_gr_files_identical(tmp_path, sym, weighted):
    a = gg.HostGraph.rmat(10, 8, seed=9, symmetric=sym)
    b = oracle.RmatGraph(10, 8, seed=9, symmetric=sym)
    if weighted:
        a.add_weights(gg.W_INT32, seed=5, lo=1, hi=100)
        b.add_weights(False, seed=5, lo=1, hi=100)
    pa, pb = str(tmp_path / "a.gr"), str(tmp_path / "b.gr")
    a.write_gr(pa)
    b.write_gr(pb)
    for suffix in ([""] if sym else ["", "_t"]):
        with open(pa + suffix, "rb") as fa, open(pb + suffix, "rb") as fb:
            assert fa.read() == fb.read(), suffix
    assert os.path.exists(pb + "_t") != sym


def test_csc_matches_sort():
    hg = gg.HostGraph.rmat(11, 16, seed=7, symmetric=False).add_weights(gg.W_INT32, seed=1)
    off, idx = hg.offsets.astype(np.int64), hg.indices.astype(np.int64)
    src = np.repeat(np.arange(hg.n, dtype=np.int64), np.diff(off))
    order = np.lexsort((src, idx))
    in_off, in_idx, in_w = oracle.csc_of(hg.offsets, hg.indices, hg.weights.astype(np.float64))
    assert np.array_equal(in_idx, src[order])
    assert np.array_equal(in_w, hg.weights[order].astype(np.float64))
    assert np.array_equal(in_off[1:], np.cumsum(np.bincount(idx, minlength=hg.n)))
    t = hg.transpose()
    assert np.array_equal(in_off, t.offsets) and np.array_equal(in_idx, t.indices)


@pytest.mark.parametrize("sym,bit", [(False, False), (False, True), (True, False)])
def test_pagerank_edge_count(sym, bit):
    """The reference-arm edge count equals the full restatement's."""
    r = oracle.RmatGraph(12, 16, seed=21, symmetric=sym)
    og = oracle.Graph(r.offsets, r.indices, symmetric=sym)
    _, st = og.pagerank(10, bit)
    assert st.rounds == 10
    assert og.pagerank_edges(10, bit) == (st.edges_traversed, st.rounds)
