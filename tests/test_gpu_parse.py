"""The PBBS text reader with the body parsed on the GPU
(gg_host_graph_read_gpu) gives the host reader's graph, and fails where the
host reader fails, also when numbers straddle its chunk boundaries."""
import os
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same(a, b):
    assert (a.n, a.m, a.symmetric, a.weight_type) == (b.n, b.m, b.symmetric, b.weight_type)
    np.testing.assert_array_equal(a.offsets, b.offsets)
    np.testing.assert_array_equal(a.indices, b.indices)
    if a.weights is None:
        assert b.weights is None
    else:
        np.testing.assert_array_equal(a.weights, b.weights)


@pytest.mark.parametrize("chunk", [0, 7, 64, 4096])
@pytest.mark.parametrize("sym,weighted", [(True, False), (False, True), (False, False)])
def test_matches_host_reader(gg, sym, weighted, chunk):
    g = gg.HostGraph.rmat(11, 8, seed=3, symmetric=sym)
    if weighted:
        g.add_weights(gg.W_INT32, seed=2, lo=1, hi=100000)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "g.adj")
        g.write_adj(p)
        host = gg.HostGraph.read(p, symmetric=sym, weighted=weighted)
        dev = gg.HostGraph.read_gpu(p, symmetric=sym, weighted=weighted, chunk_bytes=chunk)
        _same(dev, host)
        if not sym:
            _same(gg.HostGraph.read_gpu(p + "_t", weighted=weighted, chunk_bytes=chunk),
                  gg.HostGraph.read(p + "_t", weighted=weighted))


def test_irregular_whitespace_negative_weights_and_trailing_text(gg):
    body = "WeightedAdjacencyGraph\r\n 4\t5\n0 2  2\n\n4\n1 3\t\t0 2 3\n-7 12 0 2147483647 -2147483648\nextra tokens"
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "w.adj")
        open(p, "w").write(body)
        host = gg.HostGraph.read(p, weighted=True)
        for chunk in (0, 1, 3, 16):
            _same(gg.HostGraph.read_gpu(p, weighted=True, chunk_bytes=chunk), host)
        np.testing.assert_array_equal(host.weights, [-7, 12, 0, 2147483647, -2147483648])


@pytest.mark.parametrize("body", [
    "AdjacencyGraph\n3\n2\n0\n1\n",              # truncated
    "AdjacencyGraph\n3\n2\n0\n1\n2\n0\n5\n",     # neighbour out of range
    "AdjacencyGraph\n3\n2\n0\n3\n1\n0\n1\n",     # offset above m
    "AdjacencyGraph\n3\n2\n0\n2\n1\n0\n1\n",     # offsets not monotone
    "AdjacencyGraph\n3\n2\n0\n1\n1\n0x\n1\n",    # not a number
    "NotAGraph\n1\n0\n0\n",
])
def test_rejects_what_the_host_reader_rejects(gg, body):
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "bad.adj")
        open(p, "w").write(body)
        with pytest.raises(gg.GGError) as e1:
            gg.HostGraph.read(p)
        for chunk in (0, 2):
            with pytest.raises(gg.GGError) as e2:
                gg.HostGraph.read_gpu(p, chunk_bytes=chunk)
            assert "FORMAT" in str(e2.value) and "FORMAT" in str(e1.value)


def test_binary_files_and_built_graph(gg, orc):
    g = gg.HostGraph.rmat(10, 16, seed=4, symmetric=False)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "g.gr")
        g.write_gr(p)
        _same(gg.HostGraph.read_gpu(p, binary=True), gg.HostGraph.read(p, binary=True))
        q = os.path.join(d, "g.adj")
        g.write_adj(q)
        h = gg.HostGraph.read_gpu(q)
        G = gg.Graph(h, partitions=16)
        np.testing.assert_array_equal(G.bfs(3)[1], orc.Graph.from_host(g).bfs(3)[1])
