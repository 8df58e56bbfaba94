"""VEBO on the GPU (gg_vebo_gpu) against the reference's own VEBO tool
(graphtools/VEBO.C, tests/golden/vebo.npz) and against the host restatement
(gg_vebo) on larger graphs, bit for bit: offsets, neighbour lists, weights,
the permutation and the partition sizes."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "vebo.npz")
CASES = ["rmat10_P8", "rmat10_P3", "rmat12_P64", "rmat11sym_P16"]


@pytest.mark.parametrize("name", CASES)
def test_vebo_gpu_matches_reference_tool(gg, name):
    gd = np.load(GOLD)
    hg = gg.HostGraph.from_csr(gd[f"{name}_in_offsets"].astype(np.uint32), gd[f"{name}_in_indices"].astype(np.uint32),
                               symmetric=bool(gd[f"{name}_sym"]))
    out, new_of_old, sizes = hg.vebo_gpu(int(gd[f"{name}_P"]))
    np.testing.assert_array_equal(out.offsets.astype(np.int64), gd[f"{name}_offsets"])
    np.testing.assert_array_equal(out.indices.astype(np.int64), gd[f"{name}_indices"])
    assert np.array_equal(np.sort(new_of_old), np.arange(hg.n)) and sizes.sum() == hg.n


@pytest.mark.parametrize("scale,sym,P,weights", [(16, False, 384, True), (15, True, 64, False), (14, False, 3, False),
                                                 (12, False, 4096, False)])
def test_vebo_gpu_equals_host(gg, scale, sym, P, weights):
    hg = gg.HostGraph.rmat(scale, 16, seed=scale + 7, symmetric=sym)
    if weights:
        hg.add_weights(gg.W_INT32, seed=3, lo=1, hi=100)
    try:
        a, na, sa = hg.vebo(P)
    except gg.GGError as e:  # the reference's zero-degree fill fails: the GPU form must fail the same way
        with pytest.raises(gg.GGError) as e2:
            hg.vebo_gpu(P)
        assert e2.value.code == e.code
        return
    b, nb, sb = hg.vebo_gpu(P)
    np.testing.assert_array_equal(a.offsets, b.offsets)
    np.testing.assert_array_equal(a.indices, b.indices)
    np.testing.assert_array_equal(na, nb)
    np.testing.assert_array_equal(sa, sb)
    if weights:
        np.testing.assert_array_equal(a.weights, b.weights)


def test_vebo_gpu_graph_traverses_like_host(gg, orc):
    """A graph prepared on the GPU and built with -o gives the host-prepared one's BFS."""
    hg = gg.HostGraph.rmat(14, 16, seed=9, symmetric=True)
    b, _, _ = hg.vebo_gpu(16)
    og = orc.Graph.from_host(b)
    g = gg.Graph(b, partitions=16, relabel=True)
    _, lev, _ = g.bfs(3)
    np.testing.assert_array_equal(lev, og.bfs(3)[1])
