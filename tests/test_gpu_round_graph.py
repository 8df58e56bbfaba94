"""BellmanFord, Components and PageRankDelta with their runs of dense COO
rounds replayed as one CUDA graph (GG_TUNE_ROUND_GRAPH, the default) against
the host-driven loop and the oracle: identical distances and labels,
PageRankDelta's ranks within its tolerance (1e-4 relative L1: its pull sums
in FP32 in an order that varies from run to run), including the hand-back
to the host when a frontier leaves the dense COO pull (sparse push or CSC
pull) and the return from the host to the graph.

Round counts and traversed edges are not compared: within a round both
applications read values that other threads of the same round may already
have lowered (BellmanFord's distances in the pull and the push, Components'
IDs in the push), as the reference's parallel edgeMap does, so the
intermediate frontiers depend on timing while the fixed point does not."""
import numpy as np
import pytest

from conftest import PR_MAX_ABS, ok_partitions, rel_l1

PRD_REL_L1 = 1e-4

pytestmark = pytest.mark.gpu


def weighted(gg, hg, seed=3):
    return hg.add_weights(gg.W_INT32, seed=seed, lo=1, hi=100)


CASES = {
    "rmat14_dir": lambda gg: weighted(gg, gg.HostGraph.rmat(14, 16, seed=61, symmetric=False)),
    "rmat14_sym": lambda gg: weighted(gg, gg.HostGraph.rmat(14, 16, seed=62, symmetric=True)),
    "grid96": lambda gg: weighted(gg, gg.HostGraph.grid(96, 0.002, seed=5)),
    "er": lambda gg: weighted(gg, gg.HostGraph.er(1 << 13, 1 << 17, seed=7)),
}


def run_both(gg, g, fn):
    g.set_tuning(gg.TUNE_ROUND_GRAPH, 1)
    a = fn()
    g.set_tuning(gg.TUNE_ROUND_GRAPH, 0)
    b = fn()
    g.set_tuning(gg.TUNE_ROUND_GRAPH, 1)
    return a, b


@pytest.mark.parametrize("vorder", [0, 1])
@pytest.mark.parametrize("policy", [0, 2])
@pytest.mark.parametrize("name", sorted(CASES))
def test_round_graph_matches_host_loop_and_oracle(gg, orc, name, policy, vorder):
    hg = CASES[name](gg)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16), vertex_order=vorder)
    og = orc.Graph.from_host(hg)
    assert g.get_tuning(gg.TUNE_ROUND_GRAPH) == 1
    g.set_dense_policy(policy)
    for start in (0, 77):
        (d1, r1), (d0, r0) = run_both(gg, g, lambda: g.bellman_ford(start))
        np.testing.assert_array_equal(d1, d0)
        np.testing.assert_array_equal(d1, og.bellman_ford(start)[0])
        assert 1 <= r1.rounds <= hg.n and r1.edges_traversed > 0
    (i1, c1), (i0, c0) = run_both(gg, g, g.components)
    np.testing.assert_array_equal(i1, i0)
    np.testing.assert_array_equal(i1, og.cc()[0])
    assert 1 <= c1.rounds <= hg.n
    (p1, q1), (p0, q0) = run_both(gg, g, g.pagerank_delta)
    o, ost = og.pagerank_delta()
    for r in (p1, p0):
        assert rel_l1(r, o) <= PRD_REL_L1, rel_l1(r, o)
        assert np.abs(r.astype(np.float64) - o).max() <= PR_MAX_ABS
    assert 1 <= q1.rounds <= 10 * ost.rounds


def test_round_graph_buffers_stay_with_the_graph(gg, orc):
    """The first call with the switch on allocates the loop's two bitmaps and
    two n-entry arrays once per application; later calls reuse them, and a
    destroyed graph releases them."""
    hg = CASES["rmat14_dir"](gg)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16))
    g.set_dense_policy(2)
    base = g.info().device_bytes
    g.bellman_ford(0)
    after_bf = g.info().device_bytes
    n, words = hg.n, (hg.n + 31) // 32
    assert after_bf - base >= 2 * 4 * (n + 4) + 2 * 4 * (words + 4)
    g.bellman_ford(77)
    assert g.info().device_bytes == after_bf
    g.components()
    after_cc = g.info().device_bytes
    assert after_cc > after_bf
    g.pagerank_delta()
    assert g.info().device_bytes >= after_cc + 4 * 4 * (n + 4) + 3 * 4 * (words + 4)
    with pytest.raises(gg.GGError):
        g.set_tuning(gg.TUNE_ROUND_GRAPH, 2)
    g.close()
