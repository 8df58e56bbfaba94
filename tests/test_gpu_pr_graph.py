"""PageRank iterations replayed as one CUDA graph (GG_TUNE_PR_GRAPH, the
default) against the host-driven loop and the oracle: the same iteration
counts and traversed edges, ranks within the PageRank tolerance, stops on
max_iter and on L1 < eps decided on the device, and the hand-back to the host
loop when an output frontier leaves the dense COO pull."""
import numpy as np
import pytest

from conftest import PR_MAX_ABS, PR_REL_L1, ok_partitions, rel_l1

pytestmark = pytest.mark.gpu


def graph_kernels(gg, g, rounds):
    """Kernels of a run that the captured graph finished: the initial pass,
    then per iteration the pull, the check and, unless the pull's commits ran
    the vertex step over every vertex, one more pass (the uncovered ranges,
    or the epilogue); and the one-warp kernels that write the loop's control
    block before the graph and read it back after."""
    fused = g.get_tuning(gg.TUNE_COO_KERNEL) > 0
    per_iter = 2 if fused and g.info().num_coo_gaps == 0 else 3
    return 1 + per_iter * rounds + 2


def check_ranks(r, o):
    assert rel_l1(r, o) <= PR_REL_L1, rel_l1(r, o)
    assert np.abs(r.astype(np.float64) - o).max() <= PR_MAX_ABS


def funnel(gg, core=1024, leaves=60000, seed=3):
    """A small random core (8 out-edges per vertex) fed by many leaves with one
    out-edge each and no in-edges: after the first iteration the output is the
    core alone, whose edgeMap is below the COO pull's m/2 rule."""
    rng = np.random.default_rng(seed)
    rows = []
    for _ in range(core):
        rows.append(np.unique(rng.integers(0, core, 8)))
    for _ in range(leaves):
        rows.append(rng.integers(0, core, 1))
    off = np.zeros(len(rows) + 1, np.uint32)
    off[1:] = np.cumsum([len(r) for r in rows])
    return gg.HostGraph.from_csr(off, np.concatenate(rows).astype(np.uint32))


@pytest.mark.parametrize("sym", [False, True])
def test_graph_loop_matches_host_loop(gg, orc, sym):
    hg = gg.HostGraph.rmat(14, 16, seed=21, symmetric=sym)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 32))
    og = orc.Graph.from_host(hg)
    assert g.get_tuning(gg.TUNE_PR_GRAPH) == 1
    for bit in (False, True):
        for iters in (1, 2, 3, 10, 200):  # 200: L1 < eps ends the loop first
            o, ost = og.pagerank(iters, bit)
            g.set_tuning(gg.TUNE_PR_GRAPH, 1)
            r, st = g.pagerank(iters, bit)
            assert g.get_tuning(gg.TUNE_PR_GRAPH) == 1  # the driver took the graph
            assert st.kernels == graph_kernels(gg, g, st.rounds)
            g.set_tuning(gg.TUNE_PR_GRAPH, 0)
            r0, st0 = g.pagerank(iters, bit)
            if iters <= 10:
                assert st.rounds == st0.rounds == ost.rounds
                assert st.edges_traversed == st0.edges_traversed == ost.edges_traversed
                check_ranks(r, o)
                check_ranks(r0, o)
            elif sym or bit:
                # these converge: L1 < 1e-7 is met near the FP32 rounding floor of
                # the L1 sum (about 2^-24 of the ranks' total), so the stopping
                # iteration may differ from the FP64 oracle's by a few
                assert max(st.rounds, st0.rounds) < 200
                assert abs(st.rounds - ost.rounds) <= 4 and abs(st0.rounds - ost.rounds) <= 4
                check_ranks(r, o)
                check_ranks(r0, o)
            else:  # directed PageRank without bit keeps moving: max_iter ends it
                assert st.rounds == st0.rounds == ost.rounds == 200
                assert st.edges_traversed == st0.edges_traversed == ost.edges_traversed
                assert rel_l1(r, r0.astype(np.float64)) <= PR_REL_L1


def test_graph_loop_recaptured_after_knob_changes(gg, orc):
    """The captured loop follows the COO kernel, bit_all and transpose()."""
    hg = gg.HostGraph.rmat(13, 16, seed=8)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 32))
    og = orc.Graph.from_host(hg)
    o, _ = og.pagerank(10)
    for kernel in (6, 1, 0, 6):
        g.set_tuning(gg.TUNE_COO_KERNEL, kernel)
        r, st = g.pagerank(10)
        assert st.kernels == graph_kernels(gg, g, st.rounds)
        check_ranks(r, o)
    ob, _ = og.pagerank(10, True)
    r, _ = g.pagerank(10, True)
    check_ranks(r, ob)
    # after transpose() the ranks follow the transposed graph's CSR degrees
    g.transpose()
    g.set_tuning(gg.TUNE_PR_GRAPH, 0)
    r0, st0 = g.pagerank(10)
    g.set_tuning(gg.TUNE_PR_GRAPH, 1)
    r, st = g.pagerank(10)
    assert st.rounds == st0.rounds and st.edges_traversed == st0.edges_traversed
    assert rel_l1(r, r0.astype(np.float64)) <= PR_REL_L1
    g.transpose()
    r, _ = g.pagerank(10)
    check_ranks(r, o)


@pytest.mark.parametrize("div", [20, 1])
def test_graph_loop_hands_back_to_host(gg, orc, div):
    """The first output (the core) takes the CSC pull (div 20) or the sparse
    push (div 1): the graph stops after iteration 1 and the host loop goes on
    from its buffers and output bitmap."""
    hg = funnel(gg)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 8))
    assert g.info().num_coo_gaps > 0  # the leaves: the vertex step's separate pass runs
    og = orc.Graph.from_host(hg)
    g.set_tuning(gg.TUNE_SPARSE_DIV, div)
    for bit in (False, True):
        o, ost = og.pagerank(10, bit) if div == 20 else (None, None)
        r, st = g.pagerank(10, bit)
        assert g.get_tuning(gg.TUNE_PR_GRAPH) == 1
        assert st.kernels != graph_kernels(gg, g, st.rounds)  # the host loop ran too
        g.set_tuning(gg.TUNE_PR_GRAPH, 0)
        r0, st0 = g.pagerank(10, bit)
        g.set_tuning(gg.TUNE_PR_GRAPH, 1)
        assert st.rounds == st0.rounds and st.edges_traversed == st0.edges_traversed
        assert rel_l1(r, r0.astype(np.float64)) <= PR_REL_L1
        if o is not None:
            assert st.rounds == ost.rounds and st.edges_traversed == ost.edges_traversed
            check_ranks(r, o)


def test_graph_loop_policies_and_profiling(gg, orc):
    """The COO pull pinned (policy 2) keeps the graph; the CSC pull pinned
    (policy 1) and profiling take the host loop."""
    hg = gg.HostGraph.rmat(12, 16, seed=4)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16))
    og = orc.Graph.from_host(hg)
    o, ost = og.pagerank(10)
    g.set_dense_policy(2)
    r, st = g.pagerank(10)
    assert st.kernels == graph_kernels(gg, g, st.rounds) and st.rounds == ost.rounds
    check_ranks(r, o)
    g.set_dense_policy(1)
    r, st = g.pagerank(10)
    assert st.kernels != graph_kernels(gg, g, st.rounds)
    check_ranks(r, o)
    g.set_dense_policy(0)
    g.set_profiling(True)
    r, st = g.pagerank(10)
    prof = g.profile()
    g.set_profiling(False)
    assert prof["coo_pull"]["launches"] == st.rounds  # one timed pull per iteration
    check_ranks(r, o)
    with pytest.raises(gg.GGError):
        g.set_tuning(gg.TUNE_PR_GRAPH, 2)
