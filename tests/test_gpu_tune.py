"""Autotuner: the chosen knobs are applied and results stay the oracle's."""
import numpy as np
import pytest

from conftest import PR_MAX_ABS, PR_REL_L1, ok_partitions, rel_l1

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("app", ["bfs", "pagerank", "components"])
def test_autotune_keeps_results(gg, orc, app):
    hg = gg.HostGraph.rmat(12, 16, seed=71, symmetric=False)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16))
    og = orc.Graph.from_host(hg)
    code = {"bfs": gg.APP_BFS, "pagerank": gg.APP_PAGERANK, "components": gg.APP_COMPONENTS}[app]
    trials = g.autotune(code, start=3)
    assert len(trials) >= 3
    assert all(a["ms"] <= b["ms"] for a, b in zip(trials, trials[1:]))
    best = trials[0]
    assert g.get_tuning(gg.TUNE_DENSE_POLICY) == best["dense_policy"]
    assert g.get_tuning(gg.TUNE_COO_KERNEL) == best["coo_kernel"]
    assert g.get_tuning(gg.TUNE_SPARSE_DIV) == best["sparse_div"]
    np.testing.assert_array_equal(g.bfs(3)[1], og.bfs(3)[1])
    np.testing.assert_array_equal(g.components()[0], og.cc()[0])
    r, _ = g.pagerank(10)
    o, _ = og.pagerank(10)
    assert rel_l1(r, o) <= PR_REL_L1 and np.abs(r - o).max() <= PR_MAX_ABS


def test_every_sparse_threshold_keeps_results(gg, orc):
    hg = gg.HostGraph.rmat(12, 16, seed=72, symmetric=True)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16))
    og = orc.Graph.from_host(hg)
    for div in (1, 2, 20, 1000, 1 << 20):
        g.set_tuning(gg.TUNE_SPARSE_DIV, div)
        np.testing.assert_array_equal(g.bfs(5)[1], og.bfs(5)[1])
        np.testing.assert_array_equal(g.bellman_ford(5)[0], og.bellman_ford(5)[0])
    with pytest.raises(gg.GGError):
        g.set_tuning(gg.TUNE_SPARSE_DIV, 0)


def test_autotune_build_and_k(gg):
    hg = gg.HostGraph.rmat(12, 16, seed=73, symmetric=False)
    cands = [dict(partitions=8), dict(partitions=16, tile_vertices=1024), dict(partitions=16, coo_window=1024),
             dict(partitions=100000)]  # the last one the partitioner rejects and the tuner skips
    best, trial = gg.autotune_build(hg, gg.APP_PAGERANK, 0, cands)
    assert best["partitions"] in (8, 16) and trial["ms"] > 0
    g = gg.Graph(hg, partitions=16)
    k, rate = g.autotune_ppr_k(3)
    assert k in (1, 32, 64) and rate > 0


@pytest.mark.parametrize("vorder", [0, 1])
@pytest.mark.parametrize("graph", ["rmat_sym", "grid", "rmat_dir", "tiny_sym"])
def test_union_find_components(gg, orc, graph, vorder):
    """GG_TUNE_CC_ALGO 1: union-find on symmetric graphs gives the labels of
    label propagation (the smallest id of each component) in one round;
    directed graphs keep label propagation."""
    if graph == "rmat_sym":
        hg = gg.HostGraph.rmat(13, 4, seed=77, symmetric=True)   # sparse: many components
    elif graph == "grid":
        hg = gg.HostGraph.grid(200, 0.0005, seed=6)
    elif graph == "rmat_dir":
        hg = gg.HostGraph.rmat(12, 4, seed=78, symmetric=False)
    else:
        rows = [[1, 1, 0], [0, 0, 2], [1], [4], [3], []]
        off = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.uint32)
        hg = gg.HostGraph.from_csr(off, np.array([v for r in rows for v in r], np.uint32), symmetric=True)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16), vertex_order=vorder)
    want = orc.Graph.from_host(hg).cc()[0]
    g.set_tuning(gg.TUNE_CC_ALGO, 1)
    for _ in range(2):
        ids, run = g.components()
        np.testing.assert_array_equal(ids, want)
        assert run.rounds == (1 if hg.symmetric else run.rounds)
    assert len(np.unique(want)) > 1 or graph == "grid"  # the grid is one component
    g.set_tuning(gg.TUNE_CC_ALGO, 0)
    np.testing.assert_array_equal(g.components()[0], want)
    with pytest.raises(gg.GGError):
        g.set_tuning(gg.TUNE_CC_ALGO, 2)


def test_autotune_offers_union_find(gg, orc):
    hg = gg.HostGraph.grid(300, 0.0, seed=2)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16))
    trials = g.autotune(gg.APP_COMPONENTS)
    assert any(t["cc_algo"] == 1 for t in trials)
    assert trials[0]["cc_algo"] == g.get_tuning(gg.TUNE_CC_ALGO)
    np.testing.assert_array_equal(g.components()[0], orc.Graph.from_host(hg).cc()[0])
