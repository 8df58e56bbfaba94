"""Graphs built with vertex_order = VORDER_HOT_FIRST (vertices renumbered
inside every partition, hottest sources first): every application takes and
returns the given ids and must match the oracle run on the given graph; the
low-level API speaks the device ids given by Graph.vertex_order()."""
import numpy as np
import pytest

from conftest import (PR_MAX_ABS, PR_REL_L1, golden_flags, golden_names, golden_partitions, host_graph_from_golden,
                      load_golden, ok_partitions, rel_l1)

pytestmark = pytest.mark.gpu


def check_float(a, b, rel=PR_REL_L1, mx=PR_MAX_ABS):
    assert rel_l1(a, b) <= rel, rel_l1(a, b)
    assert np.abs(np.asarray(a, np.float64) - b).max() <= mx


def check_bfs(g, og, hg, start):
    par, lev, run = g.bfs(start)
    _, olev, ost = og.bfs(start)
    np.testing.assert_array_equal(lev, olev, err_msg=f"bfs from {start}")
    assert run.rounds == ost.rounds and run.edges_traversed == ost.edges_traversed
    off, idx = hg.offsets.astype(np.int64), hg.indices
    reached = np.nonzero(lev > 0)[0]
    for v in reached[:: max(1, len(reached) // 3000)]:
        p = int(par[v])
        assert lev[p] == lev[v] - 1 and v in idx[off[p]:off[p + 1]]
    assert par[start] == start and np.all(par[lev < 0] == -1)


@pytest.mark.parametrize("name", golden_names())
def test_golden_graphs(gg, orc, name):
    """The reference's own outputs, on the renumbered device graph."""
    gd = load_golden(name)
    hg = host_graph_from_golden(gd)
    part_vertex = "vertex" in golden_flags(gd)
    g = gg.Graph(hg, partitions=golden_partitions(gd), balance=gg.BALANCE_VERTEX if part_vertex else gg.BALANCE_EDGE,
                 vertex_order=gg.VORDER_HOT_FIRST)
    og = orc.Graph.from_host(hg, part_vertex=part_vertex)
    start = int(gd["start"])
    if "BFS_levels" in gd:
        np.testing.assert_array_equal(g.bfs(start)[1], gd["BFS_levels"])
        check_bfs(g, og, hg, start)
    if "CC_ids" in gd:
        np.testing.assert_array_equal(g.components()[0], gd["CC_ids"])
    for app, bit in (("PR", False), ("PRBIT", True)):
        if f"{app}_ranks" in gd:
            check_float(g.pagerank(10, bit)[0], gd[f"{app}_ranks"])
        if f"{app}_error" in gd:
            with pytest.raises(gg.GGError):
                g.pagerank(10, bit)
    if "PRD_ranks" in gd:
        check_float(g.pagerank_delta()[0], gd["PRD_ranks"])
    if "PRC_ranks" in gd:
        check_float(g.pagerank_converge()[0], gd["PRC_ranks"])
    if "SPMV_y" in gd:
        check_float(g.spmv()[0], gd["SPMV_y"], rel=1e-6, mx=1e-6)
    if "BF_dist" in gd:
        np.testing.assert_array_equal(g.bellman_ford(start)[0], gd["BF_dist"])
    if "BC_num_paths" in gd:
        dep, npth, _ = g.bc(start)
        odep, onp, _ = og.bc(start)
        np.testing.assert_allclose(npth, onp, rtol=1e-6)
        np.testing.assert_array_equal(np.isnan(dep), np.isnan(odep))
        fin = np.isfinite(odep)
        assert rel_l1(dep[fin], odep[fin]) <= 1e-4


@pytest.fixture(scope="module", params=["sym", "dir"])
def rmat13(gg, orc, request):
    sym = request.param == "sym"
    hg = gg.HostGraph.rmat(13, 16, seed=41, symmetric=sym).add_weights(gg.W_INT32, seed=3, lo=1, hi=100)
    P = ok_partitions(hg, 32)
    g = gg.Graph(hg, partitions=P, vertex_order=gg.VORDER_HOT_FIRST)
    return hg, g, orc.Graph.from_host(hg), P


def test_map_is_the_hot_first_order(gg, rmat13):
    hg, g, _, P = rmat13
    nofo = g.vertex_order()
    want, starts = hg.hot_first_order(P)
    np.testing.assert_array_equal(nofo, want)
    np.testing.assert_array_equal(g.partition_starts(), starts)
    assert not np.array_equal(nofo, np.arange(hg.n))  # a real renumbering
    plain = gg.Graph(hg, partitions=P)
    np.testing.assert_array_equal(plain.vertex_order(), np.arange(hg.n))


@pytest.mark.parametrize("policy", [0, 1, 2])
def test_apps_match_oracle(gg, rmat13, policy):
    hg, g, og, _ = rmat13
    g.set_dense_policy(policy)
    for s in (0, 100, 4321):
        check_bfs(g, og, hg, s)
        np.testing.assert_array_equal(g.bellman_ford(s)[0], og.bellman_ford(s)[0])
        dep, npth, _ = g.bc(s)
        odep, onp, _ = og.bc(s)
        np.testing.assert_allclose(npth, onp, rtol=1e-6)
        fin = np.isfinite(odep)
        assert rel_l1(dep[fin], odep[fin]) <= 1e-4
    np.testing.assert_array_equal(g.components()[0], og.cc()[0])
    for bit in (False, True):
        check_float(g.pagerank(10, bit)[0], og.pagerank(10, bit)[0])
    check_float(g.pagerank_delta()[0], og.pagerank_delta()[0])
    r, run = g.pagerank_converge()
    o, _, ol1 = og.pagerank_converge()
    check_float(r, o)
    x = np.random.default_rng(4).random(hg.n).astype(np.float32)
    y, _ = g.spmv(x)
    check_float(y, og.spmv(x.astype(np.float64))[0], rel=1e-6, mx=1e-6 * float(np.abs(og.spmv(x)[0]).max()))
    g.set_dense_policy(0)


def test_device_loop_and_thresholds(gg, rmat13):
    hg, g, og, _ = rmat13
    for div in (2, 20, 1000):
        g.set_tuning(gg.TUNE_SPARSE_DIV, div)
        for loop in (0, 1, 2):
            g.set_tuning(gg.TUNE_DEVICE_LOOP, loop)
            check_bfs(g, og, hg, 77)
    g.set_tuning(gg.TUNE_SPARSE_DIV, 20)
    g.set_tuning(gg.TUNE_DEVICE_LOOP, 2)


def test_batched_forms(gg, rmat13):
    hg, g, og, _ = rmat13
    rng = np.random.default_rng(8)
    for k in (1, 32, 64):
        seeds = rng.integers(0, hg.n, k).astype(np.uint32)
        x, _ = g.ppr_k(k, iters=8, seeds=seeds)
        for j in range(0, k, 7):
            tele = np.zeros(hg.n)
            tele[seeds[j]] = 1.0
            check_float(x[:, j], og.ppr(8, 0.85, tele))
    tele = rng.random((hg.n, 32)).astype(np.float32)
    tele /= tele.sum(axis=0, keepdims=True)
    x, _ = g.ppr_k(32, iters=5, damping=0.8, tele=tele)
    for j in (0, 13, 31):
        check_float(x[:, j], og.ppr(5, 0.8, tele[:, j].astype(np.float64)))
    x0, _ = g.ppr_k(32, iters=0, tele=tele)
    np.testing.assert_array_equal(x0, tele)
    src = rng.integers(0, hg.n, 20).astype(np.uint32)
    lev, run = g.msbfs(src)
    trav = 0
    for j, s in enumerate(src):
        _, olev, ost = og.bfs(int(s))
        np.testing.assert_array_equal(lev[:, j], olev)
        trav += ost.edges_traversed
    assert run.edges_traversed == trav
    dep, npth, _ = g.msbc(src)
    for j, s in enumerate(src[:6]):
        odep, onp = og.bc_brandes(int(s))
        np.testing.assert_allclose(npth[:, j], onp, rtol=1e-6)
        np.testing.assert_array_equal(np.isnan(dep[:, j]), np.isnan(odep))


def test_low_level_api_speaks_device_ids(gg, rmat13):
    """One BFS level through gg_edge_map on device ids, mapped back, is the
    oracle's level-1 set."""
    hg, g, og, _ = rmat13
    nofo = g.vertex_order()
    s = 100
    par = gg.DeviceArray(g, np.int32, -1)
    lev = gg.DeviceArray(g, np.int32, -1)
    F = g.frontier_single(int(nofo[s]))
    out = g.edge_map(F, gg.F_BFS, gg.BfsArgs(par.ptr, lev.ptr, 1))
    mask_dev = out.mask().astype(bool)
    _, olev, _ = og.bfs(s)
    np.testing.assert_array_equal(mask_dev[nofo], olev == 1)


def test_per_edge_apps_refuse(gg, rmat13):
    hg, g, _, _ = rmat13
    with pytest.raises(gg.GGError) as e:
        g.bp(1, np.ones((hg.n, 2), np.float32), np.ones((hg.m, 2, 2), np.float32))
    assert "UNSUPPORTED" in str(e.value)
    with pytest.raises(gg.GGError) as e:
        gg.WeightedPageRank(g, 3)
    assert "UNSUPPORTED" in str(e.value)


@pytest.mark.parametrize("sym", [True, False])
def test_source_partitions_and_transpose(gg, orc, sym):
    hg = gg.HostGraph.rmat(12, 16, seed=43, symmetric=sym).add_weights(gg.W_INT32, seed=5, lo=1, hi=100)
    og = orc.Graph.from_host(hg)
    g = gg.Graph(hg, partitions=8, part_how=gg.PART_SOURCE, vertex_order=gg.VORDER_HOT_FIRST)
    for policy in (0, 2):
        g.set_dense_policy(policy)
        np.testing.assert_array_equal(g.bfs(9)[1], og.bfs(9)[1])
        np.testing.assert_array_equal(g.components()[0], og.cc()[0])
        np.testing.assert_array_equal(g.bellman_ford(9)[0], og.bellman_ford(9)[0])
        check_float(g.pagerank(10)[0], og.pagerank(10)[0])
    if not sym:  # transposed: the same levels as the transposed graph with its given ids
        P = ok_partitions(hg, 16)
        g2 = gg.Graph(hg, partitions=P, vertex_order=gg.VORDER_HOT_FIRST)
        g3 = gg.Graph(hg, partitions=P)
        g2.transpose()
        g3.transpose()
        for s in (5, 600):
            np.testing.assert_array_equal(g2.bfs(s)[1], g3.bfs(s)[1])
            np.testing.assert_array_equal(g2.bellman_ford(s)[0], g3.bellman_ford(s)[0])
        np.testing.assert_array_equal(g2.components()[0], g3.components()[0])


def test_autotune_build_offers_vertex_order(gg):
    hg = gg.HostGraph.rmat(12, 16, seed=44, symmetric=False)
    cands = [dict(partitions=16), dict(partitions=16, vertex_order=gg.VORDER_HOT_FIRST)]
    best, trial = gg.autotune_build(hg, gg.APP_PAGERANK, 0, cands)
    assert best["vertex_order"] in (0, 1) and trial["ms"] > 0
