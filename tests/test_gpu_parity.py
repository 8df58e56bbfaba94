"""GPU parity: every application run by the B200 engine (through the C ABI)
against the oracle on the same inputs.  Integer results bit-exact; FP32
results within the stated tolerances of the FP64 oracle."""
import numpy as np
import pytest

from conftest import (PR_MAX_ABS, PR_REL_L1, golden_flags, golden_names, golden_partitions, ok_partitions,
                      host_graph_from_golden, load_golden, rel_l1)

pytestmark = pytest.mark.gpu

BC_REL_L1 = 1e-4  # FP32 dependency accumulation over many levels vs FP64


def build(gg, hg, **kw):
    return gg.Graph(hg, **kw)


def check_bfs(gg_graph, og, start, hg):
    par, lev, st = gg_graph.bfs(start)
    _, olev, ost = og.bfs(start)
    np.testing.assert_array_equal(lev, olev)
    assert st.rounds == ost.rounds
    # parents: every reached vertex (but the source) hangs off a valid edge one level up
    off = hg.offsets.astype(np.int64)
    idx = hg.indices
    reached = np.nonzero(lev > 0)[0]
    for v in reached[:: max(1, len(reached) // 5000)]:
        p = par[v]
        assert lev[p] == lev[v] - 1
        assert v in idx[off[p]:off[p + 1]]
    assert par[start] == start and np.all(par[lev < 0] == -1)


def check_float(a, b, rel=PR_REL_L1, mx=PR_MAX_ABS):
    assert rel_l1(a, b) <= rel, rel_l1(a, b)
    assert np.abs(np.asarray(a, np.float64) - b).max() <= mx


@pytest.mark.parametrize("name", golden_names())
def test_apps_on_golden_graphs(gg, orc, name):
    gd = load_golden(name)
    hg = host_graph_from_golden(gd)
    fl = golden_flags(gd)
    part_vertex = "vertex" in fl
    g = build(gg, hg, partitions=golden_partitions(gd),
              balance=gg.BALANCE_VERTEX if part_vertex else gg.BALANCE_EDGE)
    og = orc.Graph.from_host(hg, part_vertex=part_vertex)
    start = int(gd["start"])
    if "BFS_levels" in gd:
        _, lev, _ = g.bfs(start)
        np.testing.assert_array_equal(lev, gd["BFS_levels"])  # the reference's own levels
        check_bfs(g, og, start, hg)
    if "CC_ids" in gd:
        ids, _ = g.components()
        np.testing.assert_array_equal(ids, gd["CC_ids"])
    for app, bit in (("PR", False), ("PRBIT", True)):
        if f"{app}_ranks" in gd:
            r, _ = g.pagerank(10, bit)
            check_float(r, gd[f"{app}_ranks"])
        if f"{app}_error" in gd:
            with pytest.raises(gg.GGError) as e:
                g.pagerank(10, bit)
            assert "Sizes Don't match" in str(e.value)
    if "PRD_ranks" in gd:
        r, _ = g.pagerank_delta()
        check_float(r, gd["PRD_ranks"])
    if "BC_num_paths" in gd:
        dep, npth, _ = g.bc(start)
        odep, onp, _ = og.bc(start)
        np.testing.assert_allclose(npth, onp, rtol=1e-6)
        np.testing.assert_array_equal(np.isnan(dep), np.isnan(odep))
        fin = np.isfinite(odep)
        assert rel_l1(dep[fin], odep[fin]) <= BC_REL_L1
    if "PRC_ranks" in gd:  # app/PageRankConverage.C, the reference's own output
        r, run = g.pagerank_converge()
        check_float(r, gd["PRC_ranks"])
        # FP32 L1 changes below ~1e-6 sit at the values' rounding resolution, so
        # the FP32 loop may stop a little earlier or later than the FP64 one; it
        # must not stop while the reference's change is still above that
        assert 100 >= run.rounds >= int((gd["PRC_l1"] > 1e-5).sum())
    if "SPMV_y" in gd:
        y, _ = g.spmv()
        check_float(y, gd["SPMV_y"], rel=1e-6, mx=1e-6)
    if "BF_dist" in gd:
        d, _ = g.bellman_ford(start)
        np.testing.assert_array_equal(d, gd["BF_dist"])


@pytest.fixture(scope="module", params=["sym", "dir"])
def rmat14(gg, orc, request):
    sym = request.param == "sym"
    hg = gg.HostGraph.rmat(14, 16, seed=31, symmetric=sym)
    return hg, gg.Graph(hg, partitions=ok_partitions(hg, 64)), orc.Graph.from_host(hg)


def test_bfs_cc_rmat14(rmat14):
    hg, g, og = rmat14
    for start in (0, 100, 12345):
        check_bfs(g, og, start, hg)
    ids, _ = g.components()
    oids, _ = og.cc()
    np.testing.assert_array_equal(ids, oids)


def test_pagerank_family_rmat14(rmat14):
    hg, g, og = rmat14
    for bit in (False, True):
        r, st = g.pagerank(10, bit)
        o, ost = og.pagerank(10, bit)
        check_float(r, o)
        assert st.rounds == ost.rounds
    r, _ = g.pagerank_delta()
    o, _ = og.pagerank_delta()
    check_float(r, o, rel=1e-4, mx=1e-6)


def test_bc_rmat14(rmat14):
    hg, g, og = rmat14
    dep, npth, _ = g.bc(100)
    odep, onp, _ = og.bc(100)
    np.testing.assert_allclose(npth, onp, rtol=1e-5)
    np.testing.assert_array_equal(np.isnan(dep), np.isnan(odep))
    fin = np.isfinite(odep)
    assert rel_l1(dep[fin], odep[fin]) <= BC_REL_L1


@pytest.mark.parametrize("sym", [True, False])
@pytest.mark.parametrize("wt", ["int", "float"])
def test_weighted_rmat13(gg, orc, sym, wt):
    hg = gg.HostGraph.rmat(13, 16, seed=41, symmetric=sym)
    hg.add_weights(gg.W_INT32 if wt == "int" else gg.W_FLOAT32, seed=9, lo=1, hi=100)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 32))
    og = orc.Graph.from_host(hg)
    x = np.random.default_rng(1).random(hg.n).astype(np.float32)
    y, _ = g.spmv(x)
    oy, _ = og.spmv(x.astype(np.float64))
    # FP32 sums of up to thousands of terms: bound the relative error (y reaches ~1e5)
    assert rel_l1(y, oy) <= 1e-6
    nz = oy != 0
    assert np.max(np.abs(y[nz] - oy[nz]) / np.abs(oy[nz])) <= 1e-5
    assert np.all(y[~nz] == 0)
    if wt == "int":
        d, _ = g.bellman_ford(100)
        od, _ = og.bellman_ford(100)
        np.testing.assert_array_equal(d, od)


@pytest.mark.parametrize("order", ["hilbert", "csr"])
@pytest.mark.parametrize("balance", ["edge", "vertex"])
def test_build_options(gg, orc, order, balance):
    hg = gg.HostGraph.rmat(12, 16, seed=51, symmetric=True)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16), order=gg.ORDER_HILBERT if order == "hilbert" else gg.ORDER_CSR,
                 balance=gg.BALANCE_EDGE if balance == "edge" else gg.BALANCE_VERTEX, tile_vertices=512,
                 tile_edges=4096)
    og = orc.Graph.from_host(hg, part_vertex=balance == "vertex")
    assert bool(g.info().has_coo) == (balance == "edge")
    r, _ = g.pagerank(10)
    o, _ = og.pagerank(10)
    check_float(r, o)
    ids, _ = g.components()
    np.testing.assert_array_equal(ids, og.cc()[0])


def test_grid_and_er(gg, orc):
    for hg in (gg.HostGraph.grid(128, 0.001, seed=3), gg.HostGraph.er(1 << 13, 1 << 16, seed=4, symmetric=True)):
        g = gg.Graph(hg, partitions=ok_partitions(hg, 16))
        og = orc.Graph.from_host(hg)
        check_bfs(g, og, 0, hg)
        np.testing.assert_array_equal(g.components()[0], og.cc()[0])


def test_edgeless_and_tiny(gg, orc):
    hg = gg.HostGraph.from_csr(np.zeros(5, np.uint32), np.zeros(0, np.uint32), symmetric=True)
    g = gg.Graph(hg, partitions=1)
    par, lev, st = g.bfs(2)
    assert lev.tolist() == [-1, -1, 0, -1] and st.rounds == 1
    ids, _ = g.components()
    assert ids.tolist() == [0, 1, 2, 3]


@pytest.mark.parametrize("sym", [True, False])
def test_bp_matches_oracle(gg, orc, sym):
    hg = gg.HostGraph.rmat(11, 8, seed=51, symmetric=sym)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16))
    og = orc.Graph.from_host(hg)
    rng = np.random.default_rng(5)
    vp = rng.uniform(0.9, 1.1, (hg.n, 2)).astype(np.float32)
    ep = rng.uniform(0.45, 0.55, (hg.m, 2, 2)).astype(np.float32)
    for iters in (0, 1, 2, 3):
        out, run = g.bp(iters, vp, ep)
        ref = og.bp(iters, vp.astype(np.float64).ravel(), ep.astype(np.float64).ravel()).reshape(hg.n, 2)
        assert run.rounds == iters
        # unnormalised products leave FP32's range on hubs: compare inside it,
        # and require overflow / underflow where FP64 is far outside
        inside = (ref > 1e-30) & (ref < 1e30)
        assert inside.mean() > 0.5
        # a product over d in-edges of beliefs built from the previous products
        # multiplies their relative error by about d each iteration
        np.testing.assert_allclose(out[inside], ref[inside], rtol=2e-5 if iters < 2 else 1e-2)
        assert np.all(np.isinf(out[ref > 1e40]))
        assert np.all(out[ref < 1e-50] == 0)


@pytest.mark.parametrize("sym", [True, False])
def test_pagerank_converge_rmat14(gg, orc, sym):
    hg = gg.HostGraph.rmat(14, 16, seed=44, symmetric=sym)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 64))
    og = orc.Graph.from_host(hg)
    for max_iter in (1, 5, 100):
        r, run = g.pagerank_converge(max_iter)
        o, oit, l1 = og.pagerank_converge(max_iter)
        check_float(r, o)
        assert abs(float(r.sum()) - 1.0) <= 1e-5  # renormalised every iteration
        assert max_iter >= run.rounds >= int((l1 > 1e-5).sum())


def test_vebo_graph_with_relabel_partitions(gg, orc):
    """A VEBO-relabelled graph built with -o (partition boundaries at degree
    rises) traverses to the same results, under the permutation."""
    hg = gg.HostGraph.rmat(13, 16, seed=46, symmetric=False)
    vg, new_of_old, _ = hg.vebo(32)
    g = gg.Graph(vg, partitions=ok_partitions(vg, 32), relabel=True)
    og = orc.Graph.from_host(hg)
    _, olev, _ = og.bfs(100)
    _, lev, _ = g.bfs(int(new_of_old[100]))
    np.testing.assert_array_equal(lev[new_of_old], olev)
    r, _ = g.pagerank(10)
    o, _ = og.pagerank(10)
    check_float(r[new_of_old], o)
    # on a symmetric graph the component classes are invariant under relabelling
    hs = gg.HostGraph.rmat(12, 4, seed=47, symmetric=True)
    vs, nofo, _ = hs.vebo(16)
    cn = gg.Graph(vs, partitions=ok_partitions(vs, 16), relabel=True).components()[0][nofo]
    co = orc.Graph.from_host(hs).cc()[0]
    assert len(set(zip(co.tolist(), cn.tolist()))) == len(set(co.tolist())) == len(set(cn.tolist()))


@pytest.mark.parametrize("sym", [True, False])
def test_apps_with_source_partitions(gg, orc, sym):
    """-P source: COO partitions of sources, dense COO steps with atomic updates."""
    hg = gg.HostGraph.rmat(13, 16, seed=48, symmetric=sym).add_weights(gg.W_INT32, seed=4, lo=1, hi=100)
    g = gg.Graph(hg, partitions=8, part_how=gg.PART_SOURCE)
    assert g.info().has_coo
    og = orc.Graph.from_host(hg)
    for policy in (0, 2):  # reference rule, and every dense step through the COO
        g.set_dense_policy(policy)
        np.testing.assert_array_equal(g.bfs(9)[1], og.bfs(9)[1])
        np.testing.assert_array_equal(g.components()[0], og.cc()[0])
        np.testing.assert_array_equal(g.bellman_ford(9)[0], og.bellman_ford(9)[0])
        r, _ = g.pagerank(10)
        o, _ = og.pagerank(10)
        check_float(r, o)
        y, _ = g.spmv()
        check_float(y, og.spmv()[0], rel=1e-6, mx=1e-6 * float(np.abs(og.spmv()[0]).max()))


@pytest.mark.parametrize("loop", [0, 2])
@pytest.mark.parametrize("kernel", [0, 1, 2, 3])
def test_bfs_early_exit_kernels(gg, rmat14, kernel, loop):
    """Every form of the bottom-up (early-exit) dense step, from the host
    (device loop 0) and inside the all-levels launch (2), gives the oracle's
    levels; parents are frontier in-neighbours one level up."""
    hg, g, og = rmat14
    keep = g.get_tuning(gg.TUNE_DEVICE_LOOP)
    keep_kernel = g.get_tuning(gg.TUNE_EARLY_KERNEL)
    g.set_tuning(gg.TUNE_EARLY_KERNEL, kernel)
    g.set_tuning(gg.TUNE_DEVICE_LOOP, loop)
    g.set_dense_policy(1)  # every dense level takes the early-exit CSC pull
    try:
        for start in (0, 100, 12345):
            check_bfs(g, og, start, hg)
    finally:
        g.set_tuning(gg.TUNE_EARLY_KERNEL, keep_kernel)
        g.set_tuning(gg.TUNE_DEVICE_LOOP, keep)
        g.set_dense_policy(0)


@pytest.mark.parametrize("div", [0, 256, 1 << 30])
def test_bfs_dense_levels_pushed_into_bitmap(gg, rmat14, div):
    """Dense BFS levels from a small frontier run top-down into the output
    bitmap (GG_TUNE_PUSH_DENSE_DIV; 2^30 takes every dense level that way,
    0 none): the oracle's levels and traversed-edge counts either way."""
    hg, g, og = rmat14
    g.set_tuning(gg.TUNE_PUSH_DENSE_DIV, div)
    g.set_dense_policy(1)
    try:
        for start in (0, 100, 12345):
            check_bfs(g, og, start, hg)
            _, _, st = g.bfs(start)
            assert st.edges_traversed == og.bfs(start)[2].edges_traversed
    finally:
        g.set_tuning(gg.TUNE_PUSH_DENSE_DIV, 0)
        g.set_dense_policy(0)


@pytest.mark.parametrize("ctas", [0, 1, 4, 16])
def test_bfs_every_level_on_device(gg, rmat14, ctas):
    """GG_TUNE_DEVICE_LOOP 2 runs the whole BFS in one cooperative launch
    (bottom-up dense levels, top-down sparse ones, the direction rule and the
    bitmap-to-queue conversion on the device): the oracle's levels, rounds
    and traversed edges, at any grid size (GG_TUNE_LOOP_CTAS, capped by
    occupancy; 0 the default per loop)."""
    hg, g, og = rmat14
    g.set_tuning(gg.TUNE_DEVICE_LOOP, 2)
    g.set_tuning(gg.TUNE_LOOP_CTAS, ctas)
    try:
        for start in (0, 100, 12345):
            check_bfs(g, og, start, hg)
            _, _, st = g.bfs(start)
            assert st.edges_traversed == og.bfs(start)[2].edges_traversed
        for div in (1, 1000):  # every level dense / every level sparse
            g.set_tuning(gg.TUNE_SPARSE_DIV, div)
            check_bfs(g, og, 100, hg)
    finally:
        g.set_tuning(gg.TUNE_SPARSE_DIV, 20)
        g.set_tuning(gg.TUNE_DEVICE_LOOP, 2)
        g.set_tuning(gg.TUNE_LOOP_CTAS, 0)
