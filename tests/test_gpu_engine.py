"""Engine-level GPU tests through the C ABI: vertexSubset conversions, the
edgeMap direction switch, and every edgeMap kernel (sparse push, CSC pull,
partitioned-COO pull) forced in turn against the oracle."""
import ctypes as C

import numpy as np
import pytest

from conftest import ok_partitions

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sym12(gg, orc):
    hg = gg.HostGraph.rmat(12, 16, seed=61, symmetric=True)
    return hg, gg.Graph(hg, partitions=ok_partitions(hg, 16), tile_vertices=256, tile_edges=2048), orc.Graph.from_host(hg)


def test_frontier_conversions(gg, sym12):
    hg, g, _ = sym12
    rng = np.random.default_rng(0)
    mask = (rng.random(hg.n) < 0.1).astype(np.uint8)
    f = g.frontier_from_mask(mask)
    deg = hg.degrees().astype(np.int64)
    assert f.stats() == (int(mask.sum()), int(deg[mask == 1].sum()))
    f.to_sparse()
    assert f.repr() & 2
    np.testing.assert_array_equal(f.mask(), mask)
    verts = np.nonzero(mask)[0].astype(np.uint32)[::-1].copy()
    h = g.frontier_from_list(verts)
    assert h.stats() == f.stats()
    h.to_dense()
    np.testing.assert_array_equal(h.mask(), mask)
    a = g.frontier_all()
    assert a.stats() == (hg.n, hg.m) and a.repr() == 4
    s = g.frontier_single(7)
    assert s.stats() == (1, int(deg[7]))


@pytest.mark.parametrize("force", ["none", "sparse", "csc", "coo"])
def test_bfs_levels_with_forced_kernel(gg, sym12, force):
    hg, g, og = sym12
    flags = {"none": 0, "sparse": gg.EM_FORCE_SPARSE, "csc": gg.EM_FORCE_CSC, "coo": gg.EM_FORCE_COO}[force]
    par = gg.DeviceArray(g, np.int32, -1)
    lev = gg.DeviceArray(g, np.int32, -1)
    init_p = np.full(hg.n, -1, np.int32)
    init_p[3] = 3
    par.upload(init_p)
    init_l = np.full(hg.n, -1, np.int32)
    init_l[3] = 0
    lev.upload(init_l)
    F = g.frontier_single(3)
    rnd = 0
    kinds = set()
    while F.stats()[0] > 0:
        rnd += 1
        args = gg.BfsArgs(par.ptr, lev.ptr, rnd)
        F = g.edge_map(F, gg.F_BFS, args, -1, flags)
        kinds.add(g.last_edge_map_stats().kind)
    _, olev, _ = og.bfs(3)
    np.testing.assert_array_equal(lev.download(), olev)
    expect = {"sparse": {1}, "csc": {2}, "coo": {3}}.get(force)
    if expect:
        assert kinds - {0} == expect


@pytest.mark.parametrize("force", ["sparse", "csc", "coo"])
def test_cc_with_forced_kernel(gg, sym12, force):
    hg, g, og = sym12
    flags = {"sparse": gg.EM_FORCE_SPARSE, "csc": gg.EM_FORCE_CSC, "coo": gg.EM_FORCE_COO}[force]
    ids = gg.DeviceArray(g, np.int32, np.arange(hg.n, dtype=np.int32))
    prev = gg.DeviceArray(g, np.int32, 0)
    args = gg.CcArgs(ids.ptr, prev.ptr)
    F = g.frontier_all()
    rounds = 0
    while F.stats()[0] > 0 and rounds < 1000:
        gg.check(gg.lib.gg_vertex_map(g.h, F.h, 101, C.cast(C.byref(args), C.c_void_p)), "vertex_map")
        F = g.edge_map(F, gg.F_CC, args, -1, flags)
        rounds += 1
    np.testing.assert_array_equal(ids.download(), og.cc()[0])


def test_direction_switch_follows_reference_thresholds(gg, sym12):
    """m_f + outdeg(F) > m/20 -> dense; > m/2 -> COO (balance=edge); else push."""
    hg, g, _ = sym12
    deg = hg.degrees().astype(np.int64)
    m = hg.m
    order = np.argsort(-deg, kind="stable")
    csum = np.cumsum(deg[order]) + np.arange(1, hg.n + 1)
    low = order[-1:][deg[order[-1:]] > 0] if deg[order[-1]] > 0 else order[deg[order] > 0][-1:]
    mid = order[:np.searchsorted(csum, m // 4) + 1]
    full = np.arange(hg.n)
    for verts in (low, mid, full):
        par = gg.DeviceArray(g, np.int32, -1)
        F = g.frontier_from_list(verts.astype(np.uint32))
        fm, oe = F.stats()
        g.edge_map(F, gg.F_BFS, gg.BfsArgs(par.ptr, None, 1))
        kind = g.last_edge_map_stats().kind
        want = 1 if fm + oe <= m // 20 else (3 if fm + oe > m // 2 else 2)
        assert kind == want, (fm, oe, m)


def test_empty_result_cannot_be_mapped_again(gg, sym12):
    """An edgeMap whose frontier has no out-edges returns empty() with 0 rows;
    mapping it again fails like the reference (ligra-numa.h:937-942)."""
    hg, g, _ = sym12
    deg = hg.degrees()
    iso = int(np.nonzero(deg == 0)[0][0])
    par = gg.DeviceArray(g, np.int32, -1)
    F = g.frontier_single(iso)
    E = g.edge_map(F, gg.F_BFS, gg.BfsArgs(par.ptr, None, 1))
    assert E.stats() == (0, 0)
    with pytest.raises(gg.GGError) as e:
        g.edge_map(E, gg.F_BFS, gg.BfsArgs(par.ptr, None, 2))
    assert "Sizes Don't match" in str(e.value)


@pytest.mark.parametrize("coo_window", [0, 1024, 100000])
@pytest.mark.parametrize("coo_kernel", [0, 1, 2, 3, 4, 5, 6, 7])
def test_apps_with_each_coo_kernel(gg, orc, coo_kernel, coo_window):
    """Every COO pull variant (CTA ring, per-warp direct, per-warp 2/3-stage
    rings, lane-contiguous, prefetch, merged runs with and without cache
    hints) on every window order gives the oracle's results
    when all dense steps use the COO."""
    from conftest import PR_MAX_ABS, PR_REL_L1, rel_l1
    hg = gg.HostGraph.rmat(12, 16, seed=81, symmetric=False).add_weights(gg.W_INT32, seed=2, lo=1, hi=100)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16), tile_vertices=1024, coo_window=coo_window)
    assert g.get_tuning(gg.TUNE_COO_KERNEL) == (4 if coo_window else 7)
    g.set_dense_policy(2)
    g.set_tuning(gg.TUNE_COO_KERNEL, coo_kernel)
    assert g.get_tuning(gg.TUNE_COO_KERNEL) == coo_kernel
    og = orc.Graph.from_host(hg)
    r, _ = g.pagerank(10)
    o, _ = og.pagerank(10)
    assert rel_l1(r, o) <= PR_REL_L1 and np.abs(r - o).max() <= PR_MAX_ABS
    np.testing.assert_array_equal(g.components()[0], og.cc()[0])
    np.testing.assert_array_equal(g.bfs(7)[1], og.bfs(7)[1])
    np.testing.assert_array_equal(g.bellman_ford(7)[0], og.bellman_ford(7)[0])
    dep, npth, _ = g.bc(7)
    odep, onp, _ = og.bc(7)
    fin = np.isfinite(odep)
    assert rel_l1(dep[fin], odep[fin]) <= 1e-4


@pytest.mark.parametrize("graph", ["grid", "rmat_sym", "rmat_dir", "rmat_dir_t"])
def test_bfs_device_loop_matches_host_loop(gg, orc, graph):
    """BFS with consecutive sparse levels in one cooperative launch (1), and
    with every level in one (2), gives the per-level host loop's levels, level
    count and traversed edges (and the oracle's), for every push/pull
    threshold.  Transposed graphs take mode 1's path under mode 2."""
    if graph == "grid":
        hg = gg.HostGraph.grid(96, 0.002, seed=5)
    else:
        hg = gg.HostGraph.rmat(12, 8, seed=17, symmetric=graph == "rmat_sym")
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16))
    oh = hg
    if graph == "rmat_dir_t":
        g.transpose()
        oh = hg.transpose()
    og = orc.Graph.from_host(oh)
    assert g.get_tuning(gg.TUNE_DEVICE_LOOP) == 2
    for div in (20, 2, 1000):
        g.set_tuning(gg.TUNE_SPARSE_DIV, div)
        for start, loop in ((0, 1), (77, 1), (0, 2), (77, 2)):
            g.set_tuning(gg.TUNE_DEVICE_LOOP, loop)
            par, lev, run = g.bfs(start)
            g.set_tuning(gg.TUNE_DEVICE_LOOP, 0)
            par0, lev0, run0 = g.bfs(start)
            np.testing.assert_array_equal(lev, lev0)
            assert run.rounds == run0.rounds and run.edges_traversed == run0.edges_traversed
            if graph != "rmat_dir_t":
                # after transpose() the dense COO levels keep the reference's
                # untransposed COO, which a fresh graph of the transpose does not
                _, olev, ost = og.bfs(start)
                np.testing.assert_array_equal(lev, olev)
                assert run.rounds == ost.rounds and run.edges_traversed == ost.edges_traversed
            reached = lev >= 0
            # every reached vertex other than the source has a parent one level up
            p = par[reached & (lev > 0)]
            assert np.all(lev[p] == lev[reached & (lev > 0)] - 1)


@pytest.mark.parametrize("kernel", [1, 6, 7])
@pytest.mark.parametrize("force", ["coo", "csc", "sparse"])
def test_spmv_edge_map_without_output(gg, sym12, force, kernel):
    """GG_EM_NO_OUTPUT keeps the SPMV sums; the dense COO pull then returns an
    empty output instead of building it."""
    hg, g, _ = sym12
    keep = g.get_tuning(gg.TUNE_COO_KERNEL)
    g.set_tuning(gg.TUNE_COO_KERNEL, kernel)
    flags = {"sparse": gg.EM_FORCE_SPARSE, "csc": gg.EM_FORCE_CSC, "coo": gg.EM_FORCE_COO}[force]
    x = gg.DeviceArray(g, np.float32, np.random.default_rng(1).random(hg.n, dtype=np.float32))
    y0 = gg.DeviceArray(g, np.float32, 0)
    y1 = gg.DeviceArray(g, np.float32, 0)
    F = g.frontier_all()
    out0 = g.edge_map(F, gg.F_SPMV, gg.PairArgs(x.ptr, y0.ptr), -1, flags)
    out1 = g.edge_map(F, gg.F_SPMV, gg.PairArgs(x.ptr, y1.ptr), -1, flags | gg.EM_NO_OUTPUT)
    # the order of shared-memory accumulations varies from run to run
    np.testing.assert_allclose(y0.download(), y1.download(), rtol=2e-6)
    if force == "coo":
        assert out1.stats()[0] == 0 and out0.stats()[0] > 0
    g.set_tuning(gg.TUNE_COO_KERNEL, keep)
