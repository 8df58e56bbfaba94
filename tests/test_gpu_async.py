"""GG_TUNE_ASYNC_RESULTS: results bound for pinned host arrays leave on a copy
stream while the calls return; after gg_graph_synchronize every array must
hold what the synchronous calls give, also when the next call rewrites the
staging array an earlier copy still reads, and pageable arrays keep being
filled before the call returns."""
import numpy as np
import pytest

from conftest import PR_REL_L1, ok_partitions, rel_l1

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=[0, 1], ids=["given_ids", "hot_first"])
def graph(gg, request):
    hg = gg.HostGraph.rmat(14, 16, seed=12)
    hg.add_weights(gg.W_FLOAT32, seed=3)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 32), vertex_order=request.param)
    yield hg, g
    g.set_tuning(gg.TUNE_ASYNC_RESULTS, 0)


def reference_results(g, x):
    _, lev, _ = g.bfs(5)
    r10, _ = g.pagerank(10)
    r3, _ = g.pagerank(3)
    y, _ = g.spmv(x)
    ids, _ = g.components()
    return lev, r10, r3, y, ids


def test_async_results_match_sync(gg, graph):
    hg, g = graph
    n = hg.n
    x = np.random.default_rng(2).random(n, dtype=np.float32)
    g.set_tuning(gg.TUNE_ASYNC_RESULTS, 0)
    lev0, r10_0, r3_0, y0, ids0 = reference_results(g, x)
    lev7 = g.bfs(7)[1]
    g.set_tuning(gg.TUNE_ASYNC_RESULTS, 1)
    assert g.get_tuning(gg.TUNE_ASYNC_RESULTS) == 1
    par, lev = gg.PinnedArray(n, np.int32), gg.PinnedArray(n, np.int32)
    par7 = gg.PinnedArray(n, np.int32)
    r10, r3 = gg.PinnedArray(n, np.float32), gg.PinnedArray(n, np.float32)
    xin, y = gg.PinnedArray(n, np.float32), gg.PinnedArray(n, np.float32)
    xin.array[:] = x
    for rep in range(3):
        for a in (par, lev, r10, r3, y, par7):
            a.array.fill(-7)
        # back to back, no wait: both PageRank results are staged in the same
        # given-order array, both BFS parents in a third, the SpMV input and
        # the BFS levels in the second
        g.bfs(5, out=(par.array, lev.array))
        g.bfs(7, out=(par7.array, None))
        g.pagerank(10, out=r10.array)
        g.pagerank(3, out=r3.array)
        g.spmv(xin.array, out=y.array)
        ids, _ = g.components()  # pageable: filled before the call returns
        np.testing.assert_array_equal(ids, ids0)
        g.synchronize()
        np.testing.assert_array_equal(lev.array, lev0)
        reached = lev.array >= 0
        assert np.all(par.array[~reached] == -1) and np.all(par.array[reached] >= 0)
        reached7 = lev7 >= 0
        assert np.all(par7.array[~reached7] == -1) and np.all(par7.array[reached7] >= 0)
        assert rel_l1(r10.array, r10_0.astype(np.float64)) <= PR_REL_L1
        assert rel_l1(r3.array, r3_0.astype(np.float64)) <= PR_REL_L1
        assert rel_l1(r3.array, r10.array.astype(np.float64)) > 1e-4  # not the other result
        assert rel_l1(y.array, y0.astype(np.float64)) <= 1e-5


def test_async_switch(gg, graph):
    _, g = graph
    g.set_tuning(gg.TUNE_ASYNC_RESULTS, 1)
    g.set_tuning(gg.TUNE_ASYNC_RESULTS, 0)
    assert g.get_tuning(gg.TUNE_ASYNC_RESULTS) == 0
    with pytest.raises(gg.GGError):
        g.set_tuning(gg.TUNE_ASYNC_RESULTS, 2)
    g.synchronize()


def test_staged_spmv_input(gg, graph):
    """gg_spmv_stage_input uploads SpMV's input on the copy stream while the
    preceding call still runs; gg_spmv_staged then gives gg_spmv's result.
    Staging into the array a BFS level output also uses gives the input up,
    and staging needs the asynchronous mode."""
    hg, g = graph
    n = hg.n
    x = np.random.default_rng(8).random(n, dtype=np.float32)
    g.set_tuning(gg.TUNE_ASYNC_RESULTS, 0)
    y0, _ = g.spmv(x)
    with pytest.raises(gg.GGError) as e:
        g.spmv_stage_input(x)
    assert e.value.code == gg.ERR_UNSUPPORTED
    g.set_tuning(gg.TUNE_ASYNC_RESULTS, 1)
    xp, yp, rp = gg.PinnedArray(n, np.float32), gg.PinnedArray(n, np.float32), gg.PinnedArray(n, np.float32)
    xp.array[:] = x
    for _ in range(3):  # back to back, as a serving loop stages each request's input
        g.bfs(5)
        g.spmv_stage_input(xp.array)
        g.pagerank(10, out=rp.array)  # runs while the input uploads
        _, run = g.spmv_staged(out=yp.array)
        g.synchronize()
        np.testing.assert_allclose(yp.array, y0, rtol=1e-6, atol=1e-7 * np.abs(y0).max())
        assert run.edges_traversed == hg.m
    g.spmv_stage_input(xp.array)
    lev = gg.PinnedArray(n, np.int32)
    g.bfs(5, out=(np.empty(n, np.int32), lev.array))  # levels are staged in the same array
    with pytest.raises(gg.GGError) as e:
        g.spmv_staged(out=yp.array)
    assert e.value.code == gg.ERR_INVALID_ARG
    g.synchronize()
