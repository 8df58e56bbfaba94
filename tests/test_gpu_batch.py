"""Batched traversals on the GPU against the FP64 oracle."""
import numpy as np
import pytest

from conftest import ok_partitions, rel_l1

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("sym", [True, False])
@pytest.mark.parametrize("k", [1, 32, 64])
def test_ppr_k_matches_oracle_per_column(gg, orc, sym, k):
    hg = gg.HostGraph.rmat(12, 16, seed=91, symmetric=sym)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16))
    og = orc.Graph.from_host(hg)
    rng = np.random.default_rng(5)
    seeds = rng.integers(0, hg.n, k).astype(np.uint32)
    x, run = g.ppr_k(k, iters=20, damping=0.85, seeds=seeds)
    assert x.shape == (hg.n, k) and run.rounds == 20
    for j in range(k):
        tele = np.zeros(hg.n)
        tele[seeds[j]] = 1.0
        o = og.ppr(20, 0.85, tele)
        assert rel_l1(x[:, j], o) <= 1e-5, j
        assert np.abs(x[:, j] - o).max() <= 1e-6


def test_ppr_k_dense_teleport(gg, orc):
    hg = gg.HostGraph.rmat(11, 16, seed=92, symmetric=False)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16))
    og = orc.Graph.from_host(hg)
    tele = np.random.default_rng(6).random((hg.n, 32)).astype(np.float32)
    tele /= tele.sum(axis=0, keepdims=True)
    x, _ = g.ppr_k(32, iters=7, damping=0.8, tele=tele)
    for j in range(32):
        o = og.ppr(7, 0.8, tele[:, j].astype(np.float64))
        assert rel_l1(x[:, j], o) <= 1e-5


@pytest.fixture(scope="module", params=["sym", "dir"])
def rmat12(gg, orc, request):
    hg = gg.HostGraph.rmat(12, 16, seed=93, symmetric=request.param == "sym")
    return hg, gg.Graph(hg, partitions=ok_partitions(hg, 32)), orc.Graph.from_host(hg)


@pytest.mark.parametrize("k", [64, 5])
def test_msbfs_levels_bit_exact(rmat12, k):
    hg, g, og = rmat12
    src = np.random.default_rng(k).integers(0, hg.n, k).astype(np.uint32)
    src[-1] = src[0]  # duplicate sources are allowed
    lev, run = g.msbfs(src)
    assert lev.shape == (hg.n, k)
    trav = 0
    for j, s in enumerate(src):
        _, olev, ost = og.bfs(int(s))
        np.testing.assert_array_equal(lev[:, j], olev, err_msg=f"source {s}")
        trav += ost.edges_traversed
    assert run.edges_traversed == trav


def test_msbfs_transposed(gg, orc):
    hg = gg.HostGraph.rmat(11, 8, seed=94, symmetric=False)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16))
    g.transpose()
    og = orc.Graph.from_host(hg.transpose())
    src = np.arange(0, 640, 10, dtype=np.uint32)
    lev, _ = g.msbfs(src)
    for j, s in enumerate(src):
        np.testing.assert_array_equal(lev[:, j], og.bfs(int(s))[1])


@pytest.mark.parametrize("k", [64, 7])
def test_msbc_matches_brandes(rmat12, k):
    hg, g, og = rmat12
    src = np.random.default_rng(100 + k).integers(0, hg.n, k).astype(np.uint32)
    dep, npth, _ = g.msbc(src)
    for j, s in enumerate(src):
        odep, onp = og.bc_brandes(int(s))
        np.testing.assert_allclose(npth[:, j], onp, rtol=1e-6)
        np.testing.assert_array_equal(np.isnan(dep[:, j]), np.isnan(odep))
        fin = np.isfinite(odep)
        assert rel_l1(dep[fin, j], odep[fin]) <= 1e-4, s


@pytest.mark.parametrize("div", [1, 20, 1 << 20])
def test_multi_source_push_and_pull_levels(gg, orc, rmat12, div):
    """Sparse levels push the frontier's out-edges, dense ones pull; every
    level pushed (div 1), the reference's rule (20) and every level pulled
    (2^20) give the oracle's levels and path counts."""
    hg, g, og = rmat12
    g.set_tuning(gg.TUNE_SPARSE_DIV, div)
    src = np.random.default_rng(div).integers(0, hg.n, 40).astype(np.uint32)
    src[5] = src[9]
    lev, run = g.msbfs(src)
    dep, npth, _ = g.msbc(src[:12])
    g.set_tuning(gg.TUNE_SPARSE_DIV, 20)
    trav = 0
    for j, s in enumerate(src):
        _, olev, ost = og.bfs(int(s))
        np.testing.assert_array_equal(lev[:, j], olev, err_msg=f"source {s}")
        trav += ost.edges_traversed
    assert run.edges_traversed == trav
    for j, s in enumerate(src[:12]):
        odep, onp = og.bc_brandes(int(s))
        np.testing.assert_allclose(npth[:, j], onp, rtol=1e-6)
        np.testing.assert_array_equal(np.isnan(dep[:, j]), np.isnan(odep))
        fin = np.isfinite(odep)
        assert rel_l1(dep[fin, j], odep[fin]) <= 1e-4, s


def test_msbc_equals_single_source_on_symmetric(gg, orc):
    hg = gg.HostGraph.rmat(11, 16, seed=95, symmetric=True)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16))
    src = np.array([0, 3, 100, 2047], np.uint32)
    dep, npth, _ = g.msbc(src)
    for j, s in enumerate(src):
        d1, n1, _ = g.bc(int(s))
        np.testing.assert_allclose(npth[:, j], n1, rtol=1e-6)
        fin = np.isfinite(d1)
        np.testing.assert_array_equal(np.isnan(dep[:, j]), np.isnan(d1))
        assert rel_l1(dep[fin, j], d1[fin]) <= 1e-5


def _batch_graphs(gg, count, seed):
    rng = np.random.default_rng(seed)
    hgs = []
    for i in range(count):
        kind = i % 5
        if kind == 3:
            hgs.append(gg.HostGraph.grid(int(rng.integers(4, 40)), 0.01, seed=int(i)))
        elif kind == 4:
            hgs.append(gg.HostGraph.er(int(rng.integers(1, 300)), int(rng.integers(0, 900)), seed=int(i)))
        else:
            hgs.append(gg.HostGraph.rmat(int(rng.integers(4, 13)), int(rng.integers(2, 33)), seed=1000 + i,
                                         symmetric=bool(kind % 2)))
    return hgs


def test_batch_bfs_matches_oracle(gg, orc):
    hgs = _batch_graphs(gg, 60, 7)
    b = gg.GraphBatch(hgs)
    rng = np.random.default_rng(3)
    for rep in range(2):  # the second call replays the captured launch with new sources
        src = np.array([0 if rep == 0 else int(rng.integers(0, h.n)) for h in hgs], np.uint32)
        lev, run = b.bfs(src)
        trav = 0
        for h, s, lv in zip(hgs, src, b.split(lev)):
            _, olev, ost = orc.Graph.from_host(h).bfs(int(s))
            np.testing.assert_array_equal(lv, olev)
            trav += ost.edges_traversed
        assert run.edges_traversed == trav
    b.close()


def test_batch_rejects_bad_source(gg):
    hgs = [gg.HostGraph.rmat(5, 4, seed=1), gg.HostGraph.rmat(6, 4, seed=2)]
    b = gg.GraphBatch(hgs)
    with pytest.raises(gg.GGError):
        b.bfs(np.array([0, 64], np.uint32))
    b.close()
