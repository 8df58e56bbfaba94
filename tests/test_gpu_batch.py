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
