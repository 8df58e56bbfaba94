"""Weighted PageRank / SPMV forward and adjoint on the GPU against the FP64
oracle adjoint and FP64 central finite differences."""
import numpy as np
import pytest

from conftest import ok_partitions, rel_l1

pytestmark = pytest.mark.gpu


def _setup(gg, scale, sym, seed, normalize):
    hg = gg.HostGraph.rmat(scale, 16, seed=seed, symmetric=sym)
    rng = np.random.default_rng(seed)
    w = rng.uniform(0, 1, hg.m).astype(np.float32)
    w[w == 0] = 0.5
    if not normalize:  # column-normalised input weights (sum over each source's out-edges = 1)
        deg = np.diff(hg.offsets.astype(np.int64))
        src = np.repeat(np.arange(hg.n), deg)
        tot = np.zeros(hg.n)
        np.add.at(tot, src, w.astype(np.float64))
        w = (w / tot[src]).astype(np.float32)
    tele = rng.uniform(0, 1, hg.n)
    tele = (tele / tele.sum()).astype(np.float32)
    c = rng.standard_normal(hg.n).astype(np.float32)
    return hg, w, tele, c


@pytest.mark.parametrize("normalize", [False, True])
@pytest.mark.parametrize("sym", [True, False])
@pytest.mark.parametrize("every", [5, 1, 7])
def test_adjoint_matches_fp64_adjoint(gg, orc, sym, normalize, every):
    hg, w, tele, c = _setup(gg, 12, sym, 31, normalize)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16))
    og = orc.Graph.from_host(hg)
    iters = 30
    wpr = gg.WeightedPageRank(g, iters, 0.85, every, normalize)
    x, _ = wpr.forward(w, tele)
    ox = og.wpr_forward(w, tele, iters, 0.85, normalize)
    assert rel_l1(x, ox) <= 1e-5
    assert np.abs(x - ox).max() <= 1e-6
    gw, gt, g0, _ = wpr.backward(c)
    ogw, ogt, og0 = og.wpr_backward(w, tele, iters, 0.85, c, normalize)
    for a, b in ((gw, ogw), (gt, ogt), (g0, og0)):
        assert np.linalg.norm(a - b) <= 1e-4 * np.linalg.norm(b)
    np.testing.assert_allclose(gw, ogw, rtol=1e-3, atol=1e-4 * np.abs(ogw).max())
    wpr.close()


def test_adjoint_matches_finite_differences(gg, orc):
    hg, w, tele, c = _setup(gg, 11, False, 32, True)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16))
    og = orc.Graph.from_host(hg)
    iters = 30
    wpr = gg.WeightedPageRank(g, iters, 0.85, 5, True)
    wpr.forward(w, tele)
    gw, gt, _, _ = wpr.backward(c)
    w64, t64, c64 = w.astype(np.float64), tele.astype(np.float64), c.astype(np.float64)
    rng = np.random.default_rng(9)
    edges = rng.choice(hg.m, 256, replace=False)
    fd = np.empty(len(edges))
    h = 1e-6
    for i, e in enumerate(edges):
        wp, wm = w64.copy(), w64.copy()
        wp[e] += h
        wm[e] -= h
        fd[i] = (c64 @ og.wpr_forward(wp, t64, iters, 0.85, True) - c64 @ og.wpr_forward(wm, t64, iters, 0.85, True)) / (2 * h)
    assert np.linalg.norm(gw[edges] - fd) <= 1e-4 * np.linalg.norm(fd)
    verts = rng.choice(hg.n, 32, replace=False)
    for v in verts:
        tp, tm = t64.copy(), t64.copy()
        tp[v] += h
        tm[v] -= h
        f = (c64 @ og.wpr_forward(w64, tp, iters, 0.85, True) - c64 @ og.wpr_forward(w64, tm, iters, 0.85, True)) / (2 * h)
        assert abs(gt[v] - f) <= 1e-4 * max(abs(f), np.abs(gt).max())
    wpr.close()


def test_spmv_adjoint(gg, orc):
    hg, w, _, c = _setup(gg, 12, False, 33, False)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16))
    og = orc.Graph.from_host(hg)
    xin = np.random.default_rng(3).uniform(0, 1, hg.n).astype(np.float32)
    zero = np.zeros(hg.n, np.float32)
    spmv = gg.WeightedPageRank(g, 1, 1.0, 1, False)
    y, _ = spmv.forward(w, zero, x0=xin)
    oy = og.wpr_forward(w, zero, 1, 1.0, x0=xin)
    np.testing.assert_allclose(y, oy, rtol=1e-5, atol=1e-6 * np.abs(oy).max())
    gw, _, gx, _ = spmv.backward(c)
    ogw, _, ogx = og.wpr_backward(w, zero, 1, 1.0, c, x0=xin)
    np.testing.assert_allclose(gx, ogx, rtol=1e-5, atol=1e-5 * np.abs(ogx).max())
    np.testing.assert_allclose(gw, ogw, rtol=1e-5, atol=1e-6 * np.abs(ogw).max())


def test_torch_autograd_function(gg, orc):
    torch = pytest.importorskip("torch")
    from torch_wpr import weighted_pagerank

    hg, w, tele, c = _setup(gg, 11, True, 34, False)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16))
    og = orc.Graph.from_host(hg)
    eng = gg.WeightedPageRank(g, 30, 0.85, 5, False)
    wt = torch.tensor(w, requires_grad=True)
    tt = torch.tensor(tele, requires_grad=True)
    loss = (torch.tensor(c) * weighted_pagerank(wt, tt, eng)).sum()
    loss.backward()
    ogw, ogt, _ = og.wpr_backward(w, tele, 30, 0.85, c)
    assert np.linalg.norm(wt.grad.numpy() - ogw) <= 1e-4 * np.linalg.norm(ogw)
    assert np.linalg.norm(tt.grad.numpy() - ogt) <= 1e-4 * np.linalg.norm(ogt)
