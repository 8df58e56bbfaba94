"""The FP64 weighted-PageRank adjoint of the oracle against central finite
differences of the oracle's own forward."""
import numpy as np
import pytest


@pytest.mark.parametrize("normalize", [False, True])
@pytest.mark.parametrize("sym", [True, False])
def test_oracle_adjoint_matches_finite_differences(gg, orc, normalize, sym):
    hg = gg.HostGraph.rmat(7, 8, seed=21, symmetric=sym)
    og = orc.Graph.from_host(hg)
    rng = np.random.default_rng(4)
    w = rng.uniform(0.05, 1.0, hg.m)
    tele = rng.uniform(0, 1, hg.n)
    tele /= tele.sum()
    x0 = rng.uniform(0, 1, hg.n)
    c = rng.standard_normal(hg.n)
    iters, d = 6, 0.85

    def loss(w_, t_, x_):
        return float(c @ og.wpr_forward(w_, t_, iters, d, normalize, x0=x_))

    gw, gt, g0 = og.wpr_backward(w, tele, iters, d, c, normalize, x0=x0)
    h = 1e-6
    # central differences lose about eps * |L| / h to rounding
    fd_tol = 1e-6 + 4e-16 * abs(loss(w, tele, x0)) / h
    for e in rng.choice(hg.m, 40, replace=False):
        wp, wm = w.copy(), w.copy()
        wp[e] += h
        wm[e] -= h
        fd = (loss(wp, tele, x0) - loss(wm, tele, x0)) / (2 * h)
        assert abs(fd - gw[e]) <= fd_tol * max(1.0, abs(fd)), e
    for v in rng.choice(hg.n, 10, replace=False):
        tp, tm = tele.copy(), tele.copy()
        tp[v] += h
        tm[v] -= h
        assert abs((loss(w, tp, x0) - loss(w, tm, x0)) / (2 * h) - gt[v]) <= fd_tol * max(1.0, abs(gt[v]))
        xp, xm = x0.copy(), x0.copy()
        xp[v] += h
        xm[v] -= h
        assert abs((loss(w, tele, xp) - loss(w, tele, xm)) / (2 * h) - g0[v]) <= fd_tol * max(1.0, abs(g0[v]))


def test_weighted_form_reduces_to_pagerank_and_spmv(gg, orc):
    hg = gg.HostGraph.rmat(8, 8, seed=22, symmetric=True)
    og = orc.Graph.from_host(hg)
    deg = np.diff(hg.offsets.astype(np.int64))
    w = np.repeat(1.0 / np.maximum(deg, 1), deg)  # 1/outdeg per out-edge
    tele = np.full(hg.n, 1.0 / hg.n)
    x = og.wpr_forward(w, tele, 10, 0.85)
    ref, _ = og.pagerank(10, bit_all=True)
    np.testing.assert_allclose(x, ref, rtol=1e-12, atol=1e-15)
    xin = np.random.default_rng(1).uniform(0, 1, hg.n)
    wr = np.random.default_rng(2).uniform(0, 1, hg.m)
    y = og.wpr_forward(wr, np.zeros(hg.n), 1, 1.0, x0=xin)
    yref = np.zeros(hg.n)
    src = np.repeat(np.arange(hg.n), deg)
    np.add.at(yref, hg.indices, wr * xin[src])
    np.testing.assert_allclose(y, yref, rtol=1e-12)
