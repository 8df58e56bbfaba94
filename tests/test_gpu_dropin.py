"""GraphGrind's own application sources, compiled unchanged against the
source-compatible front end (include/ligra_b200.h in place of
ligra-numa.h, include/ligra_b200_main.h as parallel_main), run on the GPU
and checked against the oracle.

The programs are built by `make -C graphgrind_b200 apps` from the reference
tree's app/*.C (where that tree is present); their Compute() loops (for
example app/BFS.C:77-101, app/PageRank.C:102-150, app/Components.C:101-126)
run edgeMap / vertexMap / vertexFilter on the device with the applications'
own functor structs.  Each program's results are the arrays its Compute()
frees, written in dump mode (LIGRA_B200_DUMP)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel_l1

pytestmark = pytest.mark.gpu

APPDIR = os.path.join(ROOT, "graphgrind_b200", "_build", "apps")
APPS = ("BFS", "PageRank", "PageRankBit", "Components", "PageRankDelta", "SPMV", "BellmanFord")


def _bin(app):
    p = os.path.join(APPDIR, app)
    if not os.path.exists(p):
        pytest.skip(f"{p} not built (make -C graphgrind_b200 apps needs the GraphGrind source tree)")
    return p


def _run(app, path, flags, tmp_path, start=100):
    dump = str(tmp_path / f"{app}.dump")
    if os.path.exists(dump):
        os.remove(dump)
    env = dict(os.environ, LIGRA_B200_DUMP=dump)
    p = subprocess.run([_bin(app), *flags, "-rounds", "1", "-r", str(start), path], capture_output=True, text=True,
                       env=env, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    assert "Running : " in p.stdout and "Average : " in p.stdout
    import oracle
    return oracle.read_dump(dump)


@pytest.fixture(scope="module", params=["sym", "dir"])
def graphs(gg, orc, request, tmp_path_factory):
    sym = request.param == "sym"
    d = tmp_path_factory.mktemp("dropin")
    hg = gg.HostGraph.rmat(14, 16, seed=41, symmetric=sym)
    hw = gg.HostGraph.rmat(14, 16, seed=41, symmetric=sym).add_weights(gg.W_INT32, seed=5, lo=1, hi=100)
    pu, pw = str(d / "g.adj"), str(d / "gw.adj")
    hg.write_adj(pu)
    hw.write_adj(pw)
    flags = (["-s"] if sym else []) + ["-c", "16"]
    og = orc.Graph.from_host(hg)
    ow = orc.Graph.from_host(hw)
    return sym, hg, og, ow, pu, pw, flags, d


def test_bfs(graphs):
    sym, hg, og, _, pu, _, flags, d = graphs
    par = _run("BFS", pu, flags, d)["del0"]  # Parents
    _, olev, _ = og.bfs(100)
    np.testing.assert_array_equal(par >= 0, olev >= 0)
    assert par[100] == 100
    off = hg.offsets.astype(np.int64)
    for v in np.nonzero(olev > 0)[0]:
        p = int(par[v])
        assert olev[p] == olev[v] - 1 and v in hg.indices[off[p]:off[p + 1]]


@pytest.mark.parametrize("app,bit", [("PageRank", False), ("PageRankBit", True)])
def test_pagerank(graphs, app, bit):
    _, _, og, _, pu, _, flags, d = graphs
    ranks = _run(app, pu, flags, d)["del0"]  # p_curr after the final swap
    o, _ = og.pagerank(10, bit)
    assert rel_l1(ranks, o) <= 1e-12 and np.abs(ranks - o).max() <= 1e-15


def test_components(graphs):
    _, _, og, _, pu, _, flags, d = graphs
    ids = _run("Components", pu, flags, d)["del0"]  # IDs
    oids, _ = og.cc()
    np.testing.assert_array_equal(ids, oids)


def test_pagerank_delta(graphs):
    _, _, og, _, pu, _, flags, d = graphs
    p = _run("PageRankDelta", pu, flags, d)["del0"]  # p
    o, _ = og.pagerank_delta()
    assert rel_l1(p, o) <= 1e-9


def test_spmv(graphs):
    _, _, _, ow, _, pw, flags, d = graphs
    y = _run("SPMV", pw, flags, d)["del0"]  # p_next after the swap
    oy, _ = ow.spmv()
    assert rel_l1(y, oy) <= 1e-12


def test_bellman_ford(graphs):
    _, _, _, ow, _, pw, flags, d = graphs
    dist = _run("BellmanFord", pw, flags, d)["del1"]  # ShortestPathLen (Visited is freed first)
    od, _ = ow.bellman_ford(100)
    np.testing.assert_array_equal(dist, od)
