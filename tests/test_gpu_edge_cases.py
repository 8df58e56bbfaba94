"""Edge cases on the GPU against the oracle: edgeless and one-vertex graphs,
self-loops, repeated edges (with their own weights), rows given unsorted,
sinks and isolated vertices, through every application, the batched entry
points, the weighted-PageRank adjoint and -P source partitions.  Where the
oracle (like the reference) aborts on a graph, the device must return an
error rather than a result."""
import numpy as np
import pytest

from conftest import PR_MAX_ABS, PR_REL_L1, rel_l1

pytestmark = pytest.mark.gpu


def _csr(n, rows, weights=None):
    off = np.zeros(n + 1, np.uint32)
    off[1:] = np.cumsum([len(r) for r in rows])
    idx = np.array([v for r in rows for v in r], np.uint32)
    w = None if weights is None else np.array([x for r in weights for x in r], np.int32)
    return off, idx, w


def _weights(rows, symmetric):
    """1..9 per edge; on a symmetric graph the k-th copy of u->v and the k-th
    copy of v->u share a weight."""
    out = []
    for u, r in enumerate(rows):
        seen = {}
        ws = []
        for v in r:
            k = seen.get(v, 0)
            seen[v] = k + 1
            a, b = (min(u, v), max(u, v)) if symmetric else (u, v)
            ws.append(1 + (a * 7 + b * 13 + k * 5) % 9)
        out.append(ws)
    return out


TINY = {
    "edgeless5_dir": (5, [[]] * 5, False),
    "edgeless5_sym": (5, [[]] * 5, True),
    "one_vertex": (1, [[]], True),
    "one_loop_dir": (1, [[0]], False),
    "one_loop_sym": (1, [[0]], True),
    "two_loops_dir": (2, [[0, 0], []], False),
    "multi_dir": (7, [[1, 1, 2, 0], [2, 2, 2], [3], [], [4, 4, 5], [1, 0], []], False),
    "multi_sym": (6, [[1, 1, 3], [0, 0, 2], [1, 2], [0, 4], [3], []], True),
    "multi_sym_unsorted": (6, [[3, 1, 1], [2, 0, 0], [2, 1], [4, 0], [3], []], True),
}


def _medium_rows(symmetric, seed=61):
    """An RMAT-10 graph with repeated edges on every third vertex, self-loops
    on every fifth, and every seventh row reversed (unsorted)."""
    import graphgrind_b200 as gg
    hg = gg.HostGraph.rmat(10, 8, seed=seed, symmetric=symmetric)
    off, idx = hg.offsets.astype(np.int64), hg.indices
    n = hg.n
    if symmetric:
        pairs = [(u, int(v)) for u in range(n) for v in idx[off[u]:off[u + 1]] if u < v]
        extra = [p for i, p in enumerate(pairs) if p[0] % 3 == 0 and i % 2 == 0]
        loops = [(u, u) for u in range(0, n, 5)]
        rows = [[] for _ in range(n)]
        for u, v in pairs + extra + loops:
            rows[u].append(v)
            if u != v:
                rows[v].append(u)
        rows = [sorted(r) for r in rows]
        # a symmetric graph's rows are its in-edge lists: keep them sorted
        # (weighted PageRank needs that), repeated edges and loops included
        return n, rows
    rows = []
    for u in range(n):
        r = [int(v) for v in idx[off[u]:off[u + 1]]]
        if u % 3 == 0:
            r = r + r[:2]
        if u % 5 == 0:
            r = r + [u]
        r.sort()
        if u % 7 == 0:
            r = r[::-1]
        rows.append(r)
    return n, rows


def _host(gg, n, rows, symmetric, weighted=True):
    off, idx, w = _csr(n, rows, _weights(rows, symmetric) if weighted else None)
    return gg.HostGraph.from_csr(off, idx, w, symmetric=symmetric)


def _partitions(gg, hg, preferred, part_how=0):
    outd = hg.degrees()
    ind = hg.transpose().degrees() if not hg.symmetric else outd
    for P in range(preferred, 0, -1):
        try:
            gg.partition_sizes(ind, outd, hg.m, P, 0, part_how, False)
            return P
        except gg.GGError:
            continue
    raise AssertionError("no partition count accepted")


def _case(gg, orc, name):
    if name in TINY:
        n, rows, sym = TINY[name]
        pref = 4
    else:
        sym = name.endswith("sym")
        n, rows = _medium_rows(sym)
        pref = 16
    hg = _host(gg, n, rows, sym)
    return hg, orc.Graph.from_host(hg), pref


CASES = list(TINY) + ["medium_multi_dir", "medium_multi_sym"]


def _starts(hg):
    return list(range(hg.n)) if hg.n <= 8 else [0, 1, 5, 99, hg.n - 1]


def _oracle_or_none(fn, *a, **k):
    try:
        return fn(*a, **k)
    except AssertionError:  # the oracle aborts where the reference does
        return None


def _close(a, b, rel=PR_REL_L1, mx=PR_MAX_ABS):
    b = np.asarray(b, np.float64)
    assert rel_l1(a, b) <= rel, rel_l1(a, b)
    assert np.abs(np.asarray(a, np.float64) - b).max() <= mx * max(1.0, float(np.abs(b).max()))


def _check_parents(par, lev, hg, start):
    off, idx = hg.offsets.astype(np.int64), hg.indices
    for v in np.nonzero(lev > 0)[0]:
        p = int(par[v])
        assert lev[p] == lev[v] - 1 and v in idx[off[p]:off[p + 1]]
    assert par[start] == start and np.all(par[lev < 0] == -1)


@pytest.mark.parametrize("vorder", [0, 1])
@pytest.mark.parametrize("policy", [0, 1, 2])
@pytest.mark.parametrize("name", CASES)
def test_traversals(gg, orc, name, policy, vorder):
    """BFS (parents valid, levels bit-exact), Components, BellmanFord and BC,
    on the given ids and renumbered hottest-first."""
    hg, og, pref = _case(gg, orc, name)
    g = gg.Graph(hg, partitions=_partitions(gg, hg, pref), vertex_order=vorder)
    g.set_dense_policy(policy)
    ids, _ = g.components()
    np.testing.assert_array_equal(ids, og.cc()[0])
    for s in _starts(hg):
        par, lev, run = g.bfs(s)
        _, olev, ost = og.bfs(s)
        np.testing.assert_array_equal(lev, olev, err_msg=f"bfs from {s}")
        _check_parents(par, lev, hg, s)
        assert run.rounds == ost.rounds
        d, _ = g.bellman_ford(s)
        np.testing.assert_array_equal(d, og.bellman_ford(s)[0], err_msg=f"bellman-ford from {s}")
        dep, npth, _ = g.bc(s)
        odep, onp, _ = og.bc(s)
        np.testing.assert_allclose(npth, onp, rtol=1e-6)
        np.testing.assert_array_equal(np.isnan(dep), np.isnan(odep))
        fin = np.isfinite(odep)
        assert rel_l1(dep[fin], odep[fin]) <= 1e-4


@pytest.mark.parametrize("loop", [0, 1, 2])
@pytest.mark.parametrize("name", CASES)
def test_device_loop_modes(gg, orc, name, loop):
    """BFS with one host round trip per level (0), with runs of sparse levels
    in one cooperative launch (1) and with every level in one (2, the
    default) gives the oracle's levels, rounds and traversed edges, with
    valid parents."""
    hg, og, pref = _case(gg, orc, name)
    g = gg.Graph(hg, partitions=_partitions(gg, hg, pref))
    g.set_tuning(gg.TUNE_DEVICE_LOOP, loop)
    for s in _starts(hg):
        par, lev, run = g.bfs(s)
        _, olev, ost = og.bfs(s)
        np.testing.assert_array_equal(lev, olev, err_msg=f"bfs from {s}")
        _check_parents(par, lev, hg, s)
        assert run.rounds == ost.rounds and run.edges_traversed == ost.edges_traversed


@pytest.mark.parametrize("vorder", [0, 1])
@pytest.mark.parametrize("name", CASES)
def test_rank_apps(gg, orc, name, vorder):
    """PageRank, PageRankBit, PageRankDelta, SPMV and PageRankConverage."""
    hg, og, pref = _case(gg, orc, name)
    g = gg.Graph(hg, partitions=_partitions(gg, hg, pref), vertex_order=vorder)
    for bit in (False, True):
        o = _oracle_or_none(og.pagerank, 10, bit)
        if o is None:
            with pytest.raises(gg.GGError):
                g.pagerank(10, bit)
        else:
            _close(g.pagerank(10, bit)[0], o[0])
    o = _oracle_or_none(og.pagerank_delta)
    if o is None:
        with pytest.raises(gg.GGError):
            g.pagerank_delta()
    else:
        _close(g.pagerank_delta()[0], o[0])
    y, _ = g.spmv()
    _close(y, og.spmv()[0], rel=1e-6, mx=1e-6)
    x = np.random.default_rng(3).uniform(-1, 1, hg.n).astype(np.float32)
    y, _ = g.spmv(x)  # signed terms cancel: FP32 error is relative to the sum of |terms|
    _close(y, og.spmv(x.astype(np.float64))[0], rel=1e-5, mx=1e-5)
    o = _oracle_or_none(og.pagerank_converge)
    if o is None:
        with pytest.raises(gg.GGError):
            g.pagerank_converge()
    else:
        r, run = g.pagerank_converge()
        _close(r, o[0])
        assert 100 >= run.rounds >= int((o[2] > 1e-5).sum())


@pytest.mark.parametrize("vorder", [0, 1])
@pytest.mark.parametrize("name", CASES)
def test_batched_traversals(gg, orc, name, vorder):
    """k-column personalised PageRank, multi-source BFS and BC."""
    hg, og, pref = _case(gg, orc, name)
    g = gg.Graph(hg, partitions=_partitions(gg, hg, pref), vertex_order=vorder)
    rng = np.random.default_rng(7)
    for k in (1, 32, 64):
        seeds = rng.integers(0, hg.n, k).astype(np.uint32)
        x, run = g.ppr_k(k, iters=9, damping=0.85, seeds=seeds)
        assert run.rounds == 9
        for j in range(k):
            tele = np.zeros(hg.n)
            tele[seeds[j]] = 1.0
            _close(x[:, j], og.ppr(9, 0.85, tele))
    x0, _ = g.ppr_k(32, iters=0, seeds=np.zeros(32, np.uint32))
    assert np.all(x0[0] == 1.0) and np.all(x0[1:] == 0.0)
    src = np.array(_starts(hg) * 3, np.uint32)[:64]
    lev, run = g.msbfs(src)
    trav = 0
    for j, s in enumerate(src):
        _, olev, ost = og.bfs(int(s))
        np.testing.assert_array_equal(lev[:, j], olev, err_msg=f"msbfs source {s}")
        trav += ost.edges_traversed
    assert run.edges_traversed == trav
    dep, npth, _ = g.msbc(src)
    for j, s in enumerate(src):
        odep, onp = og.bc_brandes(int(s))
        np.testing.assert_allclose(npth[:, j], onp, rtol=1e-6)
        np.testing.assert_array_equal(np.isnan(dep[:, j]), np.isnan(odep))
        fin = np.isfinite(odep)
        np.testing.assert_allclose(dep[fin, j], odep[fin], rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("name", CASES)
def test_bp(gg, orc, name):
    hg, og, pref = _case(gg, orc, name)
    g = gg.Graph(hg, partitions=_partitions(gg, hg, pref))
    rng = np.random.default_rng(11)
    vp = rng.uniform(0.9, 1.1, (hg.n, 2)).astype(np.float32)
    ep = rng.uniform(0.45, 0.55, (max(hg.m, 1), 2, 2)).astype(np.float32)[:hg.m]
    for iters in (0, 1, 3):
        out, run = g.bp(iters, vp, ep)
        ref = og.bp(iters, vp.astype(np.float64).ravel(), ep.astype(np.float64).ravel()).reshape(hg.n, 2)
        assert run.rounds == iters
        # FP32 products over d in-edges: relative error grows about d-fold per
        # iteration, and hub products may leave FP32's range
        inside = (ref > 1e-30) & (ref < 1e30)
        np.testing.assert_allclose(out[inside], ref[inside], rtol=2e-5 if iters < 2 else 1e-2)


@pytest.mark.parametrize("normalize", [False, True])
@pytest.mark.parametrize("name", CASES)
def test_weighted_pagerank(gg, orc, name, normalize):
    """Repeated edges keep one weight each: forward and adjoint against the
    FP64 oracle (which walks the out-edges directly)."""
    hg, og, pref = _case(gg, orc, name)
    g = gg.Graph(hg, partitions=_partitions(gg, hg, pref))
    if name == "multi_sym_unsorted":
        with pytest.raises(gg.GGError) as e:
            gg.WeightedPageRank(g, 6, 0.85, 2, normalize)
        assert gg.ERRORS[e.value.code] == "FORMAT"
        return
    rng = np.random.default_rng(13)
    w = rng.uniform(0.2, 1.0, hg.m).astype(np.float32)
    tele = rng.uniform(0, 1, hg.n).astype(np.float32)
    tele /= tele.sum()
    c = rng.standard_normal(hg.n).astype(np.float32)
    for iters, every in ((0, 1), (1, 1), (6, 4)):
        wpr = gg.WeightedPageRank(g, iters, 0.85, every, normalize)
        x, _ = wpr.forward(w, tele)
        ox = og.wpr_forward(w, tele, iters, 0.85, normalize)
        _close(x, ox)
        gw, gt, g0, _ = wpr.backward(c)
        ogw, ogt, og0 = og.wpr_backward(w, tele, iters, 0.85, c, normalize)
        for a, b in ((gw, ogw), (gt, ogt), (g0, og0)):
            # exact zeros (a source whose out-edges all share one head) come out at
            # FP32 rounding of the terms, which scale with |grad_x|
            assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b) + 1e-6 * np.linalg.norm(c)
        wpr.close()


def test_graph_batch_of_edge_cases(gg, orc):
    """Every edge-case graph in one persistent batched BFS."""
    hosts, oracles = [], []
    for name in CASES:
        hg, og, _ = _case(gg, orc, name)
        hosts.append(hg)
        oracles.append(og)
    b = gg.GraphBatch(hosts)
    src = np.array([h.n - 1 for h in hosts], np.uint32)
    lev, run = b.bfs(src)
    trav = 0
    for part, og, s in zip(b.split(lev), oracles, src):
        _, olev, ost = og.bfs(int(s))
        np.testing.assert_array_equal(part, olev)
        trav += ost.edges_traversed
    assert run.edges_traversed == trav
    b.close()


@pytest.mark.parametrize("name", ["multi_dir", "multi_sym", "two_loops_dir", "edgeless5_dir", "medium_multi_dir",
                                  "medium_multi_sym"])
def test_source_partitions(gg, orc, name):
    """-P source on the same graphs, dense steps through the COO and the CSC."""
    hg, og, pref = _case(gg, orc, name)
    g = gg.Graph(hg, partitions=_partitions(gg, hg, pref, gg.PART_SOURCE), part_how=gg.PART_SOURCE)
    for policy in (0, 1, 2):
        g.set_dense_policy(policy)
        np.testing.assert_array_equal(g.components()[0], og.cc()[0])
        for s in _starts(hg)[:3]:
            np.testing.assert_array_equal(g.bfs(s)[1], og.bfs(s)[1])
            np.testing.assert_array_equal(g.bellman_ford(s)[0], og.bellman_ford(s)[0])
        o = _oracle_or_none(og.pagerank, 10)
        if o is None:
            with pytest.raises(gg.GGError):
                g.pagerank(10)
        else:
            _close(g.pagerank(10)[0], o[0])
        _close(g.spmv()[0], og.spmv()[0], rel=1e-6, mx=1e-6)


@pytest.mark.parametrize("kernel", [0, 1, 2, 3, 4, 5, 6, 7])
def test_coo_kernels_on_multigraph(gg, orc, kernel):
    """Every COO pull kernel on repeated edges and loops (coo_window builds
    give kernel 4 its lane-contiguous layout)."""
    hg, og, _ = _case(gg, orc, "medium_multi_dir")
    for window in (0, 512):
        g = gg.Graph(hg, partitions=_partitions(gg, hg, 16), coo_window=window)
        g.set_dense_policy(2)
        g.set_tuning(gg.TUNE_COO_KERNEL, kernel)
        _close(g.pagerank(10, True)[0], og.pagerank(10, True)[0])
        _close(g.spmv()[0], og.spmv()[0], rel=1e-6, mx=1e-6)
        np.testing.assert_array_equal(g.components()[0], og.cc()[0])
