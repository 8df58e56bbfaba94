"""Host-side library checks that need no GPU: the C ABI loads and exports
every declared symbol, generators are deterministic and clean, the
reference's file formats round-trip, device calls fail cleanly without a GPU."""
import os
import re
import tempfile

import numpy as np
import pytest

from conftest import ROOT


def _declared_symbols():
    src = open(os.path.join(ROOT, "include", "gg.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gg_[a-z0-9_]+)\s*\(", src)))


def test_exports_every_declared_symbol(gg):
    declared = _declared_symbols()
    assert len(declared) >= 40
    for name in declared:
        assert hasattr(gg.lib, name), f"libgg.so does not export {name}"
    assert set(declared) == set(gg.EXPORTED)


def test_version_and_error_string(gg):
    assert "sm_100a" in gg.version()
    with pytest.raises(gg.GGError) as e:
        gg.HostGraph.rmat(0)
    assert "INVALID_ARG" in str(e.value)


@pytest.mark.parametrize("sym", [True, False])
def test_rmat_deterministic_and_clean(gg, sym):
    a = gg.HostGraph.rmat(12, 8, seed=5, symmetric=sym)
    b = gg.HostGraph.rmat(12, 8, seed=5, symmetric=sym)
    c = gg.HostGraph.rmat(12, 8, seed=6, symmetric=sym)
    np.testing.assert_array_equal(a.offsets, b.offsets)
    np.testing.assert_array_equal(a.indices, b.indices)
    assert not np.array_equal(a.indices[:1000], c.indices[:1000])
    off = a.offsets.astype(np.int64)
    src = np.repeat(np.arange(a.n), np.diff(off))
    dst = a.indices.astype(np.int64)
    assert np.all(src != dst), "self loops"
    key = src * a.n + dst
    assert len(np.unique(key)) == len(key), "duplicates"
    for v in range(a.n):  # sorted rows
        row = dst[off[v]:off[v + 1]]
        assert np.all(row[1:] > row[:-1])
    if sym:
        rkey = dst * a.n + src
        assert np.array_equal(np.sort(key), np.sort(rkey))


def test_rmat_skew(gg):
    """a=0.57: low ids are the hubs; edge factor and scale give n = 2^scale."""
    g = gg.HostGraph.rmat(14, 16, seed=1, symmetric=False)
    assert g.n == 1 << 14
    assert 0.8 * 16 * g.n < g.m <= 16 * g.n  # duplicates of hub edges are removed
    deg = np.diff(g.transpose().offsets.astype(np.int64))
    assert deg[:64].mean() > 20 * deg[-4096:].mean()


def test_grid_and_er(gg):
    g = gg.HostGraph.grid(64, 0.001, seed=3)
    assert g.n == 64 * 64 and g.symmetric
    deg = g.degrees()
    assert deg.min() >= 2 and deg.max() <= 6
    e = gg.HostGraph.er(1 << 12, 1 << 15, seed=4)
    assert e.n == 4096 and 0.99 * (1 << 15) < e.m <= (1 << 15)


@pytest.mark.parametrize("binary", [False, True])
@pytest.mark.parametrize("sym", [True, False])
def test_file_round_trip(gg, binary, sym):
    g = gg.HostGraph.rmat(9, 8, seed=2, symmetric=sym).add_weights(gg.W_INT32, seed=1, lo=1, hi=100)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "g.gr" if binary else "g.adj")
        (g.write_gr if binary else g.write_adj)(p)
        if not sym:
            assert os.path.exists(p + "_t"), "transpose file for directed graphs"
            t = gg.HostGraph.read(p + "_t", binary=binary, symmetric=False, weighted=True)
            gt = g.transpose()
            np.testing.assert_array_equal(t.offsets, gt.offsets)
            np.testing.assert_array_equal(t.indices, gt.indices)
        h = gg.HostGraph.read(p, binary=binary, symmetric=sym, weighted=True)
        np.testing.assert_array_equal(h.offsets, g.offsets)
        np.testing.assert_array_equal(h.indices, g.indices)
        np.testing.assert_array_equal(h.weights, g.weights)


def test_reader_rejects_bad_files(gg):
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "bad.adj")
        open(p, "w").write("AdjacencyGraph\n3\n2\n0\n1\n")  # truncated
        with pytest.raises(gg.GGError) as e:
            gg.HostGraph.read(p)
        assert "FORMAT" in str(e.value)
        open(p, "w").write("NotAGraph\n1\n0\n0\n")
        with pytest.raises(gg.GGError):
            gg.HostGraph.read(p)
        q = os.path.join(d, "bad.gr")
        open(q, "wb").write(np.array([2, 0, 4, 4], np.uint64).tobytes())  # version 2
        with pytest.raises(gg.GGError):
            gg.HostGraph.read(q, binary=True)
        with pytest.raises(gg.GGError) as e:
            gg.HostGraph.read(os.path.join(d, "missing.adj"))
        assert "IO" in str(e.value)


def test_weights_are_per_undirected_edge(gg):
    g = gg.HostGraph.rmat(9, 8, seed=4, symmetric=True).add_weights(gg.W_FLOAT32, seed=2)
    w = g.weights
    assert w.dtype == np.float32 and np.all(w > 0) and np.all(w <= 1)
    off = g.offsets.astype(np.int64)
    lookup = {}
    for u in range(g.n):
        for j in range(off[u], off[u + 1]):
            lookup[(u, int(g.indices[j]))] = w[j]
    for (u, v), x in list(lookup.items())[:2000]:
        assert lookup[(v, u)] == x


def test_hilbert_key_matches_oracle(gg, orc):
    rng = np.random.default_rng(0)
    for _ in range(2000):
        ne = int(rng.integers(0, 1 << 20))
        x, y = (int(v) for v in rng.integers(0, 1 << 24, 2))
        assert gg.hilbert_key(ne, x, y) == orc.hilbert_key(ne, x, y)
    # on a full 8x8 grid the key is a bijection onto 0..63
    keys = sorted(gg.hilbert_key(64, x, y) for x in range(8) for y in range(8))
    assert keys == list(range(64))


def _no_gpu():
    try:
        import torch
        return not torch.cuda.is_available()
    except Exception:
        return True


@pytest.mark.skipif(not _no_gpu(), reason="a GPU is present")
def test_device_calls_fail_cleanly_without_gpu(gg):
    g = gg.HostGraph.rmat(6, 4, seed=1)
    with pytest.raises(gg.GGError) as e:
        gg.Graph(g, partitions=2)
    assert "NO_DEVICE" in str(e.value)
    with pytest.raises(gg.GGError) as e:
        gg.GraphBatch([g, g])
    assert "NO_DEVICE" in str(e.value)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "g.adj")
        g.write_adj(p)
        with pytest.raises(gg.GGError) as e:
            gg.HostGraph.read_gpu(p)
        assert "NO_DEVICE" in str(e.value)


@pytest.mark.parametrize("sym", [True, False])
@pytest.mark.parametrize("P,balance,part_how", [(16, 0, 0), (7, 1, 0), (16, 0, 1), (1, 0, 0)])
def test_hot_first_order(gg, sym, P, balance, part_how):
    """gg_hot_first_order: the reference's COO partitions keep their vertex
    sets, and inside each the vertices go by descending out-degree, ties by id."""
    hg = gg.HostGraph.rmat(11, 8, seed=21, symmetric=sym)
    outd = hg.degrees()
    ind = outd if sym else hg.transpose().degrees()
    coo, _ = gg.partition_sizes(ind, outd, hg.m, P, balance, part_how, False)
    nofo, starts = hg.hot_first_order(P, balance, part_how)
    np.testing.assert_array_equal(starts, np.concatenate([[0], np.cumsum(coo)]))
    oofn = np.empty(hg.n, np.int64)
    oofn[nofo] = np.arange(hg.n)
    assert sorted(nofo.tolist()) == list(range(hg.n))
    for p in range(P):
        a, b = int(starts[p]), int(starts[p + 1])
        ids = np.arange(a, b)
        want = ids[np.lexsort((ids, -outd[a:b].astype(np.int64)))]
        np.testing.assert_array_equal(oofn[a:b], want, err_msg=f"partition {p}")
