"""The partitioned COO as the device built it, downloaded through
gg_graph_coo_layout, against the reference's own partitions.

For the golden graphs the reference harness dumped every COO partition after
COOPartitionByDest + hilbert_sort (graphgrind/graph-numa.h:482-490,
1116-1143).  The device cuts each partition into CTA tiles of destination
ranges; the checks:
  * the tiles of partition p hold exactly the reference partition's edges
    (same multiset of (src, dst));
  * tiles cover disjoint destination ranges inside their partition, every
    slot's destination lies in its tile, and padding only ends a tile;
  * inside a tile the Hilbert key (the partition's grid side,
    roundUpPow2(edges of the partition)) never decreases from one 256-slot
    window to the next, and destinations never decrease inside a window;
  * with ORDER_CSR the same holds for the (src, dst) key of CSRDestSort
    (:338-350).
"""
import numpy as np
import pytest

from conftest import golden_partitions, host_graph_from_golden, load_golden

pytestmark = pytest.mark.gpu

PAD = 0xFFFFFFFF
WINDOW = 256


def _check_layout(gg, g, hg, order_key, ref=None):
    tiles, src, dst = g.coo_layout()
    starts = g.partition_starts()
    P = len(starts) - 1
    part_of = np.searchsorted(starts, tiles[:, 0], side="right") - 1
    by_part = {p: [] for p in range(P)}
    covered = np.zeros(hg.n, np.int32)
    for t, (v0, nv, e0, ne) in enumerate(tiles.astype(np.int64)):
        p = int(part_of[t])
        assert starts[p] <= v0 and v0 + nv <= starts[p + 1]
        covered[v0:v0 + nv] += 1
        s, d = src[e0:e0 + ne].astype(np.int64), dst[e0:e0 + ne].astype(np.int64)
        real = s != PAD
        k = int(real.sum())
        assert real[:k].all() and not real[k:].any() and ne - k < 8, f"tile {t}: padding inside"
        s, d = s[:k], d[:k]
        assert np.all((d >= v0) & (d < v0 + nv)), f"tile {t}: destination outside the tile"
        side = hg.offsets_in_range(starts[p], starts[p + 1])  # the partition's edge count
        keys = np.array([order_key(side, int(x), int(y)) for x, y in zip(s, d)], dtype=object)
        for w in range(0, k, WINDOW):
            kw, dw = keys[w:w + WINDOW], d[w:w + WINDOW]
            assert np.all(dw[1:] >= dw[:-1]), f"tile {t} window {w // WINDOW}: destinations out of order"
            if w + WINDOW < k:
                assert max(kw) <= min(keys[w + WINDOW:w + 2 * WINDOW]), f"tile {t}: windows out of key order"
        by_part[p].append(np.stack([s, d], 1))
    assert covered.max() <= 1
    if ref is not None:
        rsrc, rdst, bounds = ref
        for p in range(P):
            mine = np.concatenate(by_part[p]) if by_part[p] else np.zeros((0, 2), np.int64)
            theirs = np.stack([rsrc[bounds[p]:bounds[p + 1]], rdst[bounds[p]:bounds[p + 1]]], 1).astype(np.int64)
            assert len(mine) == len(theirs), f"partition {p}: {len(mine)} edges, reference {len(theirs)}"
            a = mine[np.lexsort((mine[:, 1], mine[:, 0]))]
            b = theirs[np.lexsort((theirs[:, 1], theirs[:, 0]))]
            np.testing.assert_array_equal(a, b, err_msg=f"partition {p}")
    return tiles


class _Host:
    """In-edge counts per destination range of a host graph (the Hilbert grid
    side of a partition is roundUpPow2 of its edge count)."""

    def __init__(self, hg):
        self.n = hg.n
        ind = np.bincount(hg.indices.astype(np.int64), minlength=hg.n)
        self.cum = np.concatenate([[0], np.cumsum(ind)])

    def offsets_in_range(self, a, b):
        return int(self.cum[b] - self.cum[a])


@pytest.mark.parametrize("name", ["sixnode", "rmat10_sym", "rmat10_dir", "star9", "twocomp10"])
@pytest.mark.parametrize("tile_edges", [0, 300])
def test_device_coo_matches_reference_partitions(gg, name, tile_edges):
    gd = load_golden(name)
    hg = host_graph_from_golden(gd)
    g = gg.Graph(hg, partitions=golden_partitions(gd), tile_edges=tile_edges)
    ref = (gd["parts_coo_src"], gd["parts_coo_dst"], gd["parts_coo_bounds"])
    tiles = _check_layout(gg, g, _Host(hg), gg.hilbert_key, ref)
    if tile_edges:
        assert len(tiles) >= len(g.partition_starts()) - 1
    g.close()


@pytest.mark.parametrize("sym", [True, False])
def test_device_coo_orders_on_rmat(gg, sym):
    hg = gg.HostGraph.rmat(13, 16, seed=17, symmetric=sym)
    h = _Host(hg)
    for order, key in ((gg.ORDER_HILBERT, gg.hilbert_key), (gg.ORDER_CSR, lambda side, x, y: (x << 32) | y)):
        g = gg.Graph(hg, partitions=32, order=order, tile_edges=2048)
        tiles = _check_layout(gg, g, h, key)
        assert len(tiles) > 32
        g.close()


@pytest.mark.parametrize("order", ["hilbert", "csr"])
@pytest.mark.parametrize("ctv", [8192, 16384])
def test_wide_coo_tiles(gg, orc, order, ctv):
    """COO tiles wider than the CSC tiles (coo_tile_vertices up to 16384):
    the layout keeps its guarantees and every dense-COO application gives
    the oracle's results."""
    from conftest import PR_MAX_ABS, PR_REL_L1, rel_l1
    hg = gg.HostGraph.rmat(16, 16, seed=23, symmetric=False).add_weights(gg.W_FLOAT32, seed=4)
    o = gg.ORDER_HILBERT if order == "hilbert" else gg.ORDER_CSR
    key = gg.hilbert_key if order == "hilbert" else (lambda side, x, y: (x << 32) | y)
    g = gg.Graph(hg, partitions=8, order=o, tile_edges=1 << 20, coo_tile_vertices=ctv)
    tiles = _check_layout(gg, g, _Host(hg), key)
    assert int(tiles[:, 1].max()) > 4096
    g.set_dense_policy(2)  # every dense step on the COO
    og = orc.Graph.from_host(hg)
    _, lev, _ = g.bfs(7)
    np.testing.assert_array_equal(lev, og.bfs(7)[1])
    r, _ = g.pagerank(10)
    o_r, _ = og.pagerank(10)
    assert rel_l1(r, o_r) <= PR_REL_L1 and np.abs(r - o_r).max() <= PR_MAX_ABS
    ids, _ = g.components()
    np.testing.assert_array_equal(ids, og.cc()[0])
    y, _ = g.spmv()
    oy, _ = og.spmv()
    assert rel_l1(y, oy) <= 1e-6
    g.close()
