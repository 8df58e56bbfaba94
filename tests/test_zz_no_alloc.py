"""gg_bfs_push_step_noalloc: the BFS push step for callers that cannot let
the library allocate device memory (their program owns every device buffer,
or cudaMalloc/cudaFree would stall a latency-critical loop).  Its result must
match the regular push path (gg_edge_map with GG_F_BFS, forced sparse) over
two BFS levels in a row; the second call also checks that the shared scratch
array left behind by the first call does not leak into the next one.

This file is collected last so that a run stopping at its first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

from conftest import ok_partitions

pytestmark = pytest.mark.gpu


def _ptr(dev_array):
    return C.c_void_p(dev_array.ptr.value)


def test_noalloc_push_matches_edge_map_over_two_levels(gg, orc):
    hg = gg.HostGraph.rmat(14, 16, seed=71, symmetric=True)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16))
    n = hg.n
    start = 5
    deg = hg.degrees().astype(np.int64)
    off_d, idx_d = C.c_void_p(), C.c_void_p()
    gg.check(gg.lib.gg_graph_device_arrays(g.h, C.byref(off_d), C.byref(idx_d), None, None),
             "gg_graph_device_arrays")

    init_p = np.full(n, -1, np.int32)
    init_p[start] = start
    init_l = np.full(n, -1, np.int32)
    init_l[start] = 0
    # regular path: frontier handles through gg_edge_map, push forced
    par_a = gg.DeviceArray(g, np.int32, init_p)
    lev_a = gg.DeviceArray(g, np.int32, init_l)
    # allocation-free path: caller-owned queues, counters and BFS state
    par_b = gg.DeviceArray(g, np.int32, init_p)
    lev_b = gg.DeviceArray(g, np.int32, init_l)
    q_in = gg.DeviceArray(g, np.uint32, 0)
    q_out = gg.DeviceArray(g, np.uint32, 0)
    counts = gg.DeviceArray(g, np.uint64, 0)
    q = np.zeros(n, np.uint32)
    q[0] = start
    q_in.upload(q)
    frontier_len = 1

    F = g.frontier_single(start)
    _, olev, _ = orc.Graph.from_host(hg).bfs(start)
    for rnd in (1, 2):
        F = g.edge_map(F, gg.F_BFS, gg.BfsArgs(par_a.ptr, lev_a.ptr, rnd), -1, gg.EM_FORCE_SPARSE)
        assert g.last_edge_map_stats().kind == 1
        gg.check(gg.lib.gg_bfs_push_step_noalloc(off_d, idx_d, n, _ptr(q_in), frontier_len, _ptr(par_b),
                                                  _ptr(lev_b), rnd, _ptr(q_out), _ptr(counts), None),
                 "gg_bfs_push_step_noalloc")
        cnt = counts.download()[:2]
        qo = q_out.download()[: int(cnt[0])]
        mask = F.mask()
        # same output frontier (as a set), same size and out-degree sum
        assert int(cnt[0]) == F.stats()[0] and int(cnt[1]) == F.stats()[1]
        assert len(np.unique(qo)) == len(qo)
        np.testing.assert_array_equal(np.sort(qo), np.nonzero(mask)[0].astype(np.uint32))
        # same levels (exact); parents valid (the CAS winner may differ)
        lb = lev_b.download()
        np.testing.assert_array_equal(lb, lev_a.download())
        np.testing.assert_array_equal(lb[lb >= 0], olev[lb >= 0])
        pb = par_b.download()
        off = hg.offsets.astype(np.int64)
        for v in qo[:2000]:
            p = pb[v]
            assert lb[p] == rnd - 1 and v in hg.indices[off[p]:off[p + 1]]
        assert int(cnt[1]) == int(deg[qo].sum())
        # next level input
        q_in.upload(np.concatenate([qo, np.zeros(n - len(qo), np.uint32)]))
        frontier_len = int(cnt[0])


def test_noalloc_rejects_oversized_inputs(gg):
    nil = C.c_void_p(16)  # never dereferenced: the size checks run first
    rc = gg.lib.gg_bfs_push_step_noalloc(nil, nil, (1 << 24) + 1, nil, 1, nil, nil, 1, nil, nil, None)
    assert rc == -10 and "GG_NOALLOC_MAX_VERTICES" in gg.lib.gg_last_error_string().decode()
    rc = gg.lib.gg_bfs_push_step_noalloc(nil, nil, 1 << 24, nil, (1 << 19) + 1, nil, nil, 1, nil, nil, None)
    assert rc == -10 and "GG_NOALLOC_MAX_FRONTIER" in gg.lib.gg_last_error_string().decode()
