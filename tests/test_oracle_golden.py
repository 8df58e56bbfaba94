"""The oracle (C restatement) against golden vectors produced by the reference
itself (tests/golden/make_golden.py).  CPU only."""
import numpy as np
import pytest

from conftest import golden_flags, golden_names, load_golden, rel_l1

NAMES = golden_names()


def _og(orc, gd):
    w = gd.get("weights")
    fl = golden_flags(gd)
    return orc.Graph(gd["offsets"], gd["indices"], None if w is None else w.astype(np.float64),
                     symmetric=bool(gd["symmetric"]), part_vertex="vertex" in fl)


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference(orc, name):
    gd = load_golden(name)
    og = _og(orc, gd)
    start = int(gd["start"])
    checked = 0
    if "BFS_levels" in gd:
        _, lev, _ = og.bfs(start)
        np.testing.assert_array_equal(lev, gd["BFS_levels"])
        checked += 1
    if "CC_ids" in gd:
        ids, _ = og.cc()
        np.testing.assert_array_equal(ids, gd["CC_ids"])
        checked += 1
    for app, bit in (("PR", False), ("PRBIT", True)):
        if f"{app}_ranks" in gd:
            r, _ = og.pagerank(10, bit)
            assert rel_l1(r, gd[f"{app}_ranks"]) < 1e-12
            checked += 1
        if f"{app}_error" in gd:  # the reference aborts: the oracle reports failure
            with pytest.raises(AssertionError):
                og.pagerank(10, bit)
            checked += 1
    if "PRD_ranks" in gd:
        r, _ = og.pagerank_delta()
        assert rel_l1(r, gd["PRD_ranks"]) < 1e-12
        checked += 1
    if "PRC_ranks" in gd:  # app/PageRankConverage.C: same iterations, same L1 trajectory
        r, it, l1 = og.pagerank_converge()
        assert it == len(gd["PRC_l1"])
        np.testing.assert_allclose(l1, gd["PRC_l1"], rtol=1e-10, atol=1e-13)  # sums of tiny differences
        assert rel_l1(r, gd["PRC_ranks"]) < 1e-12
        checked += 1
    if "BC_num_paths" in gd:
        dep, npth, _ = og.bc(start)
        np.testing.assert_allclose(npth, gd["BC_num_paths"], rtol=1e-6)
        ref = gd["BC_dependencies"]  # reference computes in float
        np.testing.assert_array_equal(np.isnan(dep), np.isnan(ref))
        fin = np.isfinite(ref)
        assert rel_l1(dep[fin], ref[fin]) < 1e-5
        checked += 1
    if "SPMV_y" in gd:
        y, _ = og.spmv()
        assert rel_l1(y, gd["SPMV_y"]) < 1e-12
        checked += 1
    if "BF_dist" in gd:
        d, _ = og.bellman_ford(start)
        np.testing.assert_array_equal(d, gd["BF_dist"])
        checked += 1
    assert checked > 0


@pytest.mark.parametrize("name", ["sixnode", "rmat10_sym", "rmat10_dir", "path8", "star9"])
def test_oracle_bfs_trace_matches_reference(orc, name):
    """Per-level frontier sizes and out-degree sums (d_m, num_out_edges) of
    BFS are deterministic and must match the reference's edgeMap outputs."""
    gd = load_golden(name)
    og = _og(orc, gd)
    tr = gd["BFS_trace"].reshape(-1, 3)
    _, lev, st = og.bfs(int(gd["start"]))
    assert st.rounds == len(tr)
    for r, (dense, dm, oe) in enumerate(tr, start=1):
        members = np.nonzero(lev == r)[0]
        assert len(members) == dm
        assert int(np.diff(og.out_off.astype(np.int64))[members].sum()) == oe


def test_partition_sizes_match_reference(gg, orc):
    import os
    from conftest import GOLDEN
    z = np.load(os.path.join(GOLDEN, "partitions.npz"))
    off = z["offsets"].astype(np.int64)
    n = len(off) - 1
    deg = np.diff(off).astype(np.uint32)  # symmetric: in == out
    m = int(off[-1])
    n_cases = 0
    for P in (1, 2, 8, 64, 200, 384):
        for mode in ("edge", "vertex", "relabel"):
            key = f"P{P}_{mode}"
            bal = 1 if mode == "vertex" else 0
            rel = mode == "relabel"
            rc, coo, csc = orc.partition_sizes(deg, deg, m, P, bal, 0, rel)
            if int(z[key + "_rc"]) != 0:
                assert rc != 0, key
                with pytest.raises(gg.GGError):
                    gg.partition_sizes(deg, deg, m, P, bal, 0, rel)
            else:
                assert rc == 0, key
                np.testing.assert_array_equal(coo, z[key + "_coo"], err_msg=key)
                np.testing.assert_array_equal(csc, z[key + "_csc"], err_msg=key)
                pc, ps = gg.partition_sizes(deg, deg, m, P, bal, 0, rel)
                np.testing.assert_array_equal(pc, z[key + "_coo"], err_msg=key)
                np.testing.assert_array_equal(ps, z[key + "_csc"], err_msg=key)
            n_cases += 1
    assert n_cases == 18 and n > 0


@pytest.mark.parametrize("name", ["sixnode", "rmat10_sym", "rmat10_dir", "star9", "twocomp10"])
def test_hilbert_key_orders_reference_coo(gg, orc, name):
    """The reference's Hilbert-sorted COO partitions (std::sort with
    HilbertEdgeSort) are non-decreasing under our key with the same grid side
    (roundUpPow2 of the partition's edge count), and hold exactly the edges
    whose destination lies in the partition."""
    gd = load_golden(name)
    src, dst, bounds = gd["parts_coo_src"], gd["parts_coo_dst"], gd["parts_coo_bounds"]
    starts = np.concatenate([[0], np.cumsum(gd["parts_coo_sizes"])])
    dst_all = np.asarray(gd["indices"], np.int64)
    for p in range(len(bounds) - 1):
        s, d = src[bounds[p]:bounds[p + 1]], dst[bounds[p]:bounds[p + 1]]
        ne = len(s)
        keys = [gg.hilbert_key(ne, int(x), int(y)) for x, y in zip(s, d)]
        okeys = [orc.hilbert_key(ne, int(x), int(y)) for x, y in zip(s, d)]
        assert keys == okeys
        assert all(a <= b for a, b in zip(keys, keys[1:])), f"partition {p} not ordered"
        assert np.all((d >= starts[p]) & (d < starts[p + 1]))
        assert ne == int(((dst_all >= starts[p]) & (dst_all < starts[p + 1])).sum())


def test_source_partitions_match_reference(gg, orc):
    """-P source on a directed graph: partition sizes balance out-degrees (COO)
    and the destinations' out-degrees (compressed CSC), and each COO partition
    holds the out-edges of its source range in Hilbert order."""
    import os
    from conftest import GOLDEN
    z = np.load(os.path.join(GOLDEN, "partitions_src.npz"))
    off = z["offsets"].astype(np.int64)
    idx = z["indices"].astype(np.int64)
    n, m = len(off) - 1, int(off[-1])
    outd = np.diff(off).astype(np.uint32)
    ind = np.bincount(idx, minlength=n).astype(np.uint32)
    for P in (1, 2, 8, 64):
        for how, code in (("source", 1), ("dest", 0)):
            key = f"P{P}_{how}"
            if int(z[key + "_rc"]):
                with pytest.raises(gg.GGError):
                    gg.partition_sizes(ind, outd, m, P, 0, code, False)
                continue
            pc, ps = gg.partition_sizes(ind, outd, m, P, 0, code, False)
            np.testing.assert_array_equal(pc, z[key + "_coo"], err_msg=key)
            np.testing.assert_array_equal(ps, z[key + "_csc"], err_msg=key)
            rc, oc, os_ = orc.partition_sizes(ind, outd, m, P, 0, code, False)
            assert rc == 0
            np.testing.assert_array_equal(oc, z[key + "_coo"], err_msg=key)
    src, dst, bounds = z["P8_source_coo_src"], z["P8_source_coo_dst"], z["P8_source_coo_bounds"]
    starts = np.concatenate([[0], np.cumsum(z["P8_source_coo"])])
    for p in range(len(bounds) - 1):
        s, d = src[bounds[p]:bounds[p + 1]], dst[bounds[p]:bounds[p + 1]]
        keys = [gg.hilbert_key(len(s), int(x), int(y)) for x, y in zip(s, d)]
        assert all(a <= b for a, b in zip(keys, keys[1:])), f"partition {p} not ordered"
        assert np.all((s >= starts[p]) & (s < starts[p + 1]))
        assert len(s) == int(off[starts[p + 1]] - off[starts[p]])
