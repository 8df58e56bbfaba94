"""VEBO reordering (gg_vebo) against the reference's own VEBO tool
(graphtools/VEBO.C, fixtures in tests/golden/vebo.npz made by make_golden.py)."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "vebo.npz")
CASES = ["rmat10_P8", "rmat10_P3", "rmat12_P64", "rmat11sym_P16"]


@pytest.mark.parametrize("name", CASES)
def test_vebo_matches_reference_tool(gg, name):
    gd = np.load(GOLD)
    hg = gg.HostGraph.from_csr(gd[f"{name}_in_offsets"].astype(np.uint32), gd[f"{name}_in_indices"].astype(np.uint32),
                               symmetric=bool(gd[f"{name}_sym"]))
    P = int(gd[f"{name}_P"])
    out, new_of_old, sizes = hg.vebo(P)
    np.testing.assert_array_equal(out.offsets.astype(np.int64), gd[f"{name}_offsets"])
    np.testing.assert_array_equal(out.indices.astype(np.int64), gd[f"{name}_indices"])
    # a permutation; new vertex i carries old vertex's out-edges, renamed, in order
    assert np.array_equal(np.sort(new_of_old), np.arange(hg.n))
    assert sizes.sum() == hg.n
    old_of_new = np.argsort(new_of_old)
    for i in (0, 1, hg.n // 2, hg.n - 1):
        o = old_of_new[i]
        old_nb = hg.indices[hg.offsets[o]:hg.offsets[o + 1]]
        np.testing.assert_array_equal(out.indices[out.offsets[i]:out.offsets[i + 1]], new_of_old[old_nb])


def test_vebo_balances_edges_and_carries_weights(gg):
    hg = gg.HostGraph.rmat(13, 16, seed=3, symmetric=False).add_weights(gg.W_INT32, seed=5, lo=1, hi=100)
    out, new_of_old, sizes = hg.vebo(32)
    indeg = np.bincount(out.indices, minlength=out.n)
    starts = np.concatenate([[0], np.cumsum(sizes)])
    per_part = np.array([indeg[starts[p]:starts[p + 1]].sum() for p in range(32)])
    assert per_part.max() - per_part.min() <= indeg.max()  # greedy balance within one vertex's degree
    old_of_new = np.argsort(new_of_old)
    src_old = np.repeat(np.arange(hg.n), np.diff(hg.offsets.astype(np.int64)))
    src_new = np.repeat(np.arange(out.n), np.diff(out.offsets.astype(np.int64)))
    key_old = {(int(new_of_old[s]), int(new_of_old[d])): int(w)
               for s, d, w in zip(src_old[:2000], hg.indices[:2000], hg.weights[:2000])}
    for s, d, w in zip(src_new, out.indices, out.weights):
        if (int(s), int(d)) in key_old:
            assert key_old[(int(s), int(d))] == int(w)
    assert np.array_equal(np.sort(old_of_new[src_new]), np.sort(src_old))


def test_vebo_rejects_bad_arguments(gg):
    hg = gg.HostGraph.rmat(6, 4, seed=1)
    with pytest.raises(gg.GGError):
        hg.vebo(0)
