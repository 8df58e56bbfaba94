"""The small plain-method configuration at full size, against the reference
itself: RMAT scale 18, edge factor 16, (a,b,c,d) = (.57,.19,.19,.05), seed 1,
symmetrised, self-loops and duplicates removed, 64 edge-balanced Hilbert COO
partitions, BFS from vertex 100 and PageRank (10 iterations).  The reference's
own build (oracle/_ref, compiled from its sources) is run on the same file:
the oracle must reproduce it (CPU), and the device must match it (GPU): BFS
levels bit-exact, PageRank FP32 against the reference's FP64 within relative
L1 1e-5 and max-abs 1e-6.  Skipped where the reference binaries were not
built."""
import os
import tempfile

import numpy as np
import pytest

from conftest import PR_MAX_ABS, PR_REL_L1, rel_l1

FLAGS = ["-s", "-c", "64"]
START = 100


@pytest.fixture(scope="module")
def c1(gg, orc):
    if not (orc.ref_available("BFS") and orc.ref_available("PR")):
        pytest.skip("reference binaries (oracle/_ref) not built")
    hg = gg.HostGraph.rmat(18, 16, 0.57, 0.19, 0.19, seed=1, symmetric=True)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "rmat18.adj")
        hg.write_adj(path)
        rc, bfs, err = orc.run_ref("BFS", "dump", path, os.path.join(d, "b.bin"), [*FLAGS, "-r", str(START)])
        assert rc == 0, err[-400:]
        rc, pr, err = orc.run_ref("PR", "dump", path, os.path.join(d, "p.bin"), [*FLAGS, "-r", str(START)])
        assert rc == 0, err[-400:]
    return hg, bfs, pr


def test_oracle_reproduces_reference(orc, c1):
    hg, bfs, pr = c1
    assert hg.n == 1 << 18 and 7_000_000 < hg.m < 8_000_000
    og = orc.Graph.from_host(hg)
    np.testing.assert_array_equal(og.bfs(START)[1], bfs["levels"])
    r, _ = og.pagerank(10)
    assert rel_l1(r, pr["ranks"]) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("vorder", [0, 1])
def test_device_matches_reference(gg, c1, vorder):
    hg, bfs, pr = c1
    g = gg.Graph(hg, partitions=64, vertex_order=vorder)
    _, lev, _ = g.bfs(START)
    np.testing.assert_array_equal(lev, bfs["levels"])
    r, _ = g.pagerank(10)
    assert rel_l1(r, pr["ranks"]) <= PR_REL_L1
    assert np.abs(r.astype(np.float64) - pr["ranks"]).max() <= PR_MAX_ABS
