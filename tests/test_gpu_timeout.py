"""A bounded device wait driven to expiry on a healthy graph.

The device BFS loops (GG_TUNE_DEVICE_LOOP 1: consecutive sparse levels, 2:
every level) end every level at a grid barrier whose wait is bounded.  With the budget set to 0 probes
(GG_TUNE_LOOP_WAIT_BUDGET, a test knob), every CTA that arrives before the
last one gives up at once: all CTAs return (the one that passed stops at the
next barrier), nothing waits on anything that will not come, the kernel
records the timeout and gg_bfs returns GG_ERR_TIMEOUT.  The same graph
handle then gives the oracle's levels again once the budget is restored."""
import numpy as np
import pytest

from conftest import ok_partitions

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("loop", [1, 2])
@pytest.mark.parametrize("sym", [True, False])
def test_loop_barrier_timeout_then_recovery(gg, orc, sym, loop):
    hg = gg.HostGraph.rmat(14, 16, seed=3, symmetric=sym)
    g = gg.Graph(hg, partitions=ok_partitions(hg, 16))
    og = orc.Graph.from_host(hg)
    _, olev, _ = og.bfs(100)
    assert g.get_tuning(gg.TUNE_DEVICE_LOOP) == 2
    g.set_tuning(gg.TUNE_DEVICE_LOOP, loop)
    assert g.get_tuning(gg.TUNE_LOOP_WAIT_BUDGET) == 1 << 22
    g.set_tuning(gg.TUNE_LOOP_WAIT_BUDGET, 0)
    for _ in range(2):
        with pytest.raises(gg.GGError) as e:
            g.bfs(100)
        assert e.value.code == gg.ERR_TIMEOUT
        assert "grid barrier" in str(e.value)
    g.set_tuning(gg.TUNE_LOOP_WAIT_BUDGET, 1 << 22)
    _, lev, _ = g.bfs(100)
    np.testing.assert_array_equal(lev, olev)
    ids, _ = g.components()
    oids, _ = og.cc()
    np.testing.assert_array_equal(ids, oids)
    with pytest.raises(gg.GGError):
        g.set_tuning(gg.TUNE_LOOP_WAIT_BUDGET, -1)
    g.close()
