"""Failure detection without a GPU fault: the query kernel's waits are
bounded, both the grid barrier (barrier schedule) and the completion-counter
waits (dataflow schedule).  A launch whose wait can never be satisfied gives
up after its poll limit, records the timeout in its status word, every CTA
returns, and the context stays usable (a query on it is still exact)."""
import numpy as np
import pytest

from helpers import make_grid, viewpoints

pytestmark = pytest.mark.gpu


def test_barrier_wait_runs_out_and_context_survives(gpu):
    from htrip_b200.minplus_oracle import HierarchyConfig, MinPlusOracle, selftest_barrier_timeout
    from oracle.ref import port_bfs
    status, returned, ms = selftest_barrier_timeout(0)
    assert status == 1          # the timeout was recorded
    assert returned == 4        # every CTA came back
    assert ms < 2000.0          # bounded: the waits ended on their own
    grid = make_grid("rooms", 32, 32, 3)
    dev = MinPlusOracle(HierarchyConfig(8, 2, 2))
    assert dev.build(grid)
    vps = viewpoints(grid, 12, 3)
    np.testing.assert_array_equal(dev.queryAllPairs(vps, grid), port_bfs(grid, vps))


def test_counter_wait_runs_out_and_context_survives(gpu):
    from htrip_b200.minplus_oracle import HierarchyConfig, MinPlusOracle, selftest_wait_timeout
    from oracle.ref import port_bfs
    status, returned, ms = selftest_wait_timeout(0)
    assert status == 1
    assert returned == 4
    assert ms < 2000.0
    grid = make_grid("street", 32, 32, 4)
    dev = MinPlusOracle(HierarchyConfig(8, 2, 2))
    assert dev.build(grid)
    vps = viewpoints(grid, 12, 4)
    np.testing.assert_array_equal(dev.queryAllPairs(vps, grid), port_bfs(grid, vps))
