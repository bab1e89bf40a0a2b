"""queryAllPairsIncremental's selective re-lift (tolerance 0: integer distances).

With the same viewpoints and only openings since the last call, the state's
own query arena still holds the last launch's port vectors, projections and
pair matrix; only the viewpoints whose leaf-to-root chain holds a matrix an
opening listed are re-lifted, and only their pairs recomputed (the
reference's version-stamped re-lift, src/minplus_oracle.cpp:1444-2002).
Along an exploration stream with a fixed viewpoint set, every refresh must
equal a full query on the same index and the reference's own incremental
query; builds, root growth and rebuilds fall back to a full query.
"""
import numpy as np
import pytest

from htrip_b200 import workloads as W
from oracle.ref import RefOracle, ref_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built (make -C oracle ref)")]


def _dev(b, g=2):
    from htrip_b200.minplus_oracle import HierarchyConfig, MinPlusOracle
    return MinPlusOracle(HierarchyConfig(tile_size_b=b, group_w=g, group_h=g))


@pytest.mark.parametrize("side,b,g,seed", [(256, 8, 2, 3), (128, 4, 4, 5), (256, 16, 2, 7)])
def test_selective_relift_equals_full_query_and_reference(gpu, side, b, g, seed):
    from htrip_b200.minplus_oracle import IncrementalState
    truth = W.street_grid(side, seed)
    obs, starts, batches = W.exploration_stream(truth, 4, 20, 96, 24, seed)
    ref = RefOracle(b, g)
    ref.set_grid(obs)
    assert ref.build()
    dev = _dev(b, g)
    assert dev.build(obs)
    # fixed viewpoints: the robots' starts and observed free cells (their
    # passability does not change under openings)
    vps = np.concatenate([starts, W.sample_free(obs, 28, seed + 1)]).astype(np.int32)
    state = IncrementalState()
    m = dev.queryAllPairsIncremental(vps, obs, state)
    assert state.last_mode == 1
    np.testing.assert_array_equal(m, ref.query_incremental(vps))
    modes = []
    for step, cells in enumerate(batches):
        obs[cells[:, 0], cells[:, 1]] = W.FREE
        ref.set_cells(cells, W.FREE)
        ref.open_batch(cells)
        dev.onBatchCellsOpened(cells, obs)
        m = dev.queryAllPairsIncremental(vps, obs, state)
        modes.append(state.last_mode)
        np.testing.assert_array_equal(m, dev.queryAllPairs(vps, obs), err_msg=f"step {step}")
        np.testing.assert_array_equal(m, ref.query_incremental(vps), err_msg=f"reference step {step}")
        again = dev.queryAllPairsIncremental(vps, obs, state)
        assert state.last_mode == 0              # nothing changed since: the cached matrix
        np.testing.assert_array_equal(again, m)
    assert set(modes) <= {0, 2} and 2 in modes  # openings only: cached or re-lifted, never a full query
    # non-monotone update: a full query again
    r, c = (int(x) for x in np.argwhere(obs == W.FREE)[len(np.argwhere(obs == W.FREE)) // 2])
    obs[r, c] = W.OBSTACLE
    ref.set_cells(np.array([[r, c]], np.int32), W.OBSTACLE)
    ref.cell_blocked(r, c)
    dev.onCellBlocked((r, c), obs)
    m = dev.queryAllPairsIncremental(vps, obs, state)
    assert state.last_mode == 1
    np.testing.assert_array_equal(m, ref.query_incremental(vps))
    np.testing.assert_array_equal(m, ref.bfs(vps))
