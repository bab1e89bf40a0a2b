"""Root growth (liftRoot), single-pair queryDistance and the incremental
all-pairs query against the unmodified reference (tolerance 0: integer
distances).  liftRoot parity covers the whole index (per-level digest of
every leaf D and node D_U), the query answers and later openings in the
grown area."""
import os

import numpy as np
import pytest

from helpers import make_grid, viewpoints
from htrip_b200 import workloads as W
from oracle.ref import RefOracle, ref_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built (make -C oracle ref)")]


def _dev(b, g=2):
    from htrip_b200.minplus_oracle import HierarchyConfig, MinPlusOracle
    return MinPlusOracle(HierarchyConfig(tile_size_b=b, group_w=g, group_h=g))


def _both(grid, b, g=2):
    ref = RefOracle(b, g)
    ref.set_grid(grid)
    assert ref.build()
    dev = _dev(b, g)
    assert dev.build(grid)
    return ref, dev


LIFT_CASES = [
    ("rooms", 32, 8, 2, 1),     # S 32 -> 64, H 2 -> 3
    ("street", 64, 16, 2, 2),   # S 64 -> 128
    ("noise", 16, 16, 2, 3),    # H = 0 -> 1
    ("noise", 16, 4, 4, 4),     # g = 4: S 16 -> 64
    ("maze", 32, 32, 2, 5),     # b = 32 leaves
]


@pytest.mark.parametrize("kind,side,b,g,seed", LIFT_CASES)
def test_lift_root_then_open_matches_reference(gpu, kind, side, b, g, seed):
    small = make_grid(kind, side, side, seed)
    ref, dev = _both(small, b, g)
    big_side = side * g
    truth = make_grid(kind, big_side, big_side, seed + 100)
    truth[:side, :side] = small
    obs, cells = W.withheld_open(truth, big_side * big_side // 20, seed)
    obs[:side, :side] = small               # the old area is as the index saw it
    cells = cells[(cells[:, 0] >= side) | (cells[:, 1] >= side)]
    ref.set_grid(obs)
    ref.lift_root()
    dev.liftRoot(obs)
    assert (dev.S, dev.H) == (ref.S, ref.H)
    assert dev.stateDigest() == ref.digest()
    vps = viewpoints(obs, 24, seed, include_blocked=2)
    np.testing.assert_array_equal(dev.queryAllPairs(vps, obs), ref.query(vps))
    np.testing.assert_array_equal(dev.queryAllPairs(vps, obs), ref.bfs(vps))
    # openings in the grown area
    for part in np.array_split(cells, 3):
        if len(part) == 0:
            continue
        obs[part[:, 0], part[:, 1]] = W.FREE
        ref.set_cells(part, W.FREE)
        ref.open_batch(part)
        dev.onBatchCellsOpened(part, obs)
        st = dev.last_batch_stats
        assert (st.n_touched_leaves, st.n_dirty_ancestors, st.n_pivots) == ref.stats()
        assert dev.stateDigest() == ref.digest()
        vps = viewpoints(obs, 20, seed + len(part))
        np.testing.assert_array_equal(dev.queryAllPairs(vps, obs), ref.query(vps))


def test_lift_root_with_default_empty_grid(gpu):
    grid = make_grid("rooms", 32, 32, 7)
    ref, dev = _both(grid, 8)
    ref.set_grid(np.zeros((0, 0), dtype=np.uint8))
    ref.lift_root()
    dev.liftRoot(None)
    assert (dev.S, dev.H) == (ref.S, ref.H)
    assert dev.stateDigest() == ref.digest()
    vps = viewpoints(grid, 12, 7)
    ref.set_grid(grid)
    np.testing.assert_array_equal(dev.queryAllPairs(vps, grid), ref.query(vps))


def test_query_distance_matches_reference_and_bfs(gpu):
    grid = make_grid("maze", 64, 64, 9)
    ref, dev = _both(grid, 8)
    rng = np.random.default_rng(9)
    pts = viewpoints(grid, 30, 9, include_blocked=4)
    for _ in range(60):
        s, t = pts[rng.integers(len(pts))], pts[rng.integers(len(pts))]
        d = dev.queryDistance(s, t, grid)
        assert d == ref.query_distance(s, t), (s, t)
        assert d == ref.bfs(np.array([s, t]))[0, 1]
    assert dev.queryDistance(pts[0], pts[0], grid) == ref.query_distance(pts[0], pts[0])
    assert dev.queryDistance((-1, 3), pts[0], grid) == 60000


def test_incremental_query_equals_reference_and_full(gpu):
    from htrip_b200.minplus_oracle import IncrementalState
    truth = make_grid("street", 64, 64, 12)
    obs, batches = W.withheld_open(truth, 200, 12)
    ref, dev = _both(obs, 8)
    state = IncrementalState()
    vps = viewpoints(truth, 20, 12)
    m = dev.queryAllPairsIncremental(vps, obs, state)
    assert state.last_recomputed
    np.testing.assert_array_equal(m, ref.query_incremental(vps))
    m2 = dev.queryAllPairsIncremental(vps, obs, state)
    assert not state.last_recomputed            # no update since: the cached matrix
    np.testing.assert_array_equal(m2, m)
    for part in np.array_split(batches, 4):
        obs[part[:, 0], part[:, 1]] = W.FREE
        ref.set_cells(part, W.FREE)
        ref.open_batch(part)
        dev.onBatchCellsOpened(part, obs)
        opened_vp = bool(set(map(tuple, part.tolist())) & set(map(tuple, np.asarray(vps).tolist())))
        m = dev.queryAllPairsIncremental(vps, obs, state)
        # only openings since: cached or a re-lift, unless a viewpoint's own
        # cell opened (its passability changed) or the openings ran on the
        # host path (which keeps no per-matrix stamps): a full query
        host_path = os.environ.get("HTRIP_OPEN_PATH") == "host"
        assert state.last_mode in ((1,) if opened_vp or host_path else (0, 2))
        np.testing.assert_array_equal(m, ref.query_incremental(vps))
        np.testing.assert_array_equal(m, dev.queryAllPairs(vps, obs))
    vps2 = vps[:13]                             # new viewpoint set: recomputed
    m = dev.queryAllPairsIncremental(vps2, obs, state)
    assert state.last_recomputed
    np.testing.assert_array_equal(m, ref.query_incremental(vps2))


BLOCK_CASES = [("rooms", 32, 8, 2, 21), ("street", 64, 16, 2, 22), ("noise", 64, 4, 4, 23), ("maze", 64, 8, 2, 24),
               ("noise", 16, 16, 2, 25)]


@pytest.mark.parametrize("kind,side,b,g,seed", BLOCK_CASES)
def test_blockages_match_reference(gpu, kind, side, b, g, seed):
    """onCellBlocked (Suite 6, test_exactness.cpp:473-497, blockages) and
    onBatchLeavesChanged against the reference: state, queries, BFS."""
    truth = make_grid(kind, side, side, seed)
    obs, cells = W.withheld_open(truth, side * side // 10, seed)
    ref, dev = _both(obs, b, g)
    obs[cells[:, 0], cells[:, 1]] = W.FREE          # open first, then block some cells
    ref.set_cells(cells, W.FREE)
    ref.open_batch(cells)
    dev.onBatchCellsOpened(cells, obs)
    rng = np.random.default_rng(seed)
    free = np.argwhere(obs == W.FREE)
    for p in free[rng.choice(len(free), size=4, replace=False)]:
        obs[p[0], p[1]] = W.OBSTACLE
        ref.set_cells([p], W.OBSTACLE)
        ref.cell_blocked(p[0], p[1])
        dev.onCellBlocked(p, obs)
        assert dev.stateDigest() == ref.digest()
        vps = viewpoints(obs, 16, int(p[0]) * 7 + 1, include_blocked=1)
        np.testing.assert_array_equal(dev.queryAllPairs(vps, obs), ref.query(vps))
        np.testing.assert_array_equal(dev.queryAllPairs(vps, obs), ref.bfs(vps))
    # several leaves at once
    lx = dev.num_leaf_tiles_x
    picks = free[rng.choice(len(free), size=6, replace=False)]
    obs[picks[:, 0], picks[:, 1]] = W.OBSTACLE
    ref.set_cells(picks, W.OBSTACLE)
    leaves = sorted({int(r) // b * lx + int(c) // b for r, c in picks})
    ref.leaves_changed(leaves)
    dev.onBatchLeavesChanged(leaves, obs)
    assert dev.stateDigest() == ref.digest()
    vps = viewpoints(obs, 16, seed + 5)
    np.testing.assert_array_equal(dev.queryAllPairs(vps, obs), ref.bfs(vps))
    # openings after blockages still match
    reopen = picks[:3]
    obs[reopen[:, 0], reopen[:, 1]] = W.FREE
    ref.set_cells(reopen, W.FREE)
    ref.open_batch(reopen)
    dev.onBatchCellsOpened(reopen, obs)
    assert dev.stateDigest() == ref.digest()
    np.testing.assert_array_equal(dev.queryAllPairs(vps, obs), ref.query(vps))
