"""Weighted grids (the reference's GridMap::weights) against the unmodified
reference: leaves with non-unit weights built as the reference's Dijkstra
leaf build, weighted seams and opened edges, onCellWeightChanged,
onTileWeightsChanged and liftRoot.  Checked: the whole index state (digest of
every leaf D and node D_U), batch stats, and queries against the reference's
queryAllPairs and its DijkstraOracle (tolerance 0: integer distances)."""
import numpy as np
import pytest

from helpers import make_grid, viewpoints
from htrip_b200 import workloads as W
from oracle.ref import RefOracle, ref_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built (make -C oracle ref)")]


def _weights(shape, seed, hi=9, region=None):
    """Weights 1..hi; with `region` = (r0, r1, c0, c1) only that block is
    non-unit (the other leaves keep the BFS build)."""
    rng = np.random.default_rng(seed)
    w = rng.integers(1, hi + 1, size=shape).astype(np.uint16)
    if region is not None:
        r0, r1, c0, c1 = region
        m = np.ones(shape, dtype=np.uint16)
        m[r0:r1, c0:c1] = w[r0:r1, c0:c1]
        w = m
    return w


def _both(grid, w, b, g=2):
    from htrip_b200.minplus_oracle import HierarchyConfig, MinPlusOracle
    ref = RefOracle(b, g)
    ref.set_grid(grid)
    ref.set_weights(w)
    assert ref.build()
    dev = MinPlusOracle(HierarchyConfig(tile_size_b=b, group_w=g, group_h=g))
    assert dev.build(grid, weights=w)
    return ref, dev


def _check(ref, dev, grid, k, seed):
    assert dev.stateDigest() == ref.digest()
    vps = viewpoints(grid, k, seed, include_blocked=2)
    got = dev.queryAllPairs(vps, grid)
    np.testing.assert_array_equal(got, ref.query(vps))
    np.testing.assert_array_equal(got, ref.dijkstra(vps))


BUILD_CASES = [
    ("street", 64, 8, 2, 1, None),
    ("maze", 64, 16, 2, 2, None),
    ("rooms", 64, 8, 2, 3, (8, 40, 16, 48)),   # weighted and unit leaves side by side
    ("noise", 64, 4, 4, 4, None),              # g = 4
    ("open", 64, 32, 2, 5, (0, 32, 0, 64)),    # b = 32 leaves (order 1024)
    ("noise", 40, 8, 2, 6, None),              # non-square grid padded to S = 64
]


@pytest.mark.parametrize("kind,side,b,g,seed,region", BUILD_CASES)
def test_weighted_build_matches_reference_and_dijkstra(gpu, kind, side, b, g, seed, region):
    grid = make_grid(kind, side, side if kind != "noise" or side != 40 else 24, seed)
    w = _weights(grid.shape, seed, region=region)
    ref, dev = _both(grid, w, b, g)
    _check(ref, dev, grid, 24, seed)


def test_unit_weights_equal_the_unweighted_index(gpu):
    from htrip_b200.minplus_oracle import HierarchyConfig, MinPlusOracle
    grid = make_grid("maze", 64, 64, 7)
    a = MinPlusOracle(HierarchyConfig(8, 2, 2))
    assert a.build(grid)
    b = MinPlusOracle(HierarchyConfig(8, 2, 2))
    assert b.build(grid, weights=np.ones(grid.shape, dtype=np.uint16))
    assert a.stateDigest() == b.stateDigest()


@pytest.mark.parametrize("kind,side,b,seed", [("street", 128, 8, 11), ("maze", 64, 16, 12), ("rooms", 64, 4, 13)])
def test_weighted_openings_match_reference(gpu, kind, side, b, seed):
    truth = make_grid(kind, side, side, seed)
    w = _weights(truth.shape, seed, hi=6)
    obs, cells = W.withheld_open(truth, side * side // 8, seed)
    ref, dev = _both(obs, w, b)
    for part in np.array_split(cells, 4):
        obs[part[:, 0], part[:, 1]] = W.FREE
        ref.set_cells(part, W.FREE)
        ref.open_batch(part)
        dev.onBatchCellsOpened(part, obs)
        st = dev.last_batch_stats
        assert (st.n_touched_leaves, st.n_dirty_ancestors, st.n_pivots) == ref.stats()
        _check(ref, dev, obs, 20, seed + len(part))


def test_cell_weight_changes_match_reference(gpu):
    grid = make_grid("street", 64, 64, 21)
    w = _weights(grid.shape, 21, hi=4)
    ref, dev = _both(grid, w, 8)
    mine = w.copy()
    rng = np.random.default_rng(21)
    free = np.argwhere(grid == W.FREE)
    blocked = np.argwhere(grid == W.OBSTACLE)
    changes = [(tuple(free[i]), int(rng.integers(1, 40))) for i in rng.choice(len(free), 6, replace=False)]
    changes.append((tuple(free[0]), int(mine[tuple(free[0])])))   # unchanged weight: nothing happens
    changes.append((tuple(blocked[0]), 7))                        # an obstacle's weight (INF) changes
    changes.append((tuple(free[3]), 1))                           # back to a unit weight
    changes.append((tuple(free[5]), 60000))                       # INF: edges through the cell vanish
    for (r, c), nw in changes:
        ref.cell_weight_changed(r, c, nw)
        dev.onCellWeightChanged((r, c), nw, grid, mine)
        _check(ref, dev, grid, 16, r * 64 + c)


def test_tile_weight_changes_match_reference(gpu):
    grid = make_grid("rooms", 64, 64, 31)
    w = np.ones(grid.shape, dtype=np.uint16)
    ref, dev = _both(grid, w, 8)
    rng = np.random.default_rng(31)
    tx, ty = 3, 2
    cells = [(ty * 8 + int(rng.integers(0, 8)), tx * 8 + int(rng.integers(0, 8))) for _ in range(10)]
    cells.append((0, 0))  # outside tile (3, 2): its weight is set, only tile (3, 2) is rebuilt
    ws = [int(rng.integers(2, 20)) for _ in cells]
    ref.tile_weights_changed(tx, ty, cells, ws)
    dev.onTileWeightsChanged(tx, ty, list(zip(cells, ws)), grid, w)
    assert dev.stateDigest() == ref.digest()
    vps = viewpoints(grid, 16, 31)
    np.testing.assert_array_equal(dev.queryAllPairs(vps, grid), ref.query(vps))
    # a rebuild of tile (0, 0) brings the other changed weight in as well
    ref.tile_weights_changed(0, 0, [], [])
    dev.onTileWeightsChanged(0, 0, [], grid, w)
    _check(ref, dev, grid, 16, 32)


def test_weighted_lift_root_matches_reference(gpu):
    small = make_grid("street", 32, 32, 41)
    ws = _weights(small.shape, 41, hi=5)
    ref, dev = _both(small, ws, 8)
    truth = make_grid("street", 64, 64, 42)
    truth[:32, :32] = small
    wb = _weights(truth.shape, 43, hi=5)
    wb[:32, :32] = ws
    ref.set_grid(truth)
    ref.set_weights(wb)
    ref.lift_root()
    dev.liftRoot(truth, weights=wb)
    assert (dev.S, dev.H) == (ref.S, ref.H)
    _check(ref, dev, truth, 24, 44)
