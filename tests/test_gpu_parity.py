"""GPU parity: the CUDA index against the unmodified reference (oracle/_ref).

Every comparison is bit-exact (tolerance 0): the path is integer min-plus.
State parity compares the reference's public members leaves[i].D / .S and
levels[l][n].D_U / .S_U / .child_to_ext with the device arena; query parity
compares queryAllPairs with the reference's queryAllPairs and BfsOracle.
"""
import numpy as np
import pytest

from helpers import make_grid, reveal_plan, viewpoints
from htrip_b200 import workloads as W
from oracle.ref import RefOracle, ref_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built (make -C oracle ref)")]


def _dev(b, g):
    from htrip_b200.minplus_oracle import HierarchyConfig, MinPlusOracle
    return MinPlusOracle(HierarchyConfig(tile_size_b=b, group_w=g, group_h=g))


def _build_both(grid, b, g):
    ref = RefOracle(b, g)
    ref.set_grid(grid)
    assert ref.build()
    dev = _dev(b, g)
    assert dev.build(grid)
    assert (dev.S, dev.H) == (ref.S, ref.H)
    return ref, dev


def _check_state(ref, dev, b, g):
    for i in range(ref.num_leaves()):
        np.testing.assert_array_equal(dev.leaf_D(i), ref.leaf_D(i), err_msg=f"leaf D {i}")
        np.testing.assert_array_equal(dev.leaf_S(i), ref.leaf_S(i), err_msg=f"leaf S {i}")
    for lvl in range(1, ref.H + 1):
        for n in range(ref.num_nodes(lvl)):
            np.testing.assert_array_equal(dev.node_DU(lvl, n), ref.node_DU(lvl, n), err_msg=f"D_U l{lvl} n{n}")
            np.testing.assert_array_equal(dev.node_SU(lvl, n), ref.node_SU(lvl, n), err_msg=f"S_U l{lvl} n{n}")
            for q in range(g * g):
                np.testing.assert_array_equal(dev.node_C2E(lvl, n, q), ref.node_C2E(lvl, n, q),
                                              err_msg=f"C2E l{lvl} n{n} q{q}")


def _check_query(ref, dev, grid, k, seed):
    vps = viewpoints(grid, k, seed, include_blocked=2)
    got = dev.queryAllPairs(vps, grid)
    exp = ref.query(vps)
    np.testing.assert_array_equal(got, exp)
    np.testing.assert_array_equal(got, ref.bfs(vps))


STATE_CASES = [
    ("noise", 16, 16, 8, 2, 1),
    ("rooms", 32, 32, 8, 2, 2),
    ("noise", 40, 24, 8, 2, 3),      # non-square, padded to S=64
    ("maze", 64, 64, 8, 2, 4),
    ("street", 64, 64, 16, 2, 5),
    ("noise", 32, 32, 4, 2, 6),
    ("rooms", 16, 16, 2, 2, 7),
    ("noise", 64, 64, 4, 4, 8),      # g = 4
    ("open", 32, 32, 8, 2, 9),
    ("maze", 64, 64, 32, 2, 10),     # b = 32 leaves
]


@pytest.mark.parametrize("kind,rows,cols,b,g,seed", STATE_CASES)
def test_build_state_and_query(gpu, kind, rows, cols, b, g, seed):
    grid = make_grid(kind, rows, cols, seed)
    ref, dev = _build_both(grid, b, g)
    _check_state(ref, dev, b, g)
    for k in (1, 5, 17):
        _check_query(ref, dev, grid, k, seed + k)


UPDATE_CASES = [
    ("rooms", 32, 32, 8, 2, 11, 6, 7),
    ("noise", 48, 40, 8, 2, 12, 5, 11),
    ("maze", 64, 64, 8, 2, 13, 4, 40),
    ("street", 64, 64, 16, 2, 14, 3, 64),
    ("noise", 64, 64, 4, 4, 15, 4, 20),
    ("rooms", 32, 32, 32, 2, 16, 3, 30),
]


@pytest.mark.parametrize("kind,rows,cols,b,g,seed,nb,bs", UPDATE_CASES)
def test_batch_open_state_stats_query(gpu, kind, rows, cols, b, g, seed, nb, bs):
    truth = make_grid(kind, rows, cols, seed)
    obs, batches = reveal_plan(truth, seed, nb, bs)
    ref, dev = _build_both(obs, b, g)
    for bi, cells in enumerate(batches):
        obs[cells[:, 0], cells[:, 1]] = 1
        ref.set_cells(cells, 1)
        ref.open_batch(cells)
        dev.onBatchCellsOpened(cells, obs)
        st = dev.last_batch_stats
        assert (st.n_touched_leaves, st.n_dirty_ancestors, st.n_pivots) == ref.stats(), f"stats batch {bi}"
        _check_query(ref, dev, obs, 9, seed + bi)
    _check_state(ref, dev, b, g)


def test_single_cell_open_matches(gpu):
    truth = make_grid("rooms", 32, 32, 21)
    obs, batches = reveal_plan(truth, 21, 1, 12)
    ref, dev = _build_both(obs, 8, 2)
    for r, c in batches[0]:
        obs[r, c] = 1
        ref.set_cells([[r, c]], 1)
        ref.open_cell(int(r), int(c))
        dev.onCellOpened((int(r), int(c)), obs)
    _check_state(ref, dev, 8, 2)
    _check_query(ref, dev, obs, 12, 3)


def test_known_answer_suite1_seam(gpu):
    """test_exactness.cpp:100-145: a cross-leaf seam opened at level 1 gives distance 1."""
    g = np.full((32, 32), 2, dtype=np.uint8)
    g[4, 16] = 1
    dev = _dev(8, 2)
    dev.build(g)
    g[4, 15] = 1
    dev.onCellOpened((4, 15), g)
    assert dev.queryAllPairs([[4, 15], [4, 16]], g)[0, 1] == 1
    for c in range(10, 21):
        g[4, c] = 1
        dev.onCellOpened((4, c), g)
    vps = [[4, 10], [4, 13], [4, 15], [4, 16], [4, 18], [4, 20]]
    m = dev.queryAllPairs(vps, g)
    exp = np.abs(np.subtract.outer([10, 13, 15, 16, 18, 20], [10, 13, 15, 16, 18, 20]))
    np.testing.assert_array_equal(m, exp)


def test_known_answer_suite8_tail_port(gpu):
    """test_exactness.cpp:597-667: the tail-port geometry has BFS distance 37."""
    g = np.full((32, 32), 2, dtype=np.uint8)
    g[2, 16:32] = 1
    g[2:16, 24] = 1
    g[16:21, 24] = 1
    g[20, 16:32] = 1
    g[16:32, 0:16] = 1
    dev = _dev(16, 2)
    dev.build(g)
    m = dev.queryAllPairs([[2, 24], [25, 10], [20, 20], [8, 24]], g)
    assert m[0, 1] == 37 and m[1, 0] == 37


def test_known_answer_suite12_blocked_viewpoint(gpu):
    """test_exactness.cpp:845-893: separated halves stay INF; a blocked viewpoint has an INF diagonal."""
    g = np.full((32, 32), 1, dtype=np.uint8)
    g[:, 16] = 2
    dev = _dev(16, 2)
    dev.build(g)
    vps = [[4, 4], [8, 12], [4, 20], [8, 28], [20, 16]]
    m = dev.queryAllPairs(vps, g)
    assert m[4, 4] == 60000 and (m[4] == 60000).all() and (m[:, 4] == 60000).all()
    assert m[0, 2] == 60000 and m[0, 1] == 12
    g[8, 16] = 1
    dev.onCellOpened((8, 16), g)
    m = dev.queryAllPairs(vps, g)
    assert m[0, 2] < 60000 and m[4, 4] == 60000


def test_h0_single_leaf(gpu):
    """test_exactness.cpp:763-795: S == b gives H = 0 (leaf-only index)."""
    g = np.full((16, 16), 2, dtype=np.uint8)
    g[8, 2:14] = 1
    ref, dev = _build_both(g, 16, 2)
    assert dev.H == 0
    cells = np.array([[7, 6], [6, 6], [5, 6], [4, 6], [9, 10], [10, 10], [11, 10], [12, 10]], dtype=np.int32)
    g[cells[:, 0], cells[:, 1]] = 1
    ref.set_cells(cells, 1)
    ref.open_batch(cells)
    dev.onBatchCellsOpened(cells, g)
    assert (dev.last_batch_stats.n_touched_leaves, dev.last_batch_stats.n_dirty_ancestors,
            dev.last_batch_stats.n_pivots) == ref.stats()
    _check_state(ref, dev, 16, 2)
    _check_query(ref, dev, g, 6, 1)


def test_clone_is_deep(gpu):
    truth = make_grid("rooms", 32, 32, 31)
    obs, batches = reveal_plan(truth, 31, 1, 10)
    ref, dev = _build_both(obs, 8, 2)
    snap = dev.clone()
    cells = batches[0]
    obs2 = obs.copy()
    obs2[cells[:, 0], cells[:, 1]] = 1
    dev.onBatchCellsOpened(cells, obs2)
    # the clone still answers for the old grid
    vps = viewpoints(obs, 10, 5)
    np.testing.assert_array_equal(snap.queryAllPairs(vps, obs), ref.query(vps))


def _open_both(ref, dev, obs, part):
    obs[part[:, 0], part[:, 1]] = W.FREE
    ref.set_cells(part, W.FREE)
    ref.open_batch(part)
    dev.onBatchCellsOpened(part, obs)
    st = dev.last_batch_stats
    assert (st.n_touched_leaves, st.n_dirty_ancestors, st.n_pivots) == ref.stats()
    assert dev.stateDigest() == ref.digest()


def test_batched_opening_shapes(gpu):
    """test_exactness.cpp:1029-1210: an 8-cell batch across tiles, a 28-cell
    batch, a whole 64-cell column in one batch, an H = 0 batch, and liftRoot
    after a batch; state, stats and queries against the reference."""
    truth = make_grid("noise", 64, 64, 61)
    truth[:, 37] = W.FREE                              # the column that opens at once
    rng = np.random.default_rng(61)
    free = np.argwhere(truth == W.FREE)
    free = free[free[:, 1] != 37]
    pick = free[rng.choice(len(free), 36, replace=False)]
    col = np.stack([np.arange(64), np.full(64, 37)], 1)
    obs = truth.copy()
    for part in (pick, col):
        obs[part[:, 0], part[:, 1]] = W.OBSTACLE
    ref, dev = _build_both(obs, 8, 2)
    for part in (pick[:8], pick[8:], col):         # 8 cells, 28 cells, the column
        _open_both(ref, dev, obs, part)
        _check_query(ref, dev, obs, 20, len(part))
    big = make_grid("noise", 128, 128, 62)            # liftRoot after the batches
    big[:64, :64] = obs
    ref.set_grid(big)
    ref.lift_root()
    dev.liftRoot(big)
    assert (dev.S, dev.H) == (ref.S, ref.H)
    assert dev.stateDigest() == ref.digest()
    _check_query(ref, dev, big, 24, 63)
    small = make_grid("open", 16, 16, 64)             # H = 0: one leaf
    cells = np.array([[3, 4], [3, 5], [9, 9], [15, 0]])
    small[cells[:, 0], cells[:, 1]] = W.OBSTACLE
    ref0, dev0 = _build_both(small, 16, 2)
    assert dev0.H == 0
    _open_both(ref0, dev0, small, cells)
    _check_query(ref0, dev0, small, 12, 65)
