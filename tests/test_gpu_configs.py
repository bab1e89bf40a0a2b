"""Parity at the benchmark workloads' full sizes (bit-exact, tolerance 0).

* 256x256 street grid, b=16, k=16: queryAllPairs equals the reference's
  queryAllPairs and BfsOracle; the whole index equals the reference's
  (per-level digest of every leaf D and node D_U).
* 512x512 mazes (corridor 1 and corridor 16), b=16, k=64 and k=256: same.
* Incremental opening on a 1024x1024 street grid, b=8: 400 onBatchCellsOpened
  calls of 256 cells in BFS-ring order from 16 radius-40 disks; after every
  call the index equals a fresh device build of the same grid (digest) and
  queryAllPairs over 16 robot poses + 48 frontier cells equals the rebuilt
  index's answer; the reference's own index runs the same stream, and every
  50th step its whole state, stats and answers (and BFS's) are compared.
* The same stream on a 256x256 grid checked against the reference's own
  incremental index after every call (digest, stats and query).
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


def _both(grid, b):
    ref = RefOracle(b)
    ref.set_grid(grid)
    assert ref.build()
    dev = _dev(b)
    assert dev.build(grid)
    return ref, dev


def test_street256_b16_k16(gpu):
    grid = W.street_grid(256, 1)
    ref, dev = _both(grid, 16)
    assert dev.stateDigest() == ref.digest()
    for seed in range(3):
        vps = W.sample_free(grid, 16, seed)
        got = dev.queryAllPairs(vps, grid)
        np.testing.assert_array_equal(got, ref.query(vps))
        np.testing.assert_array_equal(got, ref.bfs(vps))


@pytest.mark.parametrize("corridor", [1, 16])
def test_maze512_b16(gpu, corridor):
    grid = W.maze_grid(512, corridor, 2)
    ref, dev = _both(grid, 16)
    assert dev.stateDigest() == ref.digest()
    for k in (64, 256):
        vps = W.sample_free(grid, k, k)
        got = dev.queryAllPairs(vps, grid)
        np.testing.assert_array_equal(got, ref.query(vps))
        np.testing.assert_array_equal(got, ref.bfs(vps))
        assert got[got < 60000].max() < 60000


def _step_viewpoints(obs, starts, step):
    return np.concatenate([starts, W.frontier_cells(obs, 48, 1000 + step)]).astype(np.int32)


def test_incremental_1024_b8_every_step_equals_rebuild(gpu):
    """Every step against a device rebuild; the reference's own incremental
    index runs the same stream beside it, and every 50th step its state,
    stats and query answers are compared too (with BFS)."""
    truth = W.street_grid(1024, 3)
    obs, starts, batches = W.exploration_stream(truth, 16, 40, 256, 400, 3)
    assert len(batches) == 400
    ref, dev = _both(obs, 8)
    for step, cells in enumerate(batches):
        obs[cells[:, 0], cells[:, 1]] = W.FREE
        dev.onBatchCellsOpened(cells, obs)
        ref.set_cells(cells, W.FREE)
        ref.open_batch(cells)
        fresh = _dev(8)
        assert fresh.build(obs)
        assert dev.stateDigest() == fresh.stateDigest(), f"index differs from a rebuild after step {step}"
        vps = _step_viewpoints(obs, starts, step)
        got = dev.queryAllPairs(vps, obs)
        np.testing.assert_array_equal(got, fresh.queryAllPairs(vps, obs), err_msg=f"step {step}")
        if step % 50 == 49:
            st = dev.last_batch_stats
            assert (st.n_touched_leaves, st.n_dirty_ancestors, st.n_pivots) == ref.stats(), f"stats step {step}"
            assert dev.stateDigest() == ref.digest(), f"index differs from the reference after step {step}"
            np.testing.assert_array_equal(got, ref.query(vps), err_msg=f"reference step {step}")
            np.testing.assert_array_equal(got, ref.bfs(vps), err_msg=f"BFS step {step}")
        del fresh


def test_incremental_256_b8_against_reference(gpu):
    truth = W.street_grid(256, 4)
    obs, starts, batches = W.exploration_stream(truth, 4, 20, 256, 24, 4)
    ref, dev = _both(obs, 8)
    for step, cells in enumerate(batches):
        obs[cells[:, 0], cells[:, 1]] = W.FREE
        ref.set_cells(cells, W.FREE)
        ref.open_batch(cells)
        dev.onBatchCellsOpened(cells, obs)
        st = dev.last_batch_stats
        assert (st.n_touched_leaves, st.n_dirty_ancestors, st.n_pivots) == ref.stats(), f"stats step {step}"
        assert dev.stateDigest() == ref.digest(), f"index differs from the reference after step {step}"
        vps = np.concatenate([starts, W.frontier_cells(obs, 28, step)]).astype(np.int32)
        np.testing.assert_array_equal(dev.queryAllPairs(vps, obs), ref.query(vps), err_msg=f"step {step}")
