"""Batched openings and queries at the many-maps workload's scale (tolerance 0).

Maps of side 1024 with 32x32 leaves (the workload's largest indexes, about
3 GiB each), mixed with smaller street and maze maps and other leaf sides,
each get one opening batch (64-1024 withheld cells) and one queryAllPairs
with k up to 512.  One htrip_open_batch and one htrip_query_batch over all
of them must leave every index exactly as the same calls made one map at a
time (per-level digest of every leaf D and node D_U, last_batch_stats) and
give the same matrices; every matrix is also checked against the
reference's BfsOracle, and the indexes small enough for the reference's CPU
build are checked against the reference's own state and stats.
"""
import numpy as np
import pytest

from htrip_b200 import workloads as W
from oracle.ref import RefOracle, ref_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built (make -C oracle ref)")]

# (side, kind, parameter, b, cells opened, k, compare with the reference's index)
MAPS = [
    (1024, "street", 0.3, 32, 1024, 512, False),
    (1024, "maze", 4, 32, 700, 300, False),
    (1024, "street", 0.2, 8, 256, 64, False),
    (512, "maze", 1, 32, 900, 512, True),
    (256, "street", 0.4, 16, 64, 128, True),
    (128, "maze", 16, 8, 200, 8, True),
]


def _grid(side, kind, param, seed):
    return W.street_grid(side, seed, blocked=param) if kind == "street" else W.maze_grid(side, int(param), seed)


def test_batched_open_and_query_at_scale_equal_single_calls(gpu):
    from htrip_b200.minplus_oracle import Batch, HierarchyConfig, MinPlusOracle
    maps = []
    for i, (side, kind, param, b, m, k, with_ref) in enumerate(MAPS):
        truth = _grid(side, kind, param, 40 + i)
        obs, cells = W.withheld_open(truth, m, 50 + i)
        full = obs.copy()
        full[cells[:, 0], cells[:, 1]] = W.FREE
        vps = W.sample_free(full, k, 60 + i)
        maps.append((b, obs, cells, full, vps, with_ref))
    batched, single = [], []
    for b, obs, _, _, _, _ in maps:
        for lst in (batched, single):
            d = MinPlusOracle(HierarchyConfig(b, 2, 2))
            assert d.build(obs)
            lst.append(d)
    bt = Batch()
    bt.open([(d, cells, full) for d, (_, _, cells, full, _, _) in zip(batched, maps)])
    outs = bt.query([(d, vps, full) for d, (_, _, _, full, vps, _) in zip(batched, maps)])
    for i, (b, obs, cells, full, vps, with_ref) in enumerate(maps):
        single[i].onBatchCellsOpened(cells, full)
        st_b, st_s = batched[i].last_batch_stats, single[i].last_batch_stats
        assert (st_b.n_touched_leaves, st_b.n_dirty_ancestors, st_b.n_pivots) == \
               (st_s.n_touched_leaves, st_s.n_dirty_ancestors, st_s.n_pivots)
        assert batched[i].stateDigest() == single[i].stateDigest()
        one = single[i].queryAllPairs(vps, full)
        np.testing.assert_array_equal(outs[i], one)
        ref = RefOracle(b, 2)
        ref.set_grid(full)
        np.testing.assert_array_equal(outs[i], ref.bfs(vps))
        if with_ref:
            ref.set_grid(obs)
            assert ref.build()
            ref.set_cells(cells, W.FREE)
            ref.open_batch(cells)
            assert ref.stats() == (st_b.n_touched_leaves, st_b.n_dirty_ancestors, st_b.n_pivots)
            assert batched[i].stateDigest() == ref.digest()
            np.testing.assert_array_equal(outs[i], ref.query(vps))
        del ref
