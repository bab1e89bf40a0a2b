"""The query tile autotuner: every tile shape gives the same matrix, and the
tuner's choice is recorded for the request's bucket (tolerance 0)."""
import numpy as np
import pytest

from htrip_b200 import workloads as W
from oracle.ref import RefOracle, ref_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built (make -C oracle ref)")]


def test_every_tile_shape_is_exact_and_tuning_is_recorded(gpu):
    from htrip_b200.minplus_oracle import (HierarchyConfig, MinPlusOracle, autotune_clear, autotune_export,
                                           autotune_import)
    grid = W.maze_grid(256, 1, 5)
    dev = MinPlusOracle(HierarchyConfig(16, 2, 2))
    assert dev.build(grid)
    ref = RefOracle(16)
    ref.set_grid(grid)
    assert ref.build()
    vps = W.sample_free(grid, 100, 3)
    exp = ref.query(vps)
    autotune_clear()
    cfg, ms = dev.autotuneQuery(vps, grid, reps=3)
    assert 0 <= cfg < 4 and ms > 0
    line = autotune_export().strip()
    assert line.endswith(f" {cfg}") and len(line.split()) == 5
    np.testing.assert_array_equal(dev.queryAllPairs(vps, grid), exp)
    key = " ".join(line.split()[:4])
    for forced in range(4):
        autotune_import(f"{key} {forced}\n")
        np.testing.assert_array_equal(dev.queryAllPairs(vps, grid), exp, err_msg=f"tile shape {forced}")
    autotune_clear()
