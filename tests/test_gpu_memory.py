"""totalMemoryBytes against the unmodified reference (exact integer equality).

The reference sums the sizes of every leaf's D and S and every node's D_U,
S_U and child_to_ext (src/minplus_oracle.cpp:2116-2134).  The server admits
sessions by this number, so it must agree with the reference after build,
after openings and after liftRoot, for every leaf side and group size.
"""
import numpy as np
import pytest

from helpers import FREE, make_grid, reveal_plan
from oracle.ref import RefOracle, ref_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built (make -C oracle ref)")]

CASES = [
    ("street", 64, 8, 2, 1),
    ("maze", 64, 16, 2, 2),
    ("rooms", 96, 32, 2, 3),
    ("noise", 64, 8, 4, 4),
    ("street", 40, 16, 4, 5),
    ("noise", 16, 16, 2, 6),   # H = 0
]


@pytest.mark.parametrize("kind,side,b,g,seed", CASES)
def test_total_memory_bytes_matches_reference(gpu, kind, side, b, g, seed):
    from htrip_b200.minplus_oracle import HierarchyConfig, MinPlusOracle
    truth = make_grid(kind, side, side, seed)
    obs, batches = reveal_plan(truth, seed, 2, 40)
    ref = RefOracle(b, g)
    ref.set_grid(obs)
    assert ref.build()
    dev = MinPlusOracle(HierarchyConfig(b, g, g))
    assert dev.build(obs)
    assert dev.totalMemoryBytes() == ref.total_memory()
    for cells in batches:
        obs[cells[:, 0], cells[:, 1]] = FREE
        ref.set_cells(cells, FREE)
        ref.open_batch(cells)
        dev.onBatchCellsOpened(cells, obs)
        assert dev.totalMemoryBytes() == ref.total_memory()
    big = np.zeros((side * g, side * g), dtype=np.uint8)
    big[:side, :side] = obs
    ref.set_grid(big)
    ref.lift_root()
    dev.liftRoot(big)
    assert (dev.S, dev.H) == (ref.S, ref.H)
    assert dev.totalMemoryBytes() == ref.total_memory()
