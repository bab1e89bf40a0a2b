"""Generate the golden fixtures in tests/golden/ from the compiled reference.

Run here (where the reference sources exist): ``make -C oracle ref`` then
``python tests/golden/make_golden.py``.  Each case stores the input grid,
the opening batches and viewpoints, and the reference's outputs: the
queryAllPairs matrix after the build and after every batch, the
last_batch_stats of every batch, and a SHA-256 of the full index state
(every leaf D and node D_U, in index order) after the last batch.
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from helpers import make_grid, reveal_plan, viewpoints  # noqa: E402
from oracle.ref import RefOracle  # noqa: E402

CASES = [
    # name, kind, rows, cols, b, g, seed, n_batches, batch
    ("rooms32_b8", "rooms", 32, 32, 8, 2, 101, 4, 9),
    ("noise40x24_b8", "noise", 40, 24, 8, 2, 102, 3, 12),
    ("maze64_b8", "maze", 64, 64, 8, 2, 103, 3, 30),
    ("street64_b16", "street", 64, 64, 16, 2, 104, 3, 40),
    ("noise64_b4_g4", "noise", 64, 64, 4, 4, 105, 3, 20),
    ("rooms16_b2", "rooms", 16, 16, 2, 2, 106, 2, 6),
]


def state_hash(ref):
    h = hashlib.sha256()
    for i in range(ref.num_leaves()):
        h.update(ref.leaf_D(i).tobytes())
    for lvl in range(1, ref.H + 1):
        for n in range(ref.num_nodes(lvl)):
            h.update(ref.node_DU(lvl, n).tobytes())
    return h.hexdigest()


def main():
    for name, kind, rows, cols, b, g, seed, nb, bs in CASES:
        truth = make_grid(kind, rows, cols, seed)
        obs, batches = reveal_plan(truth, seed, nb, bs)
        vps = viewpoints(truth, 10, seed, include_blocked=2)
        ref = RefOracle(b, g)
        ref.set_grid(obs)
        assert ref.build()
        obs0 = obs.copy()
        mats = [ref.query(vps)]
        stats = []
        for cells in batches:
            obs[cells[:, 0], cells[:, 1]] = 1
            ref.set_cells(cells, 1)
            ref.open_batch(cells)
            stats.append(ref.stats())
            mats.append(ref.query(vps))
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"),
            b=b, g=g, observed0=obs0, vps=vps,
            batch_sizes=np.array([len(c) for c in batches], dtype=np.int32),
            cells=np.concatenate(batches).astype(np.int32),
            matrices=np.stack(mats), stats=np.array(stats, dtype=np.int32),
            S=ref.S, H=ref.H, state_sha256=state_hash(ref),
            total_memory=ref.total_memory())
        print(name, "S", ref.S, "H", ref.H, "stats", stats)


if __name__ == "__main__":
    main()
