"""The plain-C oracle (oracle/htrip_oracle.c) pinned against the reference.

* golden fixtures made by the compiled reference (tests/golden/make_golden.py):
  query matrices after the build and after every opening batch, the batches'
  last_batch_stats and a SHA-256 of the whole index state;
* the reference test suite's own known answers (apps/test_exactness.cpp);
* the compiled reference itself, when oracle/_ref is built.
"""
import glob
import hashlib
import os

import numpy as np
import pytest

from helpers import make_grid, reveal_plan, viewpoints
from oracle.ref import PortOracle, RefOracle, port_available, port_bfs, ref_available

pytestmark = pytest.mark.skipif(not port_available(), reason="oracle port not built (make -C oracle port)")

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def _state_hash(o, n_leaves, H):
    h = hashlib.sha256()
    for i in range(n_leaves):
        h.update(o.leaf_D(i).tobytes())
    for lvl in range(1, H + 1):
        nodes = (o.S // (o.b * o.g ** lvl)) ** 2
        for n in range(nodes):
            h.update(o.node_DU(lvl, n).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_port_matches_golden(path):
    z = np.load(path)
    obs = z["observed0"].copy()
    po = PortOracle(int(z["b"]), int(z["g"]))
    assert po.build(obs)
    assert (po.S, po.H) == (int(z["S"]), int(z["H"]))
    vps = z["vps"]
    np.testing.assert_array_equal(po.query(vps, obs), z["matrices"][0])
    off = 0
    for bi, n in enumerate(z["batch_sizes"]):
        cells = z["cells"][off:off + n]
        off += n
        obs[cells[:, 0], cells[:, 1]] = 1
        po.open_batch(cells, obs)
        assert po.stats() == tuple(z["stats"][bi])
        np.testing.assert_array_equal(po.query(vps, obs), z["matrices"][bi + 1])
        np.testing.assert_array_equal(port_bfs(obs, vps), z["matrices"][bi + 1])
    n_leaves = (po.S // po.b) ** 2
    assert _state_hash(po, n_leaves, po.H) == str(z["state_sha256"])


def test_port_known_answer_tail_port_37():
    """apps/test_exactness.cpp:597-667 (Suite 8): d((2,24),(25,10)) = 37."""
    g = np.full((32, 32), 2, dtype=np.uint8)
    g[2, 16:32] = 1
    g[2:16, 24] = 1
    g[16:21, 24] = 1
    g[20, 16:32] = 1
    g[16:32, 0:16] = 1
    po = PortOracle(16, 2)
    po.build(g)
    vps = [[2, 24], [25, 10], [20, 20], [8, 24]]
    m = po.query(vps, g)
    assert m[0, 1] == 37
    np.testing.assert_array_equal(m, port_bfs(g, vps))


def test_port_known_answer_seams():
    """apps/test_exactness.cpp:100-201 (Suites 1, 1b): level-1 and level-2 seams give 1."""
    for p1, p2 in (((4, 15), (4, 16)), ((15, 8), (16, 8))):
        g = np.full((32, 32), 2, dtype=np.uint8)
        g[p2] = 1
        po = PortOracle(8, 2)
        po.build(g)
        g[p1] = 1
        po.open_batch([p1], g)
        assert po.query([p1, p2], g)[0, 1] == 1


def test_port_blocked_viewpoint_inf():
    """apps/test_exactness.cpp:845-893 (Suite 12): blocked viewpoint row / diagonal stay INF."""
    g = np.full((32, 32), 1, dtype=np.uint8)
    g[:, 16] = 2
    po = PortOracle(16, 2)
    po.build(g)
    m = po.query([[4, 4], [8, 12], [4, 20], [8, 28], [20, 16]], g)
    assert (m[4] == 60000).all() and (m[:, 4] == 60000).all()
    assert m[0, 2] == 60000 and m[0, 1] == 12


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("kind,rows,cols,b,g,seed", [
    ("noise", 24, 40, 8, 2, 1), ("maze", 64, 64, 8, 2, 2), ("rooms", 32, 32, 4, 2, 3), ("noise", 64, 64, 4, 4, 4)])
def test_port_matches_compiled_reference(kind, rows, cols, b, g, seed):
    truth = make_grid(kind, rows, cols, seed)
    obs, batches = reveal_plan(truth, seed, 3, 14)
    ref = RefOracle(b, g)
    ref.set_grid(obs)
    ref.build()
    po = PortOracle(b, g)
    po.build(obs)
    for cells in batches:
        obs[cells[:, 0], cells[:, 1]] = 1
        ref.set_cells(cells, 1)
        ref.open_batch(cells)
        po.open_batch(cells, obs)
        assert po.stats() == ref.stats()
        vps = viewpoints(obs, 12, seed, include_blocked=2)
        np.testing.assert_array_equal(po.query(vps, obs), ref.query(vps))
    for i in range(ref.num_leaves()):
        np.testing.assert_array_equal(po.leaf_D(i), ref.leaf_D(i))
    for lvl in range(1, ref.H + 1):
        for n in range(ref.num_nodes(lvl)):
            np.testing.assert_array_equal(po.node_DU(lvl, n), ref.node_DU(lvl, n))
