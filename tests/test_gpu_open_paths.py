"""The two opening paths give the same index and statistics.

The default path runs a whole onBatchCellsOpened call as one persistent
kernel (the level loop, the work lists and the closure rounds on the
device); HTRIP_OPEN_PATH=host drives the levels from the host (an insert and
a close stage per level, pivot counts and decrease flags read back).  The
same opening stream runs through both in child processes and every step's
per-level digest, LastBatchStats and per-level work statistics must agree
(tolerance 0: integer distances); the opening parity suites run again under
the host path."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_CHILD = r"""
import sys, json, numpy as np
sys.path.insert(0, sys.argv[1])
from htrip_b200 import workloads as W
from htrip_b200.minplus_oracle import HierarchyConfig, MinPlusOracle
rows = []
for side, b, g, seed, robots, radius, batch, steps in ((256, 8, 2, 3, 4, 20, 256, 12), (128, 4, 4, 5, 2, 12, 64, 8),
                                                       (256, 16, 2, 7, 3, 24, 512, 6), (96, 32, 2, 2, 2, 10, 128, 4)):
    truth = W.street_grid(side, seed)
    obs, starts, batches = W.exploration_stream(truth, robots, radius, batch, steps, seed)
    dev = MinPlusOracle(HierarchyConfig(b, g, g))
    assert dev.build(obs)
    for c in batches:
        obs[c[:, 0], c[:, 1]] = W.FREE
        dev.onBatchCellsOpened(c, obs)
        st = dev.last_batch_stats
        rows.append({"digest": [str(x) for x in dev.stateDigest()],
                     "stats": [st.n_touched_leaves, st.n_dirty_ancestors, st.n_pivots],
                     "levels": dev.lastOpenLevels(), "work": list(dev.lastOpenWork())})
json.dump(rows, open(sys.argv[2], "w"))
"""


def test_open_paths_agree_step_by_step(gpu, tmp_path):
    outs = []
    for path in ("device", "host"):
        f = tmp_path / f"{path}.json"
        env = dict(os.environ, HTRIP_OPEN_PATH=path)
        r = subprocess.run([sys.executable, "-c", _CHILD, ROOT, str(f)], cwd=ROOT, env=env,
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
        outs.append(json.load(open(f)))
    assert len(outs[0]) == len(outs[1]) > 0
    for a, b in zip(*outs):
        assert a == b


SUITES = ("test_gpu_parity.py", "test_gpu_batch.py", "test_gpu_property.py", "test_gpu_next.py")


def test_opening_suites_under_host_path(gpu):
    env = dict(os.environ, HTRIP_OPEN_PATH="host")
    files = [os.path.join(ROOT, "tests", f) for f in SUITES]
    r = subprocess.run([sys.executable, "-m", "pytest", *files, "-q", "-x", "-p", "no:cacheprovider"], cwd=ROOT,
                       env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
