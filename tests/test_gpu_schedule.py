"""The query kernel's two schedules give the same results.  The default
(dataflow) schedule runs every unit as soon as the units it reads are done;
HTRIP_QUERY_DATAFLOW=0 separates the phases by grid barriers.  The whole
query, batch and device-planner parity suites run again in a child process
with the barrier schedule (tolerance 0: integer distances), and one query
is compared between the schedules directly."""
import os
import subprocess
import sys

import numpy as np
import pytest

from helpers import make_grid, viewpoints

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_CHILD = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
from helpers import make_grid, viewpoints
from htrip_b200.minplus_oracle import HierarchyConfig, MinPlusOracle
grid = make_grid("maze", 256, 256, 5)
dev = MinPlusOracle(HierarchyConfig(16, 2, 2))
assert dev.build(grid)
out = dev.queryAllPairs(viewpoints(grid, 200, 5, include_blocked=3), grid)
np.save(sys.argv[2], out)
"""


def test_schedules_agree_on_one_query(gpu, tmp_path):
    outs = []
    for mode in ("1", "0"):
        f = tmp_path / f"out{mode}.npy"
        env = dict(os.environ, HTRIP_QUERY_DATAFLOW=mode)
        r = subprocess.run([sys.executable, "-c", _CHILD, ROOT, str(f)], cwd=ROOT, env=env,
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
        outs.append(np.load(f))
    np.testing.assert_array_equal(outs[0], outs[1])


def test_barrier_schedule_passes_the_query_suites(gpu):
    env = dict(os.environ, HTRIP_QUERY_DATAFLOW="0")
    files = [os.path.join(ROOT, "tests", f) for f in
             ("test_gpu_parity.py", "test_gpu_batch.py", "test_gpu_devplan.py", "test_gpu_configs.py")]
    r = subprocess.run([sys.executable, "-m", "pytest", *files, "-q", "-x", "-p", "no:cacheprovider",
                        "-k", "not planned_on_the_device"], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
