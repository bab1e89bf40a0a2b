"""The query kernel's schedules give the same results.  The default
(dataflow) schedule runs every unit as soon as the units it reads are done;
HTRIP_QUERY_DATAFLOW=0 separates the phases by grid barriers.  Root project
items run in parts (split-K) when the root's child port list is long;
HTRIP_QUERY_ROOT_SPLIT=n forces n parts on every root level, so that the
small parity grids run the split path too.  The query, batch and
device-planner parity suites run again in child processes under these
settings (tolerance 0: integer distances), and one query is compared
between the schedules directly."""
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


SUITES = ("test_gpu_parity.py", "test_gpu_batch.py", "test_gpu_devplan.py", "test_gpu_configs.py")


@pytest.mark.parametrize("settings", [
    {"HTRIP_QUERY_DATAFLOW": "0"},                                   # grid barriers
    {"HTRIP_QUERY_ROOT_SPLIT": "3"},                                 # root items in 3 uneven parts
    {"HTRIP_QUERY_DATAFLOW": "0", "HTRIP_QUERY_ROOT_SPLIT": "2"},    # parts under grid barriers
], ids=["barrier", "split3", "barrier-split2"])
def test_query_suites_under_schedule(gpu, settings):
    env = dict(os.environ, **settings)
    files = [os.path.join(ROOT, "tests", f) for f in SUITES]
    r = subprocess.run([sys.executable, "-m", "pytest", *files, "-q", "-x", "-p", "no:cacheprovider",
                        "-k", "not planned_on_the_device"], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
