"""The C++20 drop-in (include/htrip/minplus_oracle.hpp, libhtrip.so).

tests/cpp/test_dropin.cpp is a C++ test executable in the style of the
reference's apps/test_*.cpp: it drives htrip::MinPlusOracle through its public
API and checks every matrix bit-exactly against the plain-C oracle in
oracle/ (BFS all-pairs and the min-plus hierarchy), exiting non-zero on any
mismatch.  Without a GPU it runs its host-only checks.
"""
import os
import subprocess

import pytest

from htrip_b200 import build as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_dropin.cpp")
ORACLE = os.path.join(ROOT, "oracle")


def _compile(tmp_path):
    B.build()
    subprocess.run(["make", "-s", "-C", ORACLE, "port"], check=True)
    exe = str(tmp_path / "test_dropin")
    cmd = [os.environ.get("CXX", "g++"), "-std=c++20", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"),
           "-I" + ORACLE, SRC, "-o", exe,
           "-L" + B.PKG, "-lhtrip", "-lhtrip_b200", "-Wl,-rpath," + B.PKG,
           "-L" + os.path.join(ORACLE, "_build"), "-loracle_port", "-Wl,-rpath," + os.path.join(ORACLE, "_build")]
    subprocess.run(cmd, check=True)
    return exe


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_dropin_compiles_and_host_checks(tmp_path):
    exe = _compile(tmp_path)
    if _has_gpu():
        pytest.skip("host-only mode checks the no-device error path; a GPU is present")
    r = subprocess.run([exe, "--no-device"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
def test_dropin_suite_on_device(gpu, tmp_path):
    exe = _compile(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "drop-in suite passed" in r.stdout
