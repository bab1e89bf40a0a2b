"""The C ABI library loads and exports every symbol include/htrip_b200.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

from htrip_b200 import build as B
from htrip_b200.minplus_oracle import EXPORTS

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "htrip_b200.h")


def declared():
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)  # drop comments
    return sorted(set(re.findall(r"\b(htrip_[A-Za-z0-9_]+)\s*\(", src)))


def test_library_builds_and_exports_header_symbols():
    lib = ctypes.CDLL(B.build())
    names = declared()
    assert names, "no declarations found"
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(EXPORTS)


def test_last_error_callable_without_device():
    lib = ctypes.CDLL(B.build())
    lib.htrip_last_error.restype = ctypes.c_char_p
    assert isinstance(lib.htrip_last_error(), bytes)


def test_no_cpu_fallback_without_a_device():
    """Without a GPU an index cannot be made and smoke() fails: there is no CPU path."""
    import pytest

    import __graft_entry__
    from htrip_b200.minplus_oracle import HierarchyConfig, HtripError, MinPlusOracle
    try:
        MinPlusOracle(HierarchyConfig(8, 2, 2))
    except HtripError as e:
        assert "no CUDA device" in str(e)
    else:
        pytest.skip("a GPU is present")
    with pytest.raises(HtripError, match="no CUDA device"):
        __graft_entry__.smoke()
