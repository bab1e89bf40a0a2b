"""The autotuner's table import / export (host logic; no GPU needed)."""
import pytest

from htrip_b200 import autotune
from htrip_b200.minplus_oracle import HtripError, autotune_clear, autotune_export, autotune_import


def test_import_export_round_trip(tmp_path):
    autotune_clear()
    autotune_import("5 4096 8 6 2\n7 8192 6 4 1\n")
    text = autotune_export()
    assert sorted(text.strip().splitlines()) == ["5 4096 8 6 2", "7 8192 6 4 1"]
    path = str(tmp_path / "tune.txt")
    autotune.save(path)
    autotune_clear()
    assert autotune_export() == ""
    assert autotune.load(path)
    assert sorted(autotune_export().strip().splitlines()) == ["5 4096 8 6 2", "7 8192 6 4 1"]
    autotune_import("5 4096 8 6 0\n")          # a later entry replaces the bucket's choice
    assert "5 4096 8 6 0" in autotune_export()
    assert not autotune.load(str(tmp_path / "missing.txt"))
    autotune_clear()


@pytest.mark.parametrize("bad", ["5 4096 8 6\n", "a b c d e\n", "5 4096 8 6 9\n", "5 4096 8 6 -1\n"])
def test_malformed_tables_are_refused(bad):
    autotune_clear()
    with pytest.raises(HtripError):
        autotune_import(bad)
    assert autotune_export() == ""
