"""Query tile autotuning with a file cache.

The query kernel has several tile shapes (viewpoint rows x columns per CTA
item).  ``tune`` times each shape on sample requests of an index and records
the fastest for the request's bucket (depth, root matrix order, log2 of the
viewpoint count, log2 of the largest root child group) in the library's
process-wide table; ``save`` / ``load`` keep the table in a text file so a
service tunes once per GPU type and reuses the choice at start-up.
"""
from __future__ import annotations

import os

from .minplus_oracle import autotune_clear, autotune_export, autotune_import


def tune(oracle, samples, reps: int = 5):
    """samples: iterable of (viewpoints, grid).  Returns [(cfg, ms), ...]."""
    return [oracle.autotuneQuery(vps, grid, reps) for vps, grid in samples]


def save(path: str):
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        f.write(autotune_export())
    os.replace(tmp, path)


def load(path: str) -> bool:
    """Merge a saved table into the process's table; False if there is no file."""
    if not os.path.exists(path):
        return False
    with open(path) as f:
        autotune_import(f.read())
    return True


def clear():
    autotune_clear()
