"""Python mirror of ``htrip::MinPlusOracle`` over the C ABI (include/htrip_b200.h).

Same names, argument meaning and error behaviour as the reference class
(include/htrip/minplus_oracle.hpp):

* ``MinPlusOracle(HierarchyConfig)``                       minplus_oracle.hpp:59
* ``build(grid) -> bool``       False on an invalid config / empty grid  :78
* ``onCellOpened(p, grid)``                                              :109
* ``onBatchCellsOpened(cells, grid)``                                    :171
* ``queryAllPairs(vps, grid, out=None, scratch=None) -> (k, k) uint16``  :337-348
* ``depth()``, ``totalMemoryBytes()``, ``last_batch_stats``, ``S``, ``H``

The index lives in HBM on one CUDA device.  There is no CPU fallback: if the
CUDA library cannot be loaded or no device is present, construction raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import build as _build

INF = 60000

_U8P = C.POINTER(C.c_uint8)
_U16P = C.POINTER(C.c_uint16)
_OBSTACLE = 2  # CellState::Obstacle (types.hpp)
_I32P = C.POINTER(C.c_int32)
_U64P = C.POINTER(C.c_uint64)


class HtripError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"htrip status {status}: {msg}")
        self.status = status


class _Config(C.Structure):
    _fields_ = [("tile_size_b", C.c_int32), ("group", C.c_int32)]


class _QueryRequest(C.Structure):
    _fields_ = [("index", C.c_void_p), ("vps", _I32P), ("k", C.c_int32), ("observed", _U8P),
                ("rows", C.c_int32), ("cols", C.c_int32), ("out", _U16P)]


class _OpenRequest(C.Structure):
    _fields_ = [("index", C.c_void_p), ("rc", _I32P), ("n", C.c_int32), ("observed", _U8P),
                ("rows", C.c_int32), ("cols", C.c_int32)]


class _ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("hbm_budget_bytes", C.c_uint64), ("max_requests_per_launch", C.c_int32),
                ("plain_per_call", C.c_int32), ("double_buffer", C.c_int32)]


class _ServerStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "launches_query", "launches_open", "requests_query", "requests_open", "evictions", "restores",
        "sessions", "resident_sessions", "resident_bytes", "budget_bytes", "busy_query_us", "busy_open_us")]


class _ServerRequest(C.Structure):
    _fields_ = [("session", C.c_int64), ("kind", C.c_int32), ("rc", _I32P), ("n", C.c_int32), ("out", _U16P)]


class _Stats(C.Structure):
    _fields_ = [("n_touched_leaves", C.c_int32), ("n_dirty_ancestors", C.c_int32), ("n_pivots", C.c_int32)]


_lib = None

EXPORTS = (
    "htrip_last_error", "htrip_create", "htrip_destroy", "htrip_clone", "htrip_build", "htrip_open_cells",
    "htrip_open_cell", "htrip_query_all_pairs", "htrip_query_all_pairs_dev", "htrip_sync", "htrip_stream",
    "htrip_shape", "htrip_last_batch_stats", "htrip_memory_bytes", "htrip_read_leaf_D", "htrip_read_leaf_S",
    "htrip_read_node_DU", "htrip_read_node_SU", "htrip_read_node_C2E", "htrip_level_dims", "htrip_query_work",
    "htrip_last_query_kernel_ms", "htrip_last_query_io", "htrip_query_all_pairs_noalloc",
    "htrip_batch_create", "htrip_batch_destroy", "htrip_query_batch", "htrip_batch_last_kernel_ms",
    "htrip_state_digest", "htrip_open_batch", "htrip_offload", "htrip_restore", "htrip_is_resident",
    "htrip_estimate_bytes", "htrip_server_last_error", "htrip_server_create", "htrip_server_destroy",
    "htrip_server_add_session", "htrip_server_remove_session", "htrip_server_submit_query",
    "htrip_server_submit_open", "htrip_server_wait", "htrip_server_get_stats", "htrip_server_run_trace",
    "htrip_measure_minplus_rate", "htrip_last_query_phases", "htrip_batch_last_phases", "htrip_last_open_work",
    "htrip_autotune_query", "htrip_autotune_export", "htrip_autotune_import", "htrip_autotune_clear",
    "htrip_lift_root", "htrip_query_distance", "htrip_incremental_create", "htrip_incremental_destroy",
    "htrip_query_all_pairs_incremental", "htrip_batch_create_priority", "htrip_cell_blocked",
    "htrip_leaves_changed", "htrip_selftest_barrier_timeout", "htrip_selftest_wait_timeout", "htrip_set_cell_weights",
    "htrip_cell_weight_changed", "htrip_tile_weights_changed", "htrip_server_wait_version",
    "htrip_last_open_levels", "htrip_set_query_work_counting", "htrip_last_query_executed",
    "htrip_last_open_trace",
)


def load_library(path: str | None = None):
    """Load (and if needed build) libhtrip_b200.so and declare its C ABI."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or _build.LIB
    if not os.path.exists(path):
        _build.build()
    lib = C.CDLL(path)
    P = C.c_void_p
    I = C.c_int32
    lib.htrip_last_error.restype = C.c_char_p
    lib.htrip_create.argtypes = [_Config, C.c_int, C.POINTER(P)]
    lib.htrip_destroy.argtypes = [P]
    lib.htrip_clone.argtypes = [P, C.POINTER(P)]
    lib.htrip_build.argtypes = [P, _U8P, I, I]
    lib.htrip_open_cells.argtypes = [P, _I32P, I, _U8P, I, I]
    lib.htrip_open_cell.argtypes = [P, I, I, _U8P, I, I]
    lib.htrip_query_all_pairs.argtypes = [P, _I32P, I, _U8P, I, I, _U16P]
    lib.htrip_query_all_pairs_dev.argtypes = [P, C.c_void_p, C.c_void_p, I, C.c_void_p]
    lib.htrip_query_all_pairs_noalloc.argtypes = [P, _I32P, I, _U8P, I, I, _U16P]
    lib.htrip_sync.argtypes = [P]
    lib.htrip_stream.restype = C.c_void_p
    lib.htrip_stream.argtypes = [P]
    lib.htrip_shape.argtypes = [P, _I32P, _I32P, _I32P]
    lib.htrip_last_batch_stats.argtypes = [P, C.POINTER(_Stats)]
    lib.htrip_memory_bytes.argtypes = [P, _U64P, _U64P]
    for f in ("htrip_read_leaf_D", "htrip_read_leaf_S"):
        getattr(lib, f).argtypes = [P, I, _U16P]
    for f in ("htrip_read_node_DU", "htrip_read_node_SU"):
        getattr(lib, f).argtypes = [P, I, I, _U16P]
    lib.htrip_read_node_C2E.argtypes = [P, I, I, I, _U16P]
    lib.htrip_level_dims.argtypes = [P, I, _I32P, _I32P, _I32P, _I32P]
    lib.htrip_query_work.argtypes = [P, _I32P, I, _U8P, I, I, _U64P, _U64P]
    lib.htrip_last_query_kernel_ms.argtypes = [P, C.POINTER(C.c_float)]
    lib.htrip_last_query_io.argtypes = [P, _U64P, _U64P]
    lib.htrip_state_digest.argtypes = [P, _U64P, I]
    lib.htrip_batch_create.argtypes = [C.c_int, C.POINTER(P)]
    lib.htrip_batch_create_priority.argtypes = [C.c_int, I, C.POINTER(P)]
    lib.htrip_batch_destroy.argtypes = [P]
    lib.htrip_query_batch.argtypes = [P, C.POINTER(_QueryRequest), I]
    lib.htrip_batch_last_kernel_ms.argtypes = [P, C.POINTER(C.c_float)]
    lib.htrip_open_batch.argtypes = [P, C.POINTER(_OpenRequest), I]
    lib.htrip_measure_minplus_rate.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double)]
    lib.htrip_last_query_phases.argtypes = [P, _U64P, I, _I32P]
    lib.htrip_last_open_work.argtypes = [P, _U64P, _U64P]
    lib.htrip_last_open_levels.argtypes = [P, C.POINTER(C.c_int64), I, _I32P]
    lib.htrip_set_query_work_counting.argtypes = [P, I]
    lib.htrip_last_open_trace.argtypes = [P, _U64P, I, _I32P]
    lib.htrip_last_query_executed.argtypes = [P, _U64P, _U64P, _U64P]
    lib.htrip_autotune_query.argtypes = [P, _I32P, I, _U8P, I, I, I, _I32P, C.POINTER(C.c_float)]
    lib.htrip_autotune_export.argtypes = [C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]
    lib.htrip_autotune_import.argtypes = [C.c_char_p]
    lib.htrip_autotune_clear.argtypes = []
    lib.htrip_lift_root.argtypes = [P, _U8P, I, I]
    lib.htrip_cell_blocked.argtypes = [P, I, I, _U8P, I, I]
    lib.htrip_selftest_barrier_timeout.argtypes = [C.c_int, _I32P, _I32P, C.POINTER(C.c_float)]
    lib.htrip_selftest_wait_timeout.argtypes = [C.c_int, _I32P, _I32P, C.POINTER(C.c_float)]
    lib.htrip_leaves_changed.argtypes = [P, _I32P, I, _U8P, I, I]
    lib.htrip_set_cell_weights.argtypes = [P, _U16P, I, I]
    lib.htrip_cell_weight_changed.argtypes = [P, I, I, C.c_uint16, _U8P, I, I]
    lib.htrip_tile_weights_changed.argtypes = [P, I, I, _I32P, _U16P, I, _U8P, I, I]
    lib.htrip_query_distance.argtypes = [P, I, I, I, I, _U8P, I, I, _U16P]
    lib.htrip_incremental_create.argtypes = [C.POINTER(P)]
    lib.htrip_incremental_destroy.argtypes = [P]
    lib.htrip_query_all_pairs_incremental.argtypes = [P, P, _I32P, I, _U8P, I, I, _U16P, _I32P]
    lib.htrip_batch_last_phases.argtypes = [P, _U64P, I, _I32P]
    lib.htrip_offload.argtypes = [P]
    lib.htrip_restore.argtypes = [P]
    lib.htrip_is_resident.argtypes = [P, _I32P]
    lib.htrip_estimate_bytes.argtypes = [_Config, I, I, _U64P]
    lib.htrip_server_last_error.restype = C.c_char_p
    lib.htrip_server_create.argtypes = [C.POINTER(_ServerConfig), C.POINTER(P)]
    lib.htrip_server_destroy.argtypes = [P]
    lib.htrip_server_add_session.argtypes = [P, _Config, _U8P, I, I, C.POINTER(C.c_int64)]
    lib.htrip_server_remove_session.argtypes = [P, C.c_int64]
    lib.htrip_server_submit_query.argtypes = [P, C.c_int64, _I32P, I, _U16P, _U64P]
    lib.htrip_server_submit_open.argtypes = [P, C.c_int64, _I32P, I, _U64P]
    lib.htrip_server_wait.argtypes = [P, C.c_uint64, C.POINTER(C.c_double)]
    lib.htrip_server_wait_version.argtypes = [P, C.c_uint64, C.POINTER(C.c_double), _U64P]
    lib.htrip_server_get_stats.argtypes = [P, C.POINTER(_ServerStats)]
    lib.htrip_server_run_trace.argtypes = [P, C.POINTER(_ServerRequest), C.POINTER(C.c_double), I,
                                           C.POINTER(C.c_double), C.POINTER(C.c_double)]
    for f in EXPORTS:
        if f not in ("htrip_last_error", "htrip_stream", "htrip_server_last_error"):
            getattr(lib, f).restype = C.c_int
    _lib = lib
    return lib


def _check(status: int):
    if status != 0:
        raise HtripError(status, _lib.htrip_last_error().decode())


def _check_server(status: int):
    if status != 0:
        raise HtripError(status, _lib.htrip_server_last_error().decode())


@dataclass
class HierarchyConfig:
    """Reference HierarchyConfig (include/htrip/types.hpp:199-225)."""
    tile_size_b: int = 16
    group_w: int = 2
    group_h: int = 2
    hybrid_k_threshold: int = 0

    def isValid(self) -> bool:
        return (self.tile_size_b > 0 and self.group_w >= 2 and self.group_h >= 2
                and self.group_w == self.group_h and self.group_w * self.group_h <= 256)


class GridMap:
    """Occupancy grid: ``observed`` is a (rows, cols) uint8 CellState array;
    ``weights`` the optional (rows, cols) uint16 traversal weights (None:
    every weight 1), as the reference's GridMap::weights."""

    def __init__(self, observed: np.ndarray, weights: np.ndarray | None = None):
        self.observed = np.ascontiguousarray(observed, dtype=np.uint8)
        self.weights = None if weights is None else np.ascontiguousarray(weights, dtype=np.uint16)

    def hasWeights(self) -> bool:
        return self.weights is not None

    @property
    def rows(self):
        return self.observed.shape[0]

    @property
    def cols(self):
        return self.observed.shape[1]

    def isPassable(self, r: int, c: int) -> bool:
        return 0 <= r < self.rows and 0 <= c < self.cols and self.observed[r, c] == 1

    def setObserved(self, r: int, c: int, state: int):
        if 0 <= r < self.rows and 0 <= c < self.cols:
            self.observed[r, c] = state


@dataclass
class LastBatchStats:
    n_touched_leaves: int = 0
    n_dirty_ancestors: int = 0
    n_pivots: int = 0


def _grid_args(grid):
    obs = grid.observed if isinstance(grid, GridMap) else np.ascontiguousarray(grid, dtype=np.uint8)
    return obs, obs.ctypes.data_as(_U8P), obs.shape[0], obs.shape[1]


def _own_weights(grid, weights, rows, cols):
    """The caller's weights array a weight change writes into: the explicit
    one, else a GridMap's (created with every weight 1 on first use, as
    GridMap::setCellWeight does)."""
    if weights is None and isinstance(grid, GridMap):
        if grid.weights is None:
            grid.weights = np.ones((rows, cols), dtype=np.uint16)
        return grid.weights
    return weights


def _grid_weights(grid, weights):
    """The weights of a call: the explicit ones, else a GridMap's own."""
    if weights is None and isinstance(grid, GridMap):
        return grid.weights
    return weights


def _rc(pts) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(pts, dtype=np.int32).reshape(-1, 2))


class MinPlusOracle:
    """B200-resident HTRIP index with the reference's MinPlusOracle interface."""

    def __init__(self, config: HierarchyConfig | None = None, device: int = 0, _handle=None):
        self.lib = load_library()
        self.config = config or HierarchyConfig()
        self.device = device
        if _handle is not None:
            self.h = _handle
        else:
            h = C.c_void_p()
            cfg = _Config(self.config.tile_size_b, self.config.group_w)
            _check(self.lib.htrip_create(cfg, device, C.byref(h)))
            self.h = h
        self.last_batch_stats = LastBatchStats()

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.htrip_destroy(h)
            self.h = None

    def clone(self) -> "MinPlusOracle":
        h = C.c_void_p()
        _check(self.lib.htrip_clone(self.h, C.byref(h)))
        o = MinPlusOracle(self.config, self.device, _handle=h)
        o.last_batch_stats = LastBatchStats(**vars(self.last_batch_stats))
        return o

    # -- build ------------------------------------------------------------
    def setCellWeights(self, weights=None):
        """Per-cell traversal weights (uint16, the grid's shape; None: every
        weight 1), the reference's GridMap::weights; build and liftRoot set
        them from their `weights` argument."""
        if weights is None:
            _check(self.lib.htrip_set_cell_weights(self.h, None, 0, 0))
            return
        w = np.ascontiguousarray(weights, dtype=np.uint16)
        self._weights_keep = w
        _check(self.lib.htrip_set_cell_weights(self.h, w.ctypes.data_as(_U16P), w.shape[0], w.shape[1]))

    def build(self, grid, weights=None) -> bool:
        """Reference build(grid); `weights` plays the grid's weights (None:
        an unweighted grid)."""
        if not self.config.isValid():
            return False
        self.setCellWeights(_grid_weights(grid, weights))
        obs, ptr, rows, cols = _grid_args(grid)
        st = self.lib.htrip_build(self.h, ptr, rows, cols)
        if st == 1:  # HTRIP_ERR_INVALID: the reference returns false
            return False
        _check(st)
        return True

    def depth(self) -> int:
        return self.H

    @property
    def S(self) -> int:
        return self._shape()[0]

    @property
    def H(self) -> int:
        return self._shape()[1]

    @property
    def num_leaf_tiles_x(self) -> int:
        return self._shape()[2]

    num_leaf_tiles_y = num_leaf_tiles_x

    def _shape(self):
        s, h, lx = C.c_int32(), C.c_int32(), C.c_int32()
        _check(self.lib.htrip_shape(self.h, C.byref(s), C.byref(h), C.byref(lx)))
        return s.value, h.value, lx.value

    # -- updates ----------------------------------------------------------
    def onBatchCellsOpened(self, cells, grid):
        rc = _rc(cells)
        obs, ptr, rows, cols = _grid_args(grid)
        _check(self.lib.htrip_open_cells(self.h, rc.ctypes.data_as(_I32P), len(rc), ptr, rows, cols))
        self._refresh_stats()

    def _refresh_stats(self):
        st = _Stats()
        _check(self.lib.htrip_last_batch_stats(self.h, C.byref(st)))
        self.last_batch_stats = LastBatchStats(st.n_touched_leaves, st.n_dirty_ancestors, st.n_pivots)

    def onCellOpened(self, p, grid):
        obs, ptr, rows, cols = _grid_args(grid)
        _check(self.lib.htrip_open_cell(self.h, int(p[0]), int(p[1]), ptr, rows, cols))

    def onCellBlocked(self, p, grid):
        """Reference onCellBlocked (the caller has made p non-Free in grid)."""
        obs, ptr, rows, cols = _grid_args(grid)
        _check(self.lib.htrip_cell_blocked(self.h, int(p[0]), int(p[1]), ptr, rows, cols))

    def onBatchLeavesChanged(self, leaf_indices, grid):
        """Reference onBatchLeavesChanged: rebuild these leaves and their ancestors."""
        li = np.ascontiguousarray(np.asarray(leaf_indices, dtype=np.int32).ravel())
        obs, ptr, rows, cols = _grid_args(grid)
        _check(self.lib.htrip_leaves_changed(self.h, li.ctypes.data_as(_I32P), len(li), ptr, rows, cols))

    def liftRoot(self, grid=None, weights=None):
        """Grow the index to S*g, H+1 (reference liftRoot); grid None = the
        reference's default empty GridMap; `weights` as in build."""
        self.setCellWeights(_grid_weights(grid, weights))
        if grid is None:
            _check(self.lib.htrip_lift_root(self.h, None, 0, 0))
            return
        obs, ptr, rows, cols = _grid_args(grid)
        _check(self.lib.htrip_lift_root(self.h, ptr, rows, cols))

    def onCellWeightChanged(self, p, new_weight, grid, weights=None):
        """Reference onCellWeightChanged: cell p's weight becomes new_weight
        (also written into `weights`, the caller's array, when given) and its
        leaf and ancestors are rebuilt."""
        obs, ptr, rows, cols = _grid_args(grid)
        r, c = int(p[0]), int(p[1])
        weights = _own_weights(grid, weights, rows, cols)
        if weights is not None and 0 <= r < rows and 0 <= c < cols:
            cur = 60000 if obs.reshape(rows, cols)[r, c] == _OBSTACLE else int(weights[r, c])  # getCellWeight
            if cur != int(new_weight):
                weights[r, c] = new_weight
        _check(self.lib.htrip_cell_weight_changed(self.h, r, c, int(new_weight), ptr, rows, cols))

    def onTileWeightsChanged(self, tx, ty, cell_weights, grid, weights=None):
        """Reference onTileWeightsChanged: cell_weights = [((r, c), w), ...];
        leaf (tx, ty) and its ancestors are rebuilt once."""
        rc = _rc([p for p, _ in cell_weights]) if cell_weights else np.zeros((0, 2), np.int32)
        ws = np.ascontiguousarray([int(w) for _, w in cell_weights], dtype=np.uint16)
        obs, ptr, rows, cols = _grid_args(grid)
        weights = _own_weights(grid, weights, rows, cols)
        if weights is not None:
            for (r, c), w in cell_weights:
                if 0 <= r < rows and 0 <= c < cols:
                    weights[r, c] = w
        _check(self.lib.htrip_tile_weights_changed(self.h, int(tx), int(ty), rc.ctypes.data_as(_I32P),
                                                   ws.ctypes.data_as(_U16P), len(ws), ptr, rows, cols))

    # -- queries ----------------------------------------------------------
    def queryAllPairs(self, viewpoints, grid, out: np.ndarray | None = None, scratch=None) -> np.ndarray:
        rc = _rc(viewpoints)
        k = len(rc)
        if out is None or out.shape != (k, k) or out.dtype != np.uint16 or not out.flags.c_contiguous:
            out = np.empty((k, k), dtype=np.uint16)
        if k == 0:
            return out
        obs, ptr, rows, cols = _grid_args(grid)
        _check(self.lib.htrip_query_all_pairs(self.h, rc.ctypes.data_as(_I32P), k, ptr, rows, cols,
                                              out.ctypes.data_as(_U16P)))
        return out

    def queryDistance(self, s, t, grid) -> int:
        """Reference queryDistance (minplus_oracle.hpp:312)."""
        obs, ptr, rows, cols = _grid_args(grid)
        out = C.c_uint16()
        _check(self.lib.htrip_query_distance(self.h, int(s[0]), int(s[1]), int(t[0]), int(t[1]), ptr, rows, cols,
                                             C.byref(out)))
        return out.value

    def queryAllPairsIncremental(self, viewpoints, grid, state: "IncrementalState",
                                 out: np.ndarray | None = None) -> np.ndarray:
        """Reference queryAllPairsIncremental: the cached matrix when nothing
        changed since `state` was filled; after openings only, a re-lift of
        the viewpoints whose leaf-to-root chain changed; else a full query.
        state.last_mode: 0 cached, 1 full query, 2 re-lift of the changed
        viewpoints (state.last_recomputed: mode != 0)."""
        rc = _rc(viewpoints)
        k = len(rc)
        if out is None or out.shape != (k, k) or out.dtype != np.uint16 or not out.flags.c_contiguous:
            out = np.empty((k, k), dtype=np.uint16)
        obs, ptr, rows, cols = _grid_args(grid)
        rec = C.c_int32()
        _check(self.lib.htrip_query_all_pairs_incremental(self.h, state.h, rc.ctypes.data_as(_I32P), k, ptr, rows,
                                                          cols, out.ctypes.data_as(_U16P), C.byref(rec)))
        state.last_mode = int(rec.value)
        state.last_recomputed = rec.value != 0
        return out

    def queryAllPairsNoAlloc(self, viewpoints, grid, out: np.ndarray | None = None) -> np.ndarray:
        """queryAllPairs through htrip_query_all_pairs_noalloc: the device
        scratch comes from the library's fixed 64 MiB array, nothing is
        allocated on the device (for callers that may not allocate)."""
        rc = _rc(viewpoints)
        k = len(rc)
        if out is None or out.shape != (k, k) or out.dtype != np.uint16 or not out.flags.c_contiguous:
            out = np.empty((k, k), dtype=np.uint16)
        if k == 0:
            return out
        obs, ptr, rows, cols = _grid_args(grid)
        _check(self.lib.htrip_query_all_pairs_noalloc(self.h, rc.ctypes.data_as(_I32P), k, ptr, rows, cols,
                                                      out.ctypes.data_as(_U16P)))
        return out

    def queryAllPairsDevice(self, vps_dev_ptr: int, passable_dev_ptr: int, k: int, out_dev_ptr: int):
        """Stream-ordered query on device-resident inputs (see htrip_query_all_pairs_dev)."""
        _check(self.lib.htrip_query_all_pairs_dev(self.h, C.c_void_p(vps_dev_ptr), C.c_void_p(passable_dev_ptr),
                                                  k, C.c_void_p(out_dev_ptr)))

    def queryWork(self, viewpoints, grid):
        """(algorithmic bytes, min-plus ops) of queryAllPairs on these viewpoints."""
        rc = _rc(viewpoints)
        obs, ptr, rows, cols = _grid_args(grid)
        b, o = C.c_uint64(), C.c_uint64()
        _check(self.lib.htrip_query_work(self.h, rc.ctypes.data_as(_I32P), len(rc), ptr, rows, cols,
                                         C.byref(b), C.byref(o)))
        return b.value, o.value

    def lastQueryKernelMs(self) -> float:
        ms = C.c_float()
        _check(self.lib.htrip_last_query_kernel_ms(self.h, C.byref(ms)))
        return ms.value

    def autotuneQuery(self, viewpoints, grid, reps: int = 5):
        """Time every query tile shape on this request; the fastest becomes the
        shape of its bucket (htrip_autotune_query).  Returns (cfg, ms)."""
        rc = _rc(viewpoints)
        obs, ptr, rows, cols = _grid_args(grid)
        cfg, ms = C.c_int32(), C.c_float()
        _check(self.lib.htrip_autotune_query(self.h, rc.ctypes.data_as(_I32P), len(rc), ptr, rows, cols, reps,
                                             C.byref(cfg), C.byref(ms)))
        return cfg.value, ms.value

    def lastOpenWork(self):
        """(algorithmic bytes, min-plus ops) of the last opening call."""
        b, o = C.c_uint64(), C.c_uint64()
        _check(self.lib.htrip_last_open_work(self.h, C.byref(b), C.byref(o)))
        return b.value, o.value

    def setQueryWorkCounting(self, on: bool):
        """Count the executed work of this index's query launches (a few atomics
        per work unit; off by default)."""
        _check(self.lib.htrip_set_query_work_counting(self.h, 1 if on else 0))

    def lastQueryExecuted(self):
        """(tile entries updated, operand rows streamed, rows skipped) of the
        last counted query launch (htrip_last_query_executed)."""
        e, r, s = C.c_uint64(), C.c_uint64(), C.c_uint64()
        _check(self.lib.htrip_last_query_executed(self.h, C.byref(e), C.byref(r), C.byref(s)))
        return e.value, r.value, s.value

    def lastOpenTrace(self):
        """Phase durations (ns) of the last device-driven opening launch."""
        buf = (C.c_uint64 * 1024)()
        n = C.c_int32()
        _check(self.lib.htrip_last_open_trace(self.h, buf, 1024, C.byref(n)))
        return [int(buf[i]) for i in range(min(n.value, 1024))]

    def lastOpenLevels(self):
        """Per level of the last opening call: (matrices, sum of pivots, largest
        pivot count, closure rounds) (htrip_last_open_levels)."""
        buf = (C.c_int64 * (4 * 32))()
        n = C.c_int32()
        _check(self.lib.htrip_last_open_levels(self.h, buf, 32, C.byref(n)))
        return [tuple(int(buf[4 * l + j]) for j in range(4)) for l in range(min(n.value, 32))]

    def lastQueryPhases(self):
        """Per-phase nanoseconds of the last query launch (htrip_last_query_phases)."""
        buf = (C.c_uint64 * 32)()
        n = C.c_int32()
        _check(self.lib.htrip_last_query_phases(self.h, buf, 32, C.byref(n)))
        return [int(buf[i]) for i in range(n.value)]

    def lastQueryIO(self):
        """(host->device, device->host) bytes copied by the last query call."""
        a, b = C.c_uint64(), C.c_uint64()
        _check(self.lib.htrip_last_query_io(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def stream(self) -> int:
        return int(self.lib.htrip_stream(self.h) or 0)

    def synchronize(self):
        _check(self.lib.htrip_sync(self.h))

    # -- accounting / state read-back ---------------------------------------
    def totalMemoryBytes(self) -> int:
        ref, dev = C.c_uint64(), C.c_uint64()
        _check(self.lib.htrip_memory_bytes(self.h, C.byref(ref), C.byref(dev)))
        return ref.value

    def deviceMemoryBytes(self) -> int:
        ref, dev = C.c_uint64(), C.c_uint64()
        _check(self.lib.htrip_memory_bytes(self.h, C.byref(ref), C.byref(dev)))
        return dev.value

    def offload(self):
        """Park the index in host memory and free its device memory (htrip_offload)."""
        _check(self.lib.htrip_offload(self.h))

    def restore(self):
        _check(self.lib.htrip_restore(self.h))

    def isResident(self) -> bool:
        r = C.c_int32()
        _check(self.lib.htrip_is_resident(self.h, C.byref(r)))
        return bool(r.value)

    def stateDigest(self):
        """Per-level checksum of every leaf D and node D_U (htrip_state_digest)."""
        n = self.H + 1
        out = (C.c_uint64 * n)()
        _check(self.lib.htrip_state_digest(self.h, out, n))
        return [int(x) for x in out]

    def level_dims(self, lvl: int):
        a = [C.c_int32() for _ in range(4)]
        _check(self.lib.htrip_level_dims(self.h, lvl, *[C.byref(x) for x in a]))
        return tuple(x.value for x in a)

    def leaf_D(self, i: int) -> np.ndarray:
        n = self.config.tile_size_b ** 2
        out = np.empty((n, n), dtype=np.uint16)
        _check(self.lib.htrip_read_leaf_D(self.h, i, out.ctypes.data_as(_U16P)))
        return out

    def leaf_S(self, i: int) -> np.ndarray:
        p = 4 * self.config.tile_size_b - 4
        out = np.empty((p, p), dtype=np.uint16)
        _check(self.lib.htrip_read_leaf_S(self.h, i, out.ctypes.data_as(_U16P)))
        return out

    def node_DU(self, lvl: int, node: int) -> np.ndarray:
        n = self.level_dims(lvl)[0]
        out = np.empty((n, n), dtype=np.uint16)
        _check(self.lib.htrip_read_node_DU(self.h, lvl, node, out.ctypes.data_as(_U16P)))
        return out

    def node_SU(self, lvl: int, node: int) -> np.ndarray:
        ne = self.level_dims(lvl)[1]
        out = np.empty((ne, ne), dtype=np.uint16)
        _check(self.lib.htrip_read_node_SU(self.h, lvl, node, out.ctypes.data_as(_U16P)))
        return out

    def node_C2E(self, lvl: int, node: int, quad: int) -> np.ndarray:
        n, ne, np_, _ = self.level_dims(lvl)
        out = np.empty(np_ * ne, dtype=np.uint16)
        _check(self.lib.htrip_read_node_C2E(self.h, lvl, node, quad, out.ctypes.data_as(_U16P)))
        return out


HTripOracle = MinPlusOracle


class IncrementalState:
    """Reference HTripIncrementalState (cache of the last incremental query)."""

    def __init__(self):
        self.lib = load_library()
        h = C.c_void_p()
        _check(self.lib.htrip_incremental_create(C.byref(h)))
        self.h = h
        self.last_recomputed = False
        self.last_mode = 0

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.htrip_incremental_destroy(h)
            self.h = None


class Batch:
    """Batched calls over many indexes of one device (htrip_batch_*).

    ``query([(oracle, viewpoints, grid), ...])`` answers every request in one
    launch of the persistent query kernel; each (k, k) result equals the
    oracle's own ``queryAllPairs`` of that request."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        self.device = device
        h = C.c_void_p()
        _check(self.lib.htrip_batch_create(device, C.byref(h)))
        self.h = h

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.htrip_batch_destroy(h)
            self.h = None

    def query(self, requests):
        reqs = (_QueryRequest * max(1, len(requests)))()
        keep, outs = [], []
        for i, (oracle, vps, grid) in enumerate(requests):
            rc = _rc(vps)
            obs, ptr, rows, cols = _grid_args(grid)
            out = np.empty((len(rc), len(rc)), dtype=np.uint16)
            keep += [rc, obs]
            outs.append(out)
            reqs[i] = _QueryRequest(oracle.h, rc.ctypes.data_as(_I32P), len(rc), ptr, rows, cols,
                                    out.ctypes.data_as(_U16P))
        _check(self.lib.htrip_query_batch(self.h, reqs, len(requests)))
        return outs

    def open(self, requests):
        """onBatchCellsOpened of every (oracle, cells, grid) request; each
        oracle's last_batch_stats is refreshed."""
        reqs = (_OpenRequest * max(1, len(requests)))()
        keep = []
        for i, (oracle, cells, grid) in enumerate(requests):
            rc = _rc(cells)
            obs, ptr, rows, cols = _grid_args(grid)
            keep += [rc, obs]
            reqs[i] = _OpenRequest(oracle.h, rc.ctypes.data_as(_I32P), len(rc), ptr, rows, cols)
        _check(self.lib.htrip_open_batch(self.h, reqs, len(requests)))
        for oracle, _, _ in requests:
            oracle._refresh_stats()

    def lastKernelMs(self) -> float:
        ms = C.c_float()
        _check(self.lib.htrip_batch_last_kernel_ms(self.h, C.byref(ms)))
        return ms.value

    def lastPhases(self):
        buf = (C.c_uint64 * 32)()
        n = C.c_int32()
        _check(self.lib.htrip_batch_last_phases(self.h, buf, 32, C.byref(n)))
        return [int(buf[i]) for i in range(n.value)]



def autotune_export() -> str:
    """The tuning table as text lines "H NP log2_k log2_group cfg"."""
    lib = load_library()
    n = C.c_size_t()
    _check(lib.htrip_autotune_export(None, 0, C.byref(n)))
    buf = C.create_string_buffer(n.value + 1)
    _check(lib.htrip_autotune_export(buf, n.value + 1, C.byref(n)))
    return buf.value.decode()


def autotune_import(text: str):
    _check(load_library().htrip_autotune_import(text.encode()))


def autotune_clear():
    _check(load_library().htrip_autotune_clear())


def selftest_barrier_timeout(device: int = 0):
    """(status, CTAs returned, ms) of a grid barrier that cannot complete."""
    lib = load_library()
    st, ret, ms = C.c_int32(), C.c_int32(), C.c_float()
    _check(lib.htrip_selftest_barrier_timeout(device, C.byref(st), C.byref(ret), C.byref(ms)))
    return st.value, ret.value, ms.value


def selftest_wait_timeout(device: int = 0):
    """(status, CTAs returned, ms) of completion-counter waits that cannot be satisfied."""
    lib = load_library()
    st, ret, ms = C.c_int32(), C.c_int32(), C.c_float()
    _check(lib.htrip_selftest_wait_timeout(device, C.byref(st), C.byref(ret), C.byref(ms)))
    return st.value, ret.value, ms.value


def minplus_rate(device: int = 0, variant: int = 0) -> float:
    """Measured register-only packed-u16 min-plus rate (entries/s) of the device."""
    lib = load_library()
    out = C.c_double()
    _check(lib.htrip_measure_minplus_rate(device, variant, C.byref(out)))
    return out.value


def estimate_bytes(config: HierarchyConfig, rows: int, cols: int) -> int:
    """Device bytes an index of this config and grid holds after build."""
    lib = load_library()
    out = C.c_uint64()
    _check(lib.htrip_estimate_bytes(_Config(config.tile_size_b, config.group_w), rows, cols, C.byref(out)))
    return out.value


class Server:
    """Request server over many resident map sessions (htrip_server_*)."""

    QUERY, OPEN = 0, 1

    def __init__(self, device: int = 0, budget_bytes: int = 0, max_per_launch: int = 0, plain: bool = False,
                 double_buffer: bool = False):
        self.lib = load_library()
        h = C.c_void_p()
        cfg = _ServerConfig(device, budget_bytes, max_per_launch, 1 if plain else 0, 1 if double_buffer else 0)
        _check_server(self.lib.htrip_server_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self._pending = {}

    def close(self):
        h = getattr(self, "h", None)
        if h:
            self.lib.htrip_server_destroy(h)
            self.h = None

    __del__ = close

    def add_session(self, config: HierarchyConfig, grid) -> int:
        obs, ptr, rows, cols = _grid_args(grid)
        sid = C.c_int64()
        _check_server(self.lib.htrip_server_add_session(self.h, _Config(config.tile_size_b, config.group_w), ptr,
                                                        rows, cols, C.byref(sid)))
        return sid.value

    def remove_session(self, sid: int):
        _check_server(self.lib.htrip_server_remove_session(self.h, sid))

    def submit_query(self, sid: int, vps):
        rc = _rc(vps)
        out = np.empty((len(rc), len(rc)), dtype=np.uint16)
        t = C.c_uint64()
        _check_server(self.lib.htrip_server_submit_query(self.h, sid, rc.ctypes.data_as(_I32P), len(rc),
                                                         out.ctypes.data_as(_U16P), C.byref(t)))
        self._pending[t.value] = (rc, out)
        return t.value, out

    def submit_open(self, sid: int, cells):
        rc = _rc(cells)
        t = C.c_uint64()
        _check_server(self.lib.htrip_server_submit_open(self.h, sid, rc.ctypes.data_as(_I32P), len(rc), C.byref(t)))
        self._pending[t.value] = (rc, None)
        return t.value

    def wait(self, ticket: int) -> float:
        lat = C.c_double()
        try:
            _check_server(self.lib.htrip_server_wait(self.h, ticket, C.byref(lat)))
        finally:
            self._pending.pop(ticket, None)
        return lat.value

    def wait_version(self, ticket: int):
        """(latency ms, version): for a query the number of the session's
        openings its result includes, for an opening its own number."""
        lat, ver = C.c_double(), C.c_uint64()
        try:
            _check_server(self.lib.htrip_server_wait_version(self.h, ticket, C.byref(lat), C.byref(ver)))
        finally:
            self._pending.pop(ticket, None)
        return lat.value, ver.value

    def stats(self) -> dict:
        st = _ServerStats()
        _check_server(self.lib.htrip_server_get_stats(self.h, C.byref(st)))
        return {n: getattr(st, n) for n, _ in _ServerStats._fields_}

    def run_trace(self, requests, arrival_s):
        """requests: list of (session, kind, rc); open-loop submission at
        arrival_s[i] seconds.  Returns (outs, latency_ms array, wall_s);
        outs[i] is the (k, k) matrix of a query, None for an opening."""
        n = len(requests)
        arr = (_ServerRequest * max(1, n))()
        keep, outs = [], []
        for i, (sid, kind, rc) in enumerate(requests):
            rc = _rc(rc)
            out = np.empty((len(rc), len(rc)), dtype=np.uint16) if kind == self.QUERY else None
            keep.append(rc)
            outs.append(out)
            arr[i] = _ServerRequest(sid, kind, rc.ctypes.data_as(_I32P), len(rc),
                                    out.ctypes.data_as(_U16P) if out is not None else None)
        t = np.ascontiguousarray(arrival_s, dtype=np.float64)
        lat = np.empty(n, dtype=np.float64)
        wall = C.c_double()
        _check_server(self.lib.htrip_server_run_trace(self.h, arr, t.ctypes.data_as(C.POINTER(C.c_double)), n,
                                                      lat.ctypes.data_as(C.POINTER(C.c_double)), C.byref(wall)))
        return outs, lat, wall.value
