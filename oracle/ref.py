"""ctypes bindings to the CPU checkers (TEST INFRASTRUCTURE ONLY).

* ``RefOracle``  - the unmodified reference ``htrip::MinPlusOracle`` and
  ``htrip::BfsOracle`` (oracle/_ref/libhtrip_ref.so, built by oracle/Makefile
  from the reference sources).
* ``PortOracle`` - the plain-C restatement of the same algorithm
  (oracle/_build/liboracle_port.so, built from oracle/htrip_oracle.c).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arm import this module.  The product (htrip_b200) never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libhtrip_ref.so")
PORT_SO = os.path.join(HERE, "_build", "liboracle_port.so")

_P = C.c_void_p
_I = C.c_int
_U8P = C.POINTER(C.c_uint8)
_U16P = C.POINTER(C.c_uint16)
_I32P = C.POINTER(C.c_int32)


def _p(a, t):
    return a.ctypes.data_as(t)


def _rc(pts) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(pts, dtype=np.int32).reshape(-1, 2))


_ref_lib = None


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def _load_ref():
    global _ref_lib
    if _ref_lib is None:
        lib = C.CDLL(REF_SO)
        lib.ref_create.restype = _P
        lib.ref_create.argtypes = [_I, _I]
        lib.ref_destroy.argtypes = [_P]
        lib.ref_clone.restype = _P
        lib.ref_clone.argtypes = [_P]
        lib.ref_set_grid.argtypes = [_P, _U8P, _I, _I]
        lib.ref_set_cells.argtypes = [_P, _I32P, _I, _I]
        lib.ref_build.restype = _I
        lib.ref_build.argtypes = [_P]
        lib.ref_open_batch.argtypes = [_P, _I32P, _I]
        lib.ref_open_cell.argtypes = [_P, _I, _I]
        lib.ref_lift_root.argtypes = [_P]
        lib.ref_cell_blocked.argtypes = [_P, _I, _I]
        lib.ref_leaves_changed.argtypes = [_P, _I32P, _I]
        lib.ref_set_weights.argtypes = [_P, _U16P]
        lib.ref_cell_weight_changed.argtypes = [_P, _I, _I, _I]
        lib.ref_tile_weights_changed.argtypes = [_P, _I, _I, _I32P, _U16P, _I]
        lib.ref_dijkstra_all_pairs.argtypes = [_P, _I32P, _I, _U16P]
        lib.ref_query_distance.restype = _I
        lib.ref_query_distance.argtypes = [_P, _I, _I, _I, _I]
        lib.ref_query_incremental.argtypes = [_P, _I32P, _I, _U16P]
        lib.ref_query.argtypes = [_P, _I32P, _I, _U16P]
        lib.ref_time_query.restype = C.c_double
        lib.ref_time_query.argtypes = [_P, _I32P, _I, _I, _I, _U16P]
        lib.ref_bfs_all_pairs.argtypes = [_P, _I32P, _I, _U16P]
        for f in ("ref_S", "ref_H", "ref_num_leaves"):
            getattr(lib, f).restype = _I
            getattr(lib, f).argtypes = [_P]
        lib.ref_num_nodes.restype = _I
        lib.ref_num_nodes.argtypes = [_P, _I]
        lib.ref_total_memory.restype = C.c_ulonglong
        lib.ref_total_memory.argtypes = [_P]
        lib.ref_stats.argtypes = [_P, _I32P]
        lib.ref_leaf_D.restype = _I
        lib.ref_leaf_D.argtypes = [_P, _I, _U16P]
        lib.ref_leaf_S.restype = _I
        lib.ref_leaf_S.argtypes = [_P, _I, _U16P]
        lib.ref_node_DU.restype = _I
        lib.ref_node_DU.argtypes = [_P, _I, _I, _U16P]
        lib.ref_node_SU.restype = _I
        lib.ref_node_SU.argtypes = [_P, _I, _I, _U16P]
        lib.ref_digest.restype = _I
        lib.ref_digest.argtypes = [_P, C.POINTER(C.c_uint64)]
        lib.ref_node_C2E.restype = _I
        lib.ref_node_C2E.argtypes = [_P, _I, _I, _I, _U16P]
        lib.ref_node_geometry.restype = _I
        lib.ref_node_geometry.argtypes = [_P, _I, _I, _I32P, _I32P, _I32P]
        _ref_lib = lib
    return _ref_lib


class RefOracle:
    """The reference MinPlusOracle with its own GridMap copy."""

    def __init__(self, b: int, g: int = 2, _handle=None):
        self.lib = _load_ref()
        self.b, self.g = b, g
        self.h = _handle if _handle is not None else self.lib.ref_create(b, g)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_destroy(self.h)
            self.h = None

    def clone(self) -> "RefOracle":
        return RefOracle(self.b, self.g, _handle=self.lib.ref_clone(self.h))

    def set_grid(self, observed: np.ndarray):
        obs = np.ascontiguousarray(observed, dtype=np.uint8)
        self.rows, self.cols = obs.shape
        self.lib.ref_set_grid(self.h, _p(obs, _U8P), self.rows, self.cols)

    def set_cells(self, cells, state: int):
        rc = _rc(cells)
        self.lib.ref_set_cells(self.h, _p(rc, _I32P), len(rc), state)

    def build(self) -> bool:
        return bool(self.lib.ref_build(self.h))

    def open_batch(self, cells):
        rc = _rc(cells)
        self.lib.ref_open_batch(self.h, _p(rc, _I32P), len(rc))

    def open_cell(self, r: int, c: int):
        self.lib.ref_open_cell(self.h, r, c)

    def query_distance(self, s, t) -> int:
        return self.lib.ref_query_distance(self.h, int(s[0]), int(s[1]), int(t[0]), int(t[1]))

    def query_incremental(self, vps) -> np.ndarray:
        rc = _rc(vps)
        out = np.empty((len(rc), len(rc)), dtype=np.uint16)
        self.lib.ref_query_incremental(self.h, _p(rc, _I32P), len(rc), _p(out, _U16P))
        return out

    def cell_blocked(self, r: int, c: int):
        self.lib.ref_cell_blocked(self.h, int(r), int(c))

    def set_weights(self, weights):
        """The grid's traversal weights (rows x cols uint16) or None."""
        if weights is None:
            self.lib.ref_set_weights(self.h, None)
            return
        w = np.ascontiguousarray(weights, dtype=np.uint16)
        assert w.shape == (self.rows, self.cols)
        self.lib.ref_set_weights(self.h, _p(w, _U16P))

    def cell_weight_changed(self, r: int, c: int, w: int):
        self.lib.ref_cell_weight_changed(self.h, int(r), int(c), int(w))

    def tile_weights_changed(self, tx: int, ty: int, cells, weights):
        rc = _rc(cells)
        w = np.ascontiguousarray(weights, dtype=np.uint16)
        self.lib.ref_tile_weights_changed(self.h, int(tx), int(ty), _p(rc, _I32P), _p(w, _U16P), len(w))

    def dijkstra(self, vps) -> np.ndarray:
        """DijkstraOracle::queryAllPairs on the handle's grid."""
        rc = _rc(vps)
        out = np.empty((len(rc), len(rc)), dtype=np.uint16)
        self.lib.ref_dijkstra_all_pairs(self.h, _p(rc, _I32P), len(rc), _p(out, _U16P))
        return out

    def leaves_changed(self, leaves):
        li = np.ascontiguousarray(np.asarray(leaves, dtype=np.int32).ravel())
        self.lib.ref_leaves_changed(self.h, _p(li, _I32P), len(li))

    def lift_root(self):
        """MinPlusOracle::liftRoot with the handle's current grid."""
        self.lib.ref_lift_root(self.h)

    def query(self, vps) -> np.ndarray:
        rc = _rc(vps)
        out = np.empty((len(rc), len(rc)), dtype=np.uint16)
        self.lib.ref_query(self.h, _p(rc, _I32P), len(rc), _p(out, _U16P))
        return out

    def time_query(self, vps, nthreads: int, reps: int):
        rc = _rc(vps)
        out = np.empty((len(rc), len(rc)), dtype=np.uint16)
        sec = self.lib.ref_time_query(self.h, _p(rc, _I32P), len(rc), nthreads, reps, _p(out, _U16P))
        return sec, out

    def bfs(self, vps) -> np.ndarray:
        rc = _rc(vps)
        out = np.empty((len(rc), len(rc)), dtype=np.uint16)
        self.lib.ref_bfs_all_pairs(self.h, _p(rc, _I32P), len(rc), _p(out, _U16P))
        return out

    @property
    def S(self):
        return self.lib.ref_S(self.h)

    @property
    def H(self):
        return self.lib.ref_H(self.h)

    def num_leaves(self):
        return self.lib.ref_num_leaves(self.h)

    def num_nodes(self, lvl):
        return self.lib.ref_num_nodes(self.h, lvl)

    def total_memory(self):
        return int(self.lib.ref_total_memory(self.h))

    def stats(self):
        out = np.zeros(3, dtype=np.int32)
        self.lib.ref_stats(self.h, _p(out, _I32P))
        return tuple(int(x) for x in out)

    def digest(self):
        """Per-level checksum of leaves[m].D / levels[l][m].D_U (the device
        library's htrip_state_digest formula)."""
        out = (C.c_uint64 * 64)()
        n = self.lib.ref_digest(self.h, out)
        return [int(out[i]) for i in range(n)]

    def leaf_D(self, i):
        n = self.b * self.b
        out = np.empty((n, n), dtype=np.uint16)
        self.lib.ref_leaf_D(self.h, i, _p(out, _U16P))
        return out

    def leaf_S(self, i):
        p = 4 * self.b - 4
        out = np.empty((p, p), dtype=np.uint16)
        self.lib.ref_leaf_S(self.h, i, _p(out, _U16P))
        return out

    def node_DU(self, lvl, n):
        nv = self.lib.ref_node_DU(self.h, lvl, n, None)
        out = np.empty((nv, nv), dtype=np.uint16)
        self.lib.ref_node_DU(self.h, lvl, n, _p(out, _U16P))
        return out

    def node_SU(self, lvl, n):
        ne = self.lib.ref_node_SU(self.h, lvl, n, None)
        out = np.empty((ne, ne), dtype=np.uint16)
        self.lib.ref_node_SU(self.h, lvl, n, _p(out, _U16P))
        return out

    def node_C2E(self, lvl, n, q):
        cnt = self.lib.ref_node_C2E(self.h, lvl, n, q, None)
        out = np.empty(cnt, dtype=np.uint16)
        self.lib.ref_node_C2E(self.h, lvl, n, q, _p(out, _U16P))
        return out


_port_lib = None


def port_available() -> bool:
    return os.path.exists(PORT_SO)


def _load_port():
    global _port_lib
    if _port_lib is None:
        lib = C.CDLL(PORT_SO)
        lib.orc_create.restype = _P
        lib.orc_create.argtypes = [_I, _I]
        lib.orc_destroy.argtypes = [_P]
        lib.orc_build.restype = _I
        lib.orc_build.argtypes = [_P, _U8P, _I, _I]
        lib.orc_open_batch.argtypes = [_P, _I32P, _I, _U8P, _I, _I]
        lib.orc_query.argtypes = [_P, _I32P, _I, _U8P, _I, _I, _U16P]
        lib.orc_stats.argtypes = [_P, _I32P]
        lib.orc_S.restype = _I
        lib.orc_S.argtypes = [_P]
        lib.orc_H.restype = _I
        lib.orc_H.argtypes = [_P]
        lib.orc_leaf_D.restype = _I
        lib.orc_leaf_D.argtypes = [_P, _I, _U16P]
        lib.orc_node_DU.restype = _I
        lib.orc_node_DU.argtypes = [_P, _I, _I, _U16P]
        lib.orc_bfs_all_pairs.argtypes = [_U8P, _I, _I, _I32P, _I, _U16P]
        _port_lib = lib
    return _port_lib


class PortOracle:
    """The plain-C restatement (oracle/htrip_oracle.c); the grid is passed per call."""

    def __init__(self, b: int, g: int = 2):
        self.lib = _load_port()
        self.b, self.g = b, g
        self.h = self.lib.orc_create(b, g)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    @staticmethod
    def _g(grid):
        obs = np.ascontiguousarray(grid, dtype=np.uint8)
        return obs, _p(obs, _U8P), obs.shape[0], obs.shape[1]

    def build(self, grid) -> bool:
        obs, ptr, r, c = self._g(grid)
        return bool(self.lib.orc_build(self.h, ptr, r, c))

    def open_batch(self, cells, grid):
        rc = _rc(cells)
        obs, ptr, r, c = self._g(grid)
        self.lib.orc_open_batch(self.h, _p(rc, _I32P), len(rc), ptr, r, c)

    def query(self, vps, grid) -> np.ndarray:
        rc = _rc(vps)
        obs, ptr, r, c = self._g(grid)
        out = np.empty((len(rc), len(rc)), dtype=np.uint16)
        self.lib.orc_query(self.h, _p(rc, _I32P), len(rc), ptr, r, c, _p(out, _U16P))
        return out

    def stats(self):
        out = np.zeros(3, dtype=np.int32)
        self.lib.orc_stats(self.h, _p(out, _I32P))
        return tuple(int(x) for x in out)

    @property
    def S(self):
        return self.lib.orc_S(self.h)

    @property
    def H(self):
        return self.lib.orc_H(self.h)

    def leaf_D(self, i):
        n = self.lib.orc_leaf_D(self.h, i, None)
        out = np.empty((n, n), dtype=np.uint16)
        self.lib.orc_leaf_D(self.h, i, _p(out, _U16P))
        return out

    def node_DU(self, lvl, node):
        n = self.lib.orc_node_DU(self.h, lvl, node, None)
        out = np.empty((n, n), dtype=np.uint16)
        self.lib.orc_node_DU(self.h, lvl, node, _p(out, _U16P))
        return out


def port_bfs(grid, vps) -> np.ndarray:
    lib = _load_port()
    obs = np.ascontiguousarray(grid, dtype=np.uint8)
    rc = _rc(vps)
    out = np.empty((len(rc), len(rc)), dtype=np.uint16)
    lib.orc_bfs_all_pairs(_p(obs, _U8P), obs.shape[0], obs.shape[1], _p(rc, _I32P), len(rc), _p(out, _U16P))
    return out
