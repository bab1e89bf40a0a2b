"""Seeded synthetic occupancy grids and request streams.

The reference measures on Moving AI maps (street maps such as Boston_0_256,
mazes such as maze512-1-0).  These generators produce grids of the same
shapes, sizes and obstacle statistics from a seed, so that every run (GPU
arm, CPU reference arm, tests) sees byte-identical inputs:

* ``street_grid``  - 1-cell obstacle border, axis-aligned obstacle rectangles
  of side U[4, 40] placed until about 30% of cells are blocked, then only the
  largest 4-connected free component is kept (the reference keeps the largest
  ground-truth component the same way, src/campaign_support.cpp:171).
* ``maze_grid``    - recursive-backtracker perfect maze; lattice cells are
  ``corridor`` x ``corridor`` blocks separated by walls of width ``wall``.
  ``maze_grid(512, 1)`` is the 512x512 width-1 maze over a 256x256 lattice;
  ``maze_grid(512, 16)`` uses 16-wide corridors with 1-cell walls (a 30x30
  lattice, the layout of maze512-16-0).
* ``exploration_stream`` - the incremental-opening workload: an initial
  observed mask made of radius-40 disks around seeded robot starts, then the
  remaining free cells in BFS-ring order from the observed boundary, in
  batches.

Cell states use the reference's ``CellState`` byte values
(include/htrip/types.hpp): 0 Unknown, 1 Free, 2 Obstacle.
"""
from __future__ import annotations

from collections import deque

import numpy as np

UNKNOWN = 0
FREE = 1
OBSTACLE = 2


def _largest_component(free: np.ndarray) -> np.ndarray:
    from scipy import ndimage

    lab, n = ndimage.label(free, structure=[[0, 1, 0], [1, 1, 1], [0, 1, 0]])
    if n == 0:
        return free
    counts = np.bincount(lab.ravel())
    counts[0] = 0
    return lab == int(np.argmax(counts))


def street_grid(side: int, seed: int, blocked: float = 0.30,
                rect_min: int = 4, rect_max: int = 40) -> np.ndarray:
    """Fully revealed street-like grid (uint8 CellState, shape (side, side))."""
    rng = np.random.default_rng(seed)
    obst = np.zeros((side, side), dtype=bool)
    obst[0, :] = obst[-1, :] = True
    obst[:, 0] = obst[:, -1] = True
    n_blocked = int(obst.sum())
    target = int(blocked * side * side)
    while n_blocked < target:
        h, w = (int(x) for x in rng.integers(rect_min, rect_max + 1, size=2))
        r0 = int(rng.integers(0, side - h + 1))
        c0 = int(rng.integers(0, side - w + 1))
        patch = obst[r0:r0 + h, c0:c0 + w]
        n_blocked += int(patch.size - patch.sum())
        patch[...] = True
    keep = _largest_component(~obst)
    return np.where(keep, FREE, OBSTACLE).astype(np.uint8)


def maze_grid(side: int, corridor: int, seed: int, wall: int = 1) -> np.ndarray:
    """Fully revealed recursive-backtracker maze (uint8 CellState)."""
    period = corridor + wall
    n = side // period
    rng = np.random.default_rng(seed)
    grid = np.full((side, side), OBSTACLE, dtype=np.uint8)
    visited = np.zeros((n, n), dtype=bool)
    # Open every lattice cell's corridor block.
    for i in range(n):
        for j in range(n):
            grid[i * period:i * period + corridor, j * period:j * period + corridor] = FREE
    # Iterative depth-first carve from a seeded start.
    start = (int(rng.integers(0, n)), int(rng.integers(0, n)))
    stack = [start]
    visited[start] = True
    steps = ((-1, 0), (1, 0), (0, -1), (0, 1))
    while stack:
        i, j = stack[-1]
        nbrs = [(i + di, j + dj) for di, dj in steps
                if 0 <= i + di < n and 0 <= j + dj < n and not visited[i + di, j + dj]]
        if not nbrs:
            stack.pop()
            continue
        ni, nj = nbrs[int(rng.integers(0, len(nbrs)))]
        visited[ni, nj] = True
        # Knock out the wall between (i, j) and (ni, nj).
        if ni == i:
            c = min(j, nj) * period + corridor
            grid[i * period:i * period + corridor, c:c + wall] = FREE
        else:
            r = min(i, ni) * period + corridor
            grid[r:r + wall, j * period:j * period + corridor] = FREE
        stack.append((ni, nj))
    return grid


def sample_free(grid: np.ndarray, k: int, seed: int) -> np.ndarray:
    """k distinct viewpoints drawn uniformly from Free cells -> int32 (k, 2) [r, c]."""
    rng = np.random.default_rng(seed)
    free = np.flatnonzero(grid.ravel() == FREE)
    idx = rng.choice(free, size=min(k, free.size), replace=False)
    cols = grid.shape[1]
    return np.stack([idx // cols, idx % cols], axis=1).astype(np.int32)


def exploration_stream(truth: np.ndarray, n_robots: int, radius: int, batch: int,
                       n_batches: int, seed: int):
    """Incremental-opening workload on a fully known ground-truth grid.

    Returns ``(observed0, starts, batches)``: the initial observed grid (Free
    inside the union of radius-``radius`` disks around ``n_robots`` seeded
    Free starts, Obstacle for ground-truth obstacles inside the disks, Unknown
    elsewhere), the robot start cells (int32 (n_robots, 2)) and a list of up
    to ``n_batches`` int32 (m, 2) arrays of cells to open, taken in BFS-ring
    order (over ground-truth Free cells) from the initially observed region.
    """
    rows, cols = truth.shape
    starts = sample_free(truth, n_robots, seed)
    rr, cc = np.mgrid[0:rows, 0:cols]
    inside = np.zeros((rows, cols), dtype=bool)
    for r, c in starts:
        inside |= (rr - r) ** 2 + (cc - c) ** 2 <= radius * radius
    observed = np.full((rows, cols), UNKNOWN, dtype=np.uint8)
    observed[inside & (truth == FREE)] = FREE
    observed[inside & (truth == OBSTACLE)] = OBSTACLE
    # BFS rings over ground-truth free cells, seeded by the observed free cells.
    seen = observed == FREE
    q = deque(zip(*np.nonzero(seen)))
    order = []
    need = batch * n_batches
    while q and len(order) < need:
        r, c = q.popleft()
        for dr, dc in ((-1, 0), (1, 0), (0, -1), (0, 1)):
            nr, nc = r + dr, c + dc
            if 0 <= nr < rows and 0 <= nc < cols and not seen[nr, nc] and truth[nr, nc] == FREE:
                seen[nr, nc] = True
                order.append((nr, nc))
                q.append((nr, nc))
    order = np.asarray(order, dtype=np.int32).reshape(-1, 2)
    batches = [order[i:i + batch] for i in range(0, min(len(order), batch * n_batches), batch)]
    return observed, starts, batches


def frontier_cells(observed: np.ndarray, k: int, seed: int) -> np.ndarray:
    """k Free cells with an Unknown 4-neighbour (exploration frontier), seeded."""
    free = observed == FREE
    unk = observed == UNKNOWN
    nb = np.zeros_like(unk)
    nb[1:, :] |= unk[:-1, :]
    nb[:-1, :] |= unk[1:, :]
    nb[:, 1:] |= unk[:, :-1]
    nb[:, :-1] |= unk[:, 1:]
    cand = np.flatnonzero((free & nb).ravel())
    if cand.size == 0:
        cand = np.flatnonzero(free.ravel())
    rng = np.random.default_rng(seed)
    idx = rng.choice(cand, size=min(k, cand.size), replace=False)
    cols = observed.shape[1]
    return np.stack([idx // cols, idx % cols], axis=1).astype(np.int32)


def batched_mix(n_maps: int, seed: int, sides=(128, 256, 512, 1024), tiles=(8, 16, 32),
                open_range=(64, 1024), k_range=(8, 512)):
    """The many-maps workload: per map a side, a generator (street grid with
    20-40% obstacles or maze with corridor width 1-16), a leaf side b, one
    opening batch of m cells (withheld from the initial observation and
    opened in one call) and one all-pairs query of k viewpoints.

    Returns a list of dicts {side, kind, param, b, seed, n_open, k}; grids
    come from ``mix_grid``."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_maps):
        side = int(rng.choice(sides))
        kind = "street" if rng.random() < 0.5 else "maze"
        param = float(rng.uniform(0.20, 0.40)) if kind == "street" else int(rng.integers(1, 17))
        out.append(dict(side=side, kind=kind, param=param, b=int(rng.choice(tiles)),
                        seed=int(rng.integers(0, 2**31 - 1)),
                        n_open=int(rng.integers(open_range[0], open_range[1] + 1)),
                        k=int(rng.integers(k_range[0], k_range[1] + 1))))
    return out


def mix_grid(spec) -> np.ndarray:
    """Ground-truth grid of one ``batched_mix`` entry."""
    if spec["kind"] == "street":
        return street_grid(spec["side"], spec["seed"], blocked=spec["param"])
    return maze_grid(spec["side"], int(spec["param"]), spec["seed"])


def withheld_open(truth: np.ndarray, n_open: int, seed: int):
    """(observed0, cells): n_open Free cells of ``truth`` drawn uniformly and
    left Unknown in observed0, to be opened in one batch (the reference's
    update benchmark withholds cells the same way, bench_update_latency.cpp:166-175)."""
    rng = np.random.default_rng(seed)
    free = np.flatnonzero(truth.ravel() == FREE)
    idx = rng.choice(free, size=min(n_open, free.size), replace=False)
    cols = truth.shape[1]
    cells = np.stack([idx // cols, idx % cols], axis=1).astype(np.int32)
    obs = truth.copy()
    obs[cells[:, 0], cells[:, 1]] = UNKNOWN
    return obs, cells


def served_trace(pools, n_req: int, rate: float, seed: int, q_frac: float = 0.7,
                 k_range=(4, 512), open_range=(1, 512)):
    """Open-loop request stream over map sessions.

    ``pools``: per session ``(truth, withheld)`` - the ground-truth grid and
    the cells still to be opened, in opening order.  Arrivals are Poisson at
    ``rate`` requests/s; a request is an all-pairs query with probability
    ``q_frac`` (k log-uniform in ``k_range``, viewpoints uniform on the
    session's ground-truth Free cells, so some may still be unobserved and
    answer INF) and otherwise an opening of the session's next m cells, m
    uniform in ``open_range`` (a query once the session has none left).

    Returns ``(requests, arrival_s)``: requests are ``(session_index, kind,
    rc)`` with kind 0 = query, 1 = opening."""
    rng = np.random.default_rng(seed)
    arrival = np.cumsum(rng.exponential(1.0 / rate, size=n_req))
    arrival -= arrival[0]
    cursor = [0] * len(pools)
    frees = [np.flatnonzero(t.ravel() == FREE) for t, _ in pools]
    out = []
    for _ in range(n_req):
        s = int(rng.integers(0, len(pools)))
        truth, withheld = pools[s]
        if rng.random() >= q_frac and cursor[s] < len(withheld):
            m = int(rng.integers(open_range[0], open_range[1] + 1))
            cells = withheld[cursor[s]:cursor[s] + m]
            cursor[s] += len(cells)
            out.append((s, 1, cells.astype(np.int32)))
            continue
        k = int(round(np.exp(rng.uniform(np.log(k_range[0]), np.log(k_range[1])))))
        idx = rng.choice(frees[s], size=min(k, frees[s].size), replace=False)
        cols = truth.shape[1]
        out.append((s, 0, np.stack([idx // cols, idx % cols], axis=1).astype(np.int32)))
    return out, arrival
