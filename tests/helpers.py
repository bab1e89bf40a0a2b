"""Shared test fixtures: small seeded grids and comparison helpers."""
from __future__ import annotations

import numpy as np

from htrip_b200 import workloads as W

FREE, OBST, UNK = W.FREE, W.OBSTACLE, W.UNKNOWN


def noise_grid(rows, cols, p_free, seed):
    rng = np.random.default_rng(seed)
    g = np.where(rng.random((rows, cols)) < p_free, FREE, OBST).astype(np.uint8)
    return g


def rooms_grid(rows, cols, room, seed):
    """Rooms of side `room` with 1-cell walls and one random door per wall."""
    rng = np.random.default_rng(seed)
    g = np.full((rows, cols), OBST, dtype=np.uint8)
    for r0 in range(0, rows, room):
        for c0 in range(0, cols, room):
            g[r0 + 1:min(r0 + room - 1, rows), c0 + 1:min(c0 + room - 1, cols)] = FREE
    for r0 in range(0, rows, room):
        for c0 in range(0, cols, room):
            if c0 + room < cols:
                dr = r0 + 1 + int(rng.integers(0, max(1, room - 2)))
                if dr < rows:
                    g[dr, c0 + room - 1:c0 + room + 1] = FREE
            if r0 + room < rows:
                dc = c0 + 1 + int(rng.integers(0, max(1, room - 2)))
                if dc < cols:
                    g[r0 + room - 1:r0 + room + 1, dc] = FREE
    return g


def make_grid(kind, rows, cols, seed):
    if kind == "noise":
        return noise_grid(rows, cols, 0.72, seed)
    if kind == "rooms":
        return rooms_grid(rows, cols, 8, seed)
    if kind == "street":
        side = max(rows, cols)
        return W.street_grid(side, seed, rect_min=2, rect_max=max(3, side // 6))[:rows, :cols].copy()
    if kind == "maze":
        side = max(rows, cols)
        return W.maze_grid(side, 1, seed)[:rows, :cols].copy()
    if kind == "open":
        return np.full((rows, cols), FREE, dtype=np.uint8)
    raise ValueError(kind)


def viewpoints(grid, k, seed, include_blocked=0):
    rng = np.random.default_rng(seed)
    free = np.flatnonzero(grid.ravel() == FREE)
    other = np.flatnonzero(grid.ravel() != FREE)
    pick = list(rng.choice(free, size=min(k, free.size), replace=False))
    if include_blocked and other.size:
        pick += list(rng.choice(other, size=min(include_blocked, other.size), replace=False))
    rng.shuffle(pick)
    cols = grid.shape[1]
    return np.array([[p // cols, p % cols] for p in pick], dtype=np.int32).reshape(-1, 2)


def reveal_plan(truth, seed, n_batches, batch):
    """Hide a random subset of free cells; return (observed0, batches)."""
    rng = np.random.default_rng(seed)
    obs = truth.copy()
    free = np.flatnonzero(truth.ravel() == FREE)
    hidden = rng.choice(free, size=min(free.size // 3, n_batches * batch), replace=False)
    cols = truth.shape[1]
    rc = np.stack([hidden // cols, hidden % cols], axis=1).astype(np.int32)
    obs[rc[:, 0], rc[:, 1]] = UNK
    batches = [rc[i:i + batch] for i in range(0, len(rc), batch)][:n_batches]
    return obs, batches
