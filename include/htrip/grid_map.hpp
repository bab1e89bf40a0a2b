// htrip_b200 C++20 drop-in: the occupancy grid the oracle reads.
//
// Mirrors the members of the reference's GridMap that MinPlusOracle and its
// callers use (include/htrip/grid_map.hpp:31-160, 221-290): rows / cols,
// the ground_truth / observed CellState arrays (row-major, one byte per
// cell), the optional traversal weights (:51-56, 258-334), bounds and index
// helpers, isPassable (observed == Free) and the observed accessors.  The map generators and file loaders of the reference
// are test fixtures there and are not part of this library.
//
// The oracle reads `observed` as a plain byte array (CellState is a uint8
// enum), so a GridMap is passed to the device layer without conversion.
#pragma once

#include <vector>

#include "types.hpp"

namespace htrip {

class GridMap {
public:
    int rows = 0;
    int cols = 0;
    std::vector<CellState> ground_truth;
    std::vector<CellState> observed;
    std::vector<dist_t> weights;  // per-cell traversal costs, row-major; empty: every weight 1

    GridMap() = default;
    GridMap(int r, int c, CellState initial_state = CellState::Unknown)
        : rows(r), cols(c),
          ground_truth(size_t(r > 0 ? r : 0) * size_t(c > 0 ? c : 0), initial_state),
          observed(size_t(r > 0 ? r : 0) * size_t(c > 0 ? c : 0), initial_state) {}

    [[nodiscard]] bool inBounds(int r, int c) const noexcept { return r >= 0 && c >= 0 && r < rows && c < cols; }
    [[nodiscard]] bool inBounds(Point p) const noexcept { return inBounds(p.r, p.c); }
    [[nodiscard]] int index(int r, int c) const noexcept { return r * cols + c; }
    [[nodiscard]] int index(Point p) const noexcept { return index(p.r, p.c); }
    [[nodiscard]] Point point(int idx) const noexcept { return Point(idx / cols, idx % cols); }

    [[nodiscard]] bool isPassable(int r, int c) const noexcept {
        return inBounds(r, c) && observed[size_t(index(r, c))] == CellState::Free;
    }
    [[nodiscard]] bool isPassable(Point p) const noexcept { return isPassable(p.r, p.c); }

    [[nodiscard]] CellState getObserved(int r, int c) const noexcept {
        return inBounds(r, c) ? observed[size_t(index(r, c))] : CellState::Obstacle;
    }
    [[nodiscard]] CellState getObserved(Point p) const noexcept { return getObserved(p.r, p.c); }
    void setObserved(int r, int c, CellState s) noexcept {
        if (inBounds(r, c)) observed[size_t(index(r, c))] = s;
    }
    void setObserved(Point p, CellState s) noexcept { setObserved(p.r, p.c, s); }

    [[nodiscard]] bool hasWeights() const noexcept { return !weights.empty(); }

    // INF outside the grid and on obstacles, else the cell's weight (1
    // without weights).
    [[nodiscard]] dist_t getCellWeight(int r, int c) const noexcept {
        if (!inBounds(r, c)) return INF;
        if (observed[size_t(index(r, c))] == CellState::Obstacle) return INF;
        if (weights.empty()) return 1;
        return weights[size_t(index(r, c))];
    }
    [[nodiscard]] dist_t getCellWeight(Point p) const noexcept { return getCellWeight(p.r, p.c); }
    // The first weight set gives every cell weight 1.
    void setCellWeight(int r, int c, dist_t w) noexcept {
        if (!inBounds(r, c)) return;
        if (weights.size() < size_t(rows) * size_t(cols)) weights.assign(size_t(rows) * size_t(cols), 1);
        weights[size_t(index(r, c))] = w;
    }
    void setCellWeight(Point p, dist_t w) noexcept { setCellWeight(p.r, p.c, w); }
    // Cost of the edge between adjacent cells u, v: INF if either weight is
    // INF or more, else max(1, (w_u + w_v) / 2).
    [[nodiscard]] dist_t edgeWeight(Point u, Point v) const noexcept {
        const dist_t wu = getCellWeight(u), wv = getCellWeight(v);
        if (wu >= INF || wv >= INF) return INF;
        const dist_t avg = dist_t((uint32_t(wu) + uint32_t(wv)) / 2);
        return avg == 0 ? dist_t(1) : avg;
    }

    // Copy one cell's ground truth into `observed` (reference
    // GridMap::revealCell, src/grid_map.cpp:231-235); false out of bounds.
    bool revealCell(Point p) {
        if (!inBounds(p)) return false;
        observed[size_t(index(p))] = ground_truth[size_t(index(p))];
        return true;
    }

    // Byte view of `observed` (0 Unknown, 1 Free, 2 Obstacle) for the C ABI.
    [[nodiscard]] const uint8_t* observedBytes() const noexcept {
        return reinterpret_cast<const uint8_t*>(observed.data());
    }
};

}  // namespace htrip
