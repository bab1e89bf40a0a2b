// htrip_b200 C++20 drop-in: the occupancy grid the oracle reads.
//
// Mirrors the members of the reference's GridMap that MinPlusOracle and its
// callers use (include/htrip/grid_map.hpp:31-160, 221-290): rows / cols,
// the ground_truth / observed CellState arrays (row-major, one byte per
// cell), bounds and index helpers, isPassable (observed == Free) and the
// observed accessors.  The map generators and file loaders of the reference
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
    std::vector<dist_t> weights;  // empty: unit weights (weighted grids are not supported by this library)

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
