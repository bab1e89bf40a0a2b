// htrip_b200 C++20 drop-in: semiring values, cells and the hierarchy config.
//
// Same names and meaning as the reference's include/htrip/types.hpp
// (ozaslan/htrip) so that code written against htrip::MinPlusOracle compiles
// unchanged against this library:
//   dist_t / INF / UNIT_STEP        types.hpp:34,45,50
//   add_dist (2 and 3 operands)     types.hpp:66-70, 87-91
//   CellState                       types.hpp:100-104
//   Point                           types.hpp:112-143
//   kMaxActiveChildren              types.hpp:191
//   HierarchyConfig                 types.hpp:199-225
// The values and the clamp-at-INF rule are an arithmetic contract, not a
// style choice: every distance this library returns is bit-identical to the
// reference's, so the constants must be the same.
#pragma once

#include <compare>
#include <cstdint>
#include <cstdlib>

namespace htrip {

// Path length in grid steps; INF marks "unreachable".
using dist_t = uint16_t;
inline constexpr dist_t INF = 60000;
inline constexpr dist_t UNIT_STEP = 1;

// Tropical product: the sum of two lengths, clamped at INF.
inline constexpr dist_t add_dist(dist_t a, dist_t b) noexcept {
    const uint32_t s = uint32_t(a) + uint32_t(b);
    return s >= INF ? INF : dist_t(s);
}
inline constexpr dist_t add_dist(dist_t a, dist_t b, dist_t c) noexcept {
    const uint32_t s = uint32_t(a) + uint32_t(b) + uint32_t(c);
    return s >= INF ? INF : dist_t(s);
}

// Occupancy belief of a cell.  Only Free is passable.
enum class CellState : uint8_t { Unknown = 0, Free = 1, Obstacle = 2 };

// Grid coordinate (row r, column c), row-major.
struct Point {
    int r = 0;
    int c = 0;
    constexpr Point() noexcept = default;
    constexpr Point(int r_, int c_) noexcept : r(r_), c(c_) {}
    constexpr bool operator==(const Point& o) const noexcept = default;
    constexpr auto operator<=>(const Point& o) const noexcept = default;
    [[nodiscard]] constexpr int manhattan(const Point& o) const noexcept {
        return (r > o.r ? r - o.r : o.r - r) + (c > o.c ? c - o.c : o.c - c);
    }
};

inline constexpr int kMaxActiveChildren = 256;

// Leaf side b and the g x g grouping of the hierarchy.  hybrid_k_threshold
// (a CPU k x BFS fallback for small k in the reference) is accepted and
// ignored: this library has no CPU fallback.
struct HierarchyConfig {
    int tile_size_b = 16;
    int group_w = 2;
    int group_h = 2;
    int hybrid_k_threshold = 0;

    [[nodiscard]] constexpr bool isQuadtree() const noexcept { return group_w == 2 && group_h == 2; }
    [[nodiscard]] constexpr bool isValid() const noexcept {
        return tile_size_b > 0 && group_w >= 2 && group_h >= 2 && group_w == group_h &&
               group_w * group_h <= kMaxActiveChildren;
    }
};

}  // namespace htrip
