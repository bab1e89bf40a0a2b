// htrip_b200 C++20 drop-in for htrip::MinPlusOracle.
//
// Same class name, members and call signatures as the reference's
// include/htrip/minplus_oracle.hpp (ozaslan/htrip), so callers compile
// unchanged; the index itself lives in the HBM of one CUDA device and every
// method calls the C ABI of include/htrip_b200.h (libhtrip_b200.so):
//
//   explicit MinPlusOracle(HierarchyConfig)              minplus_oracle.hpp:59
//   bool build(const GridMap&)                           :78
//   int depth() const                                    :83
//   leafIndex / tileIndexAtLevel / findLcaLevel          :88, :95, :370
//   void onCellOpened(Point, const GridMap&)             :109
//   void onBatchCellsOpened(const std::vector<Point>&,
//                           const GridMap&)              :171
//   void onCellBlocked(Point, const GridMap&)            :123
//   void onBatchLeavesChanged(const std::vector<int>&,
//                             const GridMap&)            :157
//   void onCellWeightChanged(Point, dist_t, GridMap&)    :132
//   void onTileWeightsChanged(int, int, cell_weights,
//                             GridMap&)                  :144
//   struct HTripQueryScratch (caller-owned, reused)      :189-238
//   struct LastBatchStats / last_batch_stats             :251-256
//   void queryAllPairs(vps, grid, out, scratch) const    :337-341
//   std::vector<dist_t> queryAllPairs(vps, grid) const   :348-349
//   void queryAllPairsIncremental(vps, grid, out, scratch,
//                                 HTripIncrementalState&) const :290-294
//   dist_t queryDistance(Point, Point, const GridMap&) const    :312
//   void liftRoot(const GridMap& = GridMap())            :380
//   size_t totalMemoryBytes() const                      :385
//   copy construction / assignment (deep copy, as the reference's
//   value-type oracle: bench_update_latency.cpp:178,186)
//
// Behaviour shared with the reference: build returns false on an invalid
// config or an empty grid; cells and viewpoints outside the grid are
// ignored / answered with INF rows; a viewpoint that is not Free has an INF
// row, column and diagonal.  Differences: the index is not a host object
// (no `leaves` / `levels` members; use numLeaves()), hybrid_k_threshold is
// ignored (there is no CPU fallback), and a CUDA failure throws DeviceError.
// A MinPlusOracle is not thread-safe; distinct oracles may be used from
// different threads (each owns a CUDA stream).
#pragma once

#include <cstddef>
#include <utility>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "grid_map.hpp"
#include "types.hpp"

struct htrip_index;  // opaque device index (include/htrip_b200.h)

namespace htrip {

// A CUDA or device-side failure inside the library (the reference has no
// failure mode there).  `status` is the htrip_status of the C ABI.
class DeviceError : public std::runtime_error {
public:
    DeviceError(int status, const std::string& msg) : std::runtime_error(msg), status(status) {}
    int status;
};

class MinPlusOracle {
public:
    HierarchyConfig config;
    int S = 0;
    int H = 0;
    int num_leaf_tiles_x = 0;
    int num_leaf_tiles_y = 0;

    struct LastBatchStats {
        int n_touched_leaves = 0;
        int n_dirty_ancestors = 0;
        int n_pivots = 0;
    };
    LastBatchStats last_batch_stats{};

    uint32_t update_counter = 0;  // incremented by every update call
    uint64_t epoch = 0;           // incremented by every build

    // Caller-owned query workspace, reused across calls so that a warm query
    // does not allocate host memory.  The device workspace belongs to the
    // oracle and is kept between calls.
    struct HTripQueryScratch {
        std::vector<int32_t> rc;  // viewpoints as (row, col) int32 pairs

        void ensureCapacity(size_t k, int /*H*/ = 0, size_t /*num_leaves*/ = 0) {
            if (rc.capacity() < 2 * k) rc.reserve(2 * k);
        }
    };
    mutable HTripQueryScratch query_scratch;  // used by the 2-argument queryAllPairs

    // Cache of queryAllPairsIncremental (the reference's field names for the
    // fields a caller reads).  The matrix is reused while the viewpoints,
    // the epoch and the update counter stay as they were.
    struct HTripIncrementalState {
        bool initialized = false;
        uint64_t epoch_seen = 0;
        uint32_t last_update_counter = 0;
        std::vector<Point> vp_pts;
        std::vector<dist_t> matrix;
    };

    // Index on CUDA device 0 with the default config (b = 16, 2 x 2 groups).
    MinPlusOracle();
    // Index on CUDA device `device`.  Throws DeviceError when no CUDA device
    // is usable (there is no CPU fallback).
    explicit MinPlusOracle(HierarchyConfig cfg, int device = 0);
    ~MinPlusOracle();
    MinPlusOracle(const MinPlusOracle& other);             // deep device-to-device copy
    MinPlusOracle& operator=(const MinPlusOracle& other);  // deep device-to-device copy
    MinPlusOracle(MinPlusOracle&& other) noexcept;
    MinPlusOracle& operator=(MinPlusOracle&& other) noexcept;

    bool build(const GridMap& grid);

    [[nodiscard]] int depth() const noexcept { return H; }
    [[nodiscard]] int leafIndex(int tx, int ty) const noexcept { return ty * num_leaf_tiles_x + tx; }
    // Row-major index of tile (tx, ty) among the level-`lvl` tiles (side b*g^lvl).
    [[nodiscard]] int tileIndexAtLevel(int lvl, int tx, int ty) const noexcept;
    // Lowest level whose node holds both cells (0: same leaf, H + 1: none).
    [[nodiscard]] int findLcaLevel(Point p1, Point p2) const noexcept;

    // The caller has already set p (or every cell of the batch) Free in
    // grid.observed.  onCellOpened leaves last_batch_stats untouched, as the
    // reference's single-cell path does.
    void onCellOpened(Point p, const GridMap& grid);
    void onBatchCellsOpened(const std::vector<Point>& newly_opened, const GridMap& grid);
    // Non-monotone updates: the caller has made the cell(s) non-Free in
    // grid.observed; the leaf (leaves) and every ancestor are rebuilt.
    void onCellBlocked(Point p, const GridMap& grid);
    void onBatchLeavesChanged(const std::vector<int>& leaf_indices, const GridMap& grid);
    // Weighted grids: build / liftRoot read grid.weights (empty: every weight
    // 1); a weight change sets it in `grid` and rebuilds the cell's leaf (the
    // given leaf) and every ancestor.  Change weights through these calls:
    // the index keeps its own copy of the weights.
    void onCellWeightChanged(Point p, dist_t new_weight, GridMap& grid);
    void onTileWeightsChanged(int tx, int ty, const std::vector<std::pair<Point, dist_t>>& cell_weights,
                              GridMap& grid);

    // k x k row-major matrix of exact 4-connected distances (INF when
    // unreachable), resized and filled by the call.
    void queryAllPairs(const std::vector<Point>& viewpoints, const GridMap& grid, std::vector<dist_t>& out_matrix,
                       HTripQueryScratch& scratch) const;
    [[nodiscard]] std::vector<dist_t> queryAllPairs(const std::vector<Point>& viewpoints,
                                                    const GridMap& grid) const;
    // Same matrix as queryAllPairs; without any update since `state` was
    // filled for the same viewpoints it is the cached one (no device work),
    // otherwise the full query runs again.
    void queryAllPairsIncremental(const std::vector<Point>& viewpoints, const GridMap& grid,
                                  std::vector<dist_t>& out_matrix, HTripQueryScratch& scratch,
                                  HTripIncrementalState& state) const;
    // Exact distance between two cells (INF if either is not passable).
    [[nodiscard]] dist_t queryDistance(Point s, Point t, const GridMap& grid) const;

    // Grows the index to S * g, H + 1: existing tiles keep their tables, the
    // new area and the new root are built from `grid`.
    void liftRoot(const GridMap& grid = GridMap());

    // The reference's accounting of the same index: bytes of every D, S,
    // D_U, S_U and child_to_ext table.
    [[nodiscard]] size_t totalMemoryBytes() const noexcept;
    // Bytes of HBM this index actually holds (arena and workspaces).
    [[nodiscard]] size_t deviceMemoryBytes() const noexcept;
    // Number of leaf tiles (the reference's leaves.size()).
    [[nodiscard]] size_t numLeaves() const noexcept {
        return size_t(num_leaf_tiles_x) * size_t(num_leaf_tiles_y);
    }
    [[nodiscard]] int device() const noexcept { return device_; }
    // The C ABI handle (for stream-ordered calls of include/htrip_b200.h).
    [[nodiscard]] htrip_index* handle() const noexcept { return h_; }

private:
    void create();
    void destroy() noexcept;
    void refreshShape();

    htrip_index* h_ = nullptr;
    int device_ = 0;
    bool built_ = false;
    mutable std::vector<int32_t> cells_;  // reused (row, col) staging of update calls
};

using HTripOracle = MinPlusOracle;

}  // namespace htrip
