// htrip::MinPlusOracle (C++20 drop-in) over the C ABI of include/htrip_b200.h.
//
// Every method forwards to libhtrip_b200.so; no arithmetic happens here.
// Reference behaviour reproduced at this layer (ozaslan/htrip):
//   build: false on an invalid config or empty grid   src/minplus_oracle.cpp:48-52
//   S / H / num_leaf_tiles_*: the sizes build derives  :54-70
//   tileIndexAtLevel / findLcaLevel                    :15-46
//   onBatchCellsOpened resets last_batch_stats         :531
//   queryAllPairs: out resized to k*k                  :940-943
//   2-argument queryAllPairs uses the member scratch   :1421-1426
#include "htrip/minplus_oracle.hpp"

#include <algorithm>
#include <utility>

#include "htrip_b200.h"

namespace htrip {

namespace {

[[noreturn]] void raise(htrip_status st, const char* what) {
    throw DeviceError(int(st), std::string(what) + ": " + htrip_last_error());
}

inline void check(htrip_status st, const char* what) {
    if (st != HTRIP_OK) raise(st, what);
}

}  // namespace

MinPlusOracle::MinPlusOracle() : MinPlusOracle(HierarchyConfig{}, 0) {}

MinPlusOracle::MinPlusOracle(HierarchyConfig cfg, int device) : config(cfg), device_(device) { create(); }

MinPlusOracle::~MinPlusOracle() { destroy(); }

void MinPlusOracle::create() {
    htrip_config c{config.tile_size_b, config.group_w};
    check(htrip_create(c, device_, &h_), "htrip_create");
}

void MinPlusOracle::destroy() noexcept {
    if (h_) htrip_destroy(h_);
    h_ = nullptr;
}

MinPlusOracle::MinPlusOracle(const MinPlusOracle& o)
    : config(o.config), S(o.S), H(o.H), num_leaf_tiles_x(o.num_leaf_tiles_x), num_leaf_tiles_y(o.num_leaf_tiles_y),
      last_batch_stats(o.last_batch_stats), update_counter(o.update_counter), epoch(o.epoch), device_(o.device_),
      built_(o.built_) {
    check(htrip_clone(o.h_, &h_), "htrip_clone");
}

MinPlusOracle& MinPlusOracle::operator=(const MinPlusOracle& o) {
    if (this == &o) return *this;
    MinPlusOracle tmp(o);
    *this = std::move(tmp);
    return *this;
}

MinPlusOracle::MinPlusOracle(MinPlusOracle&& o) noexcept
    : config(o.config), S(o.S), H(o.H), num_leaf_tiles_x(o.num_leaf_tiles_x), num_leaf_tiles_y(o.num_leaf_tiles_y),
      last_batch_stats(o.last_batch_stats), update_counter(o.update_counter), epoch(o.epoch),
      query_scratch(std::move(o.query_scratch)), h_(std::exchange(o.h_, nullptr)), device_(o.device_),
      built_(std::exchange(o.built_, false)) {}

MinPlusOracle& MinPlusOracle::operator=(MinPlusOracle&& o) noexcept {
    if (this == &o) return *this;
    destroy();
    config = o.config;
    S = o.S;
    H = o.H;
    num_leaf_tiles_x = o.num_leaf_tiles_x;
    num_leaf_tiles_y = o.num_leaf_tiles_y;
    last_batch_stats = o.last_batch_stats;
    update_counter = o.update_counter;
    epoch = o.epoch;
    query_scratch = std::move(o.query_scratch);
    h_ = std::exchange(o.h_, nullptr);
    device_ = o.device_;
    built_ = std::exchange(o.built_, false);
    return *this;
}

void MinPlusOracle::refreshShape() {
    int32_t s = 0, hh = 0, lx = 0;
    check(htrip_shape(h_, &s, &hh, &lx), "htrip_shape");
    S = s;
    H = hh;
    num_leaf_tiles_x = lx;
    num_leaf_tiles_y = lx;
}

// The grid's weights to the index (before build / liftRoot).
static void send_weights(htrip_index* h, const GridMap& grid) {
    const bool w = grid.hasWeights() && grid.weights.size() >= size_t(grid.rows) * size_t(grid.cols);
    check(htrip_set_cell_weights(h, w ? grid.weights.data() : nullptr, grid.rows, grid.cols), "set weights");
}

bool MinPlusOracle::build(const GridMap& grid) {
    if (!config.isValid()) return false;
    if (std::max(grid.rows, grid.cols) <= 0) return false;
    send_weights(h_, grid);
    const htrip_status st = htrip_build(h_, grid.observedBytes(), grid.rows, grid.cols);
    if (st == HTRIP_ERR_INVALID) return false;
    check(st, "build");
    refreshShape();
    built_ = true;
    last_batch_stats = {};
    ++epoch;
    return true;
}

int MinPlusOracle::tileIndexAtLevel(int lvl, int tx, int ty) const noexcept {
    int side = config.tile_size_b;
    for (int l = 0; l < lvl; ++l) side *= config.group_w;
    const int nx = side > 0 && S / side > 0 ? S / side : 1;
    return ty * nx + tx;
}

int MinPlusOracle::findLcaLevel(Point p1, Point p2) const noexcept {
    const int b = config.tile_size_b, g = config.group_w;
    int ax = p1.c / b, ay = p1.r / b, bx = p2.c / b, by = p2.r / b;
    if (ax == bx && ay == by) return 0;
    for (int lvl = 1; lvl <= H; ++lvl) {
        ax /= g;
        ay /= g;
        bx /= g;
        by /= g;
        if (ax == bx && ay == by) return lvl;
    }
    return H + 1;
}

void MinPlusOracle::onCellOpened(Point p, const GridMap& grid) {
    if (!built_) return;
    ++update_counter;
    check(htrip_open_cell(h_, p.r, p.c, grid.observedBytes(), grid.rows, grid.cols), "onCellOpened");
}

void MinPlusOracle::onBatchCellsOpened(const std::vector<Point>& newly_opened, const GridMap& grid) {
    last_batch_stats = {};
    if (newly_opened.empty() || !built_) return;
    ++update_counter;
    cells_.resize(2 * newly_opened.size());
    for (size_t i = 0; i < newly_opened.size(); ++i) {
        cells_[2 * i] = newly_opened[i].r;
        cells_[2 * i + 1] = newly_opened[i].c;
    }
    check(htrip_open_cells(h_, cells_.data(), int32_t(newly_opened.size()), grid.observedBytes(), grid.rows,
                           grid.cols),
          "onBatchCellsOpened");
    htrip_batch_stats st{};
    check(htrip_last_batch_stats(h_, &st), "last_batch_stats");
    last_batch_stats = {st.n_touched_leaves, st.n_dirty_ancestors, st.n_pivots};
}

void MinPlusOracle::onCellBlocked(Point p, const GridMap& grid) {
    if (!built_) return;
    ++update_counter;
    check(htrip_cell_blocked(h_, p.r, p.c, grid.observedBytes(), grid.rows, grid.cols), "onCellBlocked");
    ++epoch;  // reference minplus_oracle.cpp:300-301
}

// minplus_oracle.cpp:304-360
void MinPlusOracle::onCellWeightChanged(Point p, dist_t new_weight, GridMap& grid) {
    if (!grid.inBounds(p)) return;
    if (grid.getCellWeight(p) == new_weight) return;
    grid.setCellWeight(p, new_weight);
    if (!built_) return;
    ++update_counter;
    check(htrip_cell_weight_changed(h_, p.r, p.c, new_weight, grid.observedBytes(), grid.rows, grid.cols),
          "onCellWeightChanged");
    ++epoch;
}

// minplus_oracle.cpp:362-424
void MinPlusOracle::onTileWeightsChanged(int tx, int ty, const std::vector<std::pair<Point, dist_t>>& cell_weights,
                                         GridMap& grid) {
    if (tx < 0 || ty < 0 || tx >= num_leaf_tiles_x || ty >= num_leaf_tiles_y) return;
    std::vector<int32_t> rc;
    std::vector<uint16_t> w;
    for (const auto& [p, wt] : cell_weights) {
        if (grid.inBounds(p)) grid.setCellWeight(p, wt);
        rc.push_back(p.r);
        rc.push_back(p.c);
        w.push_back(wt);
    }
    if (!built_) return;
    ++update_counter;
    check(htrip_tile_weights_changed(h_, tx, ty, rc.data(), w.data(), int32_t(w.size()), grid.observedBytes(),
                                     grid.rows, grid.cols),
          "onTileWeightsChanged");
    ++epoch;
}

void MinPlusOracle::onBatchLeavesChanged(const std::vector<int>& leaf_indices, const GridMap& grid) {
    if (!built_ || leaf_indices.empty()) return;
    ++update_counter;
    std::vector<int32_t> li(leaf_indices.begin(), leaf_indices.end());
    check(htrip_leaves_changed(h_, li.data(), int32_t(li.size()), grid.observedBytes(), grid.rows, grid.cols),
          "onBatchLeavesChanged");
    ++epoch;  // reference propagateBatchUpward, minplus_oracle.cpp:504
}

void MinPlusOracle::queryAllPairs(const std::vector<Point>& viewpoints, const GridMap& grid,
                                  std::vector<dist_t>& out_matrix, HTripQueryScratch& scratch) const {
    const size_t k = viewpoints.size();
    if (out_matrix.size() != k * k) out_matrix.resize(k * k);
    if (k == 0) return;
    if (!built_) {  // nothing indexed yet: only a passable viewpoint reaches itself
        std::fill(out_matrix.begin(), out_matrix.end(), INF);
        for (size_t i = 0; i < k; ++i)
            if (grid.isPassable(viewpoints[i])) out_matrix[i * k + i] = 0;
        return;
    }
    scratch.ensureCapacity(k);
    scratch.rc.resize(2 * k);
    for (size_t i = 0; i < k; ++i) {
        scratch.rc[2 * i] = viewpoints[i].r;
        scratch.rc[2 * i + 1] = viewpoints[i].c;
    }
    check(htrip_query_all_pairs(h_, scratch.rc.data(), int32_t(k), grid.observedBytes(), grid.rows, grid.cols,
                                out_matrix.data()),
          "queryAllPairs");
}

std::vector<dist_t> MinPlusOracle::queryAllPairs(const std::vector<Point>& viewpoints, const GridMap& grid) const {
    std::vector<dist_t> m;
    queryAllPairs(viewpoints, grid, m, query_scratch);
    return m;
}

void MinPlusOracle::queryAllPairsIncremental(const std::vector<Point>& viewpoints, const GridMap& grid,
                                             std::vector<dist_t>& out_matrix, HTripQueryScratch& scratch,
                                             HTripIncrementalState& state) const {
    const size_t k = viewpoints.size();
    if (k == 0) {  // reference minplus_oracle.cpp:1450-1454
        out_matrix.clear();
        state.initialized = false;
        return;
    }
    const bool same = state.initialized && state.epoch_seen == epoch && state.vp_pts == viewpoints;
    if (same && state.last_update_counter == update_counter) {
        out_matrix = state.matrix;
        return;
    }
    queryAllPairs(viewpoints, grid, state.matrix, scratch);
    state.vp_pts = viewpoints;
    state.epoch_seen = epoch;
    state.last_update_counter = update_counter;
    state.initialized = true;
    out_matrix = state.matrix;
}

dist_t MinPlusOracle::queryDistance(Point s, Point t, const GridMap& grid) const {
    if (!grid.isPassable(s) || !grid.isPassable(t)) return INF;  // reference minplus_oracle.cpp:836-837
    if (s == t) return 0;
    if (!built_) return INF;
    dist_t d = INF;
    check(htrip_query_distance(h_, s.r, s.c, t.r, t.c, grid.observedBytes(), grid.rows, grid.cols, &d),
          "queryDistance");
    return d;
}

void MinPlusOracle::liftRoot(const GridMap& grid) {
    if (!built_) return;
    send_weights(h_, grid);
    check(htrip_lift_root(h_, grid.rows > 0 && grid.cols > 0 ? grid.observedBytes() : nullptr, grid.rows, grid.cols),
          "liftRoot");
    refreshShape();
    ++epoch;
}

size_t MinPlusOracle::totalMemoryBytes() const noexcept {
    uint64_t ref = 0, dev = 0;
    if (htrip_memory_bytes(h_, &ref, &dev) != HTRIP_OK) return 0;
    return size_t(ref);
}

size_t MinPlusOracle::deviceMemoryBytes() const noexcept {
    uint64_t ref = 0, dev = 0;
    if (htrip_memory_bytes(h_, &ref, &dev) != HTRIP_OK) return 0;
    return size_t(dev);
}

}  // namespace htrip
