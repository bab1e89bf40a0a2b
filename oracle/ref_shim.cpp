// C-ABI shim around the UNMODIFIED reference implementation (ozaslan/htrip).
//
// TEST INFRASTRUCTURE ONLY.  This file is compiled together with the
// reference's own sources (src/grid_map.cpp, src/leaf_tile.cpp,
// src/internal_node.cpp, src/minplus_oracle.cpp, src/bfs_oracle.cpp,
// src/dijkstra_oracle.cpp), where they lie, by oracle/Makefile into
// oracle/_ref/libhtrip_ref.so.  It is used by the parity tests, by
// __graft_entry__.smoke() and by bench.py's CPU baseline / reference arm,
// never by the product path.
//
// Every entry point forwards to the reference's public API:
//   htrip::MinPlusOracle::{build, onCellOpened, onBatchCellsOpened,
//   queryAllPairs(vps, grid, out, scratch)}   (include/htrip/minplus_oracle.hpp:78,109,171,337)
//   htrip::BfsOracle::queryAllPairs           (src/bfs_oracle.cpp:187)
//   htrip::DijkstraOracle::queryAllPairs      (weighted grids)
//   GridMap::weights, MinPlusOracle::{onCellWeightChanged, onTileWeightsChanged}
//                                             (grid_map.hpp:56, minplus_oracle.hpp:132,144)
// and reads back the public members leaves[i].D/.S and levels[l][n].D_U /
// .S_U / .child_to_ext for bitwise state comparison.
#include "htrip/bfs_oracle.hpp"
#include "htrip/dijkstra_oracle.hpp"
#include "htrip/grid_map.hpp"
#include "htrip/minplus_oracle.hpp"

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

using namespace htrip;

namespace {

struct RefHandle {
    MinPlusOracle oracle;
    GridMap grid;
    MinPlusOracle::HTripQueryScratch scratch;
    MinPlusOracle::HTripIncrementalState inc;
};

std::vector<Point> toPoints(const int32_t* rc, int n) {
    std::vector<Point> pts;
    pts.reserve(static_cast<size_t>(n > 0 ? n : 0));
    for (int i = 0; i < n; ++i) pts.push_back(Point{rc[2 * i], rc[2 * i + 1]});
    return pts;
}

}  // namespace

extern "C" {

void* ref_create(int b, int g) {
    auto* h = new RefHandle();
    h->oracle.config.tile_size_b = b;
    h->oracle.config.group_w = g;
    h->oracle.config.group_h = g;
    h->oracle.config.hybrid_k_threshold = 0;
    return h;
}

void ref_destroy(void* p) { delete static_cast<RefHandle*>(p); }

void* ref_clone(void* p) { return new RefHandle(*static_cast<RefHandle*>(p)); }

// Replace the handle's grid: observed[r*cols+c] holds CellState bytes
// (0 Unknown, 1 Free, 2 Obstacle).  Ground truth is set equal to observed.
void ref_set_grid(void* p, const uint8_t* observed, int rows, int cols) {
    auto* h = static_cast<RefHandle*>(p);
    h->grid = GridMap(rows, cols, CellState::Unknown);
    for (int i = 0; i < rows * cols; ++i) {
        h->grid.observed[static_cast<size_t>(i)] = static_cast<CellState>(observed[i]);
        h->grid.ground_truth[static_cast<size_t>(i)] = static_cast<CellState>(observed[i]);
    }
}

// Set the observed state of n cells (rc = r0,c0,r1,c1,...).
void ref_set_cells(void* p, const int32_t* rc, int n, int state) {
    auto* h = static_cast<RefHandle*>(p);
    for (int i = 0; i < n; ++i) h->grid.setObserved(rc[2 * i], rc[2 * i + 1], static_cast<CellState>(state));
}

int ref_build(void* p) {
    auto* h = static_cast<RefHandle*>(p);
    return h->oracle.build(h->grid) ? 1 : 0;
}

void ref_open_batch(void* p, const int32_t* rc, int n) {
    auto* h = static_cast<RefHandle*>(p);
    h->oracle.onBatchCellsOpened(toPoints(rc, n), h->grid);
}

// MinPlusOracle::queryDistance(s, t, grid) (minplus_oracle.hpp:312).
int ref_query_distance(void* p, int r1, int c1, int r2, int c2) {
    auto* h = static_cast<RefHandle*>(p);
    return h->oracle.queryDistance(Point{r1, c1}, Point{r2, c2}, h->grid);
}

// MinPlusOracle::queryAllPairsIncremental with the handle's persistent state
// (minplus_oracle.hpp:290-294).
void ref_query_incremental(void* p, const int32_t* rc, int k, uint16_t* out) {
    auto* h = static_cast<RefHandle*>(p);
    std::vector<dist_t> m;
    h->oracle.queryAllPairsIncremental(toPoints(rc, k), h->grid, m, h->scratch, h->inc);
    std::memcpy(out, m.data(), m.size() * sizeof(dist_t));
}

// MinPlusOracle::onCellBlocked(p, grid) (minplus_oracle.hpp:123) and
// onBatchLeavesChanged(leaves, grid) (:157) with the handle's current grid.
void ref_cell_blocked(void* p, int r, int c) {
    auto* h = static_cast<RefHandle*>(p);
    h->oracle.onCellBlocked(Point{r, c}, h->grid);
}
void ref_leaves_changed(void* p, const int32_t* leaves, int n) {
    auto* h = static_cast<RefHandle*>(p);
    h->oracle.onBatchLeavesChanged(std::vector<int>(leaves, leaves + n), h->grid);
}

// MinPlusOracle::liftRoot(grid) with the handle's current grid
// (minplus_oracle.hpp:380); an empty grid stands for the default argument.
void ref_lift_root(void* p) {
    auto* h = static_cast<RefHandle*>(p);
    h->oracle.liftRoot(h->grid);
}

// The grid's traversal weights (rows x cols of the current grid; null
// clears them: every weight 1).
void ref_set_weights(void* p, const uint16_t* w) {
    auto* h = static_cast<RefHandle*>(p);
    if (!w) {
        h->grid.weights.clear();
        return;
    }
    h->grid.weights.assign(w, w + static_cast<size_t>(h->grid.rows) * h->grid.cols);
}

// MinPlusOracle::onCellWeightChanged / onTileWeightsChanged with the
// handle's grid (they set the grid's weights themselves).
void ref_cell_weight_changed(void* p, int r, int c, int w) {
    auto* h = static_cast<RefHandle*>(p);
    h->oracle.onCellWeightChanged(Point{r, c}, static_cast<dist_t>(w), h->grid);
}
void ref_tile_weights_changed(void* p, int tx, int ty, const int32_t* rc, const uint16_t* w, int n) {
    auto* h = static_cast<RefHandle*>(p);
    std::vector<std::pair<Point, dist_t>> cw;
    for (int i = 0; i < n; ++i) cw.emplace_back(Point{rc[2 * i], rc[2 * i + 1]}, w[i]);
    h->oracle.onTileWeightsChanged(tx, ty, cw, h->grid);
}

// DijkstraOracle::queryAllPairs on the handle's grid (weighted all pairs).
void ref_dijkstra_all_pairs(void* p, const int32_t* rc, int k, uint16_t* out) {
    auto* h = static_cast<RefHandle*>(p);
    const auto mat = DijkstraOracle::queryAllPairs(h->grid, toPoints(rc, k));
    std::memcpy(out, mat.data(), mat.size() * sizeof(dist_t));
}

void ref_open_cell(void* p, int r, int c) {
    auto* h = static_cast<RefHandle*>(p);
    h->oracle.onCellOpened(Point{r, c}, h->grid);
}

void ref_query(void* p, const int32_t* rc, int k, uint16_t* out) {
    auto* h = static_cast<RefHandle*>(p);
    MinPlusOracle::HTripQueryScratch scratch;
    std::vector<dist_t> mat;
    h->oracle.queryAllPairs(toPoints(rc, k), h->grid, mat, scratch);
    std::memcpy(out, mat.data(), mat.size() * sizeof(dist_t));
}

// Time `reps` calls of the allocation-free queryAllPairs overload on each of
// `nthreads` threads (each with its own HTripQueryScratch; the oracle is only
// read).  Returns the wall time in seconds of the whole parallel section and
// writes the last matrix of thread 0 to `out` (may be null).
double ref_time_query(void* p, const int32_t* rc, int k, int nthreads, int reps, uint16_t* out) {
    auto* h = static_cast<RefHandle*>(p);
    const std::vector<Point> vps = toPoints(rc, k);
    if (nthreads < 1) nthreads = 1;
    std::vector<std::vector<dist_t>> mats(static_cast<size_t>(nthreads));
    std::vector<MinPlusOracle::HTripQueryScratch> scratch(static_cast<size_t>(nthreads));
    for (int t = 0; t < nthreads; ++t) h->oracle.queryAllPairs(vps, h->grid, mats[t], scratch[t]);
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; ++t) {
        pool.emplace_back([&, t]() {
            for (int r = 0; r < reps; ++r) h->oracle.queryAllPairs(vps, h->grid, mats[t], scratch[t]);
        });
    }
    for (auto& th : pool) th.join();
    const auto t1 = std::chrono::steady_clock::now();
    if (out) std::memcpy(out, mats[0].data(), mats[0].size() * sizeof(dist_t));
    return std::chrono::duration<double>(t1 - t0).count();
}

void ref_bfs_all_pairs(void* p, const int32_t* rc, int k, uint16_t* out) {
    auto* h = static_cast<RefHandle*>(p);
    const auto mat = BfsOracle::queryAllPairs(h->grid, toPoints(rc, k));
    std::memcpy(out, mat.data(), mat.size() * sizeof(dist_t));
}

int ref_S(void* p) { return static_cast<RefHandle*>(p)->oracle.S; }
int ref_H(void* p) { return static_cast<RefHandle*>(p)->oracle.H; }
int ref_num_leaves(void* p) { return static_cast<int>(static_cast<RefHandle*>(p)->oracle.leaves.size()); }
int ref_num_nodes(void* p, int lvl) {
    auto& o = static_cast<RefHandle*>(p)->oracle;
    if (lvl < 1 || lvl > static_cast<int>(o.levels.size())) return 0;
    return static_cast<int>(o.levels[static_cast<size_t>(lvl - 1)].size());
}
unsigned long long ref_total_memory(void* p) {
    return static_cast<unsigned long long>(static_cast<RefHandle*>(p)->oracle.totalMemoryBytes());
}
void ref_stats(void* p, int32_t* out3) {
    auto& s = static_cast<RefHandle*>(p)->oracle.last_batch_stats;
    out3[0] = s.n_touched_leaves;
    out3[1] = s.n_dirty_ancestors;
    out3[2] = s.n_pivots;
}

// Copy leaf `i`'s D (n*n) into out; returns n = b*b.
int ref_leaf_D(void* p, int i, uint16_t* out) {
    auto& L = static_cast<RefHandle*>(p)->oracle.leaves[static_cast<size_t>(i)];
    if (out) std::memcpy(out, L.D.data(), L.D.size() * sizeof(dist_t));
    return L.b * L.b;
}
// Copy leaf `i`'s S ((4b-4)^2) into out; returns 4b-4.
int ref_leaf_S(void* p, int i, uint16_t* out) {
    auto& L = static_cast<RefHandle*>(p)->oracle.leaves[static_cast<size_t>(i)];
    if (out) std::memcpy(out, L.S.data(), L.S.size() * sizeof(dist_t));
    return static_cast<int>(L.ports.size());
}
// Copy D_U of node `n` at level `lvl` (1-based); returns nV.
int ref_node_DU(void* p, int lvl, int n, uint16_t* out) {
    auto& N = static_cast<RefHandle*>(p)->oracle.levels[static_cast<size_t>(lvl - 1)][static_cast<size_t>(n)];
    if (out) std::memcpy(out, N.D_U.data(), N.D_U.size() * sizeof(dist_t));
    return static_cast<int>(N.V_U.size());
}
// Copy S_U of node; returns nExt.
int ref_node_SU(void* p, int lvl, int n, uint16_t* out) {
    auto& N = static_cast<RefHandle*>(p)->oracle.levels[static_cast<size_t>(lvl - 1)][static_cast<size_t>(n)];
    if (out) std::memcpy(out, N.S_U.data(), N.S_U.size() * sizeof(dist_t));
    return static_cast<int>(N.extPorts.size());
}
// Copy child_to_ext[q] of node (nP x nExt); returns its element count.
int ref_node_C2E(void* p, int lvl, int n, int q, uint16_t* out) {
    auto& N = static_cast<RefHandle*>(p)->oracle.levels[static_cast<size_t>(lvl - 1)][static_cast<size_t>(n)];
    const auto& m = N.child_to_ext[static_cast<size_t>(q)];
    if (out) std::memcpy(out, m.data(), m.size() * sizeof(dist_t));
    return static_cast<int>(m.size());
}
// Geometry of node: V_U points (2*nV ints), extPortIdx (nExt ints), childOffset (g*g+1 ints).
int ref_node_geometry(void* p, int lvl, int n, int32_t* vu, int32_t* ext_idx, int32_t* child_off) {
    auto& N = static_cast<RefHandle*>(p)->oracle.levels[static_cast<size_t>(lvl - 1)][static_cast<size_t>(n)];
    if (vu) for (size_t i = 0; i < N.V_U.size(); ++i) { vu[2 * i] = N.V_U[i].r; vu[2 * i + 1] = N.V_U[i].c; }
    if (ext_idx) for (size_t i = 0; i < N.extPortIdx.size(); ++i) ext_idx[i] = N.extPortIdx[i];
    if (child_off) for (size_t i = 0; i < N.childOffset.size(); ++i) child_off[i] = N.childOffset[i];
    return static_cast<int>(N.seam_candidates.size());
}

// Per-level checksum of the reference's matrices in the form the device
// library's htrip_state_digest uses: out[l] = sum mod 2^64 over matrices m
// (leaves[m].D for l = 0, levels[l-1][m].D_U above) and entries (i, j) of
// splitmix64(((m*n + i)*n + j) << 16 | value).  Returns H + 1 (the number of
// entries written).
int ref_digest(void* p, uint64_t* out) {
    auto& o = static_cast<RefHandle*>(p)->oracle;
    auto mix = [](uint64_t x) {
        x += 0x9E3779B97F4A7C15ull;
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        return x ^ (x >> 31);
    };
    auto sum = [&](const std::vector<dist_t>& D, uint64_t m, uint64_t n) {
        uint64_t acc = 0;
        for (uint64_t i = 0; i < n; ++i)
            for (uint64_t j = 0; j < n; ++j) acc += mix((((m * n + i) * n + j) << 16) | D[i * n + j]);
        return acc;
    };
    out[0] = 0;
    for (size_t m = 0; m < o.leaves.size(); ++m) {
        const uint64_t n = static_cast<uint64_t>(o.leaves[m].b) * o.leaves[m].b;
        out[0] += sum(o.leaves[m].D, m, n);
    }
    for (size_t l = 0; l < o.levels.size(); ++l) {
        out[l + 1] = 0;
        for (size_t m = 0; m < o.levels[l].size(); ++m)
            out[l + 1] += sum(o.levels[l][m].D_U, m, o.levels[l][m].V_U.size());
    }
    return static_cast<int>(o.levels.size()) + 1;
}

}  // extern "C"
