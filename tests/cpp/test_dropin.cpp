// The C++20 drop-in htrip::MinPlusOracle (include/htrip/) exercised the way
// the reference's own test executables exercise theirs (apps/test_exactness.cpp,
// apps/test_property_based.cpp): grids built here, the oracle driven through
// its public API, every k x k matrix compared bit-exactly with the checker.
//
// Checker: the plain-C restatement of the reference in oracle/ (its BFS
// all-pairs and its min-plus hierarchy, pinned against the reference's golden
// vectors elsewhere).  Exit status 0 = pass.
//
//   test_dropin              full suite on CUDA device 0
//   test_dropin --no-device  host-only checks: value types, and that the
//                            oracle refuses to run without a device
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "htrip/minplus_oracle.hpp"

extern "C" {
#include "htrip_oracle.h"
}

using namespace htrip;

namespace {

int g_fail = 0;

#define EXPECT(cond, ...)                                               \
    do {                                                                \
        if (!(cond)) {                                                  \
            ++g_fail;                                                   \
            std::fprintf(stderr, "FAIL %s:%d: ", __FILE__, __LINE__);   \
            std::fprintf(stderr, __VA_ARGS__);                          \
            std::fprintf(stderr, "\n");                                 \
        }                                                               \
    } while (0)

struct Rng {  // splitmix64
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    }
    int below(int n) { return int(next() % uint64_t(n)); }
};

GridMap noise_grid(int rows, int cols, double p_free, uint64_t seed) {
    GridMap g(rows, cols, CellState::Obstacle);
    Rng r{seed};
    for (auto& c : g.ground_truth) c = (r.next() % 1000) < p_free * 1000 ? CellState::Free : CellState::Obstacle;
    g.observed = g.ground_truth;
    return g;
}

GridMap rooms_grid(int rows, int cols, int room, uint64_t seed) {
    GridMap g(rows, cols, CellState::Obstacle);
    Rng r{seed};
    for (int y = 0; y < rows; ++y)
        for (int x = 0; x < cols; ++x)
            if (y % room != 0 && x % room != 0) g.ground_truth[size_t(g.index(y, x))] = CellState::Free;
    for (int y0 = 0; y0 < rows; y0 += room)
        for (int x0 = 0; x0 < cols; x0 += room) {
            const int dy = y0 + 1 + r.below(room - 1), dx = x0 + 1 + r.below(room - 1);
            if (dy < rows && x0 > 0) g.ground_truth[size_t(g.index(dy, x0))] = CellState::Free;
            if (dx < cols && y0 > 0) g.ground_truth[size_t(g.index(y0, dx))] = CellState::Free;
        }
    g.observed = g.ground_truth;
    return g;
}

std::vector<Point> sample_points(const GridMap& g, int k, uint64_t seed, int n_blocked) {
    std::vector<Point> free_cells, other;
    for (int i = 0; i < g.rows * g.cols; ++i)
        (g.observed[size_t(i)] == CellState::Free ? free_cells : other).push_back(g.point(i));
    Rng r{seed};
    std::vector<Point> out;
    for (int i = 0; i < k && !free_cells.empty(); ++i) {
        const int j = r.below(int(free_cells.size()));
        out.push_back(free_cells[size_t(j)]);
        free_cells.erase(free_cells.begin() + j);
    }
    for (int i = 0; i < n_blocked && !other.empty(); ++i) out.push_back(other[size_t(r.below(int(other.size())))]);
    out.push_back(Point(-3, 5));  // outside the grid: an INF row
    return out;
}

std::vector<int32_t> rc_of(const std::vector<Point>& p) {
    std::vector<int32_t> rc;
    for (auto& q : p) {
        rc.push_back(q.r);
        rc.push_back(q.c);
    }
    return rc;
}

std::vector<dist_t> bfs_matrix(const GridMap& g, const std::vector<Point>& vps) {
    std::vector<dist_t> m(vps.size() * vps.size());
    const auto rc = rc_of(vps);
    orc_bfs_all_pairs(g.observedBytes(), g.rows, g.cols, rc.data(), int(vps.size()), m.data());
    return m;
}

void expect_matrix(const std::vector<dist_t>& got, const std::vector<dist_t>& want, const char* what) {
    size_t bad = 0, first = 0;
    for (size_t i = 0; i < want.size(); ++i)
        if (got.size() != want.size() || got[i] != want[i]) {
            if (!bad) first = i;
            ++bad;
        }
    EXPECT(bad == 0 && got.size() == want.size(), "%s: %zu of %zu entries differ (first at %zu: %u vs %u)", what,
           bad, want.size(), first, unsigned(first < got.size() ? got[first] : 0), unsigned(want[first]));
}

// Suite 1 (test_exactness.cpp:100-145): a seam opened across two leaves.
void known_seam() {
    GridMap g(32, 32, CellState::Obstacle);
    g.setObserved(4, 16, CellState::Free);
    MinPlusOracle o(HierarchyConfig{8, 2, 2, 0});
    EXPECT(o.build(g), "build");
    g.setObserved(4, 15, CellState::Free);
    o.onCellOpened(Point(4, 15), g);
    EXPECT(o.queryAllPairs({Point(4, 15), Point(4, 16)}, g)[1] == 1, "seam distance");
    for (int c = 10; c <= 20; ++c) {
        g.setObserved(4, c, CellState::Free);
        o.onCellOpened(Point(4, c), g);
    }
    const std::vector<Point> vps = {Point(4, 10), Point(4, 13), Point(4, 16), Point(4, 20)};
    const auto m = o.queryAllPairs(vps, g);
    for (size_t i = 0; i < vps.size(); ++i)
        for (size_t j = 0; j < vps.size(); ++j)
            EXPECT(m[i * vps.size() + j] == std::abs(vps[i].c - vps[j].c), "corridor %zu %zu", i, j);
}

// Suite 8 (test_exactness.cpp:597-667): the tail-port geometry, BFS = 37.
void known_tail_port() {
    GridMap g(32, 32, CellState::Obstacle);
    auto fill = [&](int r0, int r1, int c0, int c1) {
        for (int r = r0; r < r1; ++r)
            for (int c = c0; c < c1; ++c) g.setObserved(r, c, CellState::Free);
    };
    fill(2, 3, 16, 32);
    fill(2, 16, 24, 25);
    fill(16, 21, 24, 25);
    fill(20, 21, 16, 32);
    fill(16, 32, 0, 16);
    MinPlusOracle o(HierarchyConfig{16, 2, 2, 0});
    EXPECT(o.build(g), "build");
    const auto m = o.queryAllPairs({Point(2, 24), Point(25, 10), Point(20, 20), Point(8, 24)}, g);
    EXPECT(m[1] == 37 && m[4] == 37, "tail port: %u %u", unsigned(m[1]), unsigned(m[4]));
}

// Suite 12 (test_exactness.cpp:845-893): separated halves, blocked viewpoint.
void known_blocked_viewpoint() {
    GridMap g(32, 32, CellState::Free);
    for (int r = 0; r < 32; ++r) g.setObserved(r, 16, CellState::Obstacle);
    MinPlusOracle o(HierarchyConfig{16, 2, 2, 0});
    EXPECT(o.build(g), "build");
    const std::vector<Point> vps = {Point(4, 4), Point(8, 12), Point(4, 20), Point(8, 28), Point(20, 16)};
    auto m = o.queryAllPairs(vps, g);
    EXPECT(m[4 * 5 + 4] == INF, "blocked diagonal");
    EXPECT(m[0 * 5 + 2] == INF && m[0 * 5 + 1] == 12, "halves %u %u", unsigned(m[2]), unsigned(m[1]));
    g.setObserved(8, 16, CellState::Free);
    o.onCellOpened(Point(8, 16), g);
    m = o.queryAllPairs(vps, g);
    EXPECT(m[2] < INF && m[4 * 5 + 4] == INF, "after opening");
}

void config_and_empty_grid() {
    MinPlusOracle o(HierarchyConfig{8, 3, 2, 0});  // g_w != g_h
    EXPECT(!o.build(GridMap(16, 16, CellState::Free)), "invalid config must not build");
    MinPlusOracle e(HierarchyConfig{8, 2, 2, 0});
    EXPECT(!e.build(GridMap(0, 0)), "empty grid must not build");
    // an unbuilt oracle: INF everywhere but the passable diagonal
    GridMap g(8, 8, CellState::Free);
    const auto m = e.queryAllPairs({Point(1, 1), Point(2, 2)}, g);
    EXPECT(m.size() == 4 && m[0] == 0 && m[1] == INF && m[3] == 0, "unbuilt query");
}

// Random grids, hidden cells revealed in batches; after every batch the
// matrix equals the checker's min-plus hierarchy and its BFS, and the batch
// statistics equal the checker's.
void random_openings(const char* kind, int rows, int cols, int b, int g, uint64_t seed, int nb, int bs) {
    GridMap truth = std::strcmp(kind, "rooms") == 0 ? rooms_grid(rows, cols, 8, seed) : noise_grid(rows, cols, 0.72, seed);
    GridMap obs = truth;
    Rng r{seed * 31 + 7};
    std::vector<Point> hidden;
    for (int i = 0; i < rows * cols; ++i)
        if (truth.observed[size_t(i)] == CellState::Free && r.below(4) == 0 && int(hidden.size()) < nb * bs)
            hidden.push_back(truth.point(i));
    for (auto& p : hidden) obs.setObserved(p, CellState::Unknown);
    MinPlusOracle dev(HierarchyConfig{b, g, g, 0});
    EXPECT(dev.build(obs), "build %s", kind);
    orc_t* chk = orc_create(b, g);
    orc_build(chk, obs.observedBytes(), rows, cols);
    EXPECT(dev.S == orc_S(chk) && dev.H == orc_H(chk), "shape S=%d H=%d", dev.S, dev.H);
    MinPlusOracle::HTripQueryScratch scratch;
    std::vector<dist_t> got;
    for (int bi = 0; bi * bs < int(hidden.size()); ++bi) {
        std::vector<Point> cells(hidden.begin() + bi * bs,
                                 hidden.begin() + std::min<size_t>(hidden.size(), size_t(bi + 1) * bs));
        for (auto& p : cells) obs.setObserved(p, CellState::Free);
        dev.onBatchCellsOpened(cells, obs);
        const auto crc = rc_of(cells);
        orc_open_batch(chk, crc.data(), int(cells.size()), obs.observedBytes(), rows, cols);
        int32_t st[3];
        orc_stats(chk, st);
        EXPECT(dev.last_batch_stats.n_touched_leaves == st[0] && dev.last_batch_stats.n_dirty_ancestors == st[1] &&
                   dev.last_batch_stats.n_pivots == st[2],
               "%s batch %d stats (%d %d %d) vs (%d %d %d)", kind, bi, dev.last_batch_stats.n_touched_leaves,
               dev.last_batch_stats.n_dirty_ancestors, dev.last_batch_stats.n_pivots, st[0], st[1], st[2]);
        const auto vps = sample_points(obs, 11, seed + uint64_t(bi), 2);
        dev.queryAllPairs(vps, obs, got, scratch);
        std::vector<dist_t> want(vps.size() * vps.size());
        const auto vrc = rc_of(vps);
        orc_query(chk, vrc.data(), int(vps.size()), obs.observedBytes(), rows, cols, want.data());
        expect_matrix(got, want, "query vs oracle hierarchy");
        expect_matrix(got, bfs_matrix(obs, vps), "query vs BFS");
    }
    orc_destroy(chk);
}

// Copies are deep: a copy taken before an update still answers for the old grid.
void copy_semantics() {
    GridMap truth = rooms_grid(32, 32, 8, 77);
    GridMap obs = truth;
    std::vector<Point> cells;
    for (int c = 1; c < 31; c += 3) cells.push_back(Point(12, c));
    for (auto& p : cells) obs.setObserved(p, CellState::Unknown);
    MinPlusOracle a(HierarchyConfig{8, 2, 2, 0});
    EXPECT(a.build(obs), "build");
    MinPlusOracle before = a;        // copy constructor
    MinPlusOracle assigned;          // copy assignment onto a default oracle
    assigned = a;
    const GridMap old = obs;
    for (auto& p : cells) obs.setObserved(p, CellState::Free);
    a.onBatchCellsOpened(cells, obs);
    const auto vps = sample_points(old, 12, 5, 0);
    expect_matrix(before.queryAllPairs(vps, old), bfs_matrix(old, vps), "copy keeps the old index");
    expect_matrix(assigned.queryAllPairs(vps, old), bfs_matrix(old, vps), "assigned copy keeps the old index");
    const auto vps2 = sample_points(obs, 12, 6, 0);
    expect_matrix(a.queryAllPairs(vps2, obs), bfs_matrix(obs, vps2), "original sees the opening");
    MinPlusOracle moved = std::move(a);
    expect_matrix(moved.queryAllPairs(vps2, obs), bfs_matrix(obs, vps2), "moved oracle");
    EXPECT(before.totalMemoryBytes() > 0 && before.totalMemoryBytes() == moved.totalMemoryBytes(), "memory bytes");
    EXPECT(before.numLeaves() == 16, "numLeaves %zu", before.numLeaves());
}

// Suite 11 (test_exactness.cpp:800-840): non-square grid padded to S.
void non_square() {
    GridMap g = noise_grid(20, 44, 0.8, 11);
    MinPlusOracle o(HierarchyConfig{8, 2, 2, 0});
    EXPECT(o.build(g), "build");
    EXPECT(o.S == 64 && o.H == 3, "S=%d H=%d", o.S, o.H);
    const auto vps = sample_points(g, 20, 3, 1);
    expect_matrix(o.queryAllPairs(vps, g), bfs_matrix(g, vps), "non-square");
    EXPECT(o.findLcaLevel(Point(0, 0), Point(0, 7)) == 0 && o.findLcaLevel(Point(0, 0), Point(0, 8)) == 1 &&
               o.findLcaLevel(Point(0, 0), Point(0, 40)) == 3,
           "lca");
    EXPECT(o.tileIndexAtLevel(1, 1, 1) == 5 && o.leafIndex(3, 2) == 19, "tile index");
}

// queryDistance (Suite 15, test_exactness.cpp:989-1023: equals the matrix
// entry), queryAllPairsIncremental (test_property_based.cpp: incremental ==
// full across openings) and liftRoot (the grown index still answers exactly).
void next_members() {
    GridMap truth = rooms_grid(32, 32, 8, 91);
    GridMap obs = truth;
    std::vector<Point> cells;
    for (int c = 1; c < 31; c += 2) cells.push_back(Point(20, c));
    for (auto& p : cells) obs.setObserved(p, CellState::Unknown);
    MinPlusOracle o(HierarchyConfig{8, 2, 2, 0});
    EXPECT(o.build(obs), "build");
    const auto vps = sample_points(truth, 14, 9, 1);
    MinPlusOracle::HTripQueryScratch scratch;
    MinPlusOracle::HTripIncrementalState state;
    std::vector<dist_t> inc, full;
    o.queryAllPairsIncremental(vps, obs, inc, scratch, state);
    expect_matrix(inc, bfs_matrix(obs, vps), "incremental first call");
    const size_t k = vps.size();
    for (size_t i = 0; i < k; ++i)
        for (size_t j = 0; j < k; ++j)
            EXPECT(o.queryDistance(vps[i], vps[j], obs) == inc[i * k + j], "queryDistance %zu %zu", i, j);
    for (auto& p : cells) obs.setObserved(p, CellState::Free);
    o.onBatchCellsOpened(cells, obs);
    o.queryAllPairsIncremental(vps, obs, inc, scratch, state);
    o.queryAllPairs(vps, obs, full, scratch);
    expect_matrix(inc, full, "incremental == full after an opening");
    expect_matrix(inc, bfs_matrix(obs, vps), "incremental vs BFS");
    EXPECT(state.initialized && state.last_update_counter == o.update_counter, "incremental state");
    // grow the root over a 64 x 64 grid whose old quadrant is unchanged
    GridMap big = rooms_grid(64, 64, 8, 92);
    for (int r = 0; r < 32; ++r)
        for (int c = 0; c < 32; ++c) big.setObserved(r, c, obs.getObserved(r, c));
    const uint64_t epoch = o.epoch;
    o.liftRoot(big);
    EXPECT(o.S == 64 && o.H == 3 && o.epoch == epoch + 1, "liftRoot shape S=%d H=%d", o.S, o.H);
    const auto vps2 = sample_points(big, 16, 10, 1);
    expect_matrix(o.queryAllPairs(vps2, big), bfs_matrix(big, vps2), "query after liftRoot");
    o.queryAllPairsIncremental(vps2, big, inc, scratch, state);
    expect_matrix(inc, bfs_matrix(big, vps2), "incremental after liftRoot (epoch changed)");
}

// Exact weighted all-pairs by a plain Dijkstra over GridMap::edgeWeight
// (the test's own checker).
std::vector<dist_t> dijkstra_matrix(const GridMap& g, const std::vector<Point>& vps) {
    const size_t k = vps.size(), n = size_t(g.rows) * g.cols;
    std::vector<dist_t> m(k * k, INF);
    std::vector<uint32_t> d(n);
    for (size_t a = 0; a < k; ++a) {
        if (!g.isPassable(vps[a])) continue;
        std::fill(d.begin(), d.end(), UINT32_MAX);
        std::vector<std::pair<uint32_t, int>> pq{{0u, g.index(vps[a])}};
        d[size_t(g.index(vps[a]))] = 0;
        while (!pq.empty()) {
            std::pop_heap(pq.begin(), pq.end(), std::greater<>());
            const auto [du, u] = pq.back();
            pq.pop_back();
            if (du > d[size_t(u)]) continue;
            const Point pu = g.point(u);
            const int dr[4] = {-1, 1, 0, 0}, dc[4] = {0, 0, -1, 1};
            for (int t = 0; t < 4; ++t) {
                const Point pv(pu.r + dr[t], pu.c + dc[t]);
                if (!g.isPassable(pv)) continue;
                const dist_t w = g.edgeWeight(pu, pv);
                if (w >= INF) continue;
                const uint32_t alt = du + w;
                if (alt < d[size_t(g.index(pv))]) {
                    d[size_t(g.index(pv))] = alt;
                    pq.push_back({alt, g.index(pv)});
                    std::push_heap(pq.begin(), pq.end(), std::greater<>());
                }
            }
        }
        for (size_t b = 0; b < k; ++b)
            if (g.isPassable(vps[b])) m[a * k + b] = dist_t(std::min<uint32_t>(d[size_t(g.index(vps[b]))], INF));
    }
    return m;
}

// Weighted grids: build, opening, onCellWeightChanged, onTileWeightsChanged.
void weighted_grid() {
    GridMap truth = rooms_grid(32, 32, 8, 93);
    uint64_t x = 93;
    for (int r = 0; r < 32; ++r)
        for (int c = 0; c < 32; ++c) {
            x = x * 6364136223846793005ull + 1442695040888963407ull;
            truth.setCellWeight(r, c, dist_t(1 + (x >> 60) % 7));
        }
    GridMap obs = truth;
    std::vector<Point> cells;
    for (int c = 1; c < 31; c += 3) cells.push_back(Point(12, c));
    for (auto& p : cells) obs.setObserved(p, CellState::Unknown);
    MinPlusOracle o(HierarchyConfig{8, 2, 2, 0});
    EXPECT(o.build(obs), "weighted build");
    const auto vps = sample_points(truth, 14, 11, 1);
    expect_matrix(o.queryAllPairs(vps, obs), dijkstra_matrix(obs, vps), "weighted build vs Dijkstra");
    for (auto& p : cells) obs.setObserved(p, CellState::Free);
    o.onBatchCellsOpened(cells, obs);
    expect_matrix(o.queryAllPairs(vps, obs), dijkstra_matrix(obs, vps), "weighted opening vs Dijkstra");
    const uint64_t epoch = o.epoch;
    o.onCellWeightChanged(vps[0], 25, obs);
    EXPECT(obs.getCellWeight(vps[0]) == 25 && o.epoch == epoch + 1, "onCellWeightChanged sets the grid");
    expect_matrix(o.queryAllPairs(vps, obs), dijkstra_matrix(obs, vps), "after onCellWeightChanged");
    o.onTileWeightsChanged(vps[1].c / 8, vps[1].r / 8, {{vps[1], dist_t(3)}, {Point(vps[1].r, vps[1].c / 8 * 8), dist_t(9)}},
                           obs);
    expect_matrix(o.queryAllPairs(vps, obs), dijkstra_matrix(obs, vps), "after onTileWeightsChanged");
}

int host_only() {
    static_assert(add_dist(INF, 0) == INF && add_dist(59999, 1) == INF && add_dist(59998, 1) == 59999);
    static_assert(add_dist(1, 2, 3) == 6 && add_dist(30000, 30000, 1) == INF);
    static_assert(HierarchyConfig{}.isValid() && !HierarchyConfig{8, 2, 3, 0}.isValid());
    static_assert(Point(1, 2).manhattan(Point(4, -2)) == 7 && Point(1, 2) < Point(1, 3));
    GridMap g(3, 4, CellState::Unknown);
    g.setObserved(1, 2, CellState::Free);
    EXPECT(g.isPassable(1, 2) && !g.isPassable(0, 0) && !g.isPassable(-1, 2), "isPassable");
    EXPECT(g.getObserved(9, 9) == CellState::Obstacle, "out of bounds is an obstacle");
    bool threw = false;
    try {
        MinPlusOracle o(HierarchyConfig{8, 2, 2, 0});
    } catch (const DeviceError& e) {
        threw = e.status == 6;  // HTRIP_ERR_NO_DEVICE
    }
    EXPECT(threw, "no device must raise DeviceError(HTRIP_ERR_NO_DEVICE)");
    return g_fail ? 1 : 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc > 1 && std::strcmp(argv[1], "--no-device") == 0) {
        const int rc = host_only();
        std::printf("%s\n", rc ? "host checks FAILED" : "host checks passed");
        return rc;
    }
    known_seam();
    known_tail_port();
    known_blocked_viewpoint();
    config_and_empty_grid();
    random_openings("rooms", 32, 32, 8, 2, 11, 5, 9);
    random_openings("noise", 48, 40, 8, 2, 12, 4, 13);
    random_openings("noise", 64, 64, 16, 2, 13, 3, 40);
    random_openings("noise", 64, 64, 4, 4, 14, 3, 25);
    random_openings("rooms", 16, 16, 16, 2, 15, 2, 6);  // H = 0
    copy_semantics();
    non_square();
    next_members();
    weighted_grid();
    std::printf("%s (%d failures)\n", g_fail ? "drop-in suite FAILED" : "drop-in suite passed", g_fail);
    return g_fail ? 1 : 0;
}
