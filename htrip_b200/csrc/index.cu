// Host side of the B200 HTRIP index: geometry tables, the device arena,
// build / update / query orchestration and the C ABI of include/htrip_b200.h.
//
// Reference call stacks mirrored here (ozaslan/htrip):
//   build               src/minplus_oracle.cpp:48-137
//   onBatchCellsOpened  src/minplus_oracle.cpp:530-729
//   onCellOpened        src/minplus_oracle.cpp:139-177 (same state as a batch of one)
//   queryAllPairs       src/minplus_oracle.cpp:934-1419
#include "../../include/htrip_b200.h"
#include "kernels.cuh"
#include "minplus.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <map>
#include <tuple>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <exception>
#include <condition_variable>
#include <thread>
#include <functional>
#include <new>
#include <numeric>
#include <string>
#include <vector>

using hb::MatSet;

namespace {

thread_local std::string g_err;

htrip_status fail(htrip_status s, const std::string& msg) {
    g_err = msg;
    return s;
}

struct CudaError {
    cudaError_t e;
    const char* what;
};

inline void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError{e, what};
}

// Canonical perimeter order of a side-s tile (reference getTilePorts,
// src/leaf_tile.cpp:11-30): top row, bottom row, left column without
// corners, right column without corners.
void port_local(int s, int p, int& r, int& c) {
    if (p < s) { r = 0; c = p; }
    else if (p < 2 * s) { r = s - 1; c = p - s; }
    else if (p < 3 * s - 2) { r = p - 2 * s + 1; c = 0; }
    else { r = p - (3 * s - 2) + 1; c = s - 1; }
}

// Inverse of port_local (reference getPortIndexInTile, internal_node.cpp:290-304).
int port_index(int r, int c, int s) {
    if (r == 0 && c >= 0 && c < s) return c;
    if (r == s - 1 && c >= 0 && c < s) return s + c;
    if (c == 0 && r > 0 && r < s - 1) return 2 * s + r - 1;
    if (c == s - 1 && r > 0 && r < s - 1) return 3 * s - 2 + r - 1;
    return -1;
}

int pad_order(int n) {
    if (n <= 64) return 64;
    if (n <= 128) return 128;
    return (n + 255) / 256 * 256;
}

// Device buffer.  A buffer that has to grow grows by at least half its size,
// so scratch that creeps up call by call is reallocated (a device-wide
// synchronisation) only a few times; a first reservation is exact.
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    void reserve(size_t m) {
        if (m <= n) return;
        if (n) m = std::max(m, n + n / 2);
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        ck(cudaMalloc(&p, m * sizeof(T)), "cudaMalloc");
        n = m;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

// Memory pool of a device for the scratch arenas (PoolBuf): it keeps what
// is given back (release threshold: never), so a growing arena reuses it.
cudaMemPool_t scratch_pool(int device) {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    std::lock_guard<std::mutex> lk(mu);
    cudaMemPool_t& pool = pools[std::clamp(device, 0, 63)];
    if (!pool) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        ck(cudaMemPoolCreate(&pool, &props), "cudaMemPoolCreate");
        uint64_t keep = UINT64_MAX;
        ck(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
    }
    return pool;
}

// Device scratch of the per-call paths (the query and update arenas): grows
// like DevBuf, but stream-ordered on the stream that uses the arena, from
// the device's scratch pool.  Growing a DevBuf frees the old block with
// cudaFree, which synchronizes the device and, with most of the GPU's memory
// held by resident indexes, measured up to 0.3 s for one call; a block freed
// to the pool is reused instead, and nothing waits.
template <class T>
struct PoolBuf {
    T* p = nullptr;
    size_t n = 0;
    void reserve(size_t m, cudaStream_t st) {
        if (m <= n) return;
        if (n) m = std::max(m, n + n / 2);
        int device = 0;
        ck(cudaGetDevice(&device), "cudaGetDevice");
        if (p) ck(cudaFreeAsync(p, st), "cudaFreeAsync");
        p = nullptr;
        n = 0;
        ck(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p), m * sizeof(T), scratch_pool(device), st),
           "cudaMallocFromPoolAsync");
        n = m;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

struct Level {
    int lvl = 0;
    int side = 0;      // tile side (b for leaves, s for nodes)
    int cs = 0;        // child side (nodes)
    int n = 0;         // logical order (b^2 or nV)
    int NP = 0;        // padded order
    int nExt = 0;      // 4*side - 4
    int nP = 0;        // ports per child (nodes)
    int nodes_x = 0;
    int nnodes = 0;
    std::vector<int> ext;    // exterior port -> matrix index
    std::vector<int> seams;  // 6 ints per seam candidate
    int nseams = 0;
    DevBuf<int> d_ext, d_seams, d_ext_inv;
    DevBuf<uint16_t> mat;
    DevBuf<uint8_t> kflag;
    DevBuf<int> klist, kcnt;
    DevBuf<uint8_t> dec;
    // device-driven openings: per matrix index, 1 = an exterior port (leaf
    // perimeter cell / node exterior port); per node, the stamp of the last
    // opening call whose update decreased its exterior block (dstamp) and of
    // the last call that put it on the level's work list (mstamp)
    DevBuf<uint8_t> d_isext;
    DevBuf<uint32_t> dstamp, mstamp;
    MatSet ms() const { return MatSet{mat.p, n, NP}; }
    void release() {
        d_ext.release(); d_seams.release(); d_ext_inv.release(); mat.release(); kflag.release();
        klist.release(); kcnt.release(); dec.release(); d_isext.release(); dstamp.release(); mstamp.release();
    }
};

inline size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// Cooperative launches (the query kernel, the opening kernel) of one device
// run one after another on the GPU, whatever stream issued them: each waits
// for an event recorded after the previous one.  Each such grid takes every
// SM, so running two at once gains nothing, and ordering them keeps two
// grids that wait on their own CTAs from holding parts of the GPU at once.
// The host only takes a short lock; nothing waits on the host.
constexpr int kCoopMaxDevices = 64;
struct CoopChain {
    std::mutex mu;
    cudaEvent_t ev = nullptr;
    cudaStream_t st = nullptr;
};
CoopChain g_coop[kCoopMaxDevices];

template <class F>
void coop_launch(int device, cudaStream_t st, F&& launch, const char* what) {
    CoopChain& c = g_coop[std::clamp(device, 0, kCoopMaxDevices - 1)];
    std::lock_guard<std::mutex> lk(c.mu);
    if (c.ev && c.st != st) ck(cudaStreamWaitEvent(st, c.ev, 0), "cooperative launch order");
    if (!c.ev) ck(cudaEventCreateWithFlags(&c.ev, cudaEventDisableTiming), "event");
    ck(launch(), what);
    ck(cudaEventRecord(c.ev, st), "cooperative launch order");
    c.st = st;
}

// Pinned host buffer (grows, never shrinks).  Pinning pages costs about a
// millisecond per allocation, so a first reservation takes at least 64 KB
// and growth at least half again.
struct HostBuf {
    unsigned char* p = nullptr;
    size_t n = 0;
    void reserve(size_t m) {
        if (m <= n) return;
        m = std::max(m, n ? n + n / 2 : (size_t)64 * 1024);
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
        ck(cudaHostAlloc(reinterpret_cast<void**>(&p), m, cudaHostAllocDefault), "cudaHostAlloc");
        n = m;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
    }
};

// Device scratch of query launches: an arena laid out per launch
// (LaunchLayout), pinned staging of its head and of the results, the grid
// size of the cooperative kernel and the events around the last launch.
struct QueryArena {
    PoolBuf<unsigned char> dev;
    HostBuf stage, outstage;
    int grid = 0;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool ev_valid = false;
    uint64_t last_h2d = 0, last_d2h = 0;
    size_t last_words = 0;  // arena offset of the last launch's words
    int last_phases = 0;
    // device-planned queries: host-mapped record the planner writes (one
    // 8-byte word: seq << 32 | status << 26 | viewpoints << 13 | largest root
    // child group), the sequence number of the last planned call and the
    // tile hint taken from it
    int* info = nullptr;
    int* info_dev = nullptr;
    int plan_seq = 0, info_k_last = 0;
    int hint_k = 0, hint_ns = 0, hint_group = 0;
    // ticket counter of the planner's blocks and its value after the last
    // planned launch
    DevBuf<unsigned> ticket;
    unsigned ticket_next = 0;
    void release() {
        dev.release();
        stage.release();
        outstage.release();
        ticket.release();
        ticket_next = 0;
        if (info) cudaFreeHost(info);
        info = info_dev = nullptr;
        plan_seq = hint_k = 0;
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        ev[0] = ev[1] = nullptr;
        ev_valid = false;
    }
};

// Scratch of update launches (build closures and openings): the device
// array of matrix descriptors with the launch's edge / seam lists and
// per-slot / per-task read-back words, exterior snapshots, closure panels
// and tile flags; pinned staging for the upload and the read-backs.
struct UpdateArena {
    PoolBuf<unsigned char> dev;
    DevBuf<uint16_t> snap;
    PoolBuf<uint16_t> panel;
    PoolBuf<uint8_t> pflags;
    HostBuf stage, rb;
    cudaEvent_t ev_cnt = nullptr;  // an opening level's pivot counts reached the host
    int open_grid = 0;             // CTAs of the persistent opening kernel
    // phase time stamps of the last device-driven opening launch (device,
    // and where they are in the arena)
    size_t trace_off = 0;
    int trace_valid = 0;
    void release() {
        dev.release();
        snap.release();
        panel.release();
        pflags.release();
        stage.release();
        rb.release();
        if (ev_cnt) cudaEventDestroy(ev_cnt);
        ev_cnt = nullptr;
        trace_valid = 0;
    }
};

}  // namespace

struct htrip_index {
    int device = 0;
    cudaStream_t stream = nullptr;
    int b = 16, g = 2;
    bool built = false;
    bool offloaded = false;  // matrices parked in host memory (htrip_offload)
    std::vector<std::vector<uint16_t>> parked;  // per level matrices, then the passability mirror
    size_t parked_pass = 0;
    uint64_t ref_bytes = 0;  // the reference's totalMemoryBytes accounting of this index
    uint64_t open_ops = 0, open_bytes = 0;  // algorithmic work of the last opening call
    // per level of the last opening call: {active matrices, sum of pivot
    // counts, largest pivot count, closure rounds}
    std::vector<std::array<int64_t, 4>> open_levels;
    // query launches of this index count their executed work (a measurement
    // mode: a few atomics per work unit)
    bool count_work = false;
    // stamp of the last device-driven opening call (per-node stamps in the
    // level arrays compare against it; never 0)
    uint32_t open_stamp = 0;
    // the level arrays' stamps were (re)allocated this many times, and this
    // many openings ran on the host-driven path (which does not stamp): an
    // incremental query that saw other values re-lifts everything
    uint64_t stamp_epoch = 0, host_opens = 0;
    // opening bucketing scratch (all -1 between calls; a call resets the
    // entries it set): slot of a touched leaf / of a seam node per level
    std::vector<int> open_leaf_slot;
    std::vector<std::vector<int>> open_seam_slot;
    uint64_t epoch = 0;           // build / root growth count (reference MinPlusOracle::epoch)
    uint64_t update_counter = 0;  // opening calls since creation
    int S = 0, H = 0, rows = 0, cols = 0, leaves_x = 0;
    std::vector<Level> L;
    DevBuf<uint8_t> pass;
    // scratch of the index's own build / opening launches
    UpdateArena u;
    // query scratch: one device arena per launch (QueryArena) plus pinned
    // host staging for its parameter block / plans and for the result
    QueryArena q;
    htrip_batch_stats stats{0, 0, 0};
    // Per-cell traversal weights (GridMap::weights, grid_map.hpp:56) as the
    // caller last gave them (wrows x wcols; empty: every weight is 1), and
    // their device mirror over S x S (null while unweighted).  Kept across
    // builds and offloads.
    std::vector<uint16_t> wgrid;
    int wrows = 0, wcols = 0;
    DevBuf<uint16_t> wts;

    ~htrip_index() {
        release();
        wts.release();
    }
    void release() {
        for (auto& l : L) l.release();
        L.clear();
        pass.release();
        u.release();
        q.release();
    }
};


// A launch context for batched calls over many indexes of one device
// (htrip_query_batch / htrip_open_batch): its own stream and query arena.
struct htrip_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    QueryArena q;
    UpdateArena u;
    ~htrip_batch() { q.release(); u.release(); }
};

namespace {

// ---------------------------------------------------------------------------
// Geometry
// ---------------------------------------------------------------------------
void make_levels(htrip_index* h) {
    const int b = h->b, g = h->g;
    h->L.clear();
    h->L.resize(h->H + 1);
    Level& L0 = h->L[0];
    L0.lvl = 0;
    L0.side = b;
    L0.n = b * b;
    L0.NP = pad_order(L0.n);
    L0.nExt = 4 * b - 4;
    L0.nodes_x = h->S / b;
    L0.nnodes = L0.nodes_x * L0.nodes_x;
    L0.ext.resize(L0.nExt);
    for (int e = 0; e < L0.nExt; ++e) {
        int r, c;
        port_local(b, e, r, c);
        L0.ext[e] = r * b + c;
    }
    int cs = b;
    for (int l = 1; l <= h->H; ++l) {
        Level& Lv = h->L[l];
        Lv.lvl = l;
        Lv.cs = cs;
        Lv.side = cs * g;
        Lv.nP = 4 * cs - 4;
        Lv.n = g * g * Lv.nP;
        Lv.NP = pad_order(Lv.n);
        Lv.nExt = 4 * Lv.side - 4;
        Lv.nodes_x = h->S / Lv.side;
        Lv.nnodes = Lv.nodes_x * Lv.nodes_x;
        // V_U coordinate lookup (node-local) -> index
        const int s = Lv.side;
        auto vidx = [&](int r, int c) -> int {
            if (r < 0 || c < 0 || r >= s || c >= s) return -1;
            const int q = (r / cs) * g + (c / cs);
            const int p = port_index(r % cs, c % cs, cs);
            return p < 0 ? -1 : q * Lv.nP + p;
        };
        Lv.ext.resize(Lv.nExt);
        for (int e = 0; e < Lv.nExt; ++e) {
            int r, c;
            port_local(s, e, r, c);
            Lv.ext[e] = vidx(r, c);
        }
        // Seam candidates: 4-adjacent V_U pairs in different children
        // (reference InternalNode ctor, internal_node.cpp:72-89).
        Lv.seams.clear();
        for (int q = 0; q < g * g; ++q) {
            const int cy = q / g, cx = q % g;
            for (int p = 0; p < Lv.nP; ++p) {
                int pr, pc;
                port_local(cs, p, pr, pc);
                const int r = cy * cs + pr, c = cx * cs + pc;
                const int u = q * Lv.nP + p;
                const int nb[2][2] = {{r, c + 1}, {r + 1, c}};
                for (auto& rc : nb) {
                    const int v = vidx(rc[0], rc[1]);
                    if (v < 0 || v / Lv.nP == q) continue;
                    Lv.seams.insert(Lv.seams.end(), {u, v, r, c, rc[0], rc[1]});
                }
            }
        }
        Lv.nseams = (int)Lv.seams.size() / 6;
        cs *= g;
    }
}

// The reference's accounting of an index of this geometry: D and S of
// every leaf, D_U, S_U and child_to_ext of every node
// (MinPlusOracle::totalMemoryBytes, minplus_oracle.cpp:2116-2134).
uint64_t reference_bytes(const htrip_index* h) {
    const Level& L0 = h->L[0];
    uint64_t ref = (uint64_t)L0.nnodes * ((uint64_t)L0.n * L0.n + (uint64_t)L0.nExt * L0.nExt) * 2;
    for (int l = 1; l <= h->H; ++l) {
        const Level& Lv = h->L[l];
        ref += (uint64_t)Lv.nnodes * ((uint64_t)Lv.n * Lv.n + (uint64_t)Lv.nExt * Lv.nExt + (uint64_t)Lv.n * Lv.nExt) * 2;
    }
    return ref;
}

// GridMap::getCellWeight (grid_map.hpp:273-278): INF outside the grid and on
// obstacles, else the caller's weight (1 without weights).
uint16_t host_cell_weight(const htrip_index* h, int r, int c, const uint8_t* obs, int rows, int cols) {
    if (r < 0 || c < 0 || r >= rows || c >= cols || obs[(size_t)r * cols + c] == 2) return hb::INF;
    if (h->wgrid.empty() || r >= h->wrows || c >= h->wcols) return 1;
    return h->wgrid[(size_t)r * h->wcols + c];
}

// The weights' device mirror over the index's S x S (1 outside the grid,
// where no cell is passable).
void upload_weights(htrip_index* h) {
    if (h->wgrid.empty()) {
        h->wts.release();
        return;
    }
    const int S = h->S;
    std::vector<uint16_t> w((size_t)S * S, 1);
    for (int r = 0; r < std::min(h->wrows, S); ++r)
        std::memcpy(w.data() + (size_t)r * S, h->wgrid.data() + (size_t)r * h->wcols,
                    std::min(h->wcols, S) * sizeof(uint16_t));
    h->wts.reserve(w.size());
    ck(cudaMemcpyAsync(h->wts.p, w.data(), w.size() * sizeof(uint16_t), cudaMemcpyHostToDevice, h->stream),
       "weights");
}

// Listed leaves holding a passable cell of weight != 1: the reference builds
// those with Dijkstra (leaf_tile.cpp:81-96, 154-192), the others with BFS.
std::vector<int> weighted_leaves(const htrip_index* h, const std::vector<int>& leaves, const uint8_t* obs, int rows,
                                 int cols) {
    std::vector<int> out;
    if (h->wgrid.empty()) return out;
    const int b = h->b;
    for (int leaf : leaves) {
        const int R0 = (leaf / h->leaves_x) * b, C0 = (leaf % h->leaves_x) * b;
        bool w = false;
        for (int r = R0; r < R0 + b && r < rows && !w; ++r)
            for (int c = C0; c < C0 + b && c < cols && !w; ++c)
                w = obs[(size_t)r * cols + c] == 1 && host_cell_weight(h, r, c, obs, rows, cols) != 1;
        if (w) out.push_back(leaf);
    }
    return out;
}

void close_matrices(htrip_index* h, Level& Lv, const std::vector<int>& act);

// Leaf matrices of the listed leaves (all when `leaves` is null) from the
// passability mirror: bit-parallel BFS, then, for leaves with non-unit
// weights, the weighted adjacency closed over its passable cells.
void build_leaves(htrip_index* h, const std::vector<int>* leaves, const uint8_t* obs, int rows, int cols) {
    cudaStream_t st = h->stream;
    Level& L0 = h->L[0];
    DevBuf<int> list;
    std::vector<int> all;
    if (!leaves) {
        all.resize(L0.nnodes);
        std::iota(all.begin(), all.end(), 0);
        hb::launch_leaf_bfs(h->pass.p, h->S, h->b, h->leaves_x, L0.nnodes, L0.ms(), st);
    } else if (!leaves->empty()) {
        list.reserve(leaves->size());
        ck(cudaMemcpyAsync(list.p, leaves->data(), leaves->size() * sizeof(int), cudaMemcpyHostToDevice, st), "list");
        hb::launch_leaf_bfs(h->pass.p, h->S, h->b, h->leaves_x, (int)leaves->size(), L0.ms(), st, list.p);
    }
    ck(cudaGetLastError(), "leaf bfs");
    const std::vector<int> wl = weighted_leaves(h, leaves ? *leaves : all, obs, rows, cols);
    if (!wl.empty()) {
        DevBuf<int> wlist;
        wlist.reserve(wl.size());
        ck(cudaMemcpyAsync(wlist.p, wl.data(), wl.size() * sizeof(int), cudaMemcpyHostToDevice, st), "list");
        hb::launch_leaf_weight_init(h->pass.p, h->wts.p, h->S, h->b, h->leaves_x, (int)wl.size(), L0.ms(),
                                    L0.kflag.p, wlist.p, st);
        ck(cudaGetLastError(), "weighted leaf init");
        close_matrices(h, L0, wl);  // synchronises before returning
        wlist.release();
    }
    ck(cudaStreamSynchronize(st), "leaf sync");
    list.release();
}

void alloc_levels(htrip_index* h) {
    for (auto& Lv : h->L) {
        Lv.mat.reserve((size_t)Lv.nnodes * Lv.NP * Lv.NP);
        Lv.d_ext.reserve(std::max(1, Lv.nExt));
        ck(cudaMemcpyAsync(Lv.d_ext.p, Lv.ext.data(), Lv.nExt * sizeof(int), cudaMemcpyHostToDevice, h->stream), "ext");
        if (Lv.nseams) {
            Lv.d_seams.reserve(Lv.seams.size());
            ck(cudaMemcpyAsync(Lv.d_seams.p, Lv.seams.data(), Lv.seams.size() * sizeof(int), cudaMemcpyHostToDevice,
                               h->stream), "seams");
        }
        if (Lv.lvl >= 1) {
            std::vector<int> inv(Lv.NP, -1);
            for (int e = 0; e < Lv.nExt; ++e) inv[Lv.ext[e]] = e;
            Lv.d_ext_inv.reserve(Lv.NP);
            ck(cudaMemcpyAsync(Lv.d_ext_inv.p, inv.data(), Lv.NP * sizeof(int), cudaMemcpyHostToDevice, h->stream),
               "ext_inv");
        }
        Lv.kflag.reserve((size_t)Lv.nnodes * Lv.NP);
        ck(cudaMemsetAsync(Lv.kflag.p, 0, (size_t)Lv.nnodes * Lv.NP, h->stream), "kflag");
        Lv.klist.reserve((size_t)Lv.nnodes * Lv.NP);
        Lv.kcnt.reserve(Lv.nnodes);
        Lv.dec.reserve(Lv.nnodes);
        // decrease flags are zero outside an opening call (each level's flags
        // are cleared by the level above once it has read them)
        ck(cudaMemsetAsync(Lv.dec.p, 0, Lv.nnodes, h->stream), "dec");
        std::vector<uint8_t> isext(Lv.NP, 0);
        for (int e = 0; e < Lv.nExt; ++e) isext[Lv.ext[e]] = 1;
        Lv.d_isext.reserve(Lv.NP);
        ck(cudaMemcpyAsync(Lv.d_isext.p, isext.data(), Lv.NP, cudaMemcpyHostToDevice, h->stream), "isext");
        Lv.dstamp.reserve(Lv.nnodes);
        Lv.mstamp.reserve(Lv.nnodes);
        ck(cudaMemsetAsync(Lv.dstamp.p, 0, Lv.nnodes * sizeof(uint32_t), h->stream), "dstamp");
        ck(cudaMemsetAsync(Lv.mstamp.p, 0, Lv.nnodes * sizeof(uint32_t), h->stream), "mstamp");
    }
    h->stamp_epoch++;
}

// Descriptor of matrix m of level Lv (an index's own level arrays).
hb::Slot level_slot(Level& Lv, Level* child, int m, int task, int root) {
    hb::Slot sl{};
    sl.mat = Lv.mat.p + (size_t)m * Lv.NP * Lv.NP;
    sl.kflag = Lv.kflag.p + (size_t)m * Lv.NP;
    sl.klist = Lv.klist.p + (size_t)m * Lv.NP;
    sl.kcnt = Lv.kcnt.p + m;
    sl.dec = Lv.dec.p + m;
    sl.child_mat = child ? child->mat.p : nullptr;
    sl.child_dec = child ? child->dec.p : nullptr;
    sl.node = m;
    sl.nodes_x = Lv.nodes_x;
    sl.child_nodes_x = child ? child->nodes_x : 0;
    sl.task = task;
    sl.root = root;
    return sl;
}

// Closure rounds of `n` slots (already uploaded at d_slots, pivots already
// compacted, counts cnt[] on the host) of order NP, in chunks that bound the
// panel scratch.  Issued on `st`, not waited for.
// Slots per closure launch: the panel scratch of a launch stays under 128 MB.
size_t closure_chunk(int NP) {
    const size_t per = (size_t)hb::kPivotChunk * NP;
    return std::max<size_t>(1, (size_t)(128u << 20) / (per * sizeof(uint16_t)));
}

// Closure of n slots over their pivot lists, rounds from r0 on: up to the
// largest count of a chunk (cnt, host copy of the slots' counts), or, with
// cnt null, round r0 alone for every chunk (the kernels return at once for
// a slot whose pivots end before the round).
void close_slots(UpdateArena& A, const hb::Slot* d_slots, const int* cnt, int n, int NP, cudaStream_t st,
                 int r0 = 0) {
    const size_t cap = closure_chunk(NP);
    for (size_t c0 = 0; c0 < (size_t)n; c0 += cap) {
        const int nc = (int)std::min(cap, (size_t)n - c0);
        int rounds = r0 + 1;
        if (cnt) {
            int maxk = 0;
            for (int i = 0; i < nc; ++i) maxk = std::max(maxk, cnt[c0 + i]);
            rounds = (maxk + hb::kPivotChunk - 1) / hb::kPivotChunk;
        }
        if (rounds <= r0) continue;
        A.panel.reserve(hb::closure_scratch_elems(NP, nc), st);
        A.pflags.reserve((size_t)nc * (NP / hb::kFlagTile), st);
        for (int r = r0; r < rounds; ++r) {
            hb::launch_closure_round(d_slots + c0, nc, NP, r, A.panel.p, A.pflags.p, st);
            ck(cudaGetLastError(), "closure round");
        }
    }
}

// Closure of the listed matrices of level `Lv` over their pivot flags
// (build and root growth).
void close_matrices(htrip_index* h, Level& Lv, const std::vector<int>& act) {
    if (act.empty()) return;
    cudaStream_t st = h->stream;
    UpdateArena& A = h->u;
    const int n = (int)act.size();
    const size_t slots_b = align256(n * sizeof(hb::Slot));
    A.stage.reserve(slots_b);
    A.rb.reserve(n * sizeof(int));
    A.dev.reserve(slots_b + n * sizeof(int), st);
    auto* hs = reinterpret_cast<hb::Slot*>(A.stage.p);
    for (int i = 0; i < n; ++i) hs[i] = level_slot(Lv, nullptr, act[i], 0, 0);
    ck(cudaMemcpyAsync(A.dev.p, A.stage.p, n * sizeof(hb::Slot), cudaMemcpyHostToDevice, st), "slots");
    const auto* ds = reinterpret_cast<const hb::Slot*>(A.dev.p);
    int* dcnt = reinterpret_cast<int*>(A.dev.p + slots_b);
    hb::launch_compact_pivots(ds, n, Lv.NP, dcnt, st);
    ck(cudaGetLastError(), "compact");
    int* cnt = reinterpret_cast<int*>(A.rb.p);
    ck(cudaMemcpyAsync(cnt, dcnt, n * sizeof(int), cudaMemcpyDeviceToHost, st), "counts");
    ck(cudaStreamSynchronize(st), "sync counts");
    close_slots(A, ds, cnt, n, Lv.NP, st);
}

// ---------------------------------------------------------------------------
// Build (reference MinPlusOracle::build, minplus_oracle.cpp:48-137)
// ---------------------------------------------------------------------------
void do_build(htrip_index* h, const uint8_t* observed, int rows, int cols) {
    const int b = h->b, g = h->g;
    int S = b;
    while (S < std::max(rows, cols)) S *= g;
    int H = 0;
    for (int t = S / b; t > 1; t /= g) ++H;
    h->release();
    h->built = false;
    h->offloaded = false;
    h->parked.clear();
    h->S = S;
    h->H = H;
    h->rows = rows;
    h->cols = cols;
    h->leaves_x = S / b;
    make_levels(h);
    h->ref_bytes = reference_bytes(h);
    alloc_levels(h);
    cudaStream_t st = h->stream;
    // Passability mirror, padded to S x S (outside the grid = not passable).
    std::vector<uint8_t> pass((size_t)S * S, 0);
    for (int r = 0; r < rows; ++r)
        for (int c = 0; c < cols; ++c) pass[(size_t)r * S + c] = observed[(size_t)r * cols + c] == 1;
    h->pass.reserve(pass.size());
    ck(cudaMemcpyAsync(h->pass.p, pass.data(), pass.size(), cudaMemcpyHostToDevice, st), "pass");
    upload_weights(h);
    build_leaves(h, nullptr, observed, rows, cols);
    for (int l = 1; l <= H; ++l) {
        Level& Lv = h->L[l];
        Level& Lc = h->L[l - 1];
        hb::launch_node_init(Lv.ms(), Lc.ms(), Lc.d_ext.p, Lv.nP, g, Lv.nodes_x, Lc.nodes_x, Lv.nnodes, st);
        ck(cudaGetLastError(), "node init");
        hb::launch_seams_build(Lv.ms(), Lv.d_seams.p, Lv.nseams, h->pass.p, S, Lv.side, Lv.nodes_x, Lv.nnodes,
                               Lv.kflag.p, st, nullptr, h->wts.p);
        ck(cudaGetLastError(), "seams build");
        std::vector<int> act(Lv.nnodes);
        std::iota(act.begin(), act.end(), 0);
        close_matrices(h, Lv, act);
    }
    ck(cudaStreamSynchronize(st), "build sync");
    h->built = true;
    h->epoch++;
}

// ---------------------------------------------------------------------------
// Root growth (reference MinPlusOracle::liftRoot, minplus_oracle.cpp:2008-2114):
// S -> S*g, H -> H+1.  Every existing leaf and node keeps its matrix (moved to
// its index in the wider level); leaves and nodes of the new area are built
// from `observed` (leaf BFS, child summaries + seams, closure), and a new
// root closes the old root and its new siblings over their seams.
// ---------------------------------------------------------------------------
void do_lift_root(htrip_index* h, const uint8_t* observed, int rows, int cols) {
    const int g = h->g, b = h->b;
    const int old_S = h->S, old_H = h->H;
    cudaStream_t st = h->stream;
    ck(cudaStreamSynchronize(st), "sync");
    std::vector<Level> old = std::move(h->L);
    h->L.clear();
    const int old_rows = h->rows, old_cols = h->cols;
    const uint64_t old_ref = h->ref_bytes;
    h->S = old_S * g;
    h->H = old_H + 1;
    h->leaves_x = h->S / b;
    h->rows = rows;
    h->cols = cols;
    try {
        make_levels(h);
        h->ref_bytes = reference_bytes(h);
        alloc_levels(h);
        // move the old matrices to their places in the wider levels
        for (int l = 0; l <= old_H; ++l) {
            Level& Ln = h->L[l];
            const Level& Lo = old[l];
            const size_t mat = (size_t)Ln.NP * Ln.NP * sizeof(uint16_t);
            ck(cudaMemcpy2DAsync(Ln.mat.p, Ln.nodes_x * mat, Lo.mat.p, Lo.nodes_x * mat, Lo.nodes_x * mat, Lo.nodes_x,
                                 cudaMemcpyDeviceToDevice, st), "move matrices");
        }
    } catch (...) {
        for (auto& l : h->L) l.release();
        h->L = std::move(old);  // the old matrices are intact
        h->S = old_S;
        h->H = old_H;
        h->leaves_x = old_S / b;
        h->rows = old_rows;
        h->cols = old_cols;
        h->ref_bytes = old_ref;
        throw;
    }
    for (auto& l : old) l.release();
    old.clear();
    const int S = h->S;
    std::vector<uint8_t> pass((size_t)S * S, 0);
    for (int r = 0; r < std::min(rows, S); ++r)
        for (int c = 0; c < std::min(cols, S); ++c) pass[(size_t)r * S + c] = observed[(size_t)r * cols + c] == 1;
    h->pass.reserve(pass.size());
    ck(cudaMemcpyAsync(h->pass.p, pass.data(), pass.size(), cudaMemcpyHostToDevice, st), "pass");
    upload_weights(h);
    // the new area of every level below the new root
    auto fresh = [&](int nodes_x, int old_nodes_x) {
        std::vector<int> v;
        for (int ty = 0; ty < nodes_x; ++ty)
            for (int tx = 0; tx < nodes_x; ++tx)
                if (tx >= old_nodes_x || ty >= old_nodes_x) v.push_back(ty * nodes_x + tx);
        return v;
    };
    DevBuf<int> list;
    {
        const std::vector<int> nl = fresh(h->L[0].nodes_x, old_S / b);
        build_leaves(h, &nl, observed, rows, cols);
    }
    for (int l = 1; l <= h->H; ++l) {
        Level& Lv = h->L[l];
        Level& Lc = h->L[l - 1];
        const std::vector<int> nn = l < h->H ? fresh(Lv.nodes_x, old_S / Lv.side) : std::vector<int>{0};
        list.reserve(nn.size());
        ck(cudaMemcpyAsync(list.p, nn.data(), nn.size() * sizeof(int), cudaMemcpyHostToDevice, st), "list");
        hb::launch_node_init(Lv.ms(), Lc.ms(), Lc.d_ext.p, Lv.nP, g, Lv.nodes_x, Lc.nodes_x, (int)nn.size(), st,
                             list.p);
        ck(cudaGetLastError(), "node init");
        hb::launch_seams_build(Lv.ms(), Lv.d_seams.p, Lv.nseams, h->pass.p, S, Lv.side, Lv.nodes_x, (int)nn.size(),
                               Lv.kflag.p, st, list.p, h->wts.p);
        ck(cudaGetLastError(), "seams build");
        close_matrices(h, Lv, nn);
        ck(cudaStreamSynchronize(st), "sync");
    }
    list.release();
    h->epoch++;
}

// ---------------------------------------------------------------------------
// Non-monotone updates (reference onCellBlocked, minplus_oracle.cpp:247-302,
// and onBatchLeavesChanged, :507-527 with propagateBatchUpward, :427-505):
// the listed leaves are rebuilt from the grid (leaf BFS) and every ancestor of
// a rebuilt tile is rebuilt from its children's summaries and its seams
// (node init + seams + closure), level by level up to the root.  Each rebuilt
// matrix is the unique closure of its region, so the index equals the one a
// full build of the same grid gives on those tiles.
// ---------------------------------------------------------------------------
// propagate_all: every ancestor of a rebuilt tile is rebuilt (onCellBlocked);
// otherwise a rebuilt node's parent is rebuilt only if the node's exterior
// summary S_U changed (propagateBatchUpward, minplus_oracle.cpp:479-498);
// the listed leaves' parents are always rebuilt.
void do_rebuild_leaves(htrip_index* h, const std::vector<int>& leaves_in, const uint8_t* observed, int rows,
                       int cols, bool propagate_all) {
    cudaStream_t st = h->stream;
    const int S = h->S, g = h->g;
    std::vector<int> cur;
    {
        std::vector<uint8_t> seen(h->L[0].nnodes, 0);
        for (int l : leaves_in)
            if (l >= 0 && l < h->L[0].nnodes && !seen[l]) { seen[l] = 1; cur.push_back(l); }
    }
    if (cur.empty()) return;
    h->update_counter++;
    // the passability mirror follows the caller's grid (leaf BFS and seams read it)
    std::vector<uint8_t> pass((size_t)S * S, 0);
    for (int r = 0; r < std::min(rows, S); ++r)
        for (int c = 0; c < std::min(cols, S); ++c) pass[(size_t)r * S + c] = observed[(size_t)r * cols + c] == 1;
    ck(cudaMemcpyAsync(h->pass.p, pass.data(), pass.size(), cudaMemcpyHostToDevice, st), "pass");
    DevBuf<int> list;
    DevBuf<hb::Slot> slots;
    DevBuf<uint8_t> changed;
    build_leaves(h, &cur, observed, rows, cols);
    for (int l = 1; l <= h->H && !cur.empty(); ++l) {
        Level& Lv = h->L[l];
        Level& Lc = h->L[l - 1];
        std::vector<int> parents;
        std::vector<uint8_t> seen(Lv.nnodes, 0);
        for (int c : cur) {
            const int p = (c / Lc.nodes_x / g) * Lv.nodes_x + (c % Lc.nodes_x) / g;
            if (!seen[p]) { seen[p] = 1; parents.push_back(p); }
        }
        const int n = (int)parents.size();
        const bool track = !propagate_all && l < h->H;  // does the next level depend on S_U changes?
        std::vector<hb::Slot> hs;
        if (track) {
            hs.resize(n);
            for (int i = 0; i < n; ++i) hs[i] = level_slot(Lv, nullptr, parents[i], 0, 0);
            slots.reserve(n);
            ck(cudaMemcpyAsync(slots.p, hs.data(), n * sizeof(hb::Slot), cudaMemcpyHostToDevice, st), "slots");
            h->u.snap.reserve((size_t)n * Lv.nExt * Lv.nExt);
            hb::launch_ext_snapshot(slots.p, n, Lv.d_ext.p, Lv.nExt, Lv.NP, h->u.snap.p, st);
            ck(cudaGetLastError(), "snapshot");
        }
        list.reserve(n);
        ck(cudaMemcpyAsync(list.p, parents.data(), n * sizeof(int), cudaMemcpyHostToDevice, st), "list");
        hb::launch_node_init(Lv.ms(), Lc.ms(), Lc.d_ext.p, Lv.nP, g, Lv.nodes_x, Lc.nodes_x, n, st, list.p);
        ck(cudaGetLastError(), "node init");
        hb::launch_seams_build(Lv.ms(), Lv.d_seams.p, Lv.nseams, h->pass.p, S, Lv.side, Lv.nodes_x, n, Lv.kflag.p,
                               st, list.p, h->wts.p);
        ck(cudaGetLastError(), "seams build");
        close_matrices(h, Lv, parents);
        if (track) {
            changed.reserve(n);
            ck(cudaMemsetAsync(changed.p, 0, n, st), "changed");
            hb::launch_ext_compare(slots.p, n, Lv.d_ext.p, Lv.nExt, Lv.NP, h->u.snap.p, changed.p, g, st, 1);
            ck(cudaGetLastError(), "compare");
            std::vector<uint8_t> ch(n);
            ck(cudaMemcpyAsync(ch.data(), changed.p, n, cudaMemcpyDeviceToHost, st), "changed d2h");
            ck(cudaStreamSynchronize(st), "sync");
            std::vector<int> next;
            for (int i = 0; i < n; ++i)
                if (ch[i]) next.push_back(parents[i]);
            cur = std::move(next);
        } else {
            ck(cudaStreamSynchronize(st), "sync");
            cur = std::move(parents);
        }
    }
    list.release();
    slots.release();
    changed.release();
}

// ---------------------------------------------------------------------------
// Batched opening (reference onBatchCellsOpened, minplus_oracle.cpp:530-729)
// ---------------------------------------------------------------------------
int find_lca_level(const htrip_index* h, int r1, int c1, int r2, int c2) {
    int t1x = c1 / h->b, t1y = r1 / h->b, t2x = c2 / h->b, t2y = r2 / h->b;
    if (t1x == t2x && t1y == t2y) return 0;
    for (int l = 1; l <= h->H; ++l) {
        t1x /= h->g; t1y /= h->g; t2x /= h->g; t2y /= h->g;
        if (t1x == t2x && t1y == t2y) return l;
    }
    return h->H + 1;
}

// V_U index of global cell (r, c) in its level-l node (findVertexIndex,
// internal_node.cpp:306-319).
int vertex_index(const Level& Lv, int g, int r, int c) {
    const int lr = r % Lv.side, lc = c % Lv.side;
    const int q = (lr / Lv.cs) * g + (lc / Lv.cs);
    const int p = port_index(lr % Lv.cs, lc % Lv.cs, Lv.cs);
    return p < 0 ? -1 : q * Lv.nP + p;
}

// One onBatchCellsOpened call of one index.  Host bucketing first
// (minplus_oracle.cpp:539-598), then the levels l = 0..H in order, each in
// two stages:
//   insert(l): leaves: the opened in-leaf edges (pivots marked); nodes: the
//              parents of children whose summary decreased plus the nodes
//              holding new seams get the decreased child entries and the seams
//              inserted; the exterior blocks are snapshotted first; the pivot
//              flags are compacted                 -> pivot counts to host
//   close(l):  blocked closure over the pivots, then the exterior blocks are
//              compared with their snapshots       -> decrease flags to host
// run_open_tasks runs any number of tasks (distinct indexes of one device)
// together: at each stage the matrices of all tasks with the same leaf side
// b (hence the same order, padding and port tables at this level) form ONE
// launch of each kernel, over a device array of matrix descriptors.
struct OpenTask {
    htrip_index* h = nullptr;
    bool record_stats = true;
    std::vector<int> leaves;                             // touched leaves, first-touch order
    std::vector<std::vector<int>> edges;                 // per touched leaf: (u, v, w) triples
    std::vector<std::vector<std::vector<int>>> seams;    // [lvl][slot]: (u, v, w) V_U triples
    std::vector<std::vector<int>> seam_nodes;
    std::vector<std::vector<int>> seam_slot;  // host path: [lvl][node] -> slot of seam_nodes, or -1
    // progress
    std::vector<int> act, cand;    // active matrices of this level / of the level below
    std::vector<uint8_t> cand_dec; // decrease flags of `cand` (read back after its close)
    int n_dirty = 0;
    int slot0 = 0;                 // the task's first slot in this stage's launch
    int task = 0;                  // the task's index in the launch
};

void open_prepare(OpenTask& T, htrip_index* h, const int32_t* rc, int n, const uint8_t* obs, int rows, int cols,
                  bool record_stats) {
    T = OpenTask();
    T.h = h;
    T.record_stats = record_stats;
    const int b = h->b, g = h->g, H = h->H, S = h->S;
    auto passable = [&](int r, int c) { return r >= 0 && c >= 0 && r < rows && c < cols && obs[(size_t)r * cols + c] == 1; };
    auto weight_ok = [&](int r, int c) {  // GridMap::getCellWeight(p) < INF (grid_map.hpp:273-278)
        return r >= 0 && c >= 0 && r < rows && c < cols && obs[(size_t)r * cols + c] != 2;
    };
    static const int dr[4] = {-1, 1, 0, 0};
    static const int dc[4] = {0, 0, -1, 1};
    Level& L0 = h->L[0];
    // node -> slot tables kept by the index (no per-call allocation of
    // level-sized tables; the entries set here are reset at the end)
    std::vector<int>& leaf_slot = h->open_leaf_slot;
    if (leaf_slot.size() != (size_t)L0.nnodes) leaf_slot.assign(L0.nnodes, -1);
    h->open_seam_slot.resize(H + 1);
    for (int l = 1; l <= H; ++l)
        if (h->open_seam_slot[l].size() != (size_t)h->L[l].nnodes) h->open_seam_slot[l].assign(h->L[l].nnodes, -1);
    T.seams.resize(H + 1);
    T.seam_nodes.resize(H + 1);
    for (int i = 0; i < n; ++i) {
        const int r = rc[2 * i], c = rc[2 * i + 1];
        if (r < 0 || c < 0 || r >= S || c >= S) continue;
        const int tx = c / b, ty = r / b, leaf = ty * h->leaves_x + tx;
        if (leaf_slot[leaf] < 0) {
            leaf_slot[leaf] = (int)T.leaves.size();
            T.leaves.push_back(leaf);
            T.edges.emplace_back();
            T.edges.back().reserve(96);  // 8 cells' 4 edges
        }
        if (!weight_ok(r, c)) continue;
        for (int d = 0; d < 4; ++d) {
            const int nr = r + dr[d], nc = c + dc[d];
            if (!passable(nr, nc)) continue;
            // GridMap::edgeWeight (leaf_tile.cpp:318-319, minplus_oracle.cpp:579-580)
            const int w = hb::edge_weight(host_cell_weight(h, r, c, obs, rows, cols),
                                          host_cell_weight(h, nr, nc, obs, rows, cols));
            if (w >= hb::INF) continue;
            if (nc / b == tx && nr / b == ty) {
                auto& e = T.edges[leaf_slot[leaf]];
                e.push_back((r - ty * b) * b + (c - tx * b));
                e.push_back((nr - ty * b) * b + (nc - tx * b));
                e.push_back(w);
            } else {
                const int lca = find_lca_level(h, r, c, nr, nc);
                if (lca < 1 || lca > H) continue;
                const Level& Lv = h->L[lca];
                const int node = (r / Lv.side) * Lv.nodes_x + (c / Lv.side);
                int& slot = h->open_seam_slot[lca][node];
                if (slot < 0) {
                    slot = (int)T.seam_nodes[lca].size();
                    T.seam_nodes[lca].push_back(node);
                    T.seams[lca].emplace_back();
                    T.seams[lca].back().reserve(48);
                }
                const int u = vertex_index(Lv, g, r, c), v = vertex_index(Lv, g, nr, nc);
                if (u >= 0 && v >= 0) {
                    T.seams[lca][slot].push_back(u);
                    T.seams[lca][slot].push_back(v);
                    T.seams[lca][slot].push_back(w);
                }
            }
        }
    }
    for (int leaf : T.leaves) leaf_slot[leaf] = -1;
    for (int l = 1; l <= H; ++l)
        for (int node : T.seam_nodes[l]) h->open_seam_slot[l][node] = -1;
    if (record_stats) h->stats = {0, 0, 0};
    h->open_ops = h->open_bytes = 0;
    h->open_levels.assign(H + 1, {0, 0, 0, 0});
}

bool open_has_work(const OpenTask& T) { return !T.leaves.empty(); }

// Active matrices of level l >= 1: parents of the children whose summary
// decreased (in first-seen order), then the nodes holding new seams.
void open_active(OpenTask& T, int l) {
    htrip_index* h = T.h;
    const int g = h->g;
    Level& Lv = h->L[l];
    Level& Lc = h->L[l - 1];
    std::vector<int> slot_of(Lv.nnodes, -1);
    T.act.clear();
    for (size_t i = 0; i < T.cand.size(); ++i) {
        if (!T.cand_dec[i]) continue;
        const int c = T.cand[i];
        const int cx = c % Lc.nodes_x, cy = c / Lc.nodes_x;
        const int p = (cy / g) * Lv.nodes_x + (cx / g);
        if (slot_of[p] < 0) { slot_of[p] = (int)T.act.size(); T.act.push_back(p); }
    }
    for (int node : T.seam_nodes[l])
        if (slot_of[node] < 0) { slot_of[node] = (int)T.act.size(); T.act.push_back(node); }
    T.n_dirty += (int)T.act.size();
}

// Runs the tasks (distinct indexes of one device, each with work) on stream
// `st` with scratch arena A.
void run_open_tasks(std::vector<OpenTask*>& tasks, UpdateArena& A, cudaStream_t st) {
    int maxH = -1;
    for (size_t t = 0; t < tasks.size(); ++t) {
        tasks[t]->task = (int)t;
        maxH = std::max(maxH, tasks[t]->h->H);
        OpenTask& T = *tasks[t];  // node -> seam slot tables of this path
        T.seam_slot.assign(T.h->H + 1, {});
        for (int l = 1; l <= T.h->H; ++l) {
            T.seam_slot[l].assign(T.h->L[l].nnodes, -1);
            for (size_t i = 0; i < T.seam_nodes[l].size(); ++i) T.seam_slot[l][T.seam_nodes[l][i]] = (int)i;
        }
    }
    const int n_tasks = (int)tasks.size();
    for (int l = 0; l <= maxH; ++l) {
        // ---- active matrices and the groups of this stage (one per leaf side b)
        std::vector<OpenTask*> live;
        for (OpenTask* T : tasks) {
            if (T->h->H < l) continue;
            if (l == 0) T->act = T->leaves;
            else open_active(*T, l);
            if (!T->act.empty()) live.push_back(T);
            else {  // nothing changes at this level; higher levels only see seams
                T->cand.clear();
                T->cand_dec.clear();
            }
        }
        if (live.empty()) continue;
        // tasks of equal (b, g) share this level's geometry: one launch per group
        auto key = [](const OpenTask* t) { return t->h->b * 1024 + t->h->g; };
        std::stable_sort(live.begin(), live.end(), [&](const OpenTask* a, const OpenTask* c) { return key(a) < key(c); });
        struct Group { int t0, t1, s0, s1; size_t snap_off; };
        std::vector<Group> groups;
        int n_slots = 0;
        size_t list_ints = 0, snap_elems = 0;
        for (size_t i = 0; i < live.size();) {
            size_t j = i;
            Group G{(int)i, 0, n_slots, 0, snap_elems};
            const Level& Lv0 = live[i]->h->L[l];
            while (j < live.size() && key(live[j]) == key(live[i])) {
                live[j]->slot0 = n_slots;
                n_slots += (int)live[j]->act.size();
                ++j;
            }
            G.t1 = (int)j;
            G.s1 = n_slots;
            snap_elems += (size_t)(G.s1 - G.s0) * Lv0.nExt * Lv0.nExt;
            groups.push_back(G);
            i = j;
        }
        for (OpenTask* T : live) {
            if (l == 0)
                for (auto& e : T->edges) list_ints += e.size();
            else
                for (int m : T->act) {
                    const int sl = T->seam_slot[l][m];
                    if (sl >= 0) list_ints += T->seams[l][sl].size();
                }
        }
        // ---- staged upload: [slots][lists][slot counts][slot dec][task pivots]
        const size_t o_list = align256(n_slots * sizeof(hb::Slot));
        const size_t o_cnt = o_list + align256(std::max<size_t>(1, list_ints) * sizeof(int));
        const size_t o_dec = o_cnt + align256(n_slots * sizeof(int));
        const size_t o_piv = o_dec + align256(n_slots);
        const size_t total = o_piv + align256(n_tasks * sizeof(int));
        A.stage.reserve(total);
        A.dev.reserve(total, st);
        A.rb.reserve(total - o_cnt);
        std::memset(A.stage.p + o_cnt, 0, total - o_cnt);
        auto* hs = reinterpret_cast<hb::Slot*>(A.stage.p);
        int* hl = reinterpret_cast<int*>(A.stage.p + o_list);
        int li = 0;  // in (u, v, w) triples
        for (OpenTask* T : live) {
            Level& Lv = T->h->L[l];
            Level* child = l >= 1 ? &T->h->L[l - 1] : nullptr;
            for (size_t i = 0; i < T->act.size(); ++i) {
                const int m = T->act[i];
                hb::Slot sl = level_slot(Lv, child, m, T->task, l == T->h->H);
                sl.list_begin = li;
                const std::vector<int>* lst = nullptr;
                if (l == 0) lst = &T->edges[i];
                else if (T->seam_slot[l][m] >= 0) lst = &T->seams[l][T->seam_slot[l][m]];
                if (lst) {
                    std::memcpy(hl + 3 * li, lst->data(), lst->size() * sizeof(int));
                    li += (int)lst->size() / 3;
                }
                sl.list_end = li;
                hs[T->slot0 + i] = sl;
            }
        }
        ck(cudaMemcpyAsync(A.dev.p, A.stage.p, total, cudaMemcpyHostToDevice, st), "open stage upload");
        const auto* ds = reinterpret_cast<const hb::Slot*>(A.dev.p);
        const int* dl = reinterpret_cast<const int*>(A.dev.p + o_list);
        int* dcnt = reinterpret_cast<int*>(A.dev.p + o_cnt);
        uint8_t* ddec = A.dev.p + o_dec;
        int* dpiv = reinterpret_cast<int*>(A.dev.p + o_piv);
        A.snap.reserve(std::max<size_t>(1, snap_elems));
        // ---- insert stage, one launch per kernel and group
        for (const Group& G : groups) {
            const htrip_index* h0 = live[G.t0]->h;
            const Level& Lv = h0->L[l];
            const int n = G.s1 - G.s0;
            hb::launch_ext_snapshot(ds + G.s0, n, Lv.d_ext.p, Lv.nExt, Lv.NP, A.snap.p + G.snap_off, st);
            if (l == 0) {
                hb::launch_leaf_edges(ds + G.s0, n, dl, Lv.NP, dpiv, st);
            } else {
                const Level& Lc = h0->L[l - 1];
                hb::launch_node_child_insert(ds + G.s0, n, Lc.d_ext.p, Lv.nP, h0->g, Lv.NP, Lc.NP, st);
                hb::launch_node_seams(ds + G.s0, n, dl, Lv.NP, st);
            }
            hb::launch_compact_pivots(ds + G.s0, n, Lv.NP, dcnt + G.s0, st);
            ck(cudaGetLastError(), "open insert");
        }
        int* hcnt = reinterpret_cast<int*>(A.rb.p);
        int* hpiv = reinterpret_cast<int*>(A.rb.p + (o_piv - o_cnt));
        uint8_t* hdec = A.rb.p + (o_dec - o_cnt);
        ck(cudaMemcpyAsync(A.rb.p, A.dev.p + o_cnt, o_dec - o_cnt, cudaMemcpyDeviceToHost, st), "counts");
        if (l == 0)
            ck(cudaMemcpyAsync(hpiv, dpiv, n_tasks * sizeof(int), cudaMemcpyDeviceToHost, st), "pivots");
        if (!A.ev_cnt) ck(cudaEventCreateWithFlags(&A.ev_cnt, cudaEventDisableTiming), "event");
        ck(cudaEventRecord(A.ev_cnt, st), "counts event");
        // ---- close stage.  Round 0 of every slot goes out before the counts
        // reach the host (slots without pivots return at once), so the GPU
        // works while the host waits; the scratch of every group is reserved
        // first (a reserve that grows would free a buffer queued kernels use).
        {
            size_t elems = 0, fl = 0;
            for (const Group& G : groups) {
                const int NP = live[G.t0]->h->L[l].NP;
                const size_t nc = std::min(closure_chunk(NP), (size_t)(G.s1 - G.s0));
                elems = std::max(elems, hb::closure_scratch_elems(NP, (int)nc));
                fl = std::max(fl, nc * (NP / hb::kFlagTile));
            }
            A.panel.reserve(elems, st);
            A.pflags.reserve(fl, st);
        }
        for (const Group& G : groups)
            close_slots(A, ds + G.s0, nullptr, G.s1 - G.s0, live[G.t0]->h->L[l].NP, st, 0);
        ck(cudaEventSynchronize(A.ev_cnt), "open insert stage");
        for (const Group& G : groups) {
            const htrip_index* h0 = live[G.t0]->h;
            const Level& Lv = h0->L[l];
            const int n = G.s1 - G.s0;
            close_slots(A, ds + G.s0, hcnt + G.s0, n, Lv.NP, st, 1);
            hb::launch_ext_compare(ds + G.s0, n, Lv.d_ext.p, Lv.nExt, Lv.NP, A.snap.p + G.snap_off, ddec + G.s0,
                                   h0->g, st);
            ck(cudaGetLastError(), "open close");
        }
        ck(cudaMemcpyAsync(hdec, ddec, n_slots, cudaMemcpyDeviceToHost, st), "decreases");
        ck(cudaStreamSynchronize(st), "open close stage");
        // ---- per task: work accounting, stats, the next level's candidates
        for (OpenTask* T : live) {
            htrip_index* h = T->h;
            const uint64_t n = (uint64_t)h->L[l].n;
            auto& lv = h->open_levels[l];
            lv[0] = (int64_t)T->act.size();
            for (size_t i = 0; i < T->act.size(); ++i) {
                const uint64_t k = (uint64_t)hcnt[T->slot0 + i];
                lv[1] += (int64_t)k;
                lv[2] = std::max<int64_t>(lv[2], (int64_t)k);
                if (!k) continue;
                h->open_ops += n * n * k;
                h->open_bytes += 4 * n * n + 4 * k * n;
            }
            lv[3] = (lv[2] + hb::kPivotChunk - 1) / hb::kPivotChunk;
            if (l == 0 && T->record_stats) {
                h->stats.n_touched_leaves = (int)T->act.size();
                h->stats.n_pivots = hpiv[T->task];
            }
            T->cand = T->act;
            T->cand_dec.assign(hdec + T->slot0, hdec + T->slot0 + T->act.size());
        }
    }
    for (OpenTask* T : tasks)
        if (T->record_stats) T->h->stats.n_dirty_ancestors = T->n_dirty;
}

// Which opening path runs: the device-driven one (default: one persistent
// launch per call, the level loop and the closure rounds on the device) or
// the host-driven one (HTRIP_OPEN_PATH=host: per level an insert and a close
// stage, with the pivot counts and the decrease flags read back to the host).
bool open_on_device() {
    static const bool dev = [] {
        const char* e = std::getenv("HTRIP_OPEN_PATH");
        return !(e && std::strcmp(e, "host") == 0);
    }();
    return dev;
}

// Device-driven openings of any number of tasks (distinct indexes of one
// device): tasks of equal (b, g) share one launch of the persistent opening
// kernel (open.cu).  Per launch the host uploads, in one copy, the task
// descriptors, every level's work list (level 0: the touched leaves with
// their opened edges; levels >= 1: the nodes with new seams, with room for
// the parents the device appends) and the edge / seam triples; the kernel
// writes each task's statistics, which come back in one copy.  One host wait
// for the whole call.
void run_open_device(std::vector<OpenTask*>& tasks, UpdateArena& A, cudaStream_t st, int device) {
    std::map<int, std::vector<OpenTask*>> groups;
    for (OpenTask* T : tasks) groups[T->h->b * 1024 + T->h->g].push_back(T);
    struct GL {
        std::vector<OpenTask*> ts;
        int maxH = 0;
        int cap[hb::kOpenMaxLevels] = {}, n_seam[hb::kOpenMaxLevels] = {};
        size_t o_tasks = 0, o_out = 0, o_words = 0, o_trace = 0, o_slots[hb::kOpenMaxLevels] = {}, o_trip = 0;
        size_t o_dchild[hb::kOpenMaxLevels] = {}, o_rec[hb::kOpenMaxLevels] = {}, o_sm = 0;
        size_t begin = 0, end = 0;
        int n_trip = 0;
    };
    std::vector<GL> gl;
    size_t off = 0, panel_elems = 1, pflag_bytes = 1;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += align256(std::max<size_t>(bytes, 1));
        return o;
    };
    for (auto& kv : groups) {
        GL g;
        g.ts = kv.second;
        for (OpenTask* T : g.ts) {
            if (T->h->H + 1 > hb::kOpenMaxLevels) throw CudaError{cudaErrorInvalidValue, "hierarchy too deep"};
            g.maxH = std::max(g.maxH, T->h->H);
        }
        // capacity of every level's list: the touched leaves, then per level
        // the seam nodes and every parent of the level below's capacity set
        for (OpenTask* T : g.ts) {
            htrip_index* h = T->h;
            std::vector<int> cur = T->leaves;
            g.cap[0] += (int)cur.size();
            for (const auto& e : T->edges) g.n_trip += (int)e.size() / 3;
            for (int l = 1; l <= h->H; ++l) {
                const Level& Lv = h->L[l];
                const Level& Lc = h->L[l - 1];
                std::vector<char> seen(Lv.nnodes, 0);
                std::vector<int> next;
                for (int node : T->seam_nodes[l]) {
                    seen[node] = 1;
                    next.push_back(node);
                }
                g.n_seam[l] += (int)T->seam_nodes[l].size();
                for (const auto& sv : T->seams[l]) g.n_trip += (int)sv.size() / 3;
                for (int c : cur) {
                    const int p = ((c / Lc.nodes_x) / h->g) * Lv.nodes_x + (c % Lc.nodes_x) / h->g;
                    if (!seen[p]) { seen[p] = 1; next.push_back(p); }
                }
                g.cap[l] += (int)next.size();
                cur = std::move(next);
            }
        }
        for (int l = 0; l <= g.maxH; ++l) {
            // every task of the group that reaches level l has the same (b, g)
            // geometry there: take it from any of them
            int np = 64;
            for (OpenTask* T : g.ts)
                if (T->h->H >= l) np = T->h->L[l].NP;
            panel_elems = std::max(panel_elems, (size_t)g.cap[l] * hb::kOpenB * np);
            pflag_bytes = std::max(pflag_bytes, (size_t)g.cap[l] * (np / 64));
        }
        g.begin = off;
        g.o_tasks = take(g.ts.size() * sizeof(hb::OpenTask));
        g.o_out = take(g.ts.size() * sizeof(hb::OpenTaskOut));
        g.o_words = take((3 * hb::kOpenMaxLevels + 4) * sizeof(int));
        g.o_trace = take(hb::kOpenTrace * sizeof(unsigned long long));
        g.o_sm = take((3 + hb::kOpenSmSlots) * sizeof(unsigned));  // zero at launch (the staging is cleared)
        for (int l = 0; l <= g.maxH; ++l) g.o_slots[l] = take((size_t)std::max(1, g.cap[l]) * sizeof(int4));
        for (int l = 1; l <= g.maxH; ++l) g.o_dchild[l] = take((size_t)std::max(1, g.cap[l - 1]) * sizeof(int4));
        for (int l = 0; l <= g.maxH; ++l) g.o_rec[l] = take((size_t)std::max(1, g.cap[l]) * sizeof(hb::OpenSlotRec));
        g.o_trip = take((size_t)g.n_trip * 3 * sizeof(int));
        g.end = off;
        gl.push_back(std::move(g));
    }
    A.dev.reserve(off, st);
    A.stage.reserve(off);
    A.rb.reserve(off);
    // two panel and flag buffers: a round's panel is made while the update
    // of the round before reads the other one
    panel_elems = (panel_elems + 127) / 128 * 128;
    pflag_bytes = (pflag_bytes + 255) / 256 * 256;
    A.panel.reserve(2 * panel_elems, st);
    A.pflags.reserve(2 * pflag_bytes, st);
    if (!A.open_grid) A.open_grid = hb::open_grid_blocks(device);
    unsigned char* base = A.dev.p;
    for (GL& g : gl) {
        unsigned char* hs = A.stage.p;
        std::memset(hs + g.begin, 0, g.end - g.begin);
        auto* hT = reinterpret_cast<hb::OpenTask*>(hs + g.o_tasks);
        auto* hO = reinterpret_cast<hb::OpenTaskOut*>(hs + g.o_out);
        int* words = reinterpret_cast<int*>(hs + g.o_words);  // count[17] maxk[17] dcount[17] status bar[3]
        int* trip = reinterpret_cast<int*>(hs + g.o_trip);
        int nt = 0;
        for (size_t t = 0; t < g.ts.size(); ++t) {
            OpenTask* T = g.ts[t];
            htrip_index* h = T->h;
            T->task = (int)t;
            if (++h->open_stamp == 0) h->open_stamp = 1;
            hb::OpenTask& d = hT[t];
            d.H = h->H;
            d.g = h->g;
            d.stamp = h->open_stamp;
            d.out = reinterpret_cast<hb::OpenTaskOut*>(base + g.o_out) + t;
            for (int l = 0; l <= h->H; ++l) {
                Level& Lv = h->L[l];
                d.lv[l] = hb::OpenTaskLevel{Lv.mat.p, Lv.kflag.p, Lv.klist.p, Lv.kcnt.p, Lv.dstamp.p, Lv.mstamp.p,
                                            Lv.nodes_x};
            }
            int seam_total = 0;
            for (int l = 1; l <= h->H; ++l) seam_total += (int)T->seam_nodes[l].size();
            hO[t].n_dirty = seam_total;
        }
        // level 0: the touched leaves of every task, each with its edges
        {
            int4* sl = reinterpret_cast<int4*>(hs + g.o_slots[0]);
            int n0 = 0;
            for (size_t t = 0; t < g.ts.size(); ++t) {
                OpenTask* T = g.ts[t];
                for (size_t i = 0; i < T->leaves.size(); ++i) {
                    const auto& e = T->edges[i];
                    std::memcpy(trip + 3 * nt, e.data(), e.size() * sizeof(int));
                    sl[n0++] = make_int4((int)t, T->leaves[i], nt, nt + (int)e.size() / 3);
                    nt += (int)e.size() / 3;
                }
            }
            words[0] = n0;
        }
        // levels >= 1: the seam nodes first, each with its seams
        for (int l = 1; l <= g.maxH; ++l) {
            int4* sl = reinterpret_cast<int4*>(hs + g.o_slots[l]);
            int n = 0;
            for (size_t t = 0; t < g.ts.size(); ++t) {
                OpenTask* T = g.ts[t];
                if (T->h->H < l) continue;
                for (size_t i = 0; i < T->seam_nodes[l].size(); ++i) {
                    const auto& sv = T->seams[l][i];
                    std::memcpy(trip + 3 * nt, sv.data(), sv.size() * sizeof(int));
                    sl[n++] = make_int4((int)t, T->seam_nodes[l][i], nt, nt + (int)sv.size() / 3);
                    nt += (int)sv.size() / 3;
                }
            }
            words[l] = n;
        }
        hb::OpenLaunch OL{};
        OL.n_tasks = (int)g.ts.size();
        OL.maxH = g.maxH;
        OL.g = g.ts[0]->h->g;
        OL.tasks = reinterpret_cast<const hb::OpenTask*>(base + g.o_tasks);
        for (int l = 0; l <= g.maxH; ++l) {
            const htrip_index* hl = nullptr;
            for (OpenTask* T : g.ts)
                if (T->h->H >= l) { hl = T->h; break; }
            const Level& Lv = hl->L[l];
            OL.geo[l].NP = Lv.NP;
            OL.geo[l].n = Lv.n;
            OL.geo[l].nExt = Lv.nExt;
            OL.geo[l].nP = Lv.nP;
            OL.geo[l].isext = Lv.d_isext.p;
            OL.geo[l].child_ext = l >= 1 ? hl->L[l - 1].d_ext.p : nullptr;
            OL.geo[l].childNP = l >= 1 ? hl->L[l - 1].NP : 0;
            OL.slots[l] = reinterpret_cast<int4*>(base + g.o_slots[l]);
            OL.dchild[l] = l >= 1 ? reinterpret_cast<int4*>(base + g.o_dchild[l]) : nullptr;
            OL.rec[l] = reinterpret_cast<hb::OpenSlotRec*>(base + g.o_rec[l]);
            OL.cap[l] = g.cap[l];
            OL.n_seam[l] = l >= 1 ? words[l] : 0;
        }
        OL.count = reinterpret_cast<int*>(base + g.o_words);
        OL.maxk = OL.count + hb::kOpenMaxLevels;
        OL.dcount = OL.count + 2 * hb::kOpenMaxLevels;
        OL.status = OL.count + 3 * hb::kOpenMaxLevels;
        OL.bar = reinterpret_cast<unsigned*>(OL.status + 1);
        OL.sm = reinterpret_cast<unsigned*>(base + g.o_sm);
        OL.triples = reinterpret_cast<const int*>(base + g.o_trip);
        OL.panel = A.panel.p;
        OL.pflags = A.pflags.p;
        OL.trace = reinterpret_cast<unsigned long long*>(base + g.o_trace);
        OL.panel_stride = panel_elems;
        OL.pflag_stride = pflag_bytes;
        ck(cudaMemcpyAsync(base + g.begin, hs + g.begin, g.end - g.begin, cudaMemcpyHostToDevice, st), "open upload");
        coop_launch(device, st, [&] { return hb::launch_open(OL, A.open_grid, st); }, "opening kernel");
        // statistics and the status word back (the trace stays on the device)
        ck(cudaMemcpyAsync(A.rb.p + g.o_out, base + g.o_out, g.o_trace - g.o_out, cudaMemcpyDeviceToHost, st),
           "open results");
        A.trace_off = g.o_trace;
        A.trace_valid = 1;
    }
    ck(cudaStreamSynchronize(st), "opening");
    for (GL& g : gl) {
        const int* words = reinterpret_cast<const int*>(A.rb.p + g.o_words);
        const int status = words[3 * hb::kOpenMaxLevels];
        if (status != 0)
            throw CudaError{cudaErrorLaunchFailure, status == 1 ? "opening kernel: a bounded barrier wait timed out"
                                                                : "opening kernel: a work list overflowed"};
        const auto* out = reinterpret_cast<const hb::OpenTaskOut*>(A.rb.p + g.o_out);
        for (size_t t = 0; t < g.ts.size(); ++t) {
            OpenTask* T = g.ts[t];
            htrip_index* h = T->h;
            const hb::OpenTaskOut& o = out[t];
            for (int l = 0; l <= h->H; ++l) {
                auto& lv = h->open_levels[l];
                lv = {o.level[l][0], o.level[l][1], o.level[l][2],
                      (o.level[l][2] + hb::kOpenB - 1) / hb::kOpenB};
            }
            h->open_ops = o.ops;
            h->open_bytes = o.bytes;
            if (T->record_stats) {
                h->stats.n_touched_leaves = (int)T->leaves.size();
                h->stats.n_pivots = o.new_pivots;
                h->stats.n_dirty_ancestors = o.n_dirty;
            }
        }
    }
}

void run_open(std::vector<OpenTask*>& tasks, UpdateArena& A, cudaStream_t st, int device) {
    if (open_on_device()) {
        run_open_device(tasks, A, st, device);
    } else {
        for (OpenTask* T : tasks) T->h->host_opens++;
        run_open_tasks(tasks, A, st);
    }
}

void do_open(htrip_index* h, const int32_t* rc, int n, const uint8_t* obs, int rows, int cols, bool record_stats) {
    h->update_counter++;
    OpenTask T;
    open_prepare(T, h, rc, n, obs, rows, cols, record_stats);
    if (!open_has_work(T)) return;
    std::vector<OpenTask*> tasks{&T};
    run_open(tasks, h->u, h->stream, h->device);
}

// ---------------------------------------------------------------------------
// Query (reference queryAllPairs, minplus_oracle.cpp:934-1419)
// ---------------------------------------------------------------------------
struct QueryPlan {
    std::vector<int> buf;
    int n_sorted = 0, k = 0;
    int ldv = 8;   // slot stride of X / Yt
    int ldm = 8;   // stride of the sorted-order M
    int cfg = 0;
    int o_vp0 = 0, o_inv = 0, o_l0 = 0, n_l0 = 0;
    struct Lvl {
        int o_groups = 0, n_groups = 0, max_group = 0, slots = 0;
        int o_items = 0, n_items = 0, split = 1;
        int o_meet = 0, n_meet = 0;
        int o_s2v = 0, o_lift = 0;
        size_t flags_off = 0;
    };
    std::vector<Lvl> lv;
    size_t flags_total = 0;
};

// Tile configuration of a query (hb::query_config_tile); the autotuner may
// override the default choice per (index shape, viewpoint count) bucket.
int choose_query_cfg(const htrip_index* h, int ns, int root_group);

// Parts per project item of level l (QueryLevel::split).  Root items are the
// longest (the root's child port list: ~1000 ports for a 256-cell child,
// against a few dozen at level 1).  Cutting one costs a unit's fixed
// overhead (a few microseconds) per extra part, which pays only while the
// root has no more items than the grid has CTAs.  On a 512 x 512 maze
// (root child ports 1020) the query kernel measured, for 1 / 2 / 4 parts:
// k = 16: 89 / 81 / 75 us, k = 64 (86 root items): 93 / 87 / 99 us,
// k = 128 (172 items): 134 / 122 / 134 us, k = 256 (344 items): 136 / 143
// / 164 us.  So: 2 parts for long root port lists (>= 256) when the items
// fit the grid.  HTRIP_QUERY_ROOT_SPLIT=n (1..8) imposes n parts on every
// root level regardless of size.
int query_split_forced() {
    static const int forced = [] {
        const char* e = std::getenv("HTRIP_QUERY_ROOT_SPLIT");
        return e ? std::clamp(std::atoi(e), 1, 8) : 0;
    }();
    return forced;
}

// The split a level may use (1: never) ...
int query_item_split(const htrip_index* h, int l) {
    if (l < 1 || l != h->H) return 1;
    if (query_split_forced()) return query_split_forced();
    return h->L[l].nP >= 256 ? 2 : 1;
}

// ... and the number of items up to which it does (the query grid's CTAs).
int query_split_items(const htrip_index* h) {
    if (query_split_forced()) return INT32_MAX;
    static std::mutex mu;
    static std::map<int, int> grid;
    std::lock_guard<std::mutex> lock(mu);
    auto it = grid.find(h->device);
    if (it == grid.end()) it = grid.emplace(h->device, hb::query_grid_blocks(h->device)).first;
    return it->second;
}

// Plans a query; force_cfg >= 0 imposes the tile configuration (requests
// that share a launch share one).
void make_plan(const htrip_index* h, const int32_t* vps, const uint8_t* pass_flags, int k, QueryPlan& P,
               int force_cfg = -1) {
    const int b = h->b, g = h->g, H = h->H;
    struct V { uint64_t key; int orig; int tx, ty; };
    std::vector<V> v;
    v.reserve(k);
    for (int i = 0; i < k; ++i) {
        if (!pass_flags[i]) continue;
        const int r = vps[2 * i], c = vps[2 * i + 1];
        const int tx = c / b, ty = r / b;
        uint64_t key = 0, mul = 1;
        int x = tx, y = ty;
        for (int l = 0; l < std::max(H, 1); ++l) {
            key += (uint64_t)((y % g) * g + (x % g)) * mul;
            mul *= (uint64_t)(g * g);
            x /= g;
            y /= g;
        }
        v.push_back({key, i, tx, ty});
    }
    std::stable_sort(v.begin(), v.end(), [](const V& a, const V& c) { return a.key < c.key; });
    const int ns = (int)v.size();
    P.n_sorted = ns;
    P.k = k;
    P.flags_total = 0;
    P.ldm = std::max(8, (ns + 7) / 8 * 8);
    P.buf.clear();
    P.o_vp0 = 0;
    P.buf.resize(4 * (size_t)ns + k);
    P.o_inv = 4 * ns;
    for (int i = 0; i < k; ++i) P.buf[P.o_inv + i] = -1;
    for (int i = 0; i < ns; ++i) {
        const int r = vps[2 * v[i].orig], c = vps[2 * v[i].orig + 1];
        P.buf[4 * i] = v[i].ty * h->leaves_x + v[i].tx;
        P.buf[4 * i + 1] = (r % b) * b + (c % b);
        P.buf[P.o_inv + v[i].orig] = i;
    }
    for (int i = 0; i < ns;) {
        int j = i;
        while (j < ns && P.buf[4 * j] == P.buf[4 * i]) ++j;
        for (int t = i; t < j; ++t) { P.buf[4 * t + 2] = i; P.buf[4 * t + 3] = j; }
        i = j;
    }
    // Child groups of every level.
    struct CG { int node, quad, start, cnt, slot0; };
    std::vector<std::vector<CG>> cgs(H + 1);
    P.lv.assign(H + 1, QueryPlan::Lvl());
    for (int l = 1; l <= H; ++l) {
        const Level& Lv = h->L[l];
        const Level& Lc = h->L[l - 1];
        QueryPlan::Lvl& Q = P.lv[l];
        int prev_child = -1;
        for (int i = 0; i < ns; ++i) {
            const int cxp = v[i].tx * b / Lc.side, cyp = v[i].ty * b / Lc.side;
            const int child = cyp * Lc.nodes_x + cxp;
            if (child != prev_child) {
                cgs[l].push_back({(cyp / g) * Lv.nodes_x + (cxp / g), (cyp % g) * g + (cxp % g), i, 0, 0});
                prev_child = child;
            }
            cgs[l].back().cnt++;
        }
        for (const CG& c : cgs[l]) Q.max_group = std::max(Q.max_group, c.cnt);
        Q.n_groups = (int)cgs[l].size();
    }
    P.cfg = force_cfg >= 0 ? force_cfg : choose_query_cfg(h, ns, H >= 1 ? P.lv[H].max_group : ns);
    const hb::QueryTile tile = hb::query_config_tile(P.cfg);
    const int RW = tile.RW, NC = tile.NCOL;
    // Slot layout: every child group's run starts on an RW boundary.
    std::vector<std::vector<int>> slot_of(H + 1);
    int max_slots = ns;
    for (int l = 1; l <= H; ++l) {
        QueryPlan::Lvl& Q = P.lv[l];
        int slot = 0;
        slot_of[l].assign(ns, 0);
        for (CG& c : cgs[l]) {
            c.slot0 = slot;
            for (int t = 0; t < c.cnt; ++t) slot_of[l][c.start + t] = slot + t;
            slot += (c.cnt + RW - 1) / RW * RW;
        }
        Q.slots = slot;
        max_slots = std::max(max_slots, slot);
        Q.flags_off = P.flags_total;
        P.flags_total += (size_t)Q.n_groups * h->L[l].nP;
    }
    P.ldv = (max_slots + 256 + 7) / 8 * 8;
    // Level-0 table: per level-1 slot {sorted index or -1, level-1 group}.
    P.o_l0 = (int)P.buf.size();
    if (H >= 1) {
        P.n_l0 = P.lv[1].slots;
        P.buf.resize(P.buf.size() + 2 * (size_t)P.n_l0, -1);
        for (int gi = 0; gi < (int)cgs[1].size(); ++gi)
            for (int t = 0; t < cgs[1][gi].cnt; ++t) {
                P.buf[P.o_l0 + 2 * (cgs[1][gi].slot0 + t)] = cgs[1][gi].start + t;
                P.buf[P.o_l0 + 2 * (cgs[1][gi].slot0 + t) + 1] = gi;
            }
    } else {
        P.n_l0 = 0;
    }
    const int target_items = 296;
    for (int l = 1; l <= H; ++l) {
        const Level& Lv = h->L[l];
        QueryPlan::Lvl& Q = P.lv[l];
        const auto& G = cgs[l];
        Q.o_groups = (int)P.buf.size();
        for (const CG& c : G) P.buf.insert(P.buf.end(), {c.node, c.quad, c.slot0, c.cnt, c.start});
        // project items; at the root a viewpoint of child q meets only
        // viewpoints of children >= q (i < j), so earlier blocks are skipped.
        Q.o_items = (int)P.buf.size();
        for (int gi = 0; gi < (int)G.size(); ++gi) {
            const int n_begin = (l == H) ? (G[gi].quad * Lv.nP) / NC * NC : 0;
            for (int m0 = 0; m0 < G[gi].cnt; m0 += RW)
                for (int n0 = n_begin; n0 < Lv.NP; n0 += NC) P.buf.insert(P.buf.end(), {gi, m0, n0});
        }
        Q.n_items = ((int)P.buf.size() - Q.o_items) / 3;
        Q.split = Q.n_items <= query_split_items(h) ? query_item_split(h, l) : 1;
        Q.o_s2v = (int)P.buf.size();
        P.buf.resize(P.buf.size() + Q.slots + NC, -1);
        for (const CG& c : G)
            for (int t = 0; t < c.cnt; ++t) P.buf[Q.o_s2v + c.slot0 + t] = c.start + t;
        // meet items: rows = RW viewpoints j of child group c2, lanes = NC
        // viewpoint slots i of the node before or in c2.
        std::vector<int> base;
        for (int gi = 0; gi < (int)G.size();) {
            int ge = gi;
            while (ge < (int)G.size() && G[ge].node == G[gi].node) ++ge;
            const int sW = G[gi].slot0;
            for (int c2 = gi; c2 < ge; ++c2) {
                const int s2 = G[c2].slot0, e2 = s2 + G[c2].cnt;
                for (int i0 = sW; i0 < e2 - 1; i0 += NC)
                    for (int jb = 0; jb < G[c2].cnt; jb += RW) {
                        const int j0 = s2 + jb, nj = std::min(RW, G[c2].cnt - jb);
                        if (i0 >= j0 + nj - 1) continue;
                        base.insert(base.end(), {i0, j0, nj, c2, G[c2].quad * Lv.nP});
                    }
            }
            gi = ge;
        }
        const int nbase = (int)base.size() / 5;
        int ks = nbase ? (target_items + nbase - 1) / nbase : 1;
        ks = std::max(1, std::min(ks, (Lv.nP + 63) / 64));
        const int kstep = ((Lv.nP + ks - 1) / ks + 31) / 32 * 32;
        Q.o_meet = (int)P.buf.size();
        for (int t = 0; t < nbase; ++t)
            for (int kb = 0; kb < Lv.nP; kb += kstep)
                P.buf.insert(P.buf.end(), {base[5 * t], base[5 * t + 1], base[5 * t + 2], base[5 * t + 3],
                                           base[5 * t + 4], kb, std::min(Lv.nP, kb + kstep)});
        Q.n_meet = ((int)P.buf.size() - Q.o_meet) / 7;
        // lift table: level-l slot -> {level-(l+1) slot, level-(l+1) group}
        if (l < H) {
            Q.o_lift = (int)P.buf.size();
            P.buf.resize(P.buf.size() + 2 * (size_t)Q.slots, 0);
            const auto& Gn = cgs[l + 1];
            for (int gn = 0; gn < (int)Gn.size(); ++gn)
                for (int t = 0; t < Gn[gn].cnt; ++t) {
                    const int i = Gn[gn].start + t;
                    P.buf[Q.o_lift + 2 * slot_of[l][i]] = Gn[gn].slot0 + t;
                    P.buf[Q.o_lift + 2 * slot_of[l][i] + 1] = gn;
                }
        }
    }
}

// ---------------------------------------------------------------------------
// Query launches.  One cooperative launch of the persistent kernel serves
// any number of planned requests of one device (indexes of any shape, any
// k).  Device scratch of a launch, every piece 256-byte aligned:
//   [QueryParams x n][unit prefix, n_phases x (n+1) ints][4 words][plans]
//       <- one host->device copy of the staged head (words start at zero)
//   [M of every request]      <- one memset to 0xFF (no pair found yet)
//   [flags + completion counters of every request]  <- one memset to 0
//   [X_0..X_{H-1} Y_1..Y_H of every request][results k*k u16 of every request]
// ---------------------------------------------------------------------------

struct QueryReq {
    const htrip_index* h;
    const QueryPlan* P;
    uint16_t* out_dev;  // result on the device; nullptr = in the arena
};

// Launch words: {status, barrier count, barrier generation, pad}, the
// executed-work counters (QueryParams::work, 3 x u64) at byte kWorkOffset,
// then the phase time stamps at byte kTraceOffset.
constexpr size_t kWorkOffset = 16;
constexpr size_t kTraceOffset = 64;
constexpr size_t kWordsBytes = kTraceOffset + (2 * hb::kMaxQueryPhases + 1) * sizeof(unsigned long long);

struct LaunchLayout {
    int n = 0, n_phases = 0;
    size_t o_params = 0, o_pre = 0, o_words = 0, head = 0;
    size_t o_M = 0, M_bytes = 0, o_flags = 0, flags_bytes = 0, o_out = 0, out_bytes = 0, total = 0;
    std::vector<size_t> plan, M, flags, ctr, ticket, part, out;
    std::vector<std::array<size_t, hb::kMaxQueryLevels + 1>> X, Y;
};

// Rows of the per-level buffers of a query on h: X_l (l < H) holds the
// exterior ports of level l, which are the child ports of level l+1; Yt_l
// (l >= 1) the columns of the level-l matrices.
size_t query_x_rows(const htrip_index* h, int l) {
    return (size_t)std::max(h->L[l].nExt, l + 1 <= h->H ? h->L[l + 1].nP : 0);
}
size_t query_y_rows(const htrip_index* h, int l) { return (size_t)std::max(h->L[l].NP, 64); }

// The persistent kernel's schedule: dataflow (default) or grid barriers
// (HTRIP_QUERY_DATAFLOW=0).
int query_dataflow_mode() {
    static const int mode = [] {
        const char* e = std::getenv("HTRIP_QUERY_DATAFLOW");
        return e && std::strcmp(e, "0") == 0 ? 0 : 1;
    }();
    return mode;
}

void check_query_shape(const htrip_index* h) {
    if (h->H > hb::kMaxQueryLevels) throw CudaError{cudaErrorInvalidValue, "hierarchy deeper than the query supports"};
    for (int l = 1; l <= h->H; ++l)
        if (h->L[l].nP > hb::query_max_ports())
            throw CudaError{cudaErrorInvalidValue, "child port count above the query kernel's list capacity"};
}

LaunchLayout layout_launch(const std::vector<QueryReq>& R) {
    LaunchLayout L;
    L.n = (int)R.size();
    for (const auto& r : R) L.n_phases = std::max(L.n_phases, r.h->H + 3);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += align256(std::max<size_t>(bytes, 1));
        return o;
    };
    L.o_params = take(R.size() * sizeof(hb::QueryParams));
    L.o_pre = take((size_t)L.n_phases * (R.size() + 1) * sizeof(int));
    L.o_words = take(kWordsBytes);
    for (const auto& r : R) L.plan.push_back(take(r.P->buf.size() * sizeof(int)));
    L.head = off;
    L.o_M = off;
    for (const auto& r : R) L.M.push_back(take((size_t)r.P->ldm * r.P->ldm * sizeof(uint32_t)));
    L.M_bytes = off - L.o_M;
    L.o_flags = off;
    for (const auto& r : R) {
        L.flags.push_back(take(r.P->flags_total));
        L.ctr.push_back(take(hb::query_counter_words(r.h->H, r.P->k) * sizeof(unsigned)));
        const QueryPlan::Lvl& root = r.P->lv[r.h->H];
        L.ticket.push_back(root.split > 1 ? take((size_t)root.n_items * sizeof(unsigned)) : 0);
    }
    L.flags_bytes = off - L.o_flags;
    for (const auto& r : R) {
        const QueryPlan::Lvl& root = r.P->lv[r.h->H];
        const hb::QueryTile tile = hb::query_config_tile(r.P->cfg);
        L.part.push_back(root.split > 1 ? take((size_t)root.n_items * root.split * tile.RW * tile.NCOL * 2) : 0);
    }
    for (const auto& r : R) {
        std::array<size_t, hb::kMaxQueryLevels + 1> x{}, y{};
        for (int l = 0; l < r.h->H; ++l) x[l] = take(query_x_rows(r.h, l) * r.P->ldv * sizeof(uint16_t));
        for (int l = 1; l <= r.h->H; ++l) y[l] = take(query_y_rows(r.h, l) * r.P->ldv * sizeof(uint16_t));
        L.X.push_back(x);
        L.Y.push_back(y);
    }
    L.o_out = off;
    for (const auto& r : R) L.out.push_back(r.out_dev ? 0 : take((size_t)r.P->k * r.P->k * sizeof(uint16_t)));
    L.out_bytes = off - L.o_out;
    L.total = off;
    return L;
}

// CTA work units of request P in every phase of the launch (the kernel's
// phase numbering, kernels.cuh QueryLaunch).
void query_units(const htrip_index* h, const QueryPlan& P, int n_phases, int* units) {
    const int H = h->H;
    for (int t = 0; t < n_phases; ++t) units[t] = 0;
    const long fill = (long)P.n_l0 * h->L[0].nExt;
    units[0] = (int)((fill + hb::kQueryL0Chunk - 1) / hb::kQueryL0Chunk) +
               (P.n_sorted + hb::kQueryThreads - 1) / hb::kQueryThreads;
    for (int t = 1; t <= H + 1; ++t)
        units[t] = (t <= H ? P.lv[t].n_items * P.lv[t].split : 0) + (t - 1 >= 1 ? P.lv[t - 1].n_meet : 0);
    units[H + 2] = (int)(((long)P.k * P.k + hb::kQueryFinChunk - 1) / hb::kQueryFinChunk);
}

hb::QueryParams make_params(const htrip_index* h, const QueryPlan& P, unsigned char* base, const LaunchLayout& L,
                            int i, uint16_t* out_dev, const uint8_t* dirty = nullptr) {
    const int H = h->H;
    const int* plan = reinterpret_cast<const int*>(base + L.plan[i]);
    uint8_t* flags = base + L.flags[i];
    hb::QueryParams Q{};
    Q.H = H;
    Q.k = P.k;
    Q.ns = P.n_sorted;
    Q.ldv = P.ldv;
    Q.ldm = P.ldm;
    Q.n_l0_slots = P.n_l0;
    Q.nExt0 = h->L[0].nExt;
    Q.cfg = P.cfg;
    Q.vp0 = plan + P.o_vp0;
    Q.inv = plan + P.o_inv;
    Q.l0 = plan + P.o_l0;
    Q.ext0 = h->L[0].d_ext.p;
    Q.leaves = h->L[0].ms();
    for (int l = 0; l < H; ++l) Q.X[l] = reinterpret_cast<uint16_t*>(base + L.X[i][l]);
    for (int l = 1; l <= H; ++l) Q.Y[l] = reinterpret_cast<uint16_t*>(base + L.Y[i][l]);
    Q.M = reinterpret_cast<uint32_t*>(base + L.M[i]);
    Q.ctr = reinterpret_cast<unsigned*>(base + L.ctr[i]);
    Q.out = out_dev;
    // executed-work counters: single-request launches of an index that counts
    Q.work = h->count_work && L.n == 1 ? reinterpret_cast<unsigned long long*>(base + L.o_words + kWorkOffset)
                                        : nullptr;
    Q.dirty = dirty;
    for (int l = 1; l <= H; ++l) {
        const Level& Lv = h->L[l];
        const QueryPlan::Lvl& PL = P.lv[l];
        hb::QueryLevel& q = Q.lv[l];
        q.D = Lv.mat.p;
        q.NP = Lv.NP;
        q.nP = Lv.nP;
        q.ext_inv = Lv.d_ext_inv.p;
        q.groups = plan + PL.o_groups;
        q.flags = flags + PL.flags_off;
        q.items = plan + PL.o_items;
        q.n_items = PL.n_items;
        q.meet = plan + PL.o_meet;
        q.n_meet = PL.n_meet;
        q.s2v = plan + PL.o_s2v;
        q.lift = l < H ? plan + PL.o_lift : nullptr;
        q.store_y = 1;
        q.split = PL.split;
        if (PL.split > 1) {
            q.part = reinterpret_cast<uint32_t*>(base + L.part[i]);
            q.ticket = reinterpret_cast<unsigned*>(base + L.ticket[i]);
        }
    }
    return Q;
}

// Stages the head of the launch into `stage` (>= L.head bytes of host
// memory), then issues on `st`: the head copy, the two presets and the
// kernel, bracketed by ev[0] / ev[1] when given.  Returns the device
// pointers of the results in `outs`.
// With `dirty` (one request; an incremental refresh in an arena that holds
// the previous launch of the same plan) the pair matrix and the finite-port
// flags are kept instead of preset, and only the units of dirty viewpoints
// work.
void issue_query_launch(cudaStream_t st, int device, int& grid, int cfg, const std::vector<QueryReq>& R,
                        const LaunchLayout& L, unsigned char* base, unsigned char* stage, const cudaEvent_t* ev,
                        std::vector<uint16_t*>& outs, const uint8_t* dirty = nullptr) {
    for (const auto& r : R) check_query_shape(r.h);
    std::memset(stage, 0, L.head);
    outs.resize(R.size());
    auto* params = reinterpret_cast<hb::QueryParams*>(stage + L.o_params);
    auto* pre = reinterpret_cast<int*>(stage + L.o_pre);
    std::vector<int> units(L.n_phases);
    for (int t = 0; t < L.n_phases; ++t) pre[(size_t)t * (L.n + 1)] = 0;
    for (int i = 0; i < L.n; ++i) {
        const QueryReq& r = R[i];
        outs[i] = r.out_dev ? r.out_dev : reinterpret_cast<uint16_t*>(base + L.out[i]);
        params[i] = make_params(r.h, *r.P, base, L, i, outs[i], dirty);
        std::memcpy(stage + L.plan[i], r.P->buf.data(), r.P->buf.size() * sizeof(int));
        query_units(r.h, *r.P, L.n_phases, units.data());
        for (int t = 0; t < L.n_phases; ++t)
            pre[(size_t)t * (L.n + 1) + i + 1] = pre[(size_t)t * (L.n + 1) + i] + units[t];
    }
    ck(cudaMemcpyAsync(base, stage, L.head, cudaMemcpyHostToDevice, st), "query launch head");
    if (!dirty) {
        ck(cudaMemsetAsync(base + L.o_M, 0xFF, L.M_bytes, st), "pair matrix preset");
        ck(cudaMemsetAsync(base + L.o_flags, 0, L.flags_bytes, st), "flag preset");
    } else {  // only the completion counters and the split items' tickets start at zero
        for (size_t i = 0; i < R.size(); ++i) {
            ck(cudaMemsetAsync(base + L.ctr[i], 0,
                               hb::query_counter_words(R[i].h->H, R[i].P->k) * sizeof(unsigned), st), "counters");
            const QueryPlan::Lvl& root = R[i].P->lv[R[i].h->H];
            if (root.split > 1) ck(cudaMemsetAsync(base + L.ticket[i], 0, (size_t)root.n_items * sizeof(unsigned), st),
                                   "tickets");
        }
    }
    if (grid == 0) grid = hb::query_grid_blocks(device);
    hb::QueryLaunch QL;
    QL.n_req = L.n;
    QL.n_phases = L.n_phases;
    QL.req = reinterpret_cast<const hb::QueryParams*>(base + L.o_params);
    QL.unit_pre = reinterpret_cast<const int*>(base + L.o_pre);
    QL.status = reinterpret_cast<int*>(base + L.o_words);
    QL.bar = reinterpret_cast<unsigned*>(base + L.o_words) + 1;
    QL.trace = reinterpret_cast<unsigned long long*>(base + L.o_words + kTraceOffset);
    QL.dataflow = query_dataflow_mode();
    // the start event after any wait for another stream's cooperative kernel
    coop_launch(device, st, [&] {
        if (ev) {
            const cudaError_t e = cudaEventRecord(ev[0], st);
            if (e != cudaSuccess) return e;
        }
        return hb::launch_query(QL, cfg, grid, st);
    }, "query kernel");
    if (ev) ck(cudaEventRecord(ev[1], st), "event");
}

// Runs the planned requests through the arena `A` on stream `st`.  Results
// whose out_dev is null are copied into host_out[i] (k*k each).  Returns
// the kernel's status word (0 ok, 1 a bounded wait timed out); synchronous.
int run_queries(QueryArena& A, int device, cudaStream_t st, const std::vector<QueryReq>& R,
                const std::vector<uint16_t*>& host_out, bool sync, const uint8_t* dirty = nullptr) {
    int cfg = 0;
    for (const auto& r : R) cfg = std::max(cfg, r.P->cfg);
    const LaunchLayout L = layout_launch(R);
    // A stream-ordered launch (sync == false) may still be reading the
    // arena or the pinned staging: wait for it before reusing or growing them.
    if (A.ev_valid) ck(cudaEventSynchronize(A.ev[1]), "previous launch");
    A.dev.reserve(L.total, st);
    A.stage.reserve(L.head);
    A.outstage.reserve(L.out_bytes + 256);
    if (!A.ev[0]) {
        ck(cudaEventCreate(&A.ev[0]), "event");
        ck(cudaEventCreate(&A.ev[1]), "event");
    }
    std::vector<uint16_t*> outs;
    issue_query_launch(st, device, A.grid, cfg, R, L, A.dev.p, A.stage.p, A.ev, outs, dirty);
    A.ev_valid = true;
    A.last_words = L.o_words;
    A.last_phases = L.n_phases;
    A.last_h2d = L.head;
    A.last_d2h = 0;
    int* status_host = reinterpret_cast<int*>(A.outstage.p + L.out_bytes);
    bool any_host = false;
    for (size_t i = 0; i < R.size(); ++i) any_host |= !R[i].out_dev && host_out[i];
    if (any_host) {
        ck(cudaMemcpyAsync(A.outstage.p, A.dev.p + L.o_out, L.out_bytes, cudaMemcpyDeviceToHost, st), "results");
        A.last_d2h += L.out_bytes;
    }
    if (!sync) return 0;
    ck(cudaMemcpyAsync(status_host, A.dev.p + L.o_words, sizeof(int), cudaMemcpyDeviceToHost, st), "status");
    A.last_d2h += sizeof(int);
    ck(cudaStreamSynchronize(st), "query sync");
    if (any_host)
        for (size_t i = 0; i < R.size(); ++i)
            if (!R[i].out_dev && host_out[i])
                std::memcpy(host_out[i], A.outstage.p + (L.out[i] - L.o_out),
                            (size_t)R[i].P->k * R[i].P->k * sizeof(uint16_t));
    return *status_host;
}

// Same-cfg planning for a launch: every request of one launch uses the
// largest tile configuration any of them would choose on its own.
void plan_common(std::vector<QueryPlan>& plans, const std::vector<const htrip_index*>& hs,
                 const std::vector<const int32_t*>& vps, const std::vector<std::vector<uint8_t>>& pf) {
    int cfg = 0;
    for (const auto& P : plans) cfg = std::max(cfg, P.cfg);
    for (size_t i = 0; i < plans.size(); ++i)
        if (plans[i].cfg != cfg) make_plan(hs[i], vps[i], pf[i].data(), plans[i].k, plans[i], cfg);
}

// Viewpoint passability as queryAllPairs decides it (minplus_oracle.cpp:961-965,
// :993-997): Free in `observed` and inside the index.
std::vector<uint8_t> viewpoint_flags(const htrip_index* h, const int32_t* vps, int k, const uint8_t* observed,
                                     int rows, int cols) {
    std::vector<uint8_t> pf(k);
    for (int i = 0; i < k; ++i) {
        const int r = vps[2 * i], c = vps[2 * i + 1];
        pf[i] = (r >= 0 && c >= 0 && r < rows && c < cols && observed[(size_t)r * cols + c] == 1 && r < h->S &&
                 c < h->S);
    }
    return pf;
}

// ---------------------------------------------------------------------------
// Query tile autotuner.  A process-wide table maps a request bucket - the
// index's depth H and root matrix order, and the base-2 logarithms of the
// viewpoint count and of the largest root child group - to the tile
// configuration (hb::query_config_tile) measured fastest for a sample of
// that bucket (htrip_autotune_query).  Buckets without an entry use the
// fixed rule.  The table is exported / imported as text lines
// "H NP log2_k log2_group cfg" (htrip_autotune_export / _import).
// ---------------------------------------------------------------------------
struct TuneKey {
    int H, NP, kb, gb;
    bool operator<(const TuneKey& o) const {
        return std::tie(H, NP, kb, gb) < std::tie(o.H, o.NP, o.kb, o.gb);
    }
};
std::mutex g_tune_mu;
std::map<TuneKey, int> g_tune;

int log2_bucket(int x) {
    int b = 0;
    while ((1 << (b + 1)) <= std::max(x, 1)) ++b;
    return b;
}

TuneKey tune_key(const htrip_index* h, int ns, int root_group) {
    return TuneKey{h->H, h->L[h->H].NP, log2_bucket(ns), log2_bucket(root_group)};
}

int choose_query_cfg(const htrip_index* h, int ns, int root_group) {
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find(tune_key(h, ns, root_group));
        if (it != g_tune.end()) return it->second;
    }
    return root_group >= 24 ? 2 : 1;
}

// ---------------------------------------------------------------------------
// Device-planned queries (plan.cu).  A single request on an index's own
// stream is planned by the device from its viewpoints, so nothing on the host
// waits for the GPU before the launch: a query with device-resident inputs
// is two launches (planner, query kernel) and no copy.  Arena layout, every
// piece 256-byte aligned:
//   [QueryParams][unit prefix][launch words][viewpoints 8k + flags k]
//   [plan ints][M][flags + completion counters][X_0..X_{H-1} Y_1..Y_H]
//   [result k*k u16, host-bound calls]
// The plan capacities are worst cases for k viewpoints, so the planner's
// overflow status (2) is a guard, not a path: a synchronous call that sees
// it replans on the host.
// ---------------------------------------------------------------------------
struct DevPlanLayout {
    hb::PlanGeom G{};
    hb::PlanLayout O{};
    size_t o_params = 0, o_pre = 0, o_words = 0, o_in = 0, o_plan = 0, o_M = 0, o_flags = 0, o_out = 0;
    size_t X[hb::kMaxQueryLevels + 1] = {}, Y[hb::kMaxQueryLevels + 1] = {}, o_ctr = 0, o_ticket = 0, o_part = 0;
    size_t total = 0;
    int root_split = 1;
    int n_phases = 0, fill_blocks = 1;
};

// Whether the device planner takes a request.  It can: k within its
// shared-memory sort, Morton codes below 2^52 (they carry the viewpoint index
// in the low 12 bits), and the query kernel's depth and port limits.  It
// does, by default, when the viewpoints are already on the device (the host
// would otherwise wait for their copy); with host viewpoints the host plans
// (its plan goes out with the viewpoints' copy anyway, and measured faster).
// HTRIP_QUERY_PLANNER=host plans every query on the host, =device every
// query it can on the device.
bool devplan_supported(const htrip_index* h, int k, bool host_inputs) {
    if (k < 1 || k > hb::plan_max_k() || h->H > hb::kMaxQueryLevels) return false;
    static const int mode = [] {
        const char* e = std::getenv("HTRIP_QUERY_PLANNER");
        if (e && std::strcmp(e, "host") == 0) return 1;
        if (e && std::strcmp(e, "device") == 0) return 2;
        return 0;
    }();
    if (mode == 1 || (mode == 0 && host_inputs)) return false;
    double codes = 1;
    for (int l = 0; l < std::max(h->H, 1); ++l) codes *= (double)h->g * h->g;
    if (codes >= 4503599627370496.0) return false;  // 2^52
    for (int l = 1; l <= h->H; ++l)
        if (h->L[l].nP > hb::query_max_ports()) return false;
    return true;
}

DevPlanLayout devplan_layout(const htrip_index* h, int k, int cfg, bool out_in_arena) {
    DevPlanLayout D;
    const hb::QueryTile tile = hb::query_config_tile(cfg);
    const long RW = tile.RW, NC = tile.NCOL;
    const int H = h->H, g = h->g;
    hb::PlanGeom& G = D.G;
    hb::PlanLayout& O = D.O;
    G.H = H;
    G.g = g;
    G.b = h->b;
    G.S = h->S;
    G.leaves_x = h->leaves_x;
    G.RW = (int)RW;
    G.NC = (int)NC;
    G.nExt0 = h->L[0].nExt;
    auto log2_exact = [](int v) {
        int sh = 0;
        while ((1 << sh) < v) ++sh;
        return (1 << sh) == v ? sh : -1;
    };
    G.g_shift = log2_exact(g);
    G.b_shift = log2_exact(h->b);
    for (int l = 0; l <= H; ++l) {
        G.side[l] = h->L[l].side;
        G.nodes_x[l] = h->L[l].nodes_x;
        G.nP[l] = h->L[l].nP;
        G.NP[l] = h->L[l].NP;
    }
    O.k = k;
    O.kpow = hb::plan_kpow(k);
    O.sort_bytes = hb::plan_sort_bytes(O.kpow);
    // plan ints; pieces start on 64-int boundaries
    size_t n = 0;
    auto take = [&](size_t ints) {
        const size_t o = n;
        n += (ints + 63) / 64 * 64;
        return (int)o;
    };
    long max_slots = k;
    size_t flags = 0;
    for (int l = 1; l <= H; ++l) {
        O.flags_off[l] = (long long)flags;
        // groups: distinct level-(l-1) nodes holding a viewpoint; slots: each
        // group's run padded to RW; a node's run spans at most g^2 groups
        const long ngr = std::min<long>(k, h->L[l - 1].nnodes);
        const long slots = k + ngr * (RW - 1);
        const long rows = (slots + RW - 1) / RW;
        const long span = std::min<long>(slots, k + (long)g * g * (RW - 1));
        const long NP = h->L[l].NP;
        O.cap_groups[l] = (int)ngr;
        O.cap_slots[l] = (int)slots;
        O.cap_items[l] = (int)(rows * ((NP + NC - 1) / NC));
        // meet base items: per group, ceil(span / NC) slot tiles x its row
        // tiles; the port split adds at most kPlanTargetItems
        O.cap_meet[l] = (int)(((span + NC - 1) / NC + 1) * rows + hb::kPlanTargetItems);
        max_slots = std::max(max_slots, slots);
        flags += (size_t)ngr * h->L[l].nP;
    }
    O.o_vp0 = take(4 * (size_t)k);
    O.o_inv = take(k);
    O.o_rec = take(hb::plan_record_ints());
    O.o_l0 = take(H >= 1 ? 2 * (size_t)O.cap_slots[1] : 0);
    for (int l = 1; l <= H; ++l) {
        O.o_groups[l] = take(5 * (size_t)O.cap_groups[l]);
        O.o_items[l] = take(3 * (size_t)O.cap_items[l]);
        O.o_meet[l] = take(7 * (size_t)O.cap_meet[l]);
        O.o_s2v[l] = take((size_t)O.cap_slots[l] + NC);
        O.o_lift[l] = l < H ? take(2 * (size_t)O.cap_slots[l]) : 0;
    }
    if (n > (size_t)INT32_MAX) throw CudaError{cudaErrorInvalidValue, "device plan larger than 2^31 ints"};
    O.cap_ldv = (int)((max_slots + 256 + 7) / 8 * 8);
    size_t off = 0;
    auto takeb = [&](size_t bytes) {
        const size_t o = off;
        off += align256(std::max<size_t>(bytes, 1));
        return o;
    };
    D.n_phases = H + 3;
    D.o_params = takeb(sizeof(hb::QueryParams));
    D.o_pre = takeb((size_t)D.n_phases * 2 * sizeof(int));
    D.o_words = takeb(kWordsBytes);
    D.o_in = takeb(9 * (size_t)k);
    D.o_plan = takeb(n * sizeof(int));
    const size_t ldm = std::max<size_t>(8, ((size_t)k + 7) / 8 * 8);
    O.M_bytes = (long long)(ldm * ldm * sizeof(uint32_t));
    D.o_M = takeb((size_t)O.M_bytes);
    // the planner's preset blocks clear the flags, the counters and the split
    // items' tickets after them
    D.root_split = H >= 1 ? query_item_split(h, H) : 1;
    G.split_items = query_split_items(h);
    const size_t ctr_at = (flags + 15) / 16 * 16;
    const size_t ticket_at = ctr_at + hb::query_counter_words(H, k) * sizeof(unsigned);
    const size_t root_items = H >= 1 ? std::min<size_t>(O.cap_items[H], (size_t)G.split_items) : 0;
    O.flags_bytes = (long long)(ticket_at + (D.root_split > 1 ? root_items * sizeof(unsigned) : 0));
    D.o_flags = takeb((size_t)O.flags_bytes);
    D.o_ctr = D.o_flags + ctr_at;
    D.o_ticket = D.o_flags + ticket_at;
    D.o_part = D.root_split > 1 ? takeb(root_items * D.root_split * RW * NC * 2) : 0;
    for (int l = 0; l < H; ++l) D.X[l] = takeb(query_x_rows(h, l) * O.cap_ldv * sizeof(uint16_t));
    for (int l = 1; l <= H; ++l) D.Y[l] = takeb(query_y_rows(h, l) * O.cap_ldv * sizeof(uint16_t));
    D.o_out = out_in_arena ? takeb((size_t)k * k * sizeof(uint16_t)) : 0;
    D.total = off;
    O.words_bytes = (int)kWordsBytes;
    // preset blocks: about 64 KB each, no more than fit beside the planner
    const size_t smem = hb::plan_smem_bytes(O.kpow);
    const long most = smem > 113 * 1024 ? 147 : 295;
    D.fill_blocks = (int)std::clamp<long>((long)((O.M_bytes + O.flags_bytes) >> 16), 1, most);
    return D;
}

// Tile of a device-planned call whose viewpoints are on the host: the same
// inputs the host planner gives choose_query_cfg (passable viewpoints and the
// largest root child group).
int devplan_cfg_host(const htrip_index* h, const int32_t* vps, const uint8_t* pf, int k) {
    const int H = h->H, g = h->g;
    std::vector<int> cnt((size_t)g * g, 0);
    int ns = 0;
    for (int i = 0; i < k; ++i) {
        if (!pf[i]) continue;
        ++ns;
        if (H >= 1) {
            const int side = h->L[H - 1].side;
            const int cx = vps[2 * i + 1] / side, cy = vps[2 * i] / side;
            ++cnt[(size_t)(cy % g) * g + cx % g];
        }
    }
    const int group = H >= 1 ? *std::max_element(cnt.begin(), cnt.end()) : ns;
    return choose_query_cfg(h, ns, group);
}

// Tile of a call whose viewpoints are on the device: the last planned call's
// record when it had the same k and has completed, else an even spread over
// the root's children.
int devplan_cfg_hint(htrip_index* h, int k) {
    QueryArena& A = h->q;
    if (A.info && A.plan_seq > 0) {
        // seq << 32 | status << 26 | viewpoints << 13 | largest root child group
        const uint64_t rec = *reinterpret_cast<const volatile uint64_t*>(A.info);
        const unsigned lo = (unsigned)rec;
        if ((int)(rec >> 32) == A.plan_seq && (lo >> 26) == 0) {
            A.hint_k = A.info_k_last;
            A.hint_ns = (int)((lo >> 13) & 0x1fff);
            A.hint_group = (int)(lo & 0x1fff);
        }
    }
    if (A.hint_k == k) return choose_query_cfg(h, A.hint_ns, A.hint_group);
    const int g2 = h->g * h->g;
    return choose_query_cfg(h, k, h->H >= 1 ? (k + g2 - 1) / g2 : k);
}

// One device-planned request on the index's stream.  Viewpoints and flags
// come from the host (staged and copied in) or from device memory.  The
// result goes to out_dev (stream-ordered, returns 0), or, with out_dev null,
// to host_out after a synchronisation; then the return value is the status
// word (0 ok, 1 a bounded wait timed out, 2 plan capacity exceeded).
int run_devplan(htrip_index* h, int k, int cfg, const int32_t* vps_host, const uint8_t* pf_host,
                const int32_t* vps_dev, const uint8_t* pf_dev, uint16_t* out_dev, uint16_t* host_out) {
    check_query_shape(h);
    QueryArena& A = h->q;
    cudaStream_t st = h->stream;
    const bool to_host = out_dev == nullptr;
    DevPlanLayout D = devplan_layout(h, k, cfg, to_host);
    if (D.total > A.dev.n) {
        if (A.ev_valid) ck(cudaEventSynchronize(A.ev[1]), "previous launch");
        A.dev.reserve(D.total, st);
    }
    if (!A.ev[0]) {
        ck(cudaEventCreate(&A.ev[0]), "event");
        ck(cudaEventCreate(&A.ev[1]), "event");
    }
    if (!A.ticket.p) {
        A.ticket.reserve(64);
        ck(cudaMemsetAsync(A.ticket.p, 0, sizeof(unsigned), st), "ticket");
        A.ticket_next = 0;
    }
    if (!A.info) {
        ck(cudaHostAlloc(reinterpret_cast<void**>(&A.info), 2 * sizeof(int), cudaHostAllocMapped), "cudaHostAlloc");
        std::memset(A.info, 0, 2 * sizeof(int));
        ck(cudaHostGetDevicePointer(reinterpret_cast<void**>(&A.info_dev), A.info, 0), "mapped record");
    }
    unsigned char* base = A.dev.p;
    if (vps_host) {
        // the staging buffer may still feed an earlier stream-ordered copy
        if (A.ev_valid) ck(cudaEventSynchronize(A.ev[1]), "previous launch");
        const size_t nb = 9 * (size_t)k;
        A.stage.reserve(nb);
        std::memcpy(A.stage.p, vps_host, 8 * (size_t)k);
        std::memcpy(A.stage.p + 8 * (size_t)k, pf_host, k);
        ck(cudaMemcpyAsync(base + D.o_in, A.stage.p, nb, cudaMemcpyHostToDevice, st), "viewpoints");
        vps_dev = reinterpret_cast<const int32_t*>(base + D.o_in);
        pf_dev = base + D.o_in + 8 * (size_t)k;
    }
    uint16_t* out = to_host ? reinterpret_cast<uint16_t*>(base + D.o_out) : out_dev;
    // parameter block template: everything the plan does not decide
    hb::QueryParams T{};
    T.H = h->H;
    T.k = k;
    T.nExt0 = h->L[0].nExt;
    T.cfg = cfg;
    T.ext0 = h->L[0].d_ext.p;
    T.leaves = h->L[0].ms();
    for (int l = 0; l < h->H; ++l) T.X[l] = reinterpret_cast<uint16_t*>(base + D.X[l]);
    for (int l = 1; l <= h->H; ++l) T.Y[l] = reinterpret_cast<uint16_t*>(base + D.Y[l]);
    T.M = reinterpret_cast<uint32_t*>(base + D.o_M);
    T.ctr = reinterpret_cast<unsigned*>(base + D.o_ctr);
    T.out = out;
    T.work = h->count_work ? reinterpret_cast<unsigned long long*>(base + D.o_words + kWorkOffset) : nullptr;
    for (int l = 1; l <= h->H; ++l) {
        const Level& Lv = h->L[l];
        T.lv[l].D = Lv.mat.p;
        T.lv[l].NP = Lv.NP;
        T.lv[l].nP = Lv.nP;
        T.lv[l].ext_inv = Lv.d_ext_inv.p;
        T.lv[l].store_y = 1;
        T.lv[l].split = l == h->H ? D.root_split : 1;
        if (T.lv[l].split > 1) {
            T.lv[l].part = reinterpret_cast<uint32_t*>(base + D.o_part);
            T.lv[l].ticket = reinterpret_cast<unsigned*>(base + D.o_ticket);
        }
    }
    hb::PlanLayout& O = D.O;
    O.plan = reinterpret_cast<int*>(base + D.o_plan);
    O.params = reinterpret_cast<hb::QueryParams*>(base + D.o_params);
    O.unit_pre = reinterpret_cast<int*>(base + D.o_pre);
    O.words = reinterpret_cast<int*>(base + D.o_words);
    O.M = T.M;
    O.flags = base + D.o_flags;
    O.info = A.info_dev;
    O.seq = ++A.plan_seq;
    O.ticket = A.ticket.p;
    O.ticket_base = A.ticket_next;
    A.info_k_last = k;
    ck(hb::launch_plan_query(vps_dev, pf_dev, D.G, O, T, D.fill_blocks, st), "query planner");
    A.ticket_next += (unsigned)std::max(h->H, 1);
    if (A.grid == 0) A.grid = hb::query_grid_blocks(h->device);
    hb::QueryLaunch QL;
    QL.n_req = 1;
    QL.n_phases = D.n_phases;
    QL.req = O.params;
    QL.unit_pre = O.unit_pre;
    QL.status = O.words;
    QL.bar = reinterpret_cast<unsigned*>(base + D.o_words) + 1;
    QL.trace = reinterpret_cast<unsigned long long*>(base + D.o_words + kTraceOffset);
    QL.dataflow = query_dataflow_mode();
    coop_launch(h->device, st, [&] {
        const cudaError_t e = cudaEventRecord(A.ev[0], st);
        return e != cudaSuccess ? e : hb::launch_query(QL, cfg, A.grid, st);
    }, "query kernel");
    ck(cudaEventRecord(A.ev[1], st), "event");
    A.ev_valid = true;
    A.last_words = D.o_words;
    A.last_phases = D.n_phases;
    A.last_h2d = vps_host ? 9 * (uint64_t)k : 0;
    A.last_d2h = 0;
    if (!to_host) return 0;
    const size_t ob = (size_t)k * k * sizeof(uint16_t);
    A.outstage.reserve(align256(ob) + 256);
    int* status_host = reinterpret_cast<int*>(A.outstage.p + align256(ob));
    ck(cudaMemcpyAsync(A.outstage.p, out, ob, cudaMemcpyDeviceToHost, st), "result");
    ck(cudaMemcpyAsync(status_host, O.words, sizeof(int), cudaMemcpyDeviceToHost, st), "status");
    A.last_d2h = ob + sizeof(int);
    ck(cudaStreamSynchronize(st), "query sync");
    if (*status_host == 0) std::memcpy(host_out, A.outstage.p, ob);
    return *status_host;
}

// ---------------------------------------------------------------------------
// Allocation-free query scratch (htrip_query_all_pairs_noalloc).
//
// Some callers cannot allocate device memory once they are running: a
// serving process whose pool allocator reserved all of HBM at start-up, or a
// real-time planning loop where cudaMalloc / cudaFree (cudaFree waits for the
// whole device) are not allowed after initialisation.  For them the query's
// device scratch (plan, port vectors, projections, pair matrix, flags,
// barrier words, parameter block and output staging) is carved from this
// fixed array instead of the index's own growable buffers.  Every GPU that
// loads this module holds the array until the process exits.
//
// In host code `g_noalloc_scratch` is only a host-side stand-in for the
// symbol; the device address is looked up once per device with
// cudaGetSymbolAddress (with that device current) and cached.
// ---------------------------------------------------------------------------
constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;  // 64 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;                                  // guards set-up and serialises calls
unsigned char* g_noalloc_ptr[kNoAllocMaxDevices] = {};    // device address per ordinal

// Device address of the scratch array on the current device `dev`
// (the first call on a device performs the look-up).
unsigned char* noalloc_scratch(int dev) {
    if (dev < 0 || dev >= kNoAllocMaxDevices) throw CudaError{cudaErrorInvalidDevice, "device ordinal above 63"};
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        ck(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(static scratch)");
        g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
    }
    return g_noalloc_ptr[dev];
}

}  // namespace

// State of queryAllPairsIncremental (reference HTripIncrementalState,
// minplus_oracle.hpp:262-293): the viewpoints and their passability, the
// index's build / root-growth epoch, its opening count and opening stamp
// when the matrix was computed, the matrix, and a query arena of its own
// that keeps the last launch's port vectors, projections, finite-port flags
// and pair matrix (the plan is kept too), so that a later refresh re-runs
// only the work of viewpoints whose leaf-to-root chain changed.
struct htrip_incremental {
    bool initialized = false;
    const htrip_index* index = nullptr;
    uint64_t epoch = 0, updates = 0, stamp_epoch = 0, host_opens = 0;
    uint32_t seen_stamp = 0;
    std::vector<int32_t> vps;
    std::vector<uint8_t> pf;
    std::vector<uint16_t> matrix;
    QueryPlan plan;
    QueryArena q;
    DevBuf<uint8_t> dirty;
    int* n_dirty = nullptr;      // host-mapped count of dirty viewpoints
    int* n_dirty_dev = nullptr;
    int device = -1;
    ~htrip_incremental() {
        if (device >= 0) cudaSetDevice(device);
        q.release();
        dirty.release();
        if (n_dirty) cudaFreeHost(n_dirty);
    }
};

// ===========================================================================
// C ABI
// ===========================================================================
#define HTRIP_GUARD_BEGIN try {
#define HTRIP_GUARD_END                                                                     \
    }                                                                                       \
    catch (const CudaError& ce) {                                                           \
        if (ce.e == cudaErrorMemoryAllocation) {                                            \
            cudaGetLastError();                                                             \
            return fail(HTRIP_ERR_OOM, std::string("out of device memory in ") + ce.what);   \
        }                                                                                   \
        return fail(HTRIP_ERR_CUDA, std::string(ce.what) + ": " + cudaGetErrorString(ce.e)); \
    }                                                                                       \
    catch (const std::bad_alloc&) {                                                         \
        return fail(HTRIP_ERR_OOM, "host allocation failed");                               \
    }

// OK when the index can serve calls: built and resident on the device.
static htrip_status ready(const htrip_index* h) {
    if (!h->built) return fail(HTRIP_ERR_NOT_BUILT, "index not built");
    if (h->offloaded) return fail(HTRIP_ERR_INVALID, "index is offloaded to host memory (htrip_restore first)");
    return HTRIP_OK;
}

extern "C" {

const char* htrip_last_error(void) { return g_err.c_str(); }

htrip_status htrip_create(htrip_config cfg, int device, htrip_index** out) {
    if (!out) return fail(HTRIP_ERR_INVALID, "null out");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(HTRIP_ERR_NO_DEVICE, "no CUDA device");
    }
    if (device < 0 || device >= ndev) return fail(HTRIP_ERR_INVALID, "bad device ordinal");
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(device), "cudaSetDevice");
    auto* h = new htrip_index();
    h->device = device;
    h->b = cfg.tile_size_b;
    h->g = cfg.group;
    ck(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream");
    *out = h;
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_destroy(htrip_index* h) {
    if (!h) return HTRIP_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    h->release();
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return HTRIP_OK;
}

htrip_status htrip_build(htrip_index* h, const uint8_t* observed, int32_t rows, int32_t cols) {
    if (!h) return fail(HTRIP_ERR_INVALID, "null handle");
    // HierarchyConfig::isValid (types.hpp:221-224) and build()'s own checks (minplus_oracle.cpp:49-52)
    const int b = h->b, g = h->g;
    if (!(b > 0 && g >= 2 && g * g <= 256)) return fail(HTRIP_ERR_INVALID, "invalid HierarchyConfig");
    if (std::max(rows, cols) <= 0) return fail(HTRIP_ERR_INVALID, "empty grid");
    if (b < 2 || b > 32) return fail(HTRIP_ERR_UNSUPPORTED, "tile_size_b must be in [2, 32]");
    if (!observed || rows < 0 || cols < 0) return fail(HTRIP_ERR_INVALID, "bad grid");
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    do_build(h, observed, rows, cols);
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_cell_blocked(htrip_index* h, int32_t r, int32_t c, const uint8_t* observed, int32_t rows,
                                int32_t cols) {
    if (!h || !observed) return fail(HTRIP_ERR_INVALID, "bad arguments");
    if (const htrip_status rs = ready(h)) return rs;
    if (r < 0 || c < 0 || r >= h->S || c >= h->S) return HTRIP_OK;  // minplus_oracle.cpp:251 (outside: ignored)
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    do_rebuild_leaves(h, {(r / h->b) * h->leaves_x + c / h->b}, observed, rows, cols, true);
    h->epoch++;  // minplus_oracle.cpp:300-301
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_leaves_changed(htrip_index* h, const int32_t* leaves, int32_t n, const uint8_t* observed,
                                  int32_t rows, int32_t cols) {
    if (!h || !observed || n < 0 || (n > 0 && !leaves)) return fail(HTRIP_ERR_INVALID, "bad arguments");
    if (const htrip_status rs = ready(h)) return rs;
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    do_rebuild_leaves(h, std::vector<int>(leaves, leaves + n), observed, rows, cols, false);
    h->epoch++;  // propagateBatchUpward ends with epoch++ (minplus_oracle.cpp:504)
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_set_cell_weights(htrip_index* h, const uint16_t* weights, int32_t rows, int32_t cols) {
    if (!h) return fail(HTRIP_ERR_INVALID, "null handle");
    if (weights && (rows <= 0 || cols <= 0)) return fail(HTRIP_ERR_INVALID, "bad weights grid");
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    if (weights) {
        h->wgrid.assign(weights, weights + (size_t)rows * cols);
        h->wrows = rows;
        h->wcols = cols;
    } else {
        h->wgrid.clear();
        h->wrows = h->wcols = 0;
    }
    if (h->built) {
        upload_weights(h);
        ck(cudaStreamSynchronize(h->stream), "weights sync");
    }
    return HTRIP_OK;
    HTRIP_GUARD_END
}

// GridMap::setCellWeight (grid_map.hpp:297-303): the first weight set gives
// every cell of the grid weight 1.
static void set_host_weight(htrip_index* h, int r, int c, uint16_t w, int rows, int cols) {
    if (h->wgrid.empty() || h->wrows != rows || h->wcols != cols) {
        std::vector<uint16_t> g((size_t)rows * cols, 1);
        for (int y = 0; y < std::min(rows, h->wrows); ++y)
            for (int x = 0; x < std::min(cols, h->wcols); ++x) g[(size_t)y * cols + x] = h->wgrid[(size_t)y * h->wcols + x];
        h->wgrid = std::move(g);
        h->wrows = rows;
        h->wcols = cols;
    }
    h->wgrid[(size_t)r * cols + c] = w;
}

htrip_status htrip_cell_weight_changed(htrip_index* h, int32_t r, int32_t c, uint16_t new_weight,
                                       const uint8_t* observed, int32_t rows, int32_t cols) {
    if (!h || !observed || rows <= 0 || cols <= 0) return fail(HTRIP_ERR_INVALID, "bad arguments");
    if (const htrip_status rs = ready(h)) return rs;
    // minplus_oracle.cpp:304-307: outside the grid, or the same weight: nothing
    if (r < 0 || c < 0 || r >= rows || c >= cols) return HTRIP_OK;
    if (host_cell_weight(h, r, c, observed, rows, cols) == new_weight) return HTRIP_OK;
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    set_host_weight(h, r, c, new_weight, rows, cols);
    upload_weights(h);
    if (r >= h->S || c >= h->S) return HTRIP_OK;  // :312 (no leaf holds the cell)
    // :314-357: the leaf rebuilt from the grid, then every ancestor
    do_rebuild_leaves(h, {(r / h->b) * h->leaves_x + c / h->b}, observed, rows, cols, true);
    h->epoch++;  // :359
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_tile_weights_changed(htrip_index* h, int32_t tx, int32_t ty, const int32_t* rc,
                                        const uint16_t* weights, int32_t n, const uint8_t* observed, int32_t rows,
                                        int32_t cols) {
    if (!h || !observed || rows <= 0 || cols <= 0 || n < 0 || (n > 0 && (!rc || !weights)))
        return fail(HTRIP_ERR_INVALID, "bad arguments");
    if (const htrip_status rs = ready(h)) return rs;
    if (tx < 0 || ty < 0 || tx >= h->leaves_x || ty >= h->leaves_x) return HTRIP_OK;  // minplus_oracle.cpp:366
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    for (int i = 0; i < n; ++i) {  // :368-373: every in-grid cell of the list, whichever tile holds it
        const int r = rc[2 * i], c = rc[2 * i + 1];
        if (r >= 0 && c >= 0 && r < rows && c < cols) set_host_weight(h, r, c, weights[i], rows, cols);
    }
    upload_weights(h);
    // :375-421: the leaf (tx, ty) rebuilt once, then every ancestor
    do_rebuild_leaves(h, {ty * h->leaves_x + tx}, observed, rows, cols, true);
    h->epoch++;  // :423
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_lift_root(htrip_index* h, const uint8_t* observed, int32_t rows, int32_t cols) {
    if (!h) return fail(HTRIP_ERR_INVALID, "null handle");
    if (const htrip_status rs = ready(h)) return rs;
    if (rows < 0 || cols < 0 || ((rows > 0 && cols > 0) && !observed)) return fail(HTRIP_ERR_INVALID, "bad grid");
    if ((int64_t)h->S * h->g > (1 << 20)) return fail(HTRIP_ERR_UNSUPPORTED, "grid side above 2^20");
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    do_lift_root(h, observed, rows > 0 && cols > 0 ? rows : 0, rows > 0 && cols > 0 ? cols : 0);
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_open_cells(htrip_index* h, const int32_t* rc, int32_t n, const uint8_t* observed, int32_t rows,
                              int32_t cols) {
    if (!h) return fail(HTRIP_ERR_INVALID, "null handle");
    if (const htrip_status rs = ready(h)) return rs;
    if (n < 0 || (n > 0 && !rc) || !observed) return fail(HTRIP_ERR_INVALID, "bad arguments");
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    do_open(h, rc, n, observed, rows, cols, true);
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_open_cell(htrip_index* h, int32_t r, int32_t c, const uint8_t* observed, int32_t rows, int32_t cols) {
    if (!h) return fail(HTRIP_ERR_INVALID, "null handle");
    if (const htrip_status rs = ready(h)) return rs;
    if (!observed) return fail(HTRIP_ERR_INVALID, "bad arguments");
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    const int32_t rc[2] = {r, c};
    do_open(h, rc, 1, observed, rows, cols, false);
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_query_all_pairs(htrip_index* h, const int32_t* vps, int32_t k, const uint8_t* observed, int32_t rows,
                                   int32_t cols, uint16_t* out) {
    if (!h) return fail(HTRIP_ERR_INVALID, "null handle");
    if (const htrip_status rs = ready(h)) return rs;
    if (k < 0 || (k > 0 && (!vps || !out)) || !observed) return fail(HTRIP_ERR_INVALID, "bad arguments");
    if (k == 0) return HTRIP_OK;
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    const std::vector<uint8_t> pf = viewpoint_flags(h, vps, k, observed, rows, cols);
    if (devplan_supported(h, k, true)) {
        const int status =
            run_devplan(h, k, devplan_cfg_host(h, vps, pf.data(), k), vps, pf.data(), nullptr, nullptr, nullptr, out);
        if (status == 1) return fail(HTRIP_ERR_CUDA, "query kernel: a bounded wait timed out");
        if (status == 0) return HTRIP_OK;
        // status 2: the plan outgrew its worst-case capacity; plan on the host
    }
    QueryPlan P;
    make_plan(h, vps, pf.data(), k, P);
    const std::vector<QueryReq> R{{h, &P, nullptr}};
    if (run_queries(h->q, h->device, h->stream, R, {out}, true) != 0)
        return fail(HTRIP_ERR_CUDA, "query kernel: a bounded wait timed out");
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_query_distance(htrip_index* h, int32_t r1, int32_t c1, int32_t r2, int32_t c2,
                                  const uint8_t* observed, int32_t rows, int32_t cols, uint16_t* out) {
    if (!h || !out || !observed) return fail(HTRIP_ERR_INVALID, "bad arguments");
    if (const htrip_status rs = ready(h)) return rs;
    const int32_t vps[4] = {r1, c1, r2, c2};
    const std::vector<uint8_t> pf = viewpoint_flags(h, vps, 2, observed, rows, cols);
    // queryDistance (minplus_oracle.cpp:834-849): INF unless both cells are
    // passable and inside the index, 0 for s == t.
    if (!pf[0] || !pf[1]) {
        *out = HTRIP_INF;
        return HTRIP_OK;
    }
    if (r1 == r2 && c1 == c2) {
        *out = 0;
        return HTRIP_OK;
    }
    uint16_t m[4];
    const htrip_status st = htrip_query_all_pairs(h, vps, 2, observed, rows, cols, m);
    if (st != HTRIP_OK) return st;
    *out = m[1];
    return HTRIP_OK;
}

htrip_status htrip_incremental_create(htrip_incremental** out) {
    if (!out) return fail(HTRIP_ERR_INVALID, "null out");
    *out = new (std::nothrow) htrip_incremental();
    return *out ? HTRIP_OK : fail(HTRIP_ERR_OOM, "host allocation failed");
}

htrip_status htrip_incremental_destroy(htrip_incremental* s) {
    delete s;
    return HTRIP_OK;
}

htrip_status htrip_query_all_pairs_incremental(htrip_index* h, htrip_incremental* s, const int32_t* vps, int32_t k,
                                               const uint8_t* observed, int32_t rows, int32_t cols, uint16_t* out,
                                               int32_t* recomputed) {
    if (!h || !s) return fail(HTRIP_ERR_INVALID, "null argument");
    if (const htrip_status rs = ready(h)) return rs;
    if (k < 0 || (k > 0 && (!vps || !out)) || !observed) return fail(HTRIP_ERR_INVALID, "bad arguments");
    if (recomputed) *recomputed = 0;
    if (k == 0) {  // minplus_oracle.cpp:1450-1454
        s->initialized = false;
        return HTRIP_OK;
    }
    const bool same_vps = s->vps.size() == 2 * (size_t)k && std::equal(vps, vps + 2 * (size_t)k, s->vps.begin());
    if (s->initialized && s->index == h && s->epoch == h->epoch && same_vps && s->updates == h->update_counter) {
        std::memcpy(out, s->matrix.data(), (size_t)k * k * sizeof(uint16_t));  // no update since: the cached matrix
        return HTRIP_OK;
    }
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    if (s->device >= 0 && s->device != h->device) {  // the arena lives on another device: start over
        s->q.release();
        s->dirty.release();
        s->initialized = false;
    }
    s->device = h->device;
    std::vector<uint8_t> pf = viewpoint_flags(h, vps, k, observed, rows, cols);
    // Every update since the last call was an opening on the device path
    // (no build, root growth, rebuild or weight change: equal epoch; no
    // host-path opening; no reallocation of the stamps): re-lift only the
    // viewpoints under matrices those openings listed.  Distances only
    // decrease under openings, so the pairs of the other viewpoints keep
    // their values and the new ones are the minimum with the old.
    const bool selective = s->initialized && s->index == h && s->epoch == h->epoch && same_vps && s->pf == pf &&
                           s->stamp_epoch == h->stamp_epoch && s->host_opens == h->host_opens;
    s->matrix.resize((size_t)k * k);
    const std::vector<QueryReq> R{{h, &s->plan, nullptr}};
    int status = 0;
    if (!selective) {
        s->initialized = false;
        make_plan(h, vps, pf.data(), k, s->plan);
        status = run_queries(s->q, h->device, h->stream, R, {s->matrix.data()}, true);
        if (recomputed) *recomputed = 1;
    } else {
        const LaunchLayout L = layout_launch(R);  // the same plan: the same layout as the last launch
        const int ns = s->plan.n_sorted;
        if (!s->n_dirty) {
            ck(cudaHostAlloc(reinterpret_cast<void**>(&s->n_dirty), sizeof(int), cudaHostAllocMapped), "cudaHostAlloc");
            ck(cudaHostGetDevicePointer(reinterpret_cast<void**>(&s->n_dirty_dev), s->n_dirty, 0), "mapped count");
        }
        *s->n_dirty = 0;
        s->dirty.reserve(std::max(1, ns));
        hb::IncrementalChain C{};
        C.H = h->H;
        C.g = h->g;
        C.leaves_x = h->leaves_x;
        for (int l = 0; l <= h->H; ++l) {
            C.mstamp[l] = h->L[l].mstamp.p;
            C.nodes_x[l] = h->L[l].nodes_x;
        }
        const int* vp0 = reinterpret_cast<const int*>(s->q.dev.p + L.plan[0]) + s->plan.o_vp0;
        hb::launch_incremental_dirty(vp0, ns, C, s->seen_stamp, s->dirty.p, s->n_dirty_dev, h->stream);
        ck(cudaGetLastError(), "dirty viewpoints");
        ck(cudaStreamSynchronize(h->stream), "dirty viewpoints");
        if (*s->n_dirty > 0) {
            status = run_queries(s->q, h->device, h->stream, R, {s->matrix.data()}, true, s->dirty.p);
            if (recomputed) *recomputed = 2;
        }
    }
    if (status != 0) return fail(HTRIP_ERR_CUDA, "query kernel: a bounded wait timed out");
    s->vps.assign(vps, vps + 2 * (size_t)k);
    s->pf = std::move(pf);
    s->index = h;
    s->epoch = h->epoch;
    s->updates = h->update_counter;
    s->stamp_epoch = h->stamp_epoch;
    s->host_opens = h->host_opens;
    s->seen_stamp = h->open_stamp;
    s->initialized = true;
    std::memcpy(out, s->matrix.data(), (size_t)k * k * sizeof(uint16_t));
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_query_all_pairs_dev(htrip_index* h, const int32_t* vps_dev, const uint8_t* passable_dev, int32_t k,
                                       uint16_t* out_dev) {
    if (!h) return fail(HTRIP_ERR_INVALID, "null handle");
    if (const htrip_status rs = ready(h)) return rs;
    if (k < 0 || (k > 0 && (!vps_dev || !passable_dev || !out_dev))) return fail(HTRIP_ERR_INVALID, "bad arguments");
    if (k == 0) return HTRIP_OK;
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    if (devplan_supported(h, k, false)) {  // planned on the device: no host round trip
        run_devplan(h, k, devplan_cfg_hint(h, k), nullptr, nullptr, vps_dev, passable_dev, out_dev, nullptr);
        return HTRIP_OK;
    }
    // Larger requests: the viewpoint plan is built on the host.
    std::vector<int32_t> vps(2 * (size_t)k);
    std::vector<uint8_t> pf(k);
    ck(cudaMemcpyAsync(vps.data(), vps_dev, vps.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream), "vps");
    ck(cudaMemcpyAsync(pf.data(), passable_dev, k, cudaMemcpyDeviceToHost, h->stream), "pf");
    ck(cudaStreamSynchronize(h->stream), "sync");
    for (int i = 0; i < k; ++i) {
        const int r = vps[2 * i], c = vps[2 * i + 1];
        if (r < 0 || c < 0 || r >= h->S || c >= h->S) pf[i] = 0;
    }
    QueryPlan P;
    make_plan(h, vps.data(), pf.data(), k, P);
    const std::vector<QueryReq> R{{h, &P, out_dev}};
    run_queries(h->q, h->device, h->stream, R, {nullptr}, false);
    h->q.last_d2h = vps.size() * sizeof(int32_t) + pf.size();
    return HTRIP_OK;
    HTRIP_GUARD_END
}

// Same query as htrip_query_all_pairs, with every piece of device scratch
// carved from the fixed module-scope array above: no cudaMalloc / cudaFree
// and no growth of the index's own buffers (host staging is pageable
// memory).  A process-wide lock is held from the first write to the array
// until the result is back on the host, so calls through this entry point
// never overlap on the GPU (calls that did overlap would race on the shared
// array).
htrip_status htrip_query_all_pairs_noalloc(htrip_index* h, const int32_t* vps, int32_t k, const uint8_t* observed,
                                           int32_t rows, int32_t cols, uint16_t* out) {
    if (!h) return fail(HTRIP_ERR_INVALID, "null handle");
    if (const htrip_status rs = ready(h)) return rs;
    if (k < 0 || (k > 0 && (!vps || !out)) || !observed) return fail(HTRIP_ERR_INVALID, "bad arguments");
    if (k == 0) return HTRIP_OK;
    const int H = h->H;
    if (H > hb::kMaxQueryLevels) return fail(HTRIP_ERR_UNSUPPORTED, "hierarchy deeper than the query supports");
    for (int l = 1; l <= H; ++l)
        if (h->L[l].nP > hb::query_max_ports())
            return fail(HTRIP_ERR_UNSUPPORTED, "child port count above the query kernel's list capacity");
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    const std::vector<uint8_t> pf = viewpoint_flags(h, vps, k, observed, rows, cols);
    QueryPlan P;
    make_plan(h, vps, pf.data(), k, P);
    const std::vector<QueryReq> R{{h, &P, nullptr}};
    const LaunchLayout L = layout_launch(R);
    if (L.total > kNoAllocScratchBytes)
        return fail(HTRIP_ERR_UNSUPPORTED, "query needs " + std::to_string(L.total) +
                                               " bytes of device scratch; the allocation-free entry point has " +
                                               std::to_string(kNoAllocScratchBytes) + " (fewer viewpoints or a smaller map)");
    std::vector<unsigned char> stage(L.head);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    unsigned char* base = noalloc_scratch(h->device);
    cudaStream_t st = h->stream;
    // Declared after the lock, so it runs before the lock is released on
    // every exit path (an exception included): once work that uses the
    // shared array is queued, the lock is not given up before that work has
    // finished, or the next caller's launch could overlap it.
    struct DrainOnExit {
        cudaStream_t st;
        bool armed = false;
        ~DrainOnExit() {
            if (armed) cudaStreamSynchronize(st);  // errors are reported by the call itself
        }
    } drain{st};
    // The array keeps the previous call's contents: the launch head (with
    // zeroed status / barrier words), the pair matrix and the flags are
    // rewritten by every call.
    std::vector<uint16_t*> outs;
    int grid = h->q.grid;
    drain.armed = true;
    issue_query_launch(st, h->device, grid, P.cfg, R, L, base, stage.data(), nullptr, outs);
    h->q.grid = grid;
    // The status word first: the caller's `out` is written only by a launch
    // whose every wait completed.
    int status = 0;
    ck(cudaMemcpyAsync(&status, base + L.o_words, sizeof(int), cudaMemcpyDeviceToHost, st), "status");
    ck(cudaStreamSynchronize(st), "query sync");
    if (status != 0) return fail(HTRIP_ERR_CUDA, "query kernel: a bounded wait timed out");
    ck(cudaMemcpyAsync(out, outs[0], (size_t)k * k * sizeof(uint16_t), cudaMemcpyDeviceToHost, st), "out");
    ck(cudaStreamSynchronize(st), "result sync");
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_batch_create(int device, htrip_batch** out) { return htrip_batch_create_priority(device, 0, out); }

htrip_status htrip_batch_create_priority(int device, int32_t high_priority, htrip_batch** out) {
    if (!out) return fail(HTRIP_ERR_INVALID, "null out");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(HTRIP_ERR_NO_DEVICE, "no CUDA device");
    }
    if (device < 0 || device >= ndev) return fail(HTRIP_ERR_INVALID, "bad device ordinal");
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(device), "cudaSetDevice");
    int lo = 0, hi = 0;  // numerically lower = higher priority
    ck(cudaDeviceGetStreamPriorityRange(&lo, &hi), "stream priority range");
    auto* b = new htrip_batch();
    b->device = device;
    if (cudaStreamCreateWithPriority(&b->stream, cudaStreamNonBlocking, high_priority ? hi : lo) != cudaSuccess) {
        delete b;
        return fail(HTRIP_ERR_CUDA, "stream creation failed");
    }
    *out = b;
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_batch_destroy(htrip_batch* b) {
    if (!b) return HTRIP_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    b->q.release();
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return HTRIP_OK;
}

htrip_status htrip_query_batch(htrip_batch* b, const htrip_query_request* reqs, int32_t n) {
    if (!b) return fail(HTRIP_ERR_INVALID, "null batch");
    if (n < 0 || (n > 0 && !reqs)) return fail(HTRIP_ERR_INVALID, "bad arguments");
    for (int i = 0; i < n; ++i) {
        const htrip_query_request& r = reqs[i];
        if (!r.index) return fail(HTRIP_ERR_INVALID, "request " + std::to_string(i) + ": null index");
        if (!r.index->built) return fail(HTRIP_ERR_NOT_BUILT, "request " + std::to_string(i) + ": index not built");
        if (r.index->offloaded) return fail(HTRIP_ERR_INVALID, "request " + std::to_string(i) + ": index offloaded");
        if (r.index->device != b->device)
            return fail(HTRIP_ERR_INVALID, "request " + std::to_string(i) + ": index on another device");
        if (r.k < 0 || (r.k > 0 && (!r.vps || !r.out)) || !r.observed)
            return fail(HTRIP_ERR_INVALID, "request " + std::to_string(i) + ": bad arguments");
    }
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(b->device), "cudaSetDevice");
    std::vector<QueryPlan> plans;
    std::vector<const htrip_index*> hs;
    std::vector<const int32_t*> vps;
    std::vector<std::vector<uint8_t>> pf;
    std::vector<uint16_t*> outs;
    for (int i = 0; i < n; ++i) {
        const htrip_query_request& r = reqs[i];
        if (r.k == 0) continue;
        hs.push_back(r.index);
        vps.push_back(r.vps);
        pf.push_back(viewpoint_flags(r.index, r.vps, r.k, r.observed, r.rows, r.cols));
        outs.push_back(r.out);
        plans.emplace_back();
        make_plan(r.index, r.vps, pf.back().data(), r.k, plans.back());
    }
    if (plans.empty()) return HTRIP_OK;
    plan_common(plans, hs, vps, pf);
    // Work queued on an index's own stream (a stream-ordered query) ends
    // before this launch reads the index.
    for (size_t i = 0; i < hs.size(); ++i) ck(cudaStreamSynchronize(hs[i]->stream), "index stream");
    std::vector<QueryReq> R;
    for (size_t i = 0; i < plans.size(); ++i) R.push_back({hs[i], &plans[i], nullptr});
    if (run_queries(b->q, b->device, b->stream, R, outs, true) != 0)
        return fail(HTRIP_ERR_CUDA, "query kernel: a bounded wait timed out");
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_open_batch(htrip_batch* b, const htrip_open_request* reqs, int32_t n) {
    if (!b) return fail(HTRIP_ERR_INVALID, "null batch");
    if (n < 0 || (n > 0 && !reqs)) return fail(HTRIP_ERR_INVALID, "bad arguments");
    for (int i = 0; i < n; ++i) {
        const htrip_open_request& r = reqs[i];
        if (!r.index) return fail(HTRIP_ERR_INVALID, "request " + std::to_string(i) + ": null index");
        if (!r.index->built) return fail(HTRIP_ERR_NOT_BUILT, "request " + std::to_string(i) + ": index not built");
        if (r.index->offloaded) return fail(HTRIP_ERR_INVALID, "request " + std::to_string(i) + ": index offloaded");
        if (r.index->device != b->device)
            return fail(HTRIP_ERR_INVALID, "request " + std::to_string(i) + ": index on another device");
        if (r.n < 0 || (r.n > 0 && !r.rc) || !r.observed)
            return fail(HTRIP_ERR_INVALID, "request " + std::to_string(i) + ": bad arguments");
    }
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(b->device), "cudaSetDevice");
    // Requests on the same index are applied in call order: request i goes
    // into wave w = the number of earlier requests on its index.
    std::vector<int> wave(n, 0);
    int n_waves = 0;
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < i; ++j)
            if (reqs[j].index == reqs[i].index) wave[i] = std::max(wave[i], wave[j] + 1);
        n_waves = std::max(n_waves, wave[i] + 1);
    }
    for (int w = 0; w < n_waves; ++w) {
        std::vector<OpenTask> tasks;
        tasks.reserve(n);
        for (int i = 0; i < n; ++i) {
            if (wave[i] != w) continue;
            const htrip_open_request& r = reqs[i];
            ck(cudaStreamSynchronize(r.index->stream), "index stream");
            r.index->update_counter++;
            tasks.emplace_back();
            open_prepare(tasks.back(), r.index, r.rc, r.n, r.observed, r.rows, r.cols, true);
        }
        std::vector<OpenTask*> work;
        for (auto& T : tasks)
            if (open_has_work(T)) work.push_back(&T);
        if (!work.empty()) run_open(work, b->u, b->stream, b->device);
    }
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_batch_last_kernel_ms(const htrip_batch* b, float* ms) {
    if (!b || !ms) return fail(HTRIP_ERR_INVALID, "null argument");
    if (!b->q.ev_valid) return fail(HTRIP_ERR_INVALID, "no launch has run");
    HTRIP_GUARD_BEGIN
    ck(cudaEventSynchronize(b->q.ev[1]), "event sync");
    ck(cudaEventElapsedTime(ms, b->q.ev[0], b->q.ev[1]), "event time");
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_clone(const htrip_index* src, htrip_index** out) {
    if (!src || !out) return fail(HTRIP_ERR_INVALID, "null argument");
    *out = nullptr;
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(src->device), "cudaSetDevice");
    if (src->offloaded) return fail(HTRIP_ERR_INVALID, "index is offloaded to host memory (htrip_restore first)");
    ck(cudaStreamSynchronize(src->stream), "sync");
    auto* h = new htrip_index();
    h->device = src->device;
    h->b = src->b;
    h->g = src->g;
    h->wgrid = src->wgrid;
    h->wrows = src->wrows;
    h->wcols = src->wcols;
    try {
        ck(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream");
        if (src->built) {
            h->S = src->S; h->H = src->H; h->rows = src->rows; h->cols = src->cols; h->leaves_x = src->leaves_x;
            make_levels(h);
            alloc_levels(h);
            for (int l = 0; l <= h->H; ++l)
                ck(cudaMemcpyAsync(h->L[l].mat.p, src->L[l].mat.p, h->L[l].mat.n * sizeof(uint16_t),
                                   cudaMemcpyDeviceToDevice, h->stream), "clone copy");
            h->pass.reserve(src->pass.n);
            ck(cudaMemcpyAsync(h->pass.p, src->pass.p, src->pass.n, cudaMemcpyDeviceToDevice, h->stream), "clone pass");
            if (src->wts.p) {
                h->wts.reserve(src->wts.n);
                ck(cudaMemcpyAsync(h->wts.p, src->wts.p, src->wts.n * sizeof(uint16_t), cudaMemcpyDeviceToDevice,
                                   h->stream), "clone weights");
            }
            ck(cudaStreamSynchronize(h->stream), "clone sync");
            h->built = true;
            h->stats = src->stats;
            h->ref_bytes = src->ref_bytes;
        }
    } catch (...) {
        htrip_destroy(h);
        throw;
    }
    *out = h;
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_query_work(const htrip_index* h, const int32_t* vps, int32_t k, const uint8_t* observed,
                              int32_t rows, int32_t cols, uint64_t* alg_bytes, uint64_t* alg_ops) {
    if (!h || !h->built || k < 0 || (k > 0 && !vps) || !observed) return fail(HTRIP_ERR_INVALID, "bad arguments");
    const int b = h->b, g = h->g, H = h->H;
    uint64_t bytes = 0, ops = 0;
    std::vector<int> tx, ty;
    for (int i = 0; i < k; ++i) {
        const int r = vps[2 * i], c = vps[2 * i + 1];
        if (r < 0 || c < 0 || r >= rows || c >= cols || observed[(size_t)r * cols + c] != 1) continue;
        tx.push_back(c / b);
        ty.push_back(r / b);
    }
    const uint64_t n = tx.size();
    bytes += n * (uint64_t)h->L[0].nExt * 2;  // level-0 port gathers
    for (int l = 1; l <= H; ++l) {
        const Level& Lv = h->L[l];
        const Level& Lc = h->L[l - 1];
        const uint64_t nP = Lv.nP, nExt = Lv.nExt;
        // viewpoint count per (node, quad)
        std::vector<std::pair<int, int>> key;
        for (size_t i = 0; i < n; ++i) {
            const int cx = tx[i] * b / Lc.side, cy = ty[i] * b / Lc.side;
            key.push_back({(cy / g) * Lv.nodes_x + cx / g, (cy % g) * g + cx % g});
        }
        std::sort(key.begin(), key.end());
        for (size_t i = 0; i < key.size();) {
            size_t j = i;
            while (j < key.size() && key[j].first == key[i].first) ++j;
            std::vector<uint64_t> cnt;  // per active child of this node
            for (size_t a = i; a < j;) {
                size_t c = a;
                while (c < j && key[c].second == key[a].second) ++c;
                cnt.push_back(c - a);
                a = c;
            }
            for (size_t a = 0; a < cnt.size(); ++a) {
                if (l < H) { bytes += nP * nExt * 2; ops += cnt[a] * nP * nExt; }
                for (size_t c = a + 1; c < cnt.size(); ++c) {
                    bytes += nP * nP * 2;
                    ops += cnt[a] * nP * nP + cnt[a] * cnt[c] * nP;
                }
                if (cnt[a] >= 2) { bytes += nP * nP * 2; ops += cnt[a] * nP * nP + cnt[a] * cnt[a] * nP; }
            }
            i = j;
        }
    }
    if (alg_bytes) *alg_bytes = bytes;
    if (alg_ops) *alg_ops = ops;
    return HTRIP_OK;
}

htrip_status htrip_state_digest(const htrip_index* h, uint64_t* out, int32_t n_out) {
    if (!h || !out) return fail(HTRIP_ERR_INVALID, "null argument");
    if (const htrip_status rs = ready(h)) return rs;
    if (n_out < h->H + 1) return fail(HTRIP_ERR_INVALID, "digest needs H + 1 entries");
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    DevBuf<unsigned long long> d;
    d.reserve(h->H + 1);
    ck(cudaMemsetAsync(d.p, 0, (h->H + 1) * sizeof(unsigned long long), h->stream), "digest preset");
    for (int l = 0; l <= h->H; ++l) hb::launch_digest(h->L[l].ms(), h->L[l].nnodes, d.p + l, h->stream);
    ck(cudaGetLastError(), "digest");
    ck(cudaMemcpyAsync(out, d.p, (h->H + 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost, h->stream), "digest d2h");
    ck(cudaStreamSynchronize(h->stream), "digest sync");
    d.release();
    return HTRIP_OK;
    HTRIP_GUARD_END
}

static htrip_status timeout_selftest(int kind, int device, int32_t* status, int32_t* ctas_returned, float* ms) {
    if (!status || !ctas_returned || !ms) return fail(HTRIP_ERR_INVALID, "null argument");
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(device), "cudaSetDevice");
    int st = 0, ret = 0;
    float t = 0.f;
    ck(kind == 0 ? hb::barrier_timeout_selftest(&st, &ret, &t) : hb::wait_timeout_selftest(&st, &ret, &t),
       "timeout self-test");
    *status = st;
    *ctas_returned = ret;
    *ms = t;
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_selftest_barrier_timeout(int device, int32_t* status, int32_t* ctas_returned, float* ms) {
    return timeout_selftest(0, device, status, ctas_returned, ms);
}

htrip_status htrip_selftest_wait_timeout(int device, int32_t* status, int32_t* ctas_returned, float* ms) {
    return timeout_selftest(1, device, status, ctas_returned, ms);
}

htrip_status htrip_measure_minplus_rate(int device, int variant, double* entries_per_s) {
    if (!entries_per_s || variant < 0 || variant > 4) return fail(HTRIP_ERR_INVALID, "bad arguments");
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(device), "cudaSetDevice");
    int sms = 0;
    ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "attribute");
    const double r = hb::measure_minplus_rate(variant, sms);
    if (r <= 0) return fail(HTRIP_ERR_CUDA, "min-plus rate kernel failed");
    *entries_per_s = r;
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_last_query_kernel_ms(const htrip_index* h, float* ms) {
    if (!h || !ms) return fail(HTRIP_ERR_INVALID, "null argument");
    if (!h->q.ev_valid) return fail(HTRIP_ERR_INVALID, "no query has run");
    HTRIP_GUARD_BEGIN
    ck(cudaEventSynchronize(h->q.ev[1]), "event sync");
    ck(cudaEventElapsedTime(ms, h->q.ev[0], h->q.ev[1]), "event time");
    return HTRIP_OK;
    HTRIP_GUARD_END
}

// ns[i] = duration of phase i; with max_n >= 2 * phases, ns[phases + i] =
// the part of it until the last CTA finished its work (the rest is the wait
// in the grid barrier).  Dataflow launches: both halves hold the time from
// the end of phase i-1's last unit to the end of phase i's last unit.
static htrip_status arena_phases(const QueryArena& A, cudaStream_t st, uint64_t* ns, int32_t max_n, int32_t* n) {
    if (!ns || !n || max_n < 0) return fail(HTRIP_ERR_INVALID, "bad arguments");
    if (!A.ev_valid) return fail(HTRIP_ERR_INVALID, "no query has run");
    HTRIP_GUARD_BEGIN
    unsigned long long t[2 * hb::kMaxQueryPhases + 1];
    ck(cudaEventSynchronize(A.ev[1]), "event sync");
    ck(cudaMemcpyAsync(t, A.dev.p + A.last_words + kTraceOffset, sizeof(t), cudaMemcpyDeviceToHost, st), "trace d2h");
    ck(cudaStreamSynchronize(st), "trace sync");
    const int P = A.last_phases;
    *n = std::min<int32_t>(max_n, P);
    for (int i = 0; i < *n; ++i) ns[i] = t[i + 1] > t[i] ? t[i + 1] - t[i] : 0;
    if (max_n >= 2 * P) {
        for (int i = 0; i < P; ++i) {
            const unsigned long long e = t[hb::kMaxQueryPhases + 1 + i];
            ns[P + i] = e > t[i] ? e - t[i] : 0;
        }
        *n = 2 * P;
    }
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_last_open_trace(htrip_index* h, uint64_t* ns, int32_t max_n, int32_t* n) {
    if (!h || (max_n > 0 && !ns)) return fail(HTRIP_ERR_INVALID, "bad arguments");
    if (!h->u.trace_valid) return fail(HTRIP_ERR_INVALID, "no device-driven opening has run on this index");
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    std::vector<unsigned long long> t(hb::kOpenTrace, 0);
    ck(cudaMemcpyAsync(t.data(), h->u.dev.p + h->u.trace_off, t.size() * sizeof(unsigned long long),
                       cudaMemcpyDeviceToHost, h->stream), "trace");
    ck(cudaStreamSynchronize(h->stream), "sync");
    int m = 0;  // phases stamped: stamps after t[0] that are set and not earlier than it
    while (m + 1 < (int)t.size() && t[m + 1] >= t[0] && t[m + 1] != 0) ++m;
    for (int i = 0; i < std::min(m, (int)max_n); ++i) ns[i] = t[i + 1] - t[i];
    if (n) *n = m;
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_set_query_work_counting(htrip_index* h, int32_t on) {
    if (!h) return fail(HTRIP_ERR_INVALID, "null handle");
    h->count_work = on != 0;
    return HTRIP_OK;
}

htrip_status htrip_last_query_executed(htrip_index* h, uint64_t* entries, uint64_t* rows, uint64_t* skipped) {
    if (!h) return fail(HTRIP_ERR_INVALID, "null handle");
    if (!h->count_work || !h->q.ev_valid) return fail(HTRIP_ERR_INVALID, "no counted query launch");
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    unsigned long long w[3] = {0, 0, 0};
    ck(cudaMemcpyAsync(w, h->q.dev.p + h->q.last_words + kWorkOffset, sizeof(w), cudaMemcpyDeviceToHost, h->stream),
       "work counters");
    ck(cudaStreamSynchronize(h->stream), "sync");
    if (entries) *entries = w[0];
    if (rows) *rows = w[1];
    if (skipped) *skipped = w[2];
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_last_query_phases(const htrip_index* h, uint64_t* ns, int32_t max_n, int32_t* n) {
    if (!h) return fail(HTRIP_ERR_INVALID, "null handle");
    return arena_phases(h->q, h->stream, ns, max_n, n);
}

htrip_status htrip_batch_last_phases(const htrip_batch* b, uint64_t* ns, int32_t max_n, int32_t* n) {
    if (!b) return fail(HTRIP_ERR_INVALID, "null batch");
    return arena_phases(b->q, b->stream, ns, max_n, n);
}

htrip_status htrip_autotune_query(htrip_index* h, const int32_t* vps, int32_t k, const uint8_t* observed,
                                  int32_t rows, int32_t cols, int32_t reps, int32_t* best_cfg, float* best_ms) {
    if (!h) return fail(HTRIP_ERR_INVALID, "null handle");
    if (const htrip_status rs = ready(h)) return rs;
    if (k <= 0 || !vps || !observed || reps <= 0) return fail(HTRIP_ERR_INVALID, "bad arguments");
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    const std::vector<uint8_t> pf = viewpoint_flags(h, vps, k, observed, rows, cols);
    QueryPlan P0;
    make_plan(h, vps, pf.data(), k, P0);
    const TuneKey key = tune_key(h, P0.n_sorted, h->H >= 1 ? P0.lv[h->H].max_group : P0.n_sorted);
    int best = -1;
    float best_t = 0.f;
    for (int cfg = 0; cfg < hb::kNumQueryConfigs; ++cfg) {
        QueryPlan P;
        make_plan(h, vps, pf.data(), k, P, cfg);
        const std::vector<QueryReq> R{{h, &P, nullptr}};
        float t = 0.f;
        for (int r = 0; r <= reps; ++r) {  // the first launch warms up and is not counted
            if (run_queries(h->q, h->device, h->stream, R, {nullptr}, true) != 0)
                return fail(HTRIP_ERR_CUDA, "query kernel: a bounded wait timed out");
            float ms = 0.f;
            ck(cudaEventElapsedTime(&ms, h->q.ev[0], h->q.ev[1]), "event time");
            if (r > 0) t = (r == 1) ? ms : std::min(t, ms);
        }
        if (best < 0 || t < best_t) {
            best = cfg;
            best_t = t;
        }
    }
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune[key] = best;
    }
    if (best_cfg) *best_cfg = best;
    if (best_ms) *best_ms = best_t;
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_autotune_export(char* buf, size_t cap, size_t* len) {
    std::string out;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        for (const auto& kv : g_tune)
            out += std::to_string(kv.first.H) + " " + std::to_string(kv.first.NP) + " " + std::to_string(kv.first.kb) +
                   " " + std::to_string(kv.first.gb) + " " + std::to_string(kv.second) + "\n";
    }
    if (len) *len = out.size();
    if (buf && cap > 0) {
        const size_t n = std::min(cap - 1, out.size());
        std::memcpy(buf, out.data(), n);
        buf[n] = 0;
        if (out.size() + 1 > cap) return fail(HTRIP_ERR_INVALID, "buffer too small");
    }
    return HTRIP_OK;
}

htrip_status htrip_autotune_import(const char* text) {
    if (!text) return fail(HTRIP_ERR_INVALID, "null text");
    std::map<TuneKey, int> add;
    const char* p = text;
    while (*p) {
        int v[5], used = 0;
        if (std::sscanf(p, "%d %d %d %d %d%n", &v[0], &v[1], &v[2], &v[3], &v[4], &used) != 5) {
            while (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t') ++p;
            if (!*p) break;
            return fail(HTRIP_ERR_INVALID, "malformed tuning line");
        }
        if (v[4] < 0 || v[4] >= hb::kNumQueryConfigs) return fail(HTRIP_ERR_INVALID, "tile configuration out of range");
        add[TuneKey{v[0], v[1], v[2], v[3]}] = v[4];
        p += used;
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (const auto& kv : add) g_tune[kv.first] = kv.second;
    return HTRIP_OK;
}

htrip_status htrip_autotune_clear(void) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune.clear();
    return HTRIP_OK;
}

htrip_status htrip_last_open_levels(const htrip_index* h, int64_t* out, int32_t max_levels, int32_t* n_levels) {
    if (!h) return fail(HTRIP_ERR_INVALID, "null handle");
    const int n = std::min<int>((int)h->open_levels.size(), std::max(0, max_levels));
    for (int l = 0; l < n; ++l)
        for (int j = 0; j < 4; ++j) out[4 * l + j] = h->open_levels[l][j];
    if (n_levels) *n_levels = (int32_t)h->open_levels.size();
    return HTRIP_OK;
}

htrip_status htrip_last_open_work(const htrip_index* h, uint64_t* alg_bytes, uint64_t* alg_ops) {
    if (!h) return fail(HTRIP_ERR_INVALID, "null handle");
    if (alg_bytes) *alg_bytes = h->open_bytes;
    if (alg_ops) *alg_ops = h->open_ops;
    return HTRIP_OK;
}

htrip_status htrip_last_query_io(const htrip_index* h, uint64_t* h2d_bytes, uint64_t* d2h_bytes) {
    if (!h) return fail(HTRIP_ERR_INVALID, "null handle");
    if (h2d_bytes) *h2d_bytes = h->q.last_h2d;
    if (d2h_bytes) *d2h_bytes = h->q.last_d2h;
    return HTRIP_OK;
}

htrip_status htrip_sync(htrip_index* h) {
    if (!h) return fail(HTRIP_ERR_INVALID, "null handle");
    HTRIP_GUARD_BEGIN
    ck(cudaStreamSynchronize(h->stream), "sync");
    return HTRIP_OK;
    HTRIP_GUARD_END
}

void* htrip_stream(htrip_index* h) { return h ? (void*)h->stream : nullptr; }

htrip_status htrip_shape(const htrip_index* h, int32_t* S, int32_t* H, int32_t* leaves_x) {
    if (!h) return fail(HTRIP_ERR_INVALID, "null handle");
    if (S) *S = h->S;
    if (H) *H = h->H;
    if (leaves_x) *leaves_x = h->leaves_x;
    return HTRIP_OK;
}

htrip_status htrip_last_batch_stats(const htrip_index* h, htrip_batch_stats* out) {
    if (!h || !out) return fail(HTRIP_ERR_INVALID, "null argument");
    *out = h->stats;
    return HTRIP_OK;
}

htrip_status htrip_offload(htrip_index* h) {
    if (!h) return fail(HTRIP_ERR_INVALID, "null handle");
    if (const htrip_status rs = ready(h)) return rs;
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    ck(cudaStreamSynchronize(h->stream), "sync");
    std::vector<std::vector<uint16_t>> parked(h->H + 2);
    for (int l = 0; l <= h->H; ++l) {
        parked[l].resize(h->L[l].mat.n);
        ck(cudaMemcpyAsync(parked[l].data(), h->L[l].mat.p, h->L[l].mat.n * sizeof(uint16_t), cudaMemcpyDeviceToHost,
                           h->stream), "offload");
    }
    parked[h->H + 1].resize((h->pass.n + 1) / 2);
    ck(cudaMemcpyAsync(parked[h->H + 1].data(), h->pass.p, h->pass.n, cudaMemcpyDeviceToHost, h->stream), "offload");
    ck(cudaStreamSynchronize(h->stream), "offload sync");
    const size_t pass_n = h->pass.n;
    h->release();  // every device buffer of the index (geometry is rebuilt on restore)
    h->parked = std::move(parked);
    h->parked_pass = pass_n;
    h->offloaded = true;
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_restore(htrip_index* h) {
    if (!h) return fail(HTRIP_ERR_INVALID, "null handle");
    if (!h->built) return fail(HTRIP_ERR_NOT_BUILT, "index not built");
    if (!h->offloaded) return HTRIP_OK;
    HTRIP_GUARD_BEGIN
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    try {
        make_levels(h);
        alloc_levels(h);
        for (int l = 0; l <= h->H; ++l)
            ck(cudaMemcpyAsync(h->L[l].mat.p, h->parked[l].data(), h->L[l].mat.n * sizeof(uint16_t),
                               cudaMemcpyHostToDevice, h->stream), "restore");
        h->pass.reserve(h->parked_pass);
        ck(cudaMemcpyAsync(h->pass.p, h->parked[h->H + 1].data(), h->parked_pass, cudaMemcpyHostToDevice, h->stream),
           "restore");
        ck(cudaStreamSynchronize(h->stream), "restore sync");
    } catch (const CudaError&) {
        h->release();  // still offloaded: the parked copy is intact
        throw;
    }
    h->parked.clear();
    h->parked.shrink_to_fit();
    h->offloaded = false;
    return HTRIP_OK;
    HTRIP_GUARD_END
}

htrip_status htrip_is_resident(const htrip_index* h, int32_t* resident) {
    if (!h || !resident) return fail(HTRIP_ERR_INVALID, "null argument");
    *resident = h->built && !h->offloaded;
    return HTRIP_OK;
}

htrip_status htrip_estimate_bytes(htrip_config cfg, int32_t rows, int32_t cols, uint64_t* device_bytes) {
    if (!device_bytes) return fail(HTRIP_ERR_INVALID, "null argument");
    const int b = cfg.tile_size_b, g = cfg.group;
    if (!(b >= 2 && b <= 32 && g >= 2 && g * g <= 256) || std::max(rows, cols) <= 0)
        return fail(HTRIP_ERR_INVALID, "invalid config or grid");
    htrip_index tmp;
    tmp.b = b;
    tmp.g = g;
    int S = b;
    while (S < std::max(rows, cols)) S *= g;
    int H = 0;
    for (int t = S / b; t > 1; t /= g) ++H;
    tmp.S = S;
    tmp.H = H;
    tmp.leaves_x = S / b;
    make_levels(&tmp);
    uint64_t bytes = (uint64_t)S * S;  // passability mirror
    for (const auto& Lv : tmp.L) {
        const uint64_t mats = (uint64_t)Lv.nnodes * Lv.NP;
        bytes += mats * Lv.NP * sizeof(uint16_t) + mats /* pivot flags */ + mats * sizeof(int) /* pivot lists */ +
                 (uint64_t)Lv.nnodes * (2 * sizeof(int) + 1) + (uint64_t)(Lv.nExt + Lv.NP + Lv.seams.size()) * sizeof(int);
    }
    *device_bytes = bytes;
    return HTRIP_OK;
    }

htrip_status htrip_memory_bytes(const htrip_index* h, uint64_t* reference_bytes, uint64_t* device_bytes) {
    if (!h) return fail(HTRIP_ERR_INVALID, "null handle");
    uint64_t ref = 0, dev = 0;
    if (h->built) {
        ref = h->ref_bytes;
        for (const auto& Lv : h->L)
            dev += (Lv.mat.n + Lv.klist.n * 2 + Lv.kcnt.n * 2) * sizeof(uint16_t) + Lv.kflag.n + Lv.dec.n +
                   (Lv.d_ext.n + Lv.d_seams.n) * sizeof(int);
        dev += h->pass.n + h->u.dev.n + h->u.snap.n * 2 + h->u.panel.n * 2 + h->u.pflags.n + h->q.dev.n +
               h->wts.n * sizeof(uint16_t);
    }
    if (reference_bytes) *reference_bytes = ref;
    if (device_bytes) *device_bytes = dev;
    return HTRIP_OK;
}

static htrip_status read_block(const htrip_index* h, int lvl, int node, const int* rows, int nr, const int* cols,
                               int nc, uint16_t* out) {
    const Level& Lv = h->L[lvl];
    DevBuf<int> idx;
    DevBuf<uint16_t> tmp;
    idx.reserve(nr + nc);
    tmp.reserve(std::max(1, nr * nc));
    cudaStream_t st = h->stream;
    ck(cudaMemcpyAsync(idx.p, rows, nr * sizeof(int), cudaMemcpyHostToDevice, st), "idx");
    ck(cudaMemcpyAsync(idx.p + nr, cols, nc * sizeof(int), cudaMemcpyHostToDevice, st), "idx");
    hb::launch_gather_block(Lv.mat.p + (size_t)node * Lv.NP * Lv.NP, Lv.NP, idx.p, nr, idx.p + nr, nc, tmp.p, st);
    ck(cudaGetLastError(), "gather");
    ck(cudaMemcpyAsync(out, tmp.p, (size_t)nr * nc * sizeof(uint16_t), cudaMemcpyDeviceToHost, st), "d2h");
    ck(cudaStreamSynchronize(st), "sync");
    idx.release();
    tmp.release();
    return HTRIP_OK;
}

static bool valid_node(const htrip_index* h, int lvl, int node) {
    return h && h->built && !h->offloaded && lvl >= 0 && lvl <= h->H && node >= 0 && node < h->L[lvl].nnodes;
}

htrip_status htrip_read_leaf_D(const htrip_index* h, int32_t leaf, uint16_t* out) {
    if (!valid_node(h, 0, leaf) || !out) return fail(HTRIP_ERR_INVALID, "bad leaf");
    HTRIP_GUARD_BEGIN
    std::vector<int> id(h->L[0].n);
    std::iota(id.begin(), id.end(), 0);
    return read_block(h, 0, leaf, id.data(), (int)id.size(), id.data(), (int)id.size(), out);
    HTRIP_GUARD_END
}

htrip_status htrip_read_leaf_S(const htrip_index* h, int32_t leaf, uint16_t* out) {
    if (!valid_node(h, 0, leaf) || !out) return fail(HTRIP_ERR_INVALID, "bad leaf");
    HTRIP_GUARD_BEGIN
    const auto& e = h->L[0].ext;
    return read_block(h, 0, leaf, e.data(), (int)e.size(), e.data(), (int)e.size(), out);
    HTRIP_GUARD_END
}

htrip_status htrip_read_node_DU(const htrip_index* h, int32_t lvl, int32_t node, uint16_t* out) {
    if (lvl < 1 || !valid_node(h, lvl, node) || !out) return fail(HTRIP_ERR_INVALID, "bad node");
    HTRIP_GUARD_BEGIN
    std::vector<int> id(h->L[lvl].n);
    std::iota(id.begin(), id.end(), 0);
    return read_block(h, lvl, node, id.data(), (int)id.size(), id.data(), (int)id.size(), out);
    HTRIP_GUARD_END
}

htrip_status htrip_read_node_SU(const htrip_index* h, int32_t lvl, int32_t node, uint16_t* out) {
    if (lvl < 1 || !valid_node(h, lvl, node) || !out) return fail(HTRIP_ERR_INVALID, "bad node");
    HTRIP_GUARD_BEGIN
    const auto& e = h->L[lvl].ext;
    return read_block(h, lvl, node, e.data(), (int)e.size(), e.data(), (int)e.size(), out);
    HTRIP_GUARD_END
}

htrip_status htrip_read_node_C2E(const htrip_index* h, int32_t lvl, int32_t node, int32_t quad, uint16_t* out) {
    if (lvl < 1 || !valid_node(h, lvl, node) || !out || quad < 0 || quad >= h->g * h->g)
        return fail(HTRIP_ERR_INVALID, "bad node");
    HTRIP_GUARD_BEGIN
    const Level& Lv = h->L[lvl];
    std::vector<int> rows(Lv.nP);
    std::iota(rows.begin(), rows.end(), quad * Lv.nP);
    return read_block(h, lvl, node, rows.data(), (int)rows.size(), Lv.ext.data(), (int)Lv.ext.size(), out);
    HTRIP_GUARD_END
}

htrip_status htrip_level_dims(const htrip_index* h, int32_t lvl, int32_t* n, int32_t* n_ext, int32_t* n_child_ports,
                              int32_t* n_nodes) {
    if (!h || !h->built || lvl < 0 || lvl > h->H) return fail(HTRIP_ERR_INVALID, "bad level");
    const Level& Lv = h->L[lvl];
    if (n) *n = Lv.n;
    if (n_ext) *n_ext = Lv.nExt;
    if (n_child_ports) *n_child_ports = Lv.nP;
    if (n_nodes) *n_nodes = Lv.nnodes;
    return HTRIP_OK;
}

}  // extern "C"
