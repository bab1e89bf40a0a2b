// queryAllPairs on the device (reference MinPlusOracle::queryAllPairs,
// src/minplus_oracle.cpp:934-1419) as ONE persistent cooperative kernel.
//
// Viewpoints are sorted by the base-g^2 Morton code of their leaf, so at
// every level the viewpoints of one node, and of one child of a node, form a
// contiguous run ("child group").  At level l each child group owns a run of
// "slots" that starts on an 8-slot (16-byte) boundary; the port vectors
// X_{l-1} (ports x slots) and the projections Yt_l (node columns x slots) are
// stored in level-l slot order.
//
// Work is cut into CTA items: a tile of RW rows x 64*CP columns of packed
// u16 accumulators.  The CTA's warps split the item's list of operand rows
// (split-K inside the CTA), each streaming its rows from L2/HBM through a
// cp.async ring in shared memory, then the partial tiles are min-reduced in
// shared memory and the epilogue is spread over the warps.  The rows of a
// warp are warp-uniform, the columns are spread over the lanes; per operand
// row the tile's RW values decide, uniformly for the warp, between skipping
// (all INF), the unclamped 2-op update (all <= 5535) and the clamped one.
// Two 256-thread CTAs per SM keep two items in flight.
//
//   level 0  X0[p][s] = leaf D[u][port p] for every viewpoint (+ finite-port
//            flags of its level-1 child group) and same-leaf pairs
//            (minplus_oracle.cpp:990-1048).
//   project Yt_l[c][s] = min_p X_{l-1}[p][s] (+) D_U[q*nP + p][c] over the ports
//            p finite for some viewpoint of the group (row compaction,
//            minplus_oracle.cpp:1185-1215).  The exterior columns are the lift
//            X_l = X_{l-1} (x) child_to_ext (:1113-1154); the epilogue writes
//            them straight into X_l (level-(l+1) slot order) with the next
//            level's flags.
//   meet     M[i][j] = min(M[i][j], min_p Yt_l[q_j*nP + p][i] (+) X_{l-1}[p][j])
//            for i < j in one node: the inter-child meets (:1157-1326) and the
//            intra-child shortcut (:1328-1411) are one formula.  Split-K items
//            combine with atomicMin on a 32-bit k x k matrix.
//
// Phases: [level 0] | [project 1] | [project 2 + meet 1] | ... |
// [project H + meet H-1] | [meet H] | [finalize]; every level has its own
// X and Yt buffers.  The default (dataflow) launch runs the units of all
// phases without a grid barrier: each unit waits for the units it reads on
// per-request completion counters, so a node's next level starts as soon as
// its own children are done instead of when the slowest CTA of the level is.
// The barrier launch (H + 2 grid barriers) stays selectable.
//
// Every sum is the exact clamped tropical product of minplus.cuh, so the
// matrix equals the reference's bit for bit.
#include "kernels.cuh"
#include "minplus.cuh"

#include <algorithm>

namespace hb {

namespace {

constexpr unsigned FULL = 0xffffffffu;

// Branch-free exact update: c' = min(c, min(b, INF - a) + a) per 16-bit lane
// for any a in [0, INF] (a == INF gives min(b, 0) + INF = INF: no change).
// aa = a in both halves.  min(b, INF - a) + a <= INF, so the packed add never
// carries across the halves.
template <int CP>
__device__ __forceinline__ void row_update(uint32_t (&acc)[CP], const uint32_t (&bv)[CP], uint32_t aa) {
    const uint32_t tt = INF2 - aa;
#pragma unroll
    for (int c = 0; c < CP; ++c) acc[c] = min2(add2(min2(bv[c], tt), aa), acc[c]);
}

constexpr int kThreads = kQueryThreads;
constexpr int kWarps = kThreads / 32;

// Operand staging: every warp keeps kPipeStages x kPipeRows operand rows in
// flight through cp.async into its own shared-memory ring, so an item's
// rows arrive at L2 / HBM throughput rather than one round trip per row.
constexpr int kPipeStages = 4;
constexpr int kPipeRows = 4;

// Words of one staged row: the lane-major B pairs (32 lanes x CP), then RW
// u16 of the A row.
template <int RW, int CP>
constexpr int pipe_slot_words() {
    return CP * 32 + RW / 2;
}
template <int RW, int CP>
constexpr int pipe_warp_words() {
    return kPipeStages * kPipeRows * pipe_slot_words<RW, CP>();
}

template <int BYTES>
__device__ __forceinline__ void cp_async(uint32_t saddr, const void* g) {
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(g) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(saddr), "l"(g), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Warp w of the CTA streams list entries t = w*U + 16*U*i + u (U =
// kPipeRows) of the compacted row list kl[0..n):
//   acc[r][c] = min over its rows p of A[p*lda + r] (+) B[p*ldb + lane pair c].
// A rows are RW consecutive u16 (16-byte aligned); B is already offset to the
// lane's CP pairs.  `pipe` is the warp's staging ring.  B0 is the warp's
// first column (16-byte aligned); each B row is copied as 16-byte chunks,
// chunks from column `bcols` on are taken from column 0 instead (their lanes'
// results are not used).  All operand copies bypass L1 (cp.async.cg): the
// X / Y rows may have been written by other CTAs of the same launch.
// Returns the number of rows the warp skipped (no finite value in the tile).
template <int RW, int CP>
__device__ __forceinline__ int warp_minplus_list(uint32_t (&acc)[RW][CP], const int* kl, int n, int warp,
                                                  const uint16_t* __restrict__ A, int lda,
                                                  const uint16_t* __restrict__ B0, int ldb, int bcols,
                                                  uint32_t* pipe) {
    constexpr int U = kPipeRows, NS = kPipeStages, SW = pipe_slot_words<RW, CP>();
    const int lane = threadIdx.x & 31;
    const int stride = kWarps * U;
    const int first = warp * U;
    const int n_it = first < n ? (n - first + stride - 1) / stride : 0;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(pipe);
    int skipped = 0;
    auto issue = [&](int it) {
        if (it < n_it) {
            const int st = it % NS;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int t = first + it * stride + u;
                if (t < n) {
                    const int row = kl[t];
                    const uint32_t slot = sbase + (uint32_t)((st * U + u) * SW) * 4u;
                    if (lane < 8 * CP) {
                        const int c8 = lane * 8 < bcols ? lane * 8 : 0;
                        cp_async<16>(slot + lane * 16, B0 + (size_t)row * ldb + c8);
                    }
                    if (lane < RW / 8) cp_async<16>(slot + CP * 128 + lane * 16, A + (size_t)row * lda + lane * 8);
                }
            }
        }
        cp_commit();
    };
#pragma unroll
    for (int st = 0; st < NS - 1; ++st) issue(st);
    for (int it = 0; it < n_it; ++it) {
        issue(it + NS - 1);
        cp_wait<NS - 1>();
        __syncwarp();
        const int st = it % NS;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (first + it * stride + u < n) {
                const uint32_t* slot = pipe + (st * U + u) * SW;
                uint32_t bv[CP];
#pragma unroll
                for (int c = 0; c < CP; ++c) bv[c] = slot[lane * CP + c];
                const uint32_t* a = slot + CP * 32;
                uint32_t aw[RW / 2];
#pragma unroll
                for (int r2 = 0; r2 < RW / 2; ++r2) aw[r2] = a[r2];
                // The row's RW values are warp-uniform: all INF -> nothing to
                // do; all <= INF_HEADROOM -> the unclamped 2-op form is exact
                // (a + b <= 65535 never wraps, and a sum >= INF loses to c);
                // otherwise the clamped form (exact for any a <= INF).
                uint32_t mx = aw[0], mn = aw[0];
#pragma unroll
                for (int r2 = 1; r2 < RW / 2; ++r2) {
                    mx = max2(mx, aw[r2]);
                    mn = min2(mn, aw[r2]);
                }
                mn = min2(mn, mn >> 16) & 0xffffu;
                mx = max2(mx, mx >> 16) & 0xffffu;
                if (mn >= INF) {
                    ++skipped;
                    continue;
                }
                if (mx <= INF_HEADROOM) {
#pragma unroll
                    for (int r2 = 0; r2 < RW / 2; ++r2) {
                        const uint32_t lo = __byte_perm(aw[r2], 0, 0x1010), hi = __byte_perm(aw[r2], 0, 0x3232);
#pragma unroll
                        for (int c = 0; c < CP; ++c) {
                            acc[2 * r2][c] = acc_fast(acc[2 * r2][c], bv[c], lo);
                            acc[2 * r2 + 1][c] = acc_fast(acc[2 * r2 + 1][c], bv[c], hi);
                        }
                    }
                } else {
#pragma unroll
                    for (int r2 = 0; r2 < RW / 2; ++r2) {
                        row_update<CP>(acc[2 * r2], bv, __byte_perm(aw[r2], 0, 0x1010));
                        row_update<CP>(acc[2 * r2 + 1], bv, __byte_perm(aw[r2], 0, 0x3232));
                    }
                }
            }
        }
        __syncwarp();
    }
    cp_wait<0>();
    return skipped;
}

// Executed-work counters of a request (QueryParams::work): each warp adds
// the rows of its share of the unit's operand list it streamed and skipped.
template <int RW, int CP>
__device__ __forceinline__ void count_work(unsigned long long* work, int n, int warp, int skipped) {
    if (!work || (threadIdx.x & 31) != 0) return;
    const int stride = kWarps * kPipeRows, first = warp * kPipeRows;
    int mine = 0;  // rows of the list this warp streamed (see warp_minplus_list)
    for (int t = first; t < n; t += stride) mine += min(kPipeRows, n - t);
    if (mine == 0) return;
    atomicAdd(work, (unsigned long long)(mine - skipped) * RW * 64 * CP);
    atomicAdd(work + 1, (unsigned long long)(mine - skipped));
    atomicAdd(work + 2, (unsigned long long)skipped);
}

// Compacts the set flags of rows [kb, ke) into kl (ascending); returns the
// count (block-wide scan; every thread gets the total).
__device__ __forceinline__ int compact_flags(const uint8_t* __restrict__ flags, int kb, int ke, int* kl, int* wsum) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n = ke - kb;
    const int per = (n + kThreads - 1) / kThreads;
    const int p0 = kb + tid * per, p1 = min(ke, p0 + per);
    int cntl = 0;
    for (int p = p0; p < p1; ++p) cntl += __ldcg(flags + p) != 0;
    int incl = cntl;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    int base = 0, total = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        if (w < warp) base += wsum[w];
        total += wsum[w];
    }
    int pos = base + incl - cntl;
    for (int p = p0; p < p1; ++p)
        if (__ldcg(flags + p)) kl[pos++] = p;
    __syncthreads();
    return total;
}

// Min-reduction of the warps' accumulators through shared memory; the
// reduced tile ends up in every warp's acc (warp 0 uses it).
template <int RW, int CP>
__device__ __forceinline__ void cta_reduce(uint32_t (&acc)[RW][CP], uint32_t* red) {
    constexpr int E = RW * CP * 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    __syncthreads();  // the staging rings alias `red`: every warp is done reading them
#pragma unroll
    for (int r = 0; r < RW; ++r)
#pragma unroll
        for (int c = 0; c < CP; ++c) red[warp * E + (r * CP + c) * 32 + lane] = acc[r][c];
    __syncthreads();
    for (int e = tid; e < E; e += kThreads) {
        uint32_t m = red[e];
#pragma unroll
        for (int w = 1; w < kWarps; ++w) m = min2(m, red[w * E + e]);
        red[e] = m;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RW; ++r)
#pragma unroll
        for (int c = 0; c < CP; ++c) acc[r][c] = red[(r * CP + c) * 32 + lane];
}

// Grid barrier over `expected` CTAs with a bounded spin (`limit` polls); a
// timeout sets *status and the kernel finishes without waiting further (the
// host reports the error).
__device__ __forceinline__ bool grid_barrier_n(unsigned* bar, int* status, unsigned expected, unsigned limit) {
    __syncthreads();
    bool ok = true;
    if (threadIdx.x == 0) {
        volatile unsigned* vgen = bar + 1;
        const unsigned gen = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(bar, 1u);
        if (arrived == expected - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            unsigned it = 0;
            while (*vgen == gen) {
                if (++it > limit) {
                    atomicExch(status, 1);
                    ok = false;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok && *(volatile int*)status == 0;
}

__device__ __forceinline__ bool grid_barrier(unsigned* bar, int* status) {
    return grid_barrier_n(bar, status, gridDim.x, 1u << 24);
}

// Self-test of the bounded wait: a barrier that expects one CTA more than the
// launch has can never complete, so every CTA gives up after `limit` polls,
// records the timeout in *status and returns.
__global__ void barrier_timeout_probe_kernel(unsigned* bar, int* status, unsigned limit, int* returned) {
    grid_barrier_n(bar, status, gridDim.x + 1, limit);
    if (threadIdx.x == 0) atomicAdd(returned, 1);
}

__device__ __forceinline__ unsigned long long global_timer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---------------------------------------------------------------------------
// Work item bodies.
// ---------------------------------------------------------------------------
// Shared memory of the persistent kernel: compacted row list (nP <= 4096
// ports), scan partials and the split-K reduction buffer.
constexpr int kMaxList = 4096 + 64;
// The staging rings (during an item's k-loop) and the split-K reduction
// buffer (after it) share one region.
template <int RW, int CP>
constexpr size_t query_smem_bytes() {
    return (size_t)kMaxList * sizeof(int) +
           std::max((size_t)kWarps * RW * CP * 32, (size_t)kWarps * pipe_warp_words<RW, CP>()) * sizeof(uint32_t);
}

// Per-item metadata staged in shared memory at the start of an item (its
// global loads overlap the k-loop): the exterior index / viewpoint of each
// tile column and the lift slot / viewpoint of each tile row.
struct ItemMeta {
    int col[256];
    int row[2][16];
};

// Split item: every part stores its reduced tile (warp 0); the part that
// completes the item's ticket folds the others into its own and returns
// true (it runs the epilogue), the others return false.
template <int RW, int CP>
__device__ bool combine_parts(const QueryLevel& L, int item, int part, uint32_t (&acc)[RW][CP]) {
    constexpr int E = RW * CP * 32;
    __shared__ int last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp == 0) {
        uint32_t* mine = L.part + ((size_t)item * L.split + part) * E;
#pragma unroll
        for (int r = 0; r < RW; ++r)
#pragma unroll
            for (int c = 0; c < CP; ++c) mine[(r * CP + c) * 32 + lane] = acc[r][c];
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned old = atomicAdd(L.ticket + item, 1u);
        last = old == (unsigned)(L.split - 1);
        __threadfence();
    }
    __syncthreads();
    if (!last) return false;
    for (int p = 0; p < L.split; ++p) {
        if (p == part) continue;
        const uint32_t* o = L.part + ((size_t)item * L.split + p) * E;
#pragma unroll
        for (int r = 0; r < RW; ++r)
#pragma unroll
            for (int c = 0; c < CP; ++c) acc[r][c] = min2(acc[r][c], __ldcg(o + (r * CP + c) * 32 + lane));
    }
    return true;
}

// project item {group, m0, n0}: tile of RW slots x 64*CP node columns; the
// CTA's warps split the group's finite ports (part `part` of L.split of
// them).  After the reduction the epilogue (Y stores and lift scatters) is
// spread over the warps.  Returns whether the item is complete.
// Incremental refresh: viewpoint j's level-l results changed (dirty[j] = 1 +
// the lowest level whose node changed, 0 for none).
__device__ __forceinline__ bool dirty_at(const uint8_t* dirty, int j, int l) {
    const int d = dirty[j];
    return d != 0 && d - 1 <= l;
}

template <int RW, int CP>
__device__ bool do_project(const QueryParams& P, const QueryLevel& L, const QueryLevel* Ln, int item, int part,
                           int l, int* kl, int* wsum, uint32_t* red, ItemMeta& im) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int* it = L.items + 3 * item;
    const int gi = it[0], m0 = it[1], n0 = it[2];
    const int* G = L.groups + 5 * gi;
    const int node = G[0], q = G[1], slot0 = G[2];
    if (P.dirty) {  // incremental refresh: rows of clean viewpoints keep their values
        int any = 0;
        for (int r = 0; r < min(RW, G[3] - m0); ++r) any |= dirty_at(P.dirty, G[4] + m0 + r, l);
        if (!any) return L.split <= 1 || part == 0;  // a skipped item counts once
    }
    const int nA = compact_flags(L.flags + (size_t)gi * L.nP, 0, L.nP, kl, wsum);
    const int kb = (int)((long)nA * part / L.split), ke = (int)((long)nA * (part + 1) / L.split);
    const uint16_t* D = L.D + (size_t)node * L.NP * L.NP + (size_t)q * L.nP * L.NP;
    const int col = n0 + lane * 2 * CP;
    const bool live_col = col < L.NP;
    const uint16_t* Xp = P.X[l - 1] + slot0 + m0;
    uint32_t acc[RW][CP];
#pragma unroll
    for (int r = 0; r < RW; ++r)
#pragma unroll
        for (int c = 0; c < CP; ++c) acc[r][c] = INF2;
    const int skipped = warp_minplus_list<RW, CP>(acc, kl + kb, ke - kb, warp, Xp, P.ldv, D + n0, L.NP, L.NP - n0,
                                                  red + warp * pipe_warp_words<RW, CP>());
    count_work<RW, CP>(P.work, ke - kb, warp, skipped);
    cta_reduce<RW, CP>(acc, red);
    if (L.split > 1 && !combine_parts<RW, CP>(L, item, part, acc)) {
        __syncthreads();  // kl / red / im are reused by the next item
        return false;
    }
    uint16_t* Y = P.Y[l];
#pragma unroll
    for (int cc = 0; cc < 2 * CP; ++cc) {
        const bool do_y = L.store_y && (cc % kWarps) == warp;
        const bool do_lift = Ln && ((2 * CP + cc) % kWarps) == warp;
        if (!live_col || (!do_y && !do_lift)) continue;
        uint16_t v[RW];
#pragma unroll
        for (int r = 0; r < RW; ++r)
            v[r] = (uint16_t)((cc & 1) ? (acc[r][cc >> 1] >> 16) : (acc[r][cc >> 1] & 0xffffu));
        if (do_y) {
            uint16_t* y = Y + (size_t)(col + cc) * P.ldv + slot0 + m0;
#pragma unroll
            for (int r8 = 0; r8 < RW / 8; ++r8) {
                uint4 o;
                o.x = v[8 * r8] | ((uint32_t)v[8 * r8 + 1] << 16);
                o.y = v[8 * r8 + 2] | ((uint32_t)v[8 * r8 + 3] << 16);
                o.z = v[8 * r8 + 4] | ((uint32_t)v[8 * r8 + 5] << 16);
                o.w = v[8 * r8 + 6] | ((uint32_t)v[8 * r8 + 7] << 16);
                reinterpret_cast<uint4*>(y)[r8] = o;
            }
        }
        if (do_lift) {  // exterior column e of this node -> X_l[e][level-(l+1) slot]
            const int e = im.col[lane * 2 * CP + cc];
            if (e >= 0) {
                uint16_t* Xn = P.X[l] + (size_t)e * P.ldv;
#pragma unroll
                for (int r = 0; r < RW; ++r) {
                    const int slot = im.row[0][r];
                    if (slot >= 0) {
                        Xn[slot] = v[r];
                        if (v[r] < INF) Ln->flags[(size_t)im.row[1][r] * Ln->nP + e] = 1;
                    }
                }
            }
        }
    }
    __syncthreads();  // kl / red / im are reused by the next item
    return true;
}

// meet item {i0, j0, nj, g2, coloff, kb, ke}: rows = RW viewpoints j of
// child group g2 (slots j0..), lanes = 64*CP viewpoint slots i (from i0).
// After the reduction warp w combines rows r = w (mod warps) into M.
template <int RW, int CP>
__device__ void do_meet(const QueryParams& P, const QueryLevel& L, int item, int l, int* kl, int* wsum,
                        uint32_t* red, ItemMeta& im) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int* it = L.meet + 7 * item;
    const int i0 = it[0], j0 = it[1], g2 = it[3], coloff = it[4], kb = it[5], ke = it[6];
    if (P.dirty) {  // incremental refresh: a pair of viewpoints clean at this level keeps its value
        int any = 0;
        for (int e = threadIdx.x; e < 64 * CP + RW; e += kThreads) {
            const int v = e < 64 * CP ? im.col[e] : im.row[0][e - 64 * CP];
            if (v >= 0) any |= dirty_at(P.dirty, v, l);
        }
        if (!__syncthreads_or(any)) return;
    }
    const int nA = compact_flags(L.flags + (size_t)g2 * L.nP, kb, ke, kl, wsum);
    const uint16_t* Xp = P.X[l - 1] + j0;
    const uint16_t* Y = P.Y[l] + (size_t)coloff * P.ldv + i0;
    uint32_t acc[RW][CP];
#pragma unroll
    for (int r = 0; r < RW; ++r)
#pragma unroll
        for (int c = 0; c < CP; ++c) acc[r][c] = INF2;
    const int skipped = warp_minplus_list<RW, CP>(acc, kl, nA, warp, Xp, P.ldv, Y, P.ldv, P.ldv - i0,
                                                  red + warp * pipe_warp_words<RW, CP>());
    count_work<RW, CP>(P.work, nA, warp, skipped);
    cta_reduce<RW, CP>(acc, red);
#pragma unroll
    for (int r = 0; r < RW; ++r) {
        if ((r % kWarps) != warp) continue;
        const int vj = im.row[0][r];
        if (vj < 0) continue;
#pragma unroll
        for (int cc = 0; cc < 2 * CP; ++cc) {
            const int vi = im.col[lane * 2 * CP + cc];
            const uint32_t v = (cc & 1) ? (acc[r][cc >> 1] >> 16) : (acc[r][cc >> 1] & 0xffffu);
            if (vi >= 0 && vi < vj && v < INF) atomicMin(&P.M[(size_t)vi * P.ldm + vj], v);
        }
    }
    __syncthreads();
}

// Metadata of unit u of phase t staged in shared memory before the unit
// waits for its inputs (none of it is produced by the launch): per tile
// column the exterior index (project, lifting levels) or viewpoint (meet),
// per tile row the lift slot and group (project) or viewpoint (meet).  The
// caller's next CTA barrier publishes it.
template <int RW, int CP>
__device__ void unit_prologue(const QueryParams& P, int t, int u, ItemMeta& im) {
    if (t < 1 || t > P.H + 1) return;
    const int tid = threadIdx.x;
    const int S = t <= P.H ? P.lv[t].split : 1;
    const int np = t <= P.H ? P.lv[t].n_items * S : 0;
    if (u < np) {
        if (t == P.H) return;  // root items lift nothing
        const QueryLevel& L = P.lv[t];
        const int* it = L.items + 3 * (u / S);
        const int gi = it[0], m0 = it[1], n0 = it[2];
        const int* G = L.groups + 5 * gi;
        const int slot0 = G[2], cnt = G[3];
        for (int e = tid; e < 64 * CP + RW; e += kThreads) {
            if (e < 64 * CP) {
                im.col[e] = n0 + e < L.NP ? L.ext_inv[n0 + e] : -1;
            } else {
                const int r = e - 64 * CP;
                const bool ok = m0 + r < cnt;
                im.row[0][r] = ok ? L.lift[2 * (slot0 + m0 + r)] : -1;
                im.row[1][r] = ok ? L.lift[2 * (slot0 + m0 + r) + 1] : -1;
            }
        }
    } else {
        const QueryLevel& L = P.lv[t - 1];
        const int* it = L.meet + 7 * (u - np);
        const int i0 = it[0], j0 = it[1], nj = it[2];
        for (int e = tid; e < 64 * CP + RW; e += kThreads) {
            if (e < 64 * CP) im.col[e] = L.s2v[i0 + e];
            else im.row[0][e - 64 * CP] = e - 64 * CP < nj ? L.s2v[j0 + e - 64 * CP] : -1;
        }
    }
}

// One CTA work unit of request P in phase t (see QueryLaunch); its
// metadata is staged (unit_prologue).  Returns
// false for a part of a split project item that did not complete it.
template <int RW, int CP>
__device__ bool run_unit(const QueryParams& P, int t, int u, int* kl, int* wsum, uint32_t* red, ItemMeta& im) {
    const int tid = threadIdx.x;
    if (t == 0) {
        // level 0: X0 in level-1 slot order (+ level-1 flags), same-leaf pairs
        const int S1 = P.n_l0_slots;
        const int total = S1 * P.nExt0;
        const int n_fill = (total + kQueryL0Chunk - 1) / kQueryL0Chunk;
        if (u < n_fill) {
            const int e1 = min(total, (u + 1) * kQueryL0Chunk);
            for (int e = u * kQueryL0Chunk + tid; e < e1; e += kThreads) {
                const int p = e / S1, s = e - p * S1;
                const int j = P.l0[2 * s];
                if (j < 0 || (P.dirty && !dirty_at(P.dirty, j, 0))) continue;
                const int* v = P.vp0 + 4 * j;
                const uint16_t d = P.leaves.base[((size_t)v[0] * P.leaves.NP + v[1]) * P.leaves.NP + P.ext0[p]];
                P.X[0][(size_t)p * P.ldv + s] = d;
                if (d < INF && P.H >= 1) P.lv[1].flags[(size_t)P.l0[2 * s + 1] * P.nExt0 + p] = 1;
            }
        } else {
            const int j = (u - n_fill) * kThreads + tid;
            // same-leaf viewpoints share their chain, hence their dirty flag
            if (j < P.ns && (!P.dirty || dirty_at(P.dirty, j, 0))) {
                const int* v = P.vp0 + 4 * j;
                const uint16_t* row = P.leaves.base + ((size_t)v[0] * P.leaves.NP + v[1]) * P.leaves.NP;
                // atomicMin: the level-1 meets (intra-child shortcuts) may
                // already have lowered the entry in a dataflow launch
                for (int jj = j + 1; jj < v[3]; ++jj) atomicMin(&P.M[(size_t)j * P.ldm + jj], (uint32_t)row[P.vp0[4 * jj + 1]]);
            }
        }
        return true;
    }
    if (t <= P.H + 1) {
        const int S = t <= P.H ? P.lv[t].split : 1;
        const int np = t <= P.H ? P.lv[t].n_items * S : 0;
        if (u < np)
            return do_project<RW, CP>(P, P.lv[t], t < P.H ? &P.lv[t + 1] : nullptr, u / S, u % S, t, kl, wsum, red,
                                      im);
        do_meet<RW, CP>(P, P.lv[t - 1], u - np, t - 1, kl, wsum, red, im);
        return true;
    }
    // t == H + 2: out[a][c] for one chunk of the k x k output
    const int kk = P.k * P.k;
    const int e1 = min(kk, (u + 1) * kQueryFinChunk);
    for (int e = u * kQueryFinChunk + tid; e < e1; e += kThreads) {
        const int a = e / P.k, c = e - a * P.k;
        const int ia = P.inv[a], ic = P.inv[c];
        uint32_t v = INF;
        if (ia >= 0 && ic >= 0) {
            if (ia == ic) v = 0;
            else v = min(__ldcg(ia < ic ? P.M + (size_t)ia * P.ldm + ic : P.M + (size_t)ic * P.ldm + ia), (uint32_t)INF);
        }
        P.out[e] = (uint16_t)v;
    }
    return true;
}

// ---------------------------------------------------------------------------
// Dataflow order.  Instead of a grid barrier after every phase, each unit
// waits for the units it reads and counts itself done on the request's
// completion counters (QueryParams::ctr):
//   project, level 1          all level-0 gather units (ctr[0])
//   project, level l >= 2     the level-(l-1) project items of its group's
//     (group g)               node: ctr[4 + l*k + g] reaches cnt_g x column
//                             tiles of level l-1 (every row of such an item
//                             lifts into group g; each item adds its rows)
//   meet, level l < H         the level-l project items of its node, i.e.
//                             the counter of the level-(l+1) group it lifts to
//   meet, level H             every root project item (ctr[2])
//   output                    every project, meet and pair unit (ctr[1])
// A project item cut into parts (QueryLevel::split) counts toward its
// consumers once, when the part that completes it has run the epilogue.
// A dependency is always a unit of an earlier phase, and the units of all
// phases are handed out in ascending order (one ticket counter), so the
// lowest unfinished unit has been handed out and has its inputs: every
// wait ends (all CTAs are resident: cooperative launch).  Data
// produced inside the launch is read through L2 only (cp.async.cg,
// ld.global.cg): the L1 of an SM may hold a line of it from before it was
// written.
// ---------------------------------------------------------------------------
constexpr unsigned kWaitPolls = 1u << 24;

// The thread that looks up and polls a unit's dependency: lane 0 of warp 1,
// so that it runs beside thread 0's fence and counts for the previous unit.
constexpr int kWaiter = 32;

// Bounded wait of the whole CTA until *c >= target: thread kWaiter polls,
// the CTA follows.  False after a timeout (recorded in *status) or when
// another CTA has recorded one.
__device__ __forceinline__ bool wait_count(const unsigned* c, unsigned target, int* status,
                                           unsigned limit = kWaitPolls) {
    int ok = 1;
    if (threadIdx.x == kWaiter) {
        const volatile unsigned* vc = c;
        const volatile int* vs = status;
        unsigned it = 0;
        while (*vc < target) {
            if (*vs != 0) {
                ok = 0;
                break;
            }
            if (++it > limit) {
                atomicExch(status, 1);
                ok = 0;
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
    }
    return __syncthreads_and(ok) != 0;
}

// Self-test of the bounded counter wait: every CTA waits for a count that
// nothing adds, gives up after `limit` polls (or once another CTA recorded
// the timeout) and returns.
__global__ void wait_timeout_probe_kernel(const unsigned* ctr, int* status, unsigned limit, int* returned) {
    wait_count(ctr, 1u, status, limit);
    if (threadIdx.x == 0) atomicAdd(returned, 1);
}

__device__ __forceinline__ unsigned col_tiles(int NP, int NC) { return (unsigned)((NP + NC - 1) / NC); }

// Waits for the inputs of unit u of phase t of request P (see above).
template <int RW, int CP>
__device__ __forceinline__ bool dep_wait(const QueryParams& P, int t, int u, int* status) {
    constexpr int NC = 64 * CP;
    if (t == 0) {  // level-0 units read nothing of the launch; the barrier
        __syncthreads();  // still orders this unit's reads of next_w before its update
        return true;
    }
    const unsigned* c = nullptr;
    unsigned target = 0;
    if (threadIdx.x == kWaiter) {
        const int H = P.H;
        if (t == H + 2) {
            target = (unsigned)((P.ns + kThreads - 1) / kThreads);
            for (int l = 1; l <= H; ++l) target += (unsigned)(P.lv[l].n_items * P.lv[l].split + P.lv[l].n_meet);
            c = P.ctr + 1;
        } else {
            const int np = t <= H ? P.lv[t].n_items * P.lv[t].split : 0;
            if (u < np) {  // project item (part) of level t
                if (t == 1) {
                    const long total = (long)P.n_l0_slots * P.nExt0;
                    target = (unsigned)((total + kQueryL0Chunk - 1) / kQueryL0Chunk);
                    c = P.ctr;
                } else {
                    const int gi = P.lv[t].items[3 * (u / P.lv[t].split)];
                    target = (unsigned)P.lv[t].groups[5 * gi + 3] * col_tiles(P.lv[t - 1].NP, NC);
                    c = P.ctr + 4 + (size_t)t * P.k + gi;
                }
            } else {  // meet item of level t - 1
                const int l = t - 1;
                if (l == H) {
                    target = (unsigned)P.lv[H].n_items;
                    c = P.ctr + 2;
                } else {
                    const int j0 = P.lv[l].meet[7 * (u - np) + 1];
                    const int pg = P.lv[l].lift[2 * j0 + 1];
                    target = (unsigned)P.lv[l + 1].groups[5 * pg + 3] * col_tiles(P.lv[l].NP, NC);
                    c = P.ctr + 4 + (size_t)(l + 1) * P.k + pg;
                }
            }
        }
    }
    // thread kWaiter alone waits (the others pass a null counter and target 0)
    return wait_count(c ? c : P.ctr, target, status);
}

// Counts unit u of phase t of request P as done, after every thread of the
// CTA has issued its stores (the fence orders them before the counts); a
// project item counts toward its consumers once complete (all its parts).
template <int RW, int CP>
__device__ __forceinline__ void dep_signal(const QueryParams& P, int t, int u, bool complete) {
    __syncthreads();
    if (threadIdx.x != 0) return;
    const int H = P.H;
    if (t == H + 2) return;
    __threadfence();
    if (t == 0) {
        const long total = (long)P.n_l0_slots * P.nExt0;
        const int n_fill = (int)((total + kQueryL0Chunk - 1) / kQueryL0Chunk);
        atomicAdd(P.ctr + (u < n_fill ? 0 : 1), 1u);
        return;
    }
    const int S = t <= H ? P.lv[t].split : 1;
    const int np = t <= H ? P.lv[t].n_items * S : 0;
    if (u < np && complete) {
        if (t == H) {
            atomicAdd(P.ctr + 2, 1u);
        } else {
            const int* it = P.lv[t].items + 3 * (u / S);
            const int* G = P.lv[t].groups + 5 * it[0];
            const int rows = min(RW, G[3] - it[1]);
            const int pg = P.lv[t].lift[2 * G[2] + 1];
            atomicAdd(P.ctr + 4 + (size_t)(t + 1) * P.k + pg, (unsigned)rows);
        }
    }
    atomicAdd(P.ctr + 1, 1u);
}

// The persistent kernel.  Barrier mode: phases separated by grid barriers;
// in each phase the CTAs stride over the units of every request of the
// launch.  Dataflow mode: one stride over the units of all phases.
template <int RW, int CP>
__global__ void __launch_bounds__(kThreads, 512 / kThreads) q_persistent_kernel(const QueryLaunch B) {
    extern __shared__ __align__(16) int qsm[];
    int* kl = qsm;
    uint32_t* red = reinterpret_cast<uint32_t*>(qsm + kMaxList);
    __shared__ int wsum[kWarps];
    __shared__ ItemMeta im;
    const bool stamp = B.trace && blockIdx.x == 0 && threadIdx.x == 0;
    if (stamp) B.trace[0] = global_timer();
    if (B.dataflow) {
        // Units are handed out in ascending order by a ticket (the barrier's
        // count word, unused here); a CTA takes its next ticket when it starts
        // a unit, so the fetch overlaps the work.
        __shared__ int next_w;
        int total = 0;
        for (int t = 0; t < B.n_phases; ++t) total += B.unit_pre[(size_t)t * (B.n_req + 1) + B.n_req];
        if (threadIdx.x == 0) next_w = (int)atomicAdd(B.bar, 1u);
        __syncthreads();
        for (;;) {
            const int w = next_w;
            if (w >= total) break;
            int t = 0, wl = w;
            for (;;) {
                const int nt = B.unit_pre[(size_t)t * (B.n_req + 1) + B.n_req];
                if (wl < nt) break;
                wl -= nt;
                ++t;
            }
            const int* pre = B.unit_pre + (size_t)t * (B.n_req + 1);
            int lo = 0, hi = B.n_req;  // pre[lo] <= wl < pre[hi]
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (pre[mid] <= wl) lo = mid;
                else hi = mid;
            }
            const QueryParams& P = B.req[lo];
            const int u = wl - pre[lo];
            unit_prologue<RW, CP>(P, t, u, im);  // overlaps the wait; the wait's barrier publishes it
            if (!dep_wait<RW, CP>(P, t, u, B.status)) return;
            // every thread has read next_w (the wait is a CTA barrier)
            const int nxt = threadIdx.x == 0 ? (int)atomicAdd(B.bar, 1u) : 0;
            const bool complete = run_unit<RW, CP>(P, t, u, kl, wsum, red, im);
            if (threadIdx.x == 0) next_w = nxt;
            dep_signal<RW, CP>(P, t, u, complete);  // begins with a CTA barrier: next_w is visible after it
            if (B.trace && threadIdx.x == 0) {
                const unsigned long long now = global_timer();
                atomicMax(B.trace + t + 1, now);
                atomicMax(B.trace + kMaxQueryPhases + 1 + t, now);
            }
        }
        return;
    }
    for (int t = 0; t < B.n_phases; ++t) {
        const int* pre = B.unit_pre + (size_t)t * (B.n_req + 1);
        const int total = pre[B.n_req];
        for (int w = blockIdx.x; w < total; w += gridDim.x) {
            int lo = 0, hi = B.n_req;  // pre[lo] <= w < pre[hi]
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (pre[mid] <= w) lo = mid;
                else hi = mid;
            }
            unit_prologue<RW, CP>(B.req[lo], t, w - pre[lo], im);
            __syncthreads();
            run_unit<RW, CP>(B.req[lo], t, w - pre[lo], kl, wsum, red, im);
        }
        if (B.trace && threadIdx.x == 0)  // the phase's last CTA to finish its units
            atomicMax(B.trace + kMaxQueryPhases + 1 + t, global_timer());
        if (t + 1 < B.n_phases && !grid_barrier(B.bar, B.status)) return;
        if (stamp) B.trace[t + 1] = global_timer();
    }
}

}  // namespace

// Tile shapes (rows RW x columns 64*CP per warp item) of the configurations
// the persistent kernel implements; the autotuner picks one per level.
QueryTile query_config_tile(int cfg) {
    static const QueryTile t[kNumQueryConfigs] = {{8, 64}, {8, 128}, {16, 128}, {8, 256}};
    return t[cfg];
}

int query_default_config(int NP, int max_group) {
    if (max_group >= 12) return 2;
    return NP >= 256 ? 1 : 0;
}

namespace {
typedef void (*QueryKernel)(const QueryLaunch);
const QueryKernel kQueryKernels[kNumQueryConfigs] = {q_persistent_kernel<8, 1>, q_persistent_kernel<8, 2>,
                                                     q_persistent_kernel<16, 2>, q_persistent_kernel<8, 4>};
const size_t kQuerySmem[kNumQueryConfigs] = {query_smem_bytes<8, 1>(), query_smem_bytes<8, 2>(),
                                             query_smem_bytes<16, 2>(), query_smem_bytes<8, 4>()};

void configure_query_kernels() {
    static bool done = false;
    if (done) return;
    for (int c = 0; c < kNumQueryConfigs; ++c)
        cudaFuncSetAttribute(kQueryKernels[c], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kQuerySmem[c]);
    done = true;
}
}  // namespace

int query_max_ports() { return kMaxList - 64; }

// Runs one 4-CTA probe launch whose waits can never be satisfied (kind 0:
// the grid barrier, expecting a fifth CTA; kind 1: a completion counter that
// nothing adds to) with a short poll limit.
static cudaError_t timeout_selftest(int kind, int* status, int* returned, float* ms) {
    // words: {status, barrier count / counter, barrier generation, CTAs returned}
    unsigned* w = nullptr;
    cudaError_t e = cudaMalloc(&w, 4 * sizeof(unsigned));
    if (e != cudaSuccess) return e;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaMemset(w, 0, 4 * sizeof(unsigned));
    cudaEventRecord(e0);
    if (kind == 0)
        barrier_timeout_probe_kernel<<<4, 64>>>(w + 1, reinterpret_cast<int*>(w), 1u << 14,
                                                reinterpret_cast<int*>(w + 3));
    else
        wait_timeout_probe_kernel<<<4, 64>>>(w + 1, reinterpret_cast<int*>(w), 1u << 14, reinterpret_cast<int*>(w + 3));
    cudaEventRecord(e1);
    e = cudaEventSynchronize(e1);
    unsigned h[4] = {0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpy(h, w, sizeof(h), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) cudaEventElapsedTime(ms, e0, e1);
    *status = (int)h[0];
    *returned = (int)h[3];
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(w);
    return e;
}

cudaError_t barrier_timeout_selftest(int* status, int* returned, float* ms) {
    return timeout_selftest(0, status, returned, ms);
}

cudaError_t wait_timeout_selftest(int* status, int* returned, float* ms) {
    return timeout_selftest(1, status, returned, ms);
}

int query_grid_blocks(int device) {
    configure_query_kernels();
    int sms = 0, per = 1 << 30;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    for (int c = 0; c < kNumQueryConfigs; ++c) {
        int p = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p, kQueryKernels[c], kThreads, kQuerySmem[c]);
        per = std::min(per, p);
    }
    return sms * std::max(1, per);
}

cudaError_t launch_query(const QueryLaunch& L, int cfg, int grid, cudaStream_t st) {
    configure_query_kernels();
    void* args[] = {const_cast<QueryLaunch*>(&L)};
    return cudaLaunchCooperativeKernel((const void*)kQueryKernels[cfg], dim3(grid), dim3(kThreads), args,
                                       kQuerySmem[cfg], st);
}

}  // namespace hb
